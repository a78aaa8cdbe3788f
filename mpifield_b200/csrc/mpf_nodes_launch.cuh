// mpf_nodes_launch.cuh -- host-side dispatch of the node kernels over dimension, weight
// kind, degree and component count; instantiated once per element type.
#pragma once
#include <algorithm>

#include "mpf_nodes.cuh"
#include "mpifield_b200.h"

namespace mpf {

// Lets a kernel take `bytes` of dynamic shared memory (its static shared memory comes on
// top, so even 48 KB needs the attribute). Set once per kernel instantiation, device and
// size: `cache` is the instantiation's own table of the largest size set per device.
template <typename K> static int allow_smem(K kernel, int bytes, int* cache) {
    if (bytes <= 0) return MPF_OK;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) device = 0;
    if (cache[device] >= bytes) return MPF_OK;
    const int st = record_cuda_error(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    if (st == MPF_OK) cache[device] = bytes;
    return st;
}

static int pick_block(const Tuning& t) {
    int block = t.block > 0 ? std::min(t.block, kMaxBlock) : kMaxBlock;
    return std::max(32, block / 32 * 32);
}

// CTAs for `nchunks` chunks: as many as fit on an SM by shared memory (1 KB reserved per
// CTA), threads and the kernel's register bound (`max_per_sm`), times the SM count.
static unsigned grid_for(int64_t nchunks, int smem, int block, int max_per_sm = 2) {
    const int by_smem = std::max(1, (228 * 1024) / (smem + 1024 + 64));
    const int per_sm = std::max(1, std::min({max_per_sm, by_smem, 2048 / block}));
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(nchunks, (int64_t)sm_count() * per_sm));
}

// Entries of the field (the gather through L1 indexes it with 32-bit offsets).
template <typename T, int NDIM> static int64_t field_entries(const NodeArgs<T>& a) {
    int64_t e = a.ncomp;
    for (int d = 0; d < NDIM; ++d) e *= a.g.ext[d];
    return e;
}

// Whether every axis is periodic (the kernels then take the code as a constant).
template <typename T, int NDIM> static bool all_periodic(const NodeArgs<T>& a) {
    for (int d = 0; d < NDIM; ++d)
        if (a.g.code[d] != PERIODIC) return false;
    return true;
}

// Whether the position rows can be bulk-copied (16-byte aligned rows).
template <typename T, int NDIM> static int bulk_positions(const NodeArgs<T>& a) {
    const uintptr_t p = reinterpret_cast<uintptr_t>(a.pos);
    return (p % 16 == 0) && (NDIM == 1 || (a.pos_stride * (int64_t)sizeof(T)) % 16 == 0) ? 1 : 0;
}

// CTAs per SM of the tile kernels by element type: the float builds hold fewer registers
// (the float tile scatter fits 80 registers, the lean gather 64, without spills) and half
// the shared memory, so they run more CTAs (2^26 markers on 256^3: float scatter 1.99 ->
// 1.52 ms at three CTAs, gather 1.17 -> 1.14 ms at four); the double builds spill there.
template <typename T> constexpr int kLeanGatherMinBlocks = sizeof(T) == 4 ? 4 : 3;
template <typename T> constexpr int kTileScatterMinBlocksOf = sizeof(T) == 4 ? 3 : kTileScatterMinBlocks;

// The lean tile gather (mpf_runs.cuh): BLOCK threads, MINB CTAs per SM, BUFFERS boxes.
// Returns MPF_ERR_ARGUMENT, launching nothing, when the boxes do not fit.
template <typename T, int NDIM, int KIND, int P, int NC, int BLOCK, int MINB, int BUFFERS>
static int run_gather_lean(NodeArgs<T> a, cudaStream_t stream) {
    int64_t box = NC;
    for (int d = 0; d < NDIM; ++d) box *= (int64_t)a.tile[d] + P;
    const int64_t bytes = BUFFERS * box * (int64_t)sizeof(T);
    if (bytes > (228 * 1024) / MINB - 2048) return MPF_ERR_ARGUMENT;
    const int smem = (int)bytes;
    a.error = device_error_word();
    if (!a.error) return MPF_ERR_CUDA;
    auto kernel = gather_lean_kernel<T, NDIM, KIND, P, NC, 0, 0, 0, BLOCK, MINB, BUFFERS>;
    int shape = 0;
    if constexpr (NDIM == 3 && P == 2) {
        if (a.tile[0] == 8 && a.tile[1] == 8 && a.tile[2] == 8) {
            kernel = gather_lean_kernel<T, NDIM, KIND, P, NC, 8, 8, 8, BLOCK, MINB, BUFFERS>;
            shape = 1;
        } else if (a.tile[0] == 4 && a.tile[1] == 4 && a.tile[2] == 64) {
            kernel = gather_lean_kernel<T, NDIM, KIND, P, NC, 4, 4, 64, BLOCK, MINB, BUFFERS>;
            shape = 2;
        }
    }
    static int cache[3][64] = {{0}};
    if (allow_smem(kernel, smem, cache[shape]) != MPF_OK) return MPF_ERR_CUDA;
    const int64_t units = (a.n + BLOCK - 1) / BLOCK;
    kernel<<<grid_for(units, smem, BLOCK, MINB), BLOCK, smem, stream>>>(a);
    count_launches(1);
    return launch_status();
}

// Gather variants for markers sorted by cell tile (periodic axes, 1-3 components, fewer
// than 2^31 field entries, the tile's box within shared memory): 0 (default) the lean
// tile gather with one box and three (double) or four (float) CTAs of 256 per SM, 6 with
// two boxes and one CTA of
// 512. Otherwise, and for unsorted markers: through L1 while the field has fewer than
// 2^31 entries, else with staged boxes; 1 staged boxes (path 1: global reads in that
// kernel); 2 through L1.
template <typename T, int NDIM, int KIND, int P, int NC>
static int run_gather(NodeArgs<T> a, const Tuning& t, cudaStream_t stream) {
    if constexpr (NC > 0) {
        if (a.tile_start && (t.variant == 0 || t.variant == 6) && t.path != 1 && all_periodic<T, NDIM>(a) &&
            field_entries<T, NDIM>(a) < ((int64_t)1 << 31)) {
            const int st = t.variant == 6 ? run_gather_lean<T, NDIM, KIND, P, NC, 512, 1, 2>(a, stream)
                                          : run_gather_lean<T, NDIM, KIND, P, NC, 256, kLeanGatherMinBlocks<T>, 1>(a, stream);
            if (st != MPF_ERR_ARGUMENT) return st;
        }
    }
    const bool l1 = t.variant != 1 && field_entries<T, NDIM>(a) < ((int64_t)1 << 31);
    const int block = l1 ? kMaxBlock : pick_block(t);
    const int CH = kMarkersPerThread * block;
    const bool direct = t.path == 1 || l1;
    const int pos_bytes = 2 * NDIM * CH * (int)sizeof(T);
    int box_bytes = direct ? 0 : (t.smem_bytes > 0 ? t.smem_bytes : 48 * 1024);
    box_bytes = std::min(box_bytes, 227 * 1024 - pos_bytes);
    const int smem = pos_bytes + box_bytes;
    a.force_global = direct ? 1 : 0;
    a.capacity = box_bytes / (int)sizeof(T);
    a.bulk = bulk_positions<T, NDIM>(a);
    a.error = device_error_word();
    if (!a.error) return MPF_ERR_CUDA;
    a.wait_limit = t.wait_limit == 0 ? kDefaultWaitLimit : std::max(t.wait_limit, 0);
    const int64_t nchunks = (a.n + CH - 1) / CH;
    if (l1) {
        // (the boundary codes stay run-time values here: a periodic-only build of this kernel
        // measured slower)
        auto kernel = gather_l1_kernel<T, NDIM, KIND, P, NC, kGatherMinBlocks, -1>;
        static int cache[64] = {0};
        if (allow_smem(kernel, smem, cache) != MPF_OK) return MPF_ERR_CUDA;
        kernel<<<grid_for(nchunks, smem, block, kGatherMinBlocks), block, smem, stream>>>(a);
    } else {
        auto kernel = gather_kernel<T, NDIM, KIND, P, NC>;
        static int cache[64] = {0};
        if (allow_smem(kernel, smem, cache) != MPF_OK) return MPF_ERR_CUDA;
        kernel<<<grid_for(nchunks, smem, block), block, smem, stream>>>(a);
    }
    count_launches(1);
    return launch_status();
}

// The segment scatter (one component): 256 threads, a chunk of 256 x K markers in padded
// rows, MINB CTAs per SM, the box in the rest of the SM's shared memory (or t.smem_bytes).
template <typename T, int NDIM, int KIND, int P, int K, int MINB>
static int run_scatter_segments(NodeArgs<T> a, const Tuning& t, cudaStream_t stream) {
    const int buf_bytes = (NDIM + 1) * kMaxBlock * (K + 1) * (int)sizeof(T);
    const bool direct = t.path == 1;
    int box_bytes = direct ? 0 : t.smem_bytes;
    if (!direct && box_bytes <= 0) box_bytes = (228 * 1024) / MINB - 2048 - buf_bytes;
    box_bytes = std::max(0, std::min(box_bytes, 227 * 1024 - buf_bytes));
    const int smem = buf_bytes + box_bytes;
    a.force_global = direct ? 1 : 0;
    a.capacity = box_bytes / (int)sizeof(T);
    a.bulk = 0;
    a.error = device_error_word();
    if (!a.error) return MPF_ERR_CUDA;
    const bool per = all_periodic<T, NDIM>(a);
    auto kernel = per ? scatter_segments_kernel<T, NDIM, KIND, P, K, MINB, PERIODIC>
                      : scatter_segments_kernel<T, NDIM, KIND, P, K, MINB, -1>;
    static int cache[2][64] = {{0}};
    if (allow_smem(kernel, smem, cache[per]) != MPF_OK) return MPF_ERR_CUDA;
    const int CH = kMaxBlock * K;
    const int64_t nchunks = (a.n + CH - 1) / CH;
    kernel<<<grid_for(nchunks, smem, kMaxBlock, MINB), kMaxBlock, smem, stream>>>(a);
    count_launches(1);
    return launch_status();
}

// The tile scatter (markers sorted by cell tile, one component, periodic axes): BLOCK
// threads, MINB CTAs per SM, each CTA an equal share of the live markers. Returns
// MPF_ERR_ARGUMENT, launching nothing, when the tile's box does not fit beside the rows.
template <typename T, int NDIM, int KIND, int P, int K, int MINB, int BLOCK>
static int run_scatter_tiles(NodeArgs<T> a, cudaStream_t stream) {
    const int buf_bytes = (NDIM + 1) * BLOCK * (K + 1) * (int)sizeof(T);
    int64_t total = 1;
    for (int d = 0; d < NDIM; ++d) {
        int64_t e = (int64_t)a.tile[d] + P;
        if (d == NDIM - 1 && (e & 1) == 0) ++e;
        total *= e;
    }
    const int64_t box_bytes = total * (int64_t)sizeof(T);
    if (box_bytes > (228 * 1024) / MINB - 2048 - buf_bytes) return MPF_ERR_ARGUMENT;
    const int smem = buf_bytes + (int)box_bytes;
    a.error = device_error_word();
    if (!a.error) return MPF_ERR_CUDA;
    // the tile shapes of the 3D quadratic stores as compile-time constants, others at run time
    auto kernel = scatter_tiles_kernel<T, NDIM, KIND, P, K, MINB, 0, 0, 0, BLOCK>;
    int shape = 0;
    if constexpr (NDIM == 3 && P == 2) {
        if (a.tile[0] == 8 && a.tile[1] == 8 && a.tile[2] == 8) {
            kernel = scatter_tiles_kernel<T, NDIM, KIND, P, K, MINB, 8, 8, 8, BLOCK>;
            shape = 1;
        } else if (a.tile[0] == 8 && a.tile[1] == 8 && a.tile[2] == 16) {
            kernel = scatter_tiles_kernel<T, NDIM, KIND, P, K, MINB, 8, 8, 16, BLOCK>;
            shape = 2;
        } else if (a.tile[0] == 4 && a.tile[1] == 4 && a.tile[2] == 64) {
            kernel = scatter_tiles_kernel<T, NDIM, KIND, P, K, MINB, 4, 4, 64, BLOCK>;
            shape = 3;
        }
    }
    static int cache[4][64] = {{0}};
    if (allow_smem(kernel, smem, cache[shape]) != MPF_OK) return MPF_ERR_CUDA;
    const int64_t units = (a.n + BLOCK - 1) / BLOCK;
    kernel<<<grid_for(units, smem, BLOCK, MINB), BLOCK, smem, stream>>>(a);
    count_launches(1);
    return launch_status();
}

// The lean tile scatter (mpf_runs.cuh: coherent lanes, per-warp tables walked by
// stencil point): BLOCK threads, MINB CTAs per SM. Returns MPF_ERR_ARGUMENT, launching
// nothing, when the box and the tables do not fit.
template <typename T, int NDIM, int KIND, int P, int BLOCK, int MINB>
static int run_scatter_lean(NodeArgs<T> a, cudaStream_t stream) {
    constexpr int SP = StencilPoints<P + 1, NDIM>::value;
    int64_t box = 1;
    for (int d = 0; d < NDIM; ++d) {
        int64_t e = (int64_t)a.tile[d] + P;
        if (d == NDIM - 1 && (e & 1) == 0) ++e;
        box *= e;
    }
    const int64_t bytes = (((box + 1) & ~1) + (int64_t)(BLOCK / 32) * 32 * (SP + 2)) * (int64_t)sizeof(T);
    if (bytes > (228 * 1024) / MINB - 2048) return MPF_ERR_ARGUMENT;
    const int smem = (int)bytes;
    a.error = device_error_word();
    if (!a.error) return MPF_ERR_CUDA;
    auto kernel = scatter_lean_kernel<T, NDIM, KIND, P, 0, 0, 0, BLOCK, MINB>;
    int shape = 0;
    if constexpr (NDIM == 3 && P == 2) {
        if (a.tile[0] == 8 && a.tile[1] == 8 && a.tile[2] == 8) {
            kernel = scatter_lean_kernel<T, NDIM, KIND, P, 8, 8, 8, BLOCK, MINB>;
            shape = 1;
        } else if (a.tile[0] == 4 && a.tile[1] == 4 && a.tile[2] == 64) {
            kernel = scatter_lean_kernel<T, NDIM, KIND, P, 4, 4, 64, BLOCK, MINB>;
            shape = 2;
        }
    }
    static int cache[3][64] = {{0}};
    if (allow_smem(kernel, smem, cache[shape]) != MPF_OK) return MPF_ERR_CUDA;
    const int64_t units = (a.n + BLOCK - 1) / BLOCK;
    kernel<<<grid_for(units, smem, BLOCK, MINB), BLOCK, smem, stream>>>(a);
    count_launches(1);
    return launch_status();
}

// Scatter variants: 0 (default) the tile scatter for markers sorted by cell tile (one
// component, periodic axes, stencils of at most 27 points, the tile's box within shared
// memory), else the segment scatter for one component and stencils of at most 27
// points, else the warp-transposed run reduction; 1 the segment scatter where it
// applies (tile order ignored); 2 the warp-transposed run reduction; 5 for markers
// sorted by cell tile the lean tile scatter (block 128: four CTAs of 128 per SM).
template <typename T, int NDIM, int KIND, int P, int NC>
static int run_scatter(NodeArgs<T> a, const Tuning& t, cudaStream_t stream) {
    constexpr int SP = StencilPoints<P + 1, NDIM>::value;
    if constexpr (NC == 1 && SP <= 27) {
        if (a.tile_start && (t.variant == 0 || t.variant == 5) && t.path != 1 && all_periodic<T, NDIM>(a)) {
            if (t.variant == 5) {
                const int st = t.block == 128 ? run_scatter_lean<T, NDIM, KIND, P, 128, 4>(a, stream)
                                              : run_scatter_lean<T, NDIM, KIND, P, 256, 2>(a, stream);
                if (st != MPF_ERR_ARGUMENT) return st;
            }
            const int st =
                run_scatter_tiles<T, NDIM, KIND, P, kSegment, kTileScatterMinBlocksOf<T>, kTileScatterBlock>(a, stream);
            if (st != MPF_ERR_ARGUMENT) return st;
        }
        if (t.variant == 3) return run_scatter_segments<T, NDIM, KIND, P, 4, 3>(a, t, stream);
        if (t.variant != 2) return run_scatter_segments<T, NDIM, KIND, P, kSegment, 2>(a, t, stream);
    }
    constexpr int ROWS = SP < 32 ? SP : 32;
    const int block = pick_block(t);
    const int CH = kMarkersPerThread * block;
    const bool direct = t.path == 1;
    int box_bytes = direct ? 0 : (t.smem_bytes > 0 ? t.smem_bytes : 40 * 1024);
    const int scratch_bytes = direct ? 0 : (block / 32) * (ROWS * 33 * (int)sizeof(T) + 32 * (int)sizeof(int));
    box_bytes = std::min(box_bytes, 227 * 1024 - scratch_bytes);
    const int smem = box_bytes + scratch_bytes;
    a.force_global = direct ? 1 : 0;
    a.capacity = box_bytes / (int)sizeof(T);
    a.bulk = 0;
    a.error = device_error_word();
    if (!a.error) return MPF_ERR_CUDA;
    auto kernel = scatter_kernel<T, NDIM, KIND, P, NC>;
    static int cache[64] = {0};
    if (allow_smem(kernel, smem, cache) != MPF_OK) return MPF_ERR_CUDA;
    const int64_t nchunks = (a.n + CH - 1) / CH;
    kernel<<<grid_for(nchunks, smem, block), block, smem, stream>>>(a);
    count_launches(1);
    return launch_status();
}

template <typename T, int NDIM, int KIND, int P>
static int run_gather_grad(const NodeArgs<T>& a, cudaStream_t stream) {
    const int block = 256;
    const int64_t blocks = std::min<int64_t>((a.n + block - 1) / block, (int64_t)sm_count() * 8);
    gather_grad_kernel<T, NDIM, KIND, P><<<(unsigned)std::max<int64_t>(blocks, 1), block, 0, stream>>>(a);
    count_launches(1);
    return launch_status();
}

// The component count as a template argument for 1-3 components, a run-time loop above.
template <typename T, int NDIM, int KIND, int P, bool SCATTER, int NC>
static int run_node(const NodeArgs<T>& a, const Tuning& t, cudaStream_t stream) {
    if constexpr (SCATTER) return run_scatter<T, NDIM, KIND, P, NC>(a, t, stream);
    else return run_gather<T, NDIM, KIND, P, NC>(a, t, stream);
}

template <typename T, int NDIM, int KIND, int P, bool SCATTER>
static int by_components(const NodeArgs<T>& a, const Tuning& t, cudaStream_t stream) {
    switch (a.ncomp) {
        case 1: return run_node<T, NDIM, KIND, P, SCATTER, 1>(a, t, stream);
        case 2: return run_node<T, NDIM, KIND, P, SCATTER, 2>(a, t, stream);
        case 3: return run_node<T, NDIM, KIND, P, SCATTER, 3>(a, t, stream);
        default: return run_node<T, NDIM, KIND, P, SCATTER, 0>(a, t, stream);
    }
}

template <typename T, int NDIM, bool SCATTER>
static int by_kind(int kind, int degree, const NodeArgs<T>& a, const Tuning& t, cudaStream_t stream) {
    if (kind == LINEAR) return by_components<T, NDIM, LINEAR, 1, SCATTER>(a, t, stream);
    if (kind == QUADRATIC) return by_components<T, NDIM, QUADRATIC, 2, SCATTER>(a, t, stream);
    switch (degree) {
        case 0: return by_components<T, NDIM, SPLINE, 0, SCATTER>(a, t, stream);
        case 1: return by_components<T, NDIM, SPLINE, 1, SCATTER>(a, t, stream);
        case 2: return by_components<T, NDIM, SPLINE, 2, SCATTER>(a, t, stream);
        case 3: return by_components<T, NDIM, SPLINE, 3, SCATTER>(a, t, stream);
    }
    return MPF_ERR_ARGUMENT;
}

template <typename T, bool SCATTER>
static int by_dimension(int kind, int degree, int ndim, const NodeArgs<T>& a, const Tuning& t,
                        cudaStream_t stream) {
    switch (ndim) {
        case 1: return by_kind<T, 1, SCATTER>(kind, degree, a, t, stream);
        case 2: return by_kind<T, 2, SCATTER>(kind, degree, a, t, stream);
        case 3: return by_kind<T, 3, SCATTER>(kind, degree, a, t, stream);
    }
    return MPF_ERR_ARGUMENT;
}

template <typename T, int NDIM>
static int grad_by_kind(int kind, int degree, const NodeArgs<T>& a, cudaStream_t stream) {
    if (kind == LINEAR) return run_gather_grad<T, NDIM, LINEAR, 1>(a, stream);
    if (kind == QUADRATIC) return run_gather_grad<T, NDIM, QUADRATIC, 2>(a, stream);
    switch (degree) {
        case 0: return run_gather_grad<T, NDIM, SPLINE, 0>(a, stream);
        case 1: return run_gather_grad<T, NDIM, SPLINE, 1>(a, stream);
        case 2: return run_gather_grad<T, NDIM, SPLINE, 2>(a, stream);
        case 3: return run_gather_grad<T, NDIM, SPLINE, 3>(a, stream);
    }
    return MPF_ERR_ARGUMENT;
}

// One dimension's node launches (op 0 gather, 1 scatter, 2 position gradient); each
// element type and dimension is instantiated in a translation unit of its own.
template <typename T, int NDIM>
int node_launch(int op, int kind, int degree, const NodeArgs<T>& a, const Tuning& t, cudaStream_t stream) {
    if (op == 0) return by_kind<T, NDIM, false>(kind, degree, a, t, stream);
    if (op == 1) return by_kind<T, NDIM, true>(kind, degree, a, t, stream);
    return grad_by_kind<T, NDIM>(kind, degree, a, stream);
}

}  // namespace mpf

// mpf_nodes.cuh -- node gather, node scatter and the position gradient of a gather.
//
// The arithmetic is that of mpifield's gather_/scatter_{linear,quadratic,spline}_{1,2,3}d
// kernels (e.g. src/mpifield/kernels/gather_spline_3d/gather_spline_3d_cuda.cu:11-53,
// scatter_spline_3d/scatter_spline_3d_cuda.cu:12-61): result(c, i) = sum_k W_k(x_i) F(k, c)
// and F(k, c) += sum_i W_k(x_i) v(c, i), with W_k the tensor product of the per-axis
// stencils of mpf_stencil.cuh, and a marker whose values are all zero skipped before its
// position is read (scatter_quadratic_3d_cuda.cu:32-38).
//
// The B200 organisation is new. A CTA takes a chunk of MPT * blockDim consecutive markers
// (coalesced SoA loads, marker i of a chunk on thread i % blockDim), keeps their
// positions in cells in registers, and reduces the chunk's bounding box of stencil nodes
// (pre-mapping coordinates, so a box may straddle a periodic seam). When the box fits in
// the CTA's shared memory -- markers sorted by cell tile -- the gather stages that box of
// the field once and evaluates every marker from shared memory, and the scatter
// accumulates the chunk into a shared box with shared-memory atomics and flushes it with
// one global atomic add per non-zero node. Otherwise (unsorted markers, a chunk that
// spans the grid) the same chunk reads and adds straight to global memory. The sum over
// the stencil is factored axis by axis (x outermost), which changes the rounding of
// the reference's sum by a few ulps, not the nodes or the weights.
#pragma once
#include <climits>

#include "mpf_internal.h"
#include "mpf_stencil.cuh"
#include "mpifield_b200.h"

namespace mpf {

extern __shared__ __align__(16) unsigned char mpf_dynamic_smem[];

constexpr int kMarkersPerThread = 4;
constexpr int kMaxBlock = 256;
// CTAs of 256 threads per SM the gather through L1 is register-bounded for.
constexpr int kGatherMinBlocks = 3;
// Consecutive markers per thread in the segment scatter, and the widest margin of its boxes.
constexpr int kSegment = 8;
constexpr int kScatterMargin = 0;
// The tile scatter's CTA: threads and resident CTAs per SM (128 registers a thread).
constexpr int kTileScatterBlock = 256;
constexpr int kTileScatterMinBlocks = 2;

template <typename T>
__device__ __forceinline__ T rel_of(const NodeArgs<T>& a, int d, int64_t i) {
    return cells_from(a.pos[d * a.pos_stride + i] - a.g.lower[d], a.g.cell[d], a.g.inv[d], a.g.pow2[d]);
}

// Block-wide min of lo[] and max of hi[] over NDIM axes, into s_lo / s_hi (which the
// caller set to INT_MAX / INT_MIN and synchronised). Every thread of the block calls it.
template <int NDIM>
__device__ __forceinline__ void block_box(const int* lo, const int* hi, int* s_lo, int* s_hi) {
#pragma unroll
    for (int d = 0; d < NDIM; ++d) {
        const int l = __reduce_min_sync(0xffffffffu, lo[d]);
        const int h = __reduce_max_sync(0xffffffffu, hi[d]);
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&s_lo[d], l);
            atomicMax(&s_hi[d], h);
        }
    }
}

// The node offsets of a stencil: off[d][a] such that node (a, b, e) is at
// (off[0][a] + off[1][b] + off[2][e]) * ncomp. Unused axes hold one zero offset.
template <int NDIM, int S, typename I>
__device__ __forceinline__ void box_offsets(const int* base, const int* lo, const int* ex,
                                            I (&off)[3][S]) {
    const I sy = NDIM > 2 ? (I)ex[2] : (I)1;
    const I sx = NDIM > 1 ? (I)ex[1] * sy : (I)1;
    const I stride[3] = {sx, sy, (I)1};
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int a = 0; a < S; ++a)
            off[d][a] = d < NDIM ? (I)(base[d] - lo[d] + a) * stride[d] : (I)0;
}

template <int NDIM, int S>
__device__ __forceinline__ void global_offsets(const int* base, const int* num, const int* code,
                                               const int* ext, int64_t (&off)[3][S]) {
    const int64_t sy = NDIM > 2 ? (int64_t)ext[2] : 1;
    const int64_t sx = NDIM > 1 ? (int64_t)ext[1] * sy : 1;
    const int64_t stride[3] = {sx, sy, 1};
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int a = 0; a < S; ++a)
            off[d][a] = d < NDIM ? (int64_t)map_node(base[d] + a, num[d], code[d]) * stride[d] : 0;
}

template <typename T, bool LDG> __device__ __forceinline__ T load(const T* p) {
    if constexpr (LDG) return __ldg(p);
    else return *p;
}

// acc[c] = sum_a wx[a] sum_b wy[b] sum_e wz[e] src[(off) * ncomp + c0 + c], c < NCC.
template <typename T, int NDIM, int S, int NCC, bool LDG, typename I>
__device__ __forceinline__ void stencil_sum(const T* __restrict__ src, const I (&off)[3][S],
                                            const T (&w)[3][S], I ncomp, int c0, T* acc) {
    constexpr int SY = NDIM > 1 ? S : 1;
    constexpr int SZ = NDIM > 2 ? S : 1;
#pragma unroll
    for (int c = 0; c < NCC; ++c) acc[c] = T(0);
#pragma unroll
    for (int a = 0; a < S; ++a) {
        T sa[NCC];
#pragma unroll
        for (int c = 0; c < NCC; ++c) sa[c] = T(0);
#pragma unroll
        for (int b = 0; b < SY; ++b) {
            T sb[NCC];
#pragma unroll
            for (int c = 0; c < NCC; ++c) sb[c] = T(0);
#pragma unroll
            for (int e = 0; e < SZ; ++e) {
                const T* p = src + (off[0][a] + off[1][b] + off[2][e]) * ncomp + c0;
#pragma unroll
                for (int c = 0; c < NCC; ++c) {
                    const T v = load<T, LDG>(p + c);
                    if constexpr (NDIM > 2) sb[c] += w[2][e] * v;
                    else sb[c] += v;
                }
            }
#pragma unroll
            for (int c = 0; c < NCC; ++c) {
                if constexpr (NDIM > 1) sa[c] += w[1][b] * sb[c];
                else sa[c] += sb[c];
            }
        }
#pragma unroll
        for (int c = 0; c < NCC; ++c) acc[c] += w[0][a] * sa[c];
    }
}

// dst[(off) * ncomp + c0 + c] += W * v[c] with atomic adds.
template <typename T, int NDIM, int S, int NCC, typename I>
__device__ __forceinline__ void stencil_add(T* dst, const I (&off)[3][S], const T (&w)[3][S],
                                            I ncomp, int c0, const T (&v)[NCC]) {
    constexpr int SY = NDIM > 1 ? S : 1;
    constexpr int SZ = NDIM > 2 ? S : 1;
#pragma unroll
    for (int a = 0; a < S; ++a) {
#pragma unroll
        for (int b = 0; b < SY; ++b) {
            const T wab = NDIM > 1 ? w[0][a] * w[1][b] : w[0][a];
#pragma unroll
            for (int e = 0; e < SZ; ++e) {
                const T wt = NDIM > 2 ? wab * w[2][e] : wab;
                T* p = dst + (off[0][a] + off[1][b] + off[2][e]) * ncomp + c0;
#pragma unroll
                for (int c = 0; c < NCC; ++c) atomicAdd(p + c, wt * v[c]);
            }
        }
    }
}

// A box of the grid in shared memory: pre-mapping node lo[d] .. lo[d] + ex[d] - 1 per
// axis, node-major with the components innermost.
struct Box {
    int lo[3];
    int ex[3];
};

// The rows of a box: every row runs along the last axis, ex[NDIM-1] * ncomp elements,
// contiguous in shared memory and (away from a periodic seam) in global memory. One warp
// per row; the row's node prefix is mapped once, the last axis per element (with no
// mapping when the row lies inside the grid). Int32 arithmetic throughout: a box holds
// at most the shared memory of a CTA.
template <int NDIM>
__device__ __forceinline__ int box_rows(const Box& b) {
    int rows = 1;
#pragma unroll
    for (int d = 0; d < NDIM - 1; ++d) rows *= b.ex[d];
    return rows;
}

template <int NDIM, typename G>
__device__ __forceinline__ int64_t row_prefix(int r, const Box& b, const G& g) {
    // global node index of (row r, last-axis node 0), before the last axis is added
    int64_t prefix = 0;
    if constexpr (NDIM == 3) {
        const int jx = r / b.ex[1];
        const int jy = r - jx * b.ex[1];
        prefix = ((int64_t)map_node(b.lo[0] + jx, g.num[0], g.code[0]) * g.ext[1] +
                  map_node(b.lo[1] + jy, g.num[1], g.code[1])) * g.ext[2];
    } else if constexpr (NDIM == 2) {
        prefix = (int64_t)map_node(b.lo[0] + r, g.num[0], g.code[0]) * g.ext[1];
    }
    return prefix;
}

// tile <- the box of the field (a gather's staging).
template <typename T, int NDIM, int NC>
__device__ __forceinline__ void stage_box(T* __restrict__ tile, const T* __restrict__ field, const Box& b,
                                          const Grid<T>& g, int ncomp_rt) {
    const int ncomp = NC > 0 ? NC : ncomp_rt;
    constexpr int L = NDIM - 1;
    const int last = b.ex[L];
    const int rowlen = last * ncomp;
    const int rows = box_rows<NDIM>(b);
    const int lane = threadIdx.x & 31;
    const int nwarps = blockDim.x >> 5;
    const bool inside = g.code[L] == CLAMPED || (b.lo[L] >= 0 && b.lo[L] + last <= g.num[L]);
    for (int r = threadIdx.x >> 5; r < rows; r += nwarps) {
        const int64_t prefix = row_prefix<NDIM>(r, b, g);
        T* dst = tile + r * rowlen;
        if (inside) {
            const T* src = field + (prefix + b.lo[L]) * ncomp;
            for (int e = lane; e < rowlen; e += 32) dst[e] = __ldg(src + e);
        } else {
            for (int e = lane; e < rowlen; e += 32) {
                const int j = e / ncomp;
                const int c = e - j * ncomp;
                dst[e] = __ldg(field + (prefix + map_node(b.lo[L] + j, g.num[L], g.code[L])) * ncomp + c);
            }
        }
    }
}

// field += the non-zero entries of the box (a scatter's flush), global atomics.
template <typename T, int NDIM, int NC>
__device__ __forceinline__ void flush_box(const T* __restrict__ tile, T* field, const Box& b, const Grid<T>& g,
                                          int ncomp_rt) {
    const int ncomp = NC > 0 ? NC : ncomp_rt;
    constexpr int L = NDIM - 1;
    const int last = b.ex[L];
    const int rowlen = last * ncomp;
    const int rows = box_rows<NDIM>(b);
    const int lane = threadIdx.x & 31;
    const int nwarps = blockDim.x >> 5;
    for (int r = threadIdx.x >> 5; r < rows; r += nwarps) {
        const int64_t prefix = row_prefix<NDIM>(r, b, g);
        const T* src = tile + r * rowlen;
        for (int e = lane; e < rowlen; e += 32) {
            const T v = src[e];
            if (v != T(0)) {
                const int j = e / ncomp;
                const int c = e - j * ncomp;
                atomicAdd(field + (prefix + map_node(b.lo[L] + j, g.num[L], g.code[L])) * ncomp + c, v);
            }
        }
    }
}

template <int NDIM>
__device__ __forceinline__ bool box_holds(const Box& b, const int* lo, const int* hi_last) {
#pragma unroll
    for (int d = 0; d < NDIM; ++d)
        if (lo[d] < b.lo[d] || hi_last[d] > b.lo[d] + b.ex[d] - 1) return false;
    return true;
}

// The box for a chunk whose stencils span pre-mapping nodes lo[d] .. hi[d] + S - 1: the
// span widened by the largest margin (2, 1 or 0 nodes a side) that still fits
// `capacity` elements, so that the next chunks of the same cell tile fall inside it.
// On a clamped-knot axis (no mapping) the box stays inside the array. Returns false
// when not even the bare span fits.
// With ODD_LAST the last axis gets an odd extent where it can (one node more), so that
// nodes of the box a whole number of rows apart fall in different shared-memory banks.
template <int NDIM, int S, typename G, bool ODD_LAST = false, int MAX_MARGIN = 2>
__device__ __forceinline__ bool choose_box(const int* lo, const int* hi, int ncomp, int capacity, const G& g,
                                           Box& b) {
    for (int margin = MAX_MARGIN; margin >= 0; --margin) {
        int64_t vol = ncomp;
#pragma unroll
        for (int d = 0; d < NDIM; ++d) {
            int first = lo[d] - margin;
            int end = hi[d] + S + margin;  // one past the last node
            if (g.code[d] == CLAMPED) {
                first = max(first, 0);
                end = min(end, g.ext[d]);
            }
            if (ODD_LAST && d == NDIM - 1 && ((end - first) & 1) == 0) {
                if (g.code[d] != CLAMPED || end < g.ext[d]) ++end;
                else if (first > 0) --first;
            }
            b.lo[d] = first;
            b.ex[d] = end - first;
            vol *= b.ex[d];
        }
        if (vol <= (int64_t)capacity) return true;
    }
    return false;
}

// The chunks of CTA `block`: a contiguous range, so that consecutive chunks of a CTA
// come from the same cell tile when the markers are sorted by tile.
__device__ __forceinline__ void chunk_range(int64_t nchunks, int64_t& first, int64_t& last) {
    const int64_t per = (nchunks + gridDim.x - 1) / gridDim.x;
    first = (int64_t)blockIdx.x * per;
    last = min(first + per, nchunks);
}

// ------------------------------------------------ bulk copies (TMA) and barriers --
//
// The gather prefetches the positions of its next chunk into shared memory with 1D bulk
// copies (cp.async.bulk, no multicast) completing on an mbarrier; every wait is bounded
// and a CTA that gives up records MPF_DEVICE_ERROR_WAIT in *a.error and leaves.


__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int limit) {
    for (int i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// Puts the positions of chunk `ci` (count markers from `first`) into rows
// buf[d * CH ...]: bulk copies of the 16-byte multiple, plain loads for the rest.
// Called by one thread; the barrier completes when the bulk bytes have landed.
template <typename T, int NDIM>
__device__ __forceinline__ void issue_positions(const NodeArgs<T>& a, T* buf, int CH, int64_t first, int count,
                                                uint64_t* bar) {
    const unsigned bytes = (unsigned)count * (unsigned)sizeof(T);
    const unsigned bulk = bytes & ~15u;
    mbar_expect_tx(bar, bulk * NDIM);
#pragma unroll
    for (int d = 0; d < NDIM; ++d)
        if (bulk) bulk_g2s(buf + d * CH, a.pos + d * a.pos_stride + first, bulk, bar);
    for (int j = bulk / sizeof(T); j < count; ++j)
#pragma unroll
        for (int d = 0; d < NDIM; ++d) buf[d * CH + j] = a.pos[d * a.pos_stride + first + j];
}

// A CTA that gave up waiting for the positions of its chunk k (buffer b): before it
// leaves, thread 0 waits for every bulk copy it issued that may still be in flight -- the
// one into buffer b and, if issued, the next chunk's into buffer b ^ 1 -- each wait
// bounded by the default limit, so that no copy lands in shared memory after the CTA
// has handed it back. Then it records MPF_DEVICE_ERROR_WAIT.
template <typename T>
__device__ __forceinline__ void drain_and_flag(const NodeArgs<T>& a, uint64_t* bars, int b, int k, bool next) {
    mbar_wait(&bars[b], (k >> 1) & 1, kDefaultWaitLimit);
    if (next) mbar_wait(&bars[b ^ 1], ((k + 1) >> 1) & 1, kDefaultWaitLimit);
    atomicOr(a.error, (unsigned)MPF_DEVICE_ERROR_WAIT);
}

template <typename T>
__device__ __forceinline__ T rel_from(const T x, const Grid<T>& g, int d) {
    return cells_from(x - g.lower[d], g.cell[d], g.inv[d], g.pow2[d]);
}

// The gather. Positions of chunk k wait in shared buffer k % 2 while the bulk copy of
// chunk k + 1 fills the other; the field box is staged as described above.
template <typename T, int NDIM, int KIND, int P, int NC>
__global__ void __launch_bounds__(kMaxBlock, 2) gather_kernel(const NodeArgs<T> a) {
    constexpr int S = P + 1;
    constexpr int NCC = NC > 0 ? NC : 1;
    constexpr int MPT = kMarkersPerThread;
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ int s_lo[3], s_hi[3];
    const int ncomp = NC > 0 ? NC : a.ncomp;
    const int CH = MPT * blockDim.x;
    T* posbuf = reinterpret_cast<T*>(mpf_dynamic_smem);  // [2][NDIM][CH]
    T* tile = posbuf + 2 * NDIM * CH;
    const int64_t nchunks = (a.n + CH - 1) / CH;
    int64_t c_first, c_last;
    chunk_range(nchunks, c_first, c_last);
    if (c_first >= c_last) return;
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (a.bulk && threadIdx.x == 0)
        issue_positions<T, NDIM>(a, posbuf, CH, c_first * CH, (int)min((int64_t)CH, a.n - c_first * CH), &bars[0]);
    Box box;
    bool have_box = false;
    for (int64_t ci = c_first; ci < c_last; ++ci) {
        const int k = (int)(ci - c_first);
        const int b = k & 1;
        const int64_t first = ci * CH;
        const int count = (int)min((int64_t)CH, a.n - first);
        T* pb = posbuf + b * NDIM * CH;
        if (a.bulk) {
            if (threadIdx.x == 0 && ci + 1 < c_last) {
                fence_proxy_async();
                issue_positions<T, NDIM>(a, posbuf + (b ^ 1) * NDIM * CH, CH, first + CH,
                                         (int)min((int64_t)CH, a.n - first - CH), &bars[b ^ 1]);
            }
            const bool late = !mbar_wait(&bars[b], (k >> 1) & 1, a.wait_limit);
            if (__syncthreads_or(late)) {
                if (threadIdx.x == 0) drain_and_flag(a, bars, b, k, ci + 1 < c_last);
                __syncthreads();
                return;
            }
        } else {
            for (int j = threadIdx.x; j < count; j += blockDim.x)
#pragma unroll
                for (int d = 0; d < NDIM; ++d) pb[d * CH + j] = a.pos[d * a.pos_stride + first + j];
            __syncthreads();
        }
        int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
#pragma unroll
        for (int m = 0; m < MPT; ++m) {
            const int j = m * blockDim.x + threadIdx.x;
            if (j < count) {
#pragma unroll
                for (int d = 0; d < NDIM; ++d) {
                    T w[S];
                    const int base = axis_stencil<T, KIND, P>(rel_from(pb[d * CH + j], a.g, d), a.g.num[d],
                                                              a.g.code[d], w);
                    lo[d] = min(lo[d], base);
                    hi[d] = max(hi[d], base);
                }
            }
        }
        bool staged = false;
        if (!a.force_global) {
            if (threadIdx.x < 3) {
                s_lo[threadIdx.x] = INT_MAX;
                s_hi[threadIdx.x] = INT_MIN;
            }
            __syncthreads();
            block_box<NDIM>(lo, hi, s_lo, s_hi);
            __syncthreads();
            int clo[3], chi[3], top[3];
#pragma unroll
            for (int d = 0; d < NDIM; ++d) {
                clo[d] = s_lo[d];
                chi[d] = s_hi[d];
                top[d] = chi[d] + S - 1;
            }
            if (have_box && box_holds<NDIM>(box, clo, top)) {
                staged = true;
            } else {
                Box nb;
                if (choose_box<NDIM, S>(clo, chi, ncomp, a.capacity, a.g, nb)) {
                    stage_box<T, NDIM, NC>(tile, a.field_in, nb, a.g, ncomp);
                    box = nb;
                    have_box = true;
                    staged = true;
                    __syncthreads();
                }
            }
        }
#pragma unroll
        for (int m = 0; m < MPT; ++m) {
            const int j = m * blockDim.x + threadIdx.x;
            if (j >= count) continue;
            const int64_t i = first + j;
            T w[3][S];
            int base[3] = {0, 0, 0};
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (d < NDIM) {
                    base[d] = axis_stencil<T, KIND, P>(rel_from(pb[d * CH + j], a.g, d), a.g.num[d], a.g.code[d],
                                                       w[d]);
                } else {
#pragma unroll
                    for (int s = 0; s < S; ++s) w[d][s] = T(s == 0);
                }
            }
            if (staged) {
                int off[3][S];
                box_offsets<NDIM, S, int>(base, box.lo, box.ex, off);
                if constexpr (NC > 0) {
                    T acc[NCC];
                    stencil_sum<T, NDIM, S, NCC, false, int>(tile, off, w, NC, 0, acc);
#pragma unroll
                    for (int c = 0; c < NCC; ++c) a.result[c * a.res_stride + i] = acc[c];
                } else {
                    for (int c = 0; c < ncomp; ++c) {
                        T acc[1];
                        stencil_sum<T, NDIM, S, 1, false, int>(tile, off, w, ncomp, c, acc);
                        a.result[c * a.res_stride + i] = acc[0];
                    }
                }
            } else {
                int64_t off[3][S];
                global_offsets<NDIM, S>(base, a.g.num, a.g.code, a.g.ext, off);
                if constexpr (NC > 0) {
                    T acc[NCC];
                    stencil_sum<T, NDIM, S, NCC, true, int64_t>(a.field_in, off, w, NC, 0, acc);
#pragma unroll
                    for (int c = 0; c < NCC; ++c) a.result[c * a.res_stride + i] = acc[c];
                } else {
                    for (int c = 0; c < ncomp; ++c) {
                        T acc[1];
                        stencil_sum<T, NDIM, S, 1, true, int64_t>(a.field_in, off, w, ncomp, c, acc);
                        a.result[c * a.res_stride + i] = acc[0];
                    }
                }
            }
        }
        // the positions buffer and the box are free once every thread is past this point
        __syncthreads();
    }
}

template <int S, int NDIM> struct StencilPoints {
    static constexpr int value = NDIM == 1 ? S : (NDIM == 2 ? S * S : S * S * S);
};


// The gather through L1: the positions of a chunk come by bulk copy as in gather_kernel,
// and each marker reads its S^ndim nodes straight from global memory with 32-bit offsets
// (the launcher uses it for fields of fewer than 2^31 entries), with no box and no
// bounding pass: in a marker store sorted by cell, the nodes of consecutive markers stay
// in L1. Bounded to MINB CTAs of 256 threads per SM.
template <typename T, int NDIM, int KIND, int P, int NC, int MINB, int UNI>
__global__ void __launch_bounds__(kMaxBlock, MINB) gather_l1_kernel(const NodeArgs<T> a) {
    constexpr int S = P + 1;
    constexpr int NCC = NC > 0 ? NC : 1;
    constexpr int MPT = kMarkersPerThread;
    __shared__ __align__(8) uint64_t bars[2];
    const int ncomp = NC > 0 ? NC : a.ncomp;
    // UNI >= 0: every axis has that boundary code (a compile-time constant)
    auto code = [&](int d) { return UNI >= 0 ? UNI : a.g.code[d]; };
    const int CH = MPT * blockDim.x;
    T* posbuf = reinterpret_cast<T*>(mpf_dynamic_smem);  // [2][NDIM][CH]
    const int64_t nchunks = (a.n + CH - 1) / CH;
    int64_t c_first, c_last;
    chunk_range(nchunks, c_first, c_last);
    if (c_first >= c_last) return;
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (a.bulk && threadIdx.x == 0)
        issue_positions<T, NDIM>(a, posbuf, CH, c_first * CH, (int)min((int64_t)CH, a.n - c_first * CH), &bars[0]);
    const int sy = NDIM > 2 ? a.g.ext[2] : 1;
    const int sx = NDIM > 1 ? a.g.ext[1] * sy : 1;
    const int stride[3] = {NDIM == 1 ? 1 : sx, NDIM == 2 ? 1 : sy, 1};
    for (int64_t ci = c_first; ci < c_last; ++ci) {
        const int k = (int)(ci - c_first);
        const int b = k & 1;
        const int64_t first = ci * CH;
        const int count = (int)min((int64_t)CH, a.n - first);
        T* pb = posbuf + b * NDIM * CH;
        if (a.bulk) {
            if (threadIdx.x == 0 && ci + 1 < c_last) {
                fence_proxy_async();
                issue_positions<T, NDIM>(a, posbuf + (b ^ 1) * NDIM * CH, CH, first + CH,
                                         (int)min((int64_t)CH, a.n - first - CH), &bars[b ^ 1]);
            }
            const bool late = !mbar_wait(&bars[b], (k >> 1) & 1, a.wait_limit);
            if (__syncthreads_or(late)) {
                if (threadIdx.x == 0) drain_and_flag(a, bars, b, k, ci + 1 < c_last);
                __syncthreads();
                return;
            }
        } else {
            for (int j = threadIdx.x; j < count; j += blockDim.x)
#pragma unroll
                for (int d = 0; d < NDIM; ++d) pb[d * CH + j] = a.pos[d * a.pos_stride + first + j];
            __syncthreads();
        }
#pragma unroll 1
        for (int m = 0; m < MPT; ++m) {
            const int j = m * blockDim.x + threadIdx.x;
            if (j >= count) continue;
            const int64_t i = first + j;
            T w[3][S];
            int off[3][S];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (d < NDIM) {
                    const int base = axis_stencil<T, KIND, P>(rel_from(pb[d * CH + j], a.g, d), a.g.num[d],
                                                              code(d), w[d]);
#pragma unroll
                    for (int s = 0; s < S; ++s) off[d][s] = map_node(base + s, a.g.num[d], code(d)) * stride[d];
                } else {
#pragma unroll
                    for (int s = 0; s < S; ++s) {
                        w[d][s] = T(s == 0);
                        off[d][s] = 0;
                    }
                }
            }
            if constexpr (NC > 0) {
                T acc[NCC];
                stencil_sum<T, NDIM, S, NCC, true, int>(a.field_in, off, w, NC, 0, acc);
#pragma unroll
                for (int c = 0; c < NCC; ++c) a.result[c * a.res_stride + i] = acc[c];
            } else {
                for (int c = 0; c < ncomp; ++c) {
                    T acc[1];
                    stencil_sum<T, NDIM, S, 1, true, int>(a.field_in, off, w, ncomp, c, acc);
                    a.result[c * a.res_stride + i] = acc[0];
                }
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------- runs of one stencil anchor --
//
// The open run of a thread in the segment and tile scatters: the weighted sums of its
// markers of one anchor, acc[(x SY + y) SZ + z] for node (x, y, z) of the stencil.

template <int NDIM, int S> struct RunShape {
    static constexpr int SY = NDIM > 1 ? S : 1;
    static constexpr int SZ = NDIM > 2 ? S : 1;
    static constexpr int SP = S * SY * SZ;
};

// acc += v w_x w_y w_z: a marker's contributions to its run.
template <typename T, int NDIM, int S>
__device__ __forceinline__ void run_add(T (&acc)[RunShape<NDIM, S>::SP], const T (&w)[3][S], T v) {
    constexpr int SY = RunShape<NDIM, S>::SY, SZ = RunShape<NDIM, S>::SZ;
    T wz[SZ];
#pragma unroll
    for (int z = 0; z < SZ; ++z) wz[z] = (NDIM > 2 ? w[2][z] : T(1)) * v;
#pragma unroll
    for (int x = 0; x < S; ++x)
#pragma unroll
        for (int y = 0; y < SY; ++y) {
            const T wxy = NDIM > 2 ? w[0][x] * w[1][y] : (NDIM > 1 ? w[0][x] * (w[1][y] * v) : w[0][x] * v);
#pragma unroll
            for (int z = 0; z < SZ; ++z) {
                T& r = acc[(x * SY + y) * SZ + z];
                r = NDIM > 2 ? fma(wxy, wz[z], r) : r + wxy;
            }
        }
}

// Adds the run anchored at box entry `at` to the box (node (x, y, z) at at + x sa + y sb +
// z se, shared-memory atomics) and empties it.
template <typename T, int NDIM, int S>
__device__ __forceinline__ void run_flush(T* box, int at, int sa, int sb, int se, T (&acc)[RunShape<NDIM, S>::SP]) {
    constexpr int SY = RunShape<NDIM, S>::SY, SZ = RunShape<NDIM, S>::SZ;
#pragma unroll
    for (int x = 0; x < S; ++x)
#pragma unroll
        for (int y = 0; y < SY; ++y)
#pragma unroll
            for (int z = 0; z < SZ; ++z) {
                atomicAdd(box + at + x * sa + y * sb + z * se, acc[(x * SY + y) * SZ + z]);
                acc[(x * SY + y) * SZ + z] = T(0);
            }
}

// The closing runs of a warp (key -1: none), added to the box. Lanes of one anchor form
// contiguous groups in a sorted store; where groups of four or more lanes occur (the dense
// cells of a beam) each group is summed across the warp first (a segmented suffix sum into
// its first lane). Every lane of the warp calls it.
template <typename T, int NDIM, int S>
__device__ __forceinline__ void run_close(T* box, int key, int sa, int sb, int se,
                                          T (&acc)[RunShape<NDIM, S>::SP]) {
    constexpr int SP = RunShape<NDIM, S>::SP;
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int tag = key >= 0 ? key : -2 - lane;
    const unsigned peers = __match_any_sync(FULL, tag);
    const int head = __ffs(peers) - 1;
    const int size = __popc(peers);
    const int biggest = __reduce_max_sync(FULL, size);
    const bool contiguous = peers == ((size == 32 ? FULL : ((1u << size) - 1u)) << head);
    if (biggest >= 4 && __all_sync(FULL, contiguous)) {
        const int last = head + size - 1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
            for (int q = 0; q < SP; ++q) {
                const T other = __shfl_down_sync(FULL, acc[q], o);
                if (lane + o <= last) acc[q] += other;
            }
        }
        if (key >= 0 && lane == head) run_flush<T, NDIM, S>(box, key, sa, sb, se, acc);
    } else if (key >= 0) {
        run_flush<T, NDIM, S>(box, key, sa, sb, se, acc);
    }
}

// 4- or 8-byte asynchronous copy global -> shared (cp.async, completion by group).
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// The segment scatter of one component (stencils of at most 27 points). A chunk is
// 256 x K consecutive markers; thread t owns the K markers t K .. t K + K - 1, which sit in
// shared memory at t (K + 1) .. (a pitch of K + 1 keeps the lanes of a warp on distinct
// banks at every step). The thread walks its markers in order and sums their weighted
// contributions in registers while the stencil anchor stays the same; on a change of
// anchor, and at the end of the segment, it adds the sum to the chunk's box in shared
// memory (27 atomic adds per run instead of 27 per marker: markers of a cell are
// consecutive in a store sorted by cell). At the end, lanes whose runs share an anchor --
// the dense cells of a beam -- are summed across the warp first. Pass 1 turns each live
// position into its cell coordinate in place and reduces the box; chunks whose box does
// not fit add to global memory marker by marker.
template <typename T, int NDIM, int KIND, int P, int K, int MINB, int UNI>
__global__ void __launch_bounds__(kMaxBlock, MINB) scatter_segments_kernel(const NodeArgs<T> a) {
    constexpr int S = P + 1;
    constexpr int SY = NDIM > 1 ? S : 1;
    constexpr int SZ = NDIM > 2 ? S : 1;
    constexpr int SP = S * SY * SZ;
    constexpr int PITCH = K + 1;
    constexpr int ROWS = NDIM + 1;
    constexpr int CH = kMaxBlock * K;
    constexpr int ROW = kMaxBlock * PITCH;
    // UNI >= 0: every axis has that boundary code (a compile-time constant)
    auto code = [&](int d) { return UNI >= 0 ? UNI : a.g.code[d]; };
    __shared__ int s_lo[3], s_hi[3], s_lo2[3], s_hi2[3];
    T* buf = reinterpret_cast<T*>(mpf_dynamic_smem);  // [ROWS][ROW]
    T* tile = buf + ROWS * ROW;
    // A periodic axis can also be measured in a frame shifted by half a period (anchor a
    // as ((a + half) mod num) + num - half, the same node modulo num): a chunk that
    // crosses the seam of the grid -- the last and the first tiles of a row -- has a short
    // span in that frame. The box takes whichever frame is shorter, per axis.
    int half[3], shifted[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < NDIM; ++d) half[d] = a.g.num[d] / 2;
    const int t = threadIdx.x;
    const int64_t nchunks = (a.n + CH - 1) / CH;
    int64_t c_first, c_last;
    chunk_range(nchunks, c_first, c_last);
    Box box;
    bool have_box = false;
    for (int64_t ci = c_first; ci < c_last; ++ci) {
        const int64_t first = ci * CH;
        const int count = (int)min((int64_t)CH, a.n - first);
        for (int j = t; j < count; j += kMaxBlock) {
            const int q = (j / K) * PITCH + j % K;
#pragma unroll
            for (int d = 0; d < NDIM; ++d) cp_async<sizeof(T)>(buf + d * ROW + q, a.pos + d * a.pos_stride + first + j);
            cp_async<sizeof(T)>(buf + NDIM * ROW + q, a.values + first + j);
        }
        cp_async_commit();
        cp_async_wait_all();
        __syncthreads();
        // pass 1: cell coordinates in place, and the box of the live markers
        const int nmine = min(K, max(0, count - t * K));
        T* mine = buf + t * PITCH;
        int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
        int lo2[3] = {INT_MAX, INT_MAX, INT_MAX}, hi2[3] = {INT_MIN, INT_MIN, INT_MIN};
#pragma unroll 1
        for (int s = 0; s < nmine; ++s) {
            if (mine[NDIM * ROW + s] == T(0)) continue;
#pragma unroll
            for (int d = 0; d < NDIM; ++d) {
                const T rel = rel_from(mine[d * ROW + s], a.g, d);
                mine[d * ROW + s] = rel;
                T w[S];
                const int base = axis_stencil<T, KIND, P>(rel, a.g.num[d], code(d), w);
                lo[d] = min(lo[d], base);
                hi[d] = max(hi[d], base);
                const int moved = wrap_index(base + half[d], a.g.num[d]);
                lo2[d] = min(lo2[d], moved);
                hi2[d] = max(hi2[d], moved);
            }
        }
        bool staged = false;
        if (!a.force_global) {
            if (t < 3) {
                s_lo[t] = INT_MAX;
                s_hi[t] = INT_MIN;
                s_lo2[t] = INT_MAX;
                s_hi2[t] = INT_MIN;
            }
            __syncthreads();
            block_box<NDIM>(lo, hi, s_lo, s_hi);
            block_box<NDIM>(lo2, hi2, s_lo2, s_hi2);
            __syncthreads();
            int clo[3], chi[3], top[3], frame[3] = {0, 0, 0};
            bool empty = false;
#pragma unroll
            for (int d = 0; d < NDIM; ++d) {
                clo[d] = s_lo[d];
                chi[d] = s_hi[d];
                if (code(d) == PERIODIC && s_hi2[d] - s_lo2[d] < chi[d] - clo[d]) {
                    frame[d] = 1;
                    clo[d] = s_lo2[d] + a.g.num[d] - half[d];
                    chi[d] = s_hi2[d] + a.g.num[d] - half[d];
                }
                top[d] = chi[d] + S - 1;
                if (chi[d] < clo[d]) empty = true;
            }
            if (empty) {  // every marker of the chunk is dead
                __syncthreads();
                continue;
            }
            bool same_frame = true;
#pragma unroll
            for (int d = 0; d < NDIM; ++d) same_frame = same_frame && frame[d] == shifted[d];
            if (have_box && same_frame && box_holds<NDIM>(box, clo, top)) {
                staged = true;
            } else {
                Box nb;
                if (choose_box<NDIM, S, Grid<T>, true, kScatterMargin>(clo, chi, 1, a.capacity, a.g, nb)) {
                    if (have_box) flush_box<T, NDIM, 1>(tile, a.field_out, box, a.g, 1);
                    __syncthreads();
                    int total = 1;
#pragma unroll
                    for (int d = 0; d < NDIM; ++d) total *= nb.ex[d];
                    for (int q = t; q < total; q += kMaxBlock) tile[q] = T(0);
                    __syncthreads();
                    box = nb;
#pragma unroll
                    for (int d = 0; d < NDIM; ++d) shifted[d] = frame[d];
                    have_box = true;
                    staged = true;
                }
            }
        }
        if (staged) {
            // box strides: node (a, b, e) of anchor key is tile[key + a sa + b sb + e se]
            int st[3];
            st[NDIM - 1] = 1;
#pragma unroll
            for (int d = NDIM - 2; d >= 0; --d) st[d] = st[d + 1] * box.ex[d + 1];
            const int sa = st[0];
            const int sb = NDIM > 1 ? st[1] : 0;
            const int se = NDIM > 2 ? st[2] : 0;
            T acc[SP];
#pragma unroll
            for (int q = 0; q < SP; ++q) acc[q] = T(0);
            int key = -1;  // the anchor of the open run, -1: none
#pragma unroll 1
            for (int s = 0; s < nmine; ++s) {
                const T v = mine[NDIM * ROW + s];
                if (v == T(0)) continue;
                T w[3][S];
                int k = 0;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    if (d < NDIM) {
                        int base = axis_stencil<T, KIND, P>(mine[d * ROW + s], a.g.num[d], code(d), w[d]);
                        if (shifted[d]) base = wrap_index(base + half[d], a.g.num[d]) + a.g.num[d] - half[d];
                        k += (base - box.lo[d]) * st[d];
                    } else {
#pragma unroll
                        for (int z = 0; z < S; ++z) w[d][z] = T(z == 0);
                    }
                }
                if (k != key && key >= 0) run_flush<T, NDIM, S>(tile, key, sa, sb, se, acc);
                run_add<T, NDIM, S>(acc, w, v);
                key = k;
            }
            run_close<T, NDIM, S>(tile, key, sa, sb, se, acc);
        } else {
            // no box: each live marker adds to global memory
#pragma unroll 1
            for (int s = 0; s < nmine; ++s) {
                const T v = mine[NDIM * ROW + s];
                if (v == T(0)) continue;
                T w[3][S];
                int base[3] = {0, 0, 0};
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    if (d < NDIM) {
                        base[d] = axis_stencil<T, KIND, P>(mine[d * ROW + s], a.g.num[d], code(d), w[d]);
                    } else {
#pragma unroll
                        for (int z = 0; z < S; ++z) w[d][z] = T(z == 0);
                    }
                }
                int64_t off[3][S];
                global_offsets<NDIM, S>(base, a.g.num, a.g.code, a.g.ext, off);
                const T vv[1] = {v};
                stencil_add<T, NDIM, S, 1, int64_t>(a.field_out, off, w, 1, 0, vv);
            }
        }
        // the buffer and the box are free once every thread is past this point
        __syncthreads();
    }
    if (have_box) flush_box<T, NDIM, 1>(tile, a.field_out, box, a.g, 1);
}

// ------------------------------------------------------- the tile scatter (sorted) --

// The tile holding rank m, searched from tile `t` (tile_start[t] <= m): the tile whose
// ranks reach past m, tile_start[t + 1] > m. A store sorted by tile mostly needs the
// next tile or the one after, so a few steps forward come first, then a binary search.
// Always a tile in [0, ntiles).
__device__ __forceinline__ int64_t tile_of(const int64_t* ts, int64_t ntiles, int64_t t, int64_t m) {
    t = min(max(t, (int64_t)0), ntiles - 1);
#pragma unroll 1
    for (int step = 0; step < 4; ++step, ++t)
        if (t + 1 >= ntiles || __ldg(ts + t + 1) > m) return t;
    int64_t lo = t, hi = ntiles - 1;  // the last tile in [t, ntiles) starting at or before m
#pragma unroll 1
    while (lo < hi) {
        const int64_t mid = lo + (hi - lo + 1) / 2;
        if (__ldg(ts + mid) <= m) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// The extents of the box of a tile (tile + P nodes per axis, the last made odd so that
// nodes a whole number of rows apart fall in different shared-memory banks).
template <int NDIM, int P>
__device__ __forceinline__ void tile_box_extents(const int* tile, int* ex) {
#pragma unroll
    for (int d = 0; d < NDIM; ++d) ex[d] = tile[d] + P;
    if ((ex[NDIM - 1] & 1) == 0) ++ex[NDIM - 1];
}

// Calls fn(e, at) for the entries e of a tile's box that this thread takes, at being the
// entry's node index in the grid. The box is row-major with extents ex; its entry
// (0, 0, 0) is the pre-mapping node lo of a grid whose axes are all periodic (num, ext).
// Thread t takes entries t, t + B, t + 2B, ... (B = blockDim.x), its box coordinates found
// once and then advanced by those of B with one carry per axis: no division per entry.
template <int NDIM, typename F>
__device__ __forceinline__ void for_box_entries(const int* lo, const int* ex, const int* num, const int* ext,
                                                F&& fn) {
    int total = 1;
#pragma unroll
    for (int d = 0; d < NDIM; ++d) total *= ex[d];
    int c[3] = {0, 0, 0}, dc[3] = {0, 0, 0};
    int q = threadIdx.x, b = blockDim.x;
#pragma unroll
    for (int d = NDIM - 1; d > 0; --d) {
        c[d] = q % ex[d];
        q /= ex[d];
        dc[d] = b % ex[d];
        b /= ex[d];
    }
    c[0] = q;
    dc[0] = b;
#pragma unroll 1
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        fn(e, [&]() {
            int64_t at = 0;
#pragma unroll
            for (int d = 0; d < NDIM; ++d) at = at * ext[d] + wrap_index(lo[d] + c[d], num[d]);
            return at;
        });
        int carry = 0;
#pragma unroll
        for (int d = NDIM - 1; d >= 0; --d) {
            c[d] += dc[d] + carry;
            carry = 0;
            if (d > 0 && c[d] >= ex[d]) {
                c[d] -= ex[d];
                carry = 1;
            }
        }
    }
}

// field += the non-zero entries of a tile's box (global atomics), and the box zeroed.
template <typename T, int NDIM>
__device__ __forceinline__ void flush_clear_box(T* box, T* field, const int* lo, const int* ex, const Grid<T>& g) {
    for_box_entries<NDIM>(lo, ex, g.num, g.ext, [&](int e, auto node) {
        const T v = box[e];
        if (v != T(0)) {
            box[e] = T(0);
            atomicAdd(field + node(), v);
        }
    });
}

}  // namespace mpf

// the lean tile kernels (they use the helpers above; the tile scatter below uses their
// piece walk)
#include "mpf_runs.cuh"

namespace mpf {

// The tile scatter: the segment scatter (above) for markers sorted by cell tile
// (mpf_sort_by_tile), one component, every axis periodic. tile_start names the ranks of
// every tile, so the CTA's share of the ranks (an equal share of the live markers, the
// tiles before the sentinel) splits at tile boundaries into pieces whose box is known
// in advance: the tile's anchors widened by the stencil, tile + P nodes per axis (the
// last axis made odd for the shared-memory banks). No box reduction, no frame choice,
// one flush per piece, fused with the zeroing. Thread t owns the t-th of 256 contiguous
// ranges of a piece, taken K markers at a time in sub-chunks (the padded rows of the
// segment scatter, thread t's markers at t (K + 1) ..), so a thread's runs carry over the
// sub-chunk boundaries and close once per piece. Runs of one anchor are summed in
// registers and added to the box as there,
// except that a run followed by the next cell along the last axis (anchor + 1, the
// usual step in a store sorted by cell) adds only the plane of its window that the
// next run does not touch and slides the rest: S^(NDIM-1) shared-memory atomics
// instead of S^NDIM, the atomics being what the kernel's time goes to. Thread 0 plans
// the sub-chunks; the plan and the loop state live in shared memory, not in the
// registers of the marker loop. A marker whose anchor is not in the piece's tile
// (tile_start not made from these positions) adds to global memory directly: the
// result never depends on the order.
struct TileLoop {
    int64_t m, m_end;  // the next rank of the CTA's share, and its end
    int64_t cur;       // the tile of the box (-1: none)
    int64_t e;         // the end of the current piece
    int64_t part, extra;
    int sub, nsub;     // sub-chunks of the current piece: done, in all
};
struct TileStep {
    int64_t first;  // the sub-chunk's first rank (with thread ranges: the piece's)
    int count;      // its markers (with thread ranges: the piece's; 0: the CTA is done)
    int sub, nsub;  // with thread ranges: the sub-chunk of the piece, and their number
    int retire;     // 1: add the box of the previous tile (first node old_lo) to the field first
    int blo[3];     // the sub-chunk's tile: its first anchor per axis
    int old_lo[3];
};

// Thread 0's plan of the next sub-chunk: tile pieces cut at tile_start (at most 2^30
// markers), each into nearly equal sub-chunks of at most ch markers, or with thread ranges
// (RANGES: the piece's markers split into blockDim.x contiguous ranges, sub-chunk s taking
// markers s ch .. s ch + ch - 1 of every range) into as many sub-chunks as the longest
// range needs.
template <int NDIM, int H, bool RANGES = false>
__device__ __forceinline__ void plan_tile_step(TileLoop& L, TileStep& st, const int64_t* ts, int64_t ntiles,
                                               const int* tiles, const int* tl, int ch) {
    st.retire = 0;
    if (L.sub >= L.nsub) {
        L.m = L.e;
        if (L.m >= L.m_end) {
            st.count = 0;
            st.retire = L.cur >= 0 ? 1 : 0;
#pragma unroll
            for (int d = 0; d < NDIM; ++d) st.old_lo[d] = st.blo[d] - H;
            L.cur = -1;
            return;
        }
        const int64_t tt = tile_of(ts, ntiles, L.cur, L.m);
        L.e = min(min(L.m_end, L.m + ((int64_t)1 << 30)), max(L.m + 1, __ldg(ts + tt + 1)));
        if (tt != L.cur) {
            st.retire = L.cur >= 0 ? 1 : 0;
            int rest = (int)tt;  // tiles number fewer than 2^31
#pragma unroll
            for (int d = NDIM - 1; d >= 0; --d) {
                st.old_lo[d] = st.blo[d] - H;
                const int c = rest % tiles[d];
                rest /= tiles[d];
                st.blo[d] = c * tl[d];
            }
            L.cur = tt;
        }
        const int n32 = (int)(L.e - L.m);  // below 2^30
        if (RANGES) {
            const int longest = n32 / (int)blockDim.x + (n32 % (int)blockDim.x != 0 ? 1 : 0);
            L.nsub = longest / ch + (longest % ch != 0 ? 1 : 0);
        } else {
            L.nsub = n32 / ch + (n32 % ch != 0 ? 1 : 0);
            L.part = n32 / L.nsub;
            L.extra = n32 - (int)L.part * L.nsub;
        }
        L.sub = 0;
    }
    if (RANGES) {
        st.first = L.m;
        st.count = (int)(L.e - L.m);
    } else {
        st.first = L.m + L.sub * L.part + min((int64_t)L.sub, L.extra);
        st.count = (int)(L.part + (L.sub < L.extra ? 1 : 0));
    }
    st.sub = L.sub;
    st.nsub = L.nsub;
    ++L.sub;
}

template <typename T, int NDIM, int KIND, int P, int K, int MINB, int TX = 0, int TY = 0, int TZ = 0,
          int BLOCK = kMaxBlock>
__global__ void __launch_bounds__(BLOCK, MINB) scatter_tiles_kernel(const NodeArgs<T> a) {
    constexpr int S = P + 1;
    constexpr int SY = NDIM > 1 ? S : 1;
    constexpr int SZ = NDIM > 2 ? S : 1;
    constexpr int SP = S * SY * SZ;
    constexpr int PITCH = K + 1;
    constexpr int ROWS = NDIM + 1;
    constexpr int ROW = BLOCK * PITCH;
    constexpr int H = P / 2;  // a stencil's anchor is its first node + H
    __shared__ TileLoop s_loop;
    __shared__ TileStep s_step;
    T* buf = reinterpret_cast<T*>(mpf_dynamic_smem);  // [ROWS][ROW]
    T* box = buf + ROWS * ROW;
    const int t = threadIdx.x;
    // the tile shape: compile-time constants where the launch fixes them (TX, TY, TZ > 0),
    // so that the box strides and every stencil offset in the box are immediates
    const int tl[3] = {TX > 0 ? TX : a.tile[0], TY > 0 ? TY : a.tile[1], TZ > 0 ? TZ : a.tile[2]};
    int ex[3] = {1, 1, 1};
    tile_box_extents<NDIM, P>(tl, ex);
    for (int q = t; q < ex[0] * ex[1] * ex[2]; q += BLOCK) box[q] = T(0);
    if (t == 0) {
        const int64_t live = min(max(__ldg(a.tile_start + a.ntiles), (int64_t)0), a.n);
        const int64_t per = (live + gridDim.x - 1) / gridDim.x;
        s_loop.m = min((int64_t)blockIdx.x * per, live);
        s_loop.m_end = min(s_loop.m + per, live);
        s_loop.e = s_loop.m;
        s_loop.cur = -1;
        s_loop.sub = s_loop.nsub = 0;
        s_loop.part = s_loop.extra = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) s_step.blo[d] = s_step.old_lo[d] = 0;
    }
    // box strides: node (x, y, z) of anchor key is box[key + x sa + y sb + z se]
    const int se = NDIM > 2 ? 1 : 0;
    const int sb = NDIM > 2 ? ex[2] : (NDIM > 1 ? 1 : 0);
    const int sa = NDIM > 2 ? ex[1] * ex[2] : (NDIM > 1 ? ex[1] : 1);
    const int st[3] = {sa, NDIM > 1 ? sb : 0, NDIM > 2 ? se : 0};
    // the open run of the thread: it carries over the sub-chunks of a piece
    T acc[SP];
#pragma unroll
    for (int q = 0; q < SP; ++q) acc[q] = T(0);
    int key = -1;  // the anchor of the open run, -1: none
#pragma unroll 1
    for (;;) {
        if (t == 0) plan_tile_step<NDIM, H, true>(s_loop, s_step, a.tile_start, a.ntiles, a.tiles, tl, K);
        // the plan is visible, the previous sub-chunk's adds are complete and its rows free
        __syncthreads();
        const int64_t first = s_step.first;
        const int count = s_step.count;
        const int sub = s_step.sub;
        const bool closing = sub + 1 >= s_step.nsub;
        if (s_step.retire) {
            const int lo[3] = {s_step.old_lo[0], s_step.old_lo[1], s_step.old_lo[2]};
            flush_clear_box<T, NDIM>(box, a.field_out, lo, ex, a.g);
            __syncthreads();
        }
        if (count == 0) break;
        const int blo[3] = {s_step.blo[0], s_step.blo[1], s_step.blo[2]};
        // the piece in BLOCK contiguous ranges (thread u: `per` markers, one more for
        // u < rem); this sub-chunk holds markers sub K .. sub K + K - 1 of every range,
        // thread u's at row position u (K + 1) + j, read by groups of K consecutive lanes
        const int per = count / BLOCK, rem = count % BLOCK;
        for (int q = t; q < BLOCK * K; q += BLOCK) {
            const int u = q / K, j = q % K;
            const int idx = sub * K + j;
            if (idx < per + (u < rem ? 1 : 0)) {
                const int64_t g = first + (int64_t)u * per + min(u, rem) + idx;
                const int at = u * PITCH + j;
#pragma unroll
                for (int d = 0; d < NDIM; ++d)
                    cp_async<sizeof(T)>(buf + d * ROW + at, a.pos + d * a.pos_stride + g);
                cp_async<sizeof(T)>(buf + NDIM * ROW + at, a.values + g);
            }
        }
        cp_async_commit();
        cp_async_wait_all();
        __syncthreads();
        const int nmine = min(K, max(0, per + (t < rem ? 1 : 0) - sub * K));
        // a run that ends: the plane of its window at the first node along the last axis is
        // complete whatever comes next, and every ending run adds it in the same
        // instructions. A run followed by the next cell along the last axis (anchor + 1, the
        // usual step in a store sorted by cell) slides its other planes down; one followed by
        // the cell after that (anchor + 2: an empty cell between) adds its second plane too
        // and slides by two; any other adds all of them and empties.
        constexpr int LASTN = NDIM == 3 ? SZ : (NDIM == 2 ? SY : S);
        constexpr int OUTER = SP / LASTN;
        auto end_run = [&](int at, int step) {
            const int shift = (step >= 1 && step < LASTN) ? step : LASTN;
#pragma unroll
            for (int l = 0; l < LASTN; ++l) {
                if (l == 0 || shift > l) {
#pragma unroll
                    for (int o = 0; o < OUTER; ++o) {
                        const int ob = NDIM == 3 ? (o / SY) * sa + (o % SY) * sb : (NDIM == 2 ? o * sa : 0);
                        atomicAdd(box + at + ob + l, acc[o * LASTN + l]);
                    }
                }
            }
            if (shift == 1) {
#pragma unroll
                for (int o = 0; o < OUTER; ++o) {
#pragma unroll
                    for (int l = 0; l + 1 < LASTN; ++l) acc[o * LASTN + l] = acc[o * LASTN + l + 1];
                    acc[o * LASTN + LASTN - 1] = T(0);
                }
            } else if (LASTN > 2 && shift == 2) {
#pragma unroll
                for (int o = 0; o < OUTER; ++o) {
#pragma unroll
                    for (int l = 0; l < LASTN; ++l) acc[o * LASTN + l] = l + 2 < LASTN ? acc[o * LASTN + l + 2] : T(0);
                }
            } else {
#pragma unroll
                for (int q = 0; q < SP; ++q) acc[q] = T(0);
            }
        };
        // the next marker's position and value are read while the current one is worked on
        T nx[4] = {T(0), T(0), T(0), T(0)};
        if (nmine > 0) {
#pragma unroll
            for (int d = 0; d <= NDIM; ++d) nx[d] = buf[d * ROW + t * PITCH];
        }
#pragma unroll 1
        for (int s = 0; s < nmine; ++s) {
            T cx[4];
#pragma unroll
            for (int d = 0; d < 4; ++d) cx[d] = nx[d];
            if (s + 1 < nmine) {
#pragma unroll
                for (int d = 0; d <= NDIM; ++d) nx[d] = buf[d * ROW + t * PITCH + s + 1];
            }
            const T v = cx[NDIM];
            if (v == T(0)) continue;
            T w[3][S];
            int base[3] = {0, 0, 0};
            int k = 0;
            bool inside = true;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (d < NDIM) {
                    const T rel = rel_from(cx[d], a.g, d);
                    base[d] = axis_stencil<T, KIND, P>(rel, a.g.num[d], PERIODIC, w[d]);
                    const int off = wrap_index(base[d] + H - blo[d], a.g.num[d]);
                    inside = inside && (unsigned)off < (unsigned)tl[d];
                    k += off * st[d];
                } else {
#pragma unroll
                    for (int z = 0; z < S; ++z) w[d][z] = T(z == 0);
                }
            }
            if (!inside) {  // not this tile's marker: straight to global memory
                int64_t goff[3][S];
                global_offsets<NDIM, S>(base, a.g.num, a.g.code, a.g.ext, goff);
                const T vv[1] = {v};
                stencil_add<T, NDIM, S, 1, int64_t>(a.field_out, goff, w, 1, 0, vv);
                continue;
            }
            if (k != key && key >= 0) end_run(key, P > 0 ? k - key : 0);
            run_add<T, NDIM, S>(acc, w, v);
            key = k;
        }
        if (!closing) continue;  // the runs go on in the piece's next sub-chunk
        run_close<T, NDIM, S>(box, key, sa, sb, se, acc);
        // every run is closed (the other lanes of a group summed into its head)
#pragma unroll
        for (int q = 0; q < SP; ++q) acc[q] = T(0);
        key = -1;
    }
    // the sentinel tile's ranks (values zero when the store was sorted) through global memory
    PieceWalk rest;
    rest.start(a.tile_start, a.ntiles, a.n);
    scatter_tail<T, NDIM, KIND, P>(a, rest.tail, rest.tail_end, BLOCK);
}

// The scatter. The markers of a chunk go to warps in contiguous runs of 32 (lane l of
// warp w, step s: marker (w * MPT + s) * 32 + l of the chunk), so that in a marker store
// sorted by cell the lanes of a warp hold markers of a few cells. For a box chunk, every
// lane writes the stencil contributions of its marker into the warp's scratch
// (a [stencil point][33] table); lane o then runs along the 32 markers summing
// contribution o over runs of markers with the same stencil base, and adds each run's
// sum to the box with one shared-memory add. Within an instruction the lanes add to
// distinct nodes, so the adds of a warp never contend.
template <typename T, int NDIM, int KIND, int P, int NC>
__global__ void __launch_bounds__(kMaxBlock, 2) scatter_kernel(const NodeArgs<T> a) {
    constexpr int S = P + 1;
    constexpr int NCC = NC > 0 ? NC : 1;
    constexpr int MPT = kMarkersPerThread;
    constexpr int SP = StencilPoints<S, NDIM>::value;
    constexpr int ROWS = SP < 32 ? SP : 32;
    constexpr int GROUPS = (SP + 31) / 32;
    constexpr int PITCH = 33;
    __shared__ int s_lo[3], s_hi[3];
    const int ncomp = NC > 0 ? NC : a.ncomp;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    const int CH = MPT * blockDim.x;
    T* tile = reinterpret_cast<T*>(mpf_dynamic_smem);
    T* scratch = tile + a.capacity + warp * (ROWS * PITCH);  // this warp's [ROWS][PITCH]
    int* bidx = reinterpret_cast<int*>(tile + a.capacity + nwarps * (ROWS * PITCH)) + warp * 32;
    const int64_t nchunks = (a.n + CH - 1) / CH;
    int64_t c_first, c_last;
    chunk_range(nchunks, c_first, c_last);
    Box box;
    bool have_box = false;  // the box holds deposits not yet flushed
    for (int64_t ci = c_first; ci < c_last; ++ci) {
        const int64_t first = ci * CH + (int64_t)warp * 32 * MPT;
        T rel[MPT][NDIM];
        T val[MPT][NCC];
        bool live[MPT];
        int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
#pragma unroll
        for (int m = 0; m < MPT; ++m) {
            const int64_t i = first + m * 32 + lane;
            live[m] = false;
            if (i < a.n) {
                // a dead marker (all values zero) deposits nothing and its position,
                // which may be non-finite, is not read
                if constexpr (NC > 0) {
#pragma unroll
                    for (int c = 0; c < NCC; ++c) {
                        val[m][c] = a.values[c * a.val_stride + i];
                        live[m] = live[m] || val[m][c] != T(0);
                    }
                } else {
                    for (int c = 0; c < ncomp; ++c) live[m] = live[m] || a.values[c * a.val_stride + i] != T(0);
                }
            }
            if (live[m]) {
#pragma unroll
                for (int d = 0; d < NDIM; ++d) {
                    rel[m][d] = rel_of(a, d, i);
                    T w[S];
                    const int b = axis_stencil<T, KIND, P>(rel[m][d], a.g.num[d], a.g.code[d], w);
                    lo[d] = min(lo[d], b);
                    hi[d] = max(hi[d], b);
                }
            }
        }
        bool staged = false;
        if (!a.force_global) {
            if (threadIdx.x < 3) {
                s_lo[threadIdx.x] = INT_MAX;
                s_hi[threadIdx.x] = INT_MIN;
            }
            __syncthreads();
            block_box<NDIM>(lo, hi, s_lo, s_hi);
            __syncthreads();
            int clo[3], chi[3], top[3];
            bool empty = false;
#pragma unroll
            for (int d = 0; d < NDIM; ++d) {
                clo[d] = s_lo[d];
                chi[d] = s_hi[d];
                top[d] = chi[d] + S - 1;
                if (chi[d] < clo[d]) empty = true;
            }
            if (empty) continue;  // no live marker in the chunk (uniform across the CTA)
            if (have_box && box_holds<NDIM>(box, clo, top)) {
                staged = true;
            } else {
                Box nb;
                if (choose_box<NDIM, S>(clo, chi, ncomp, a.capacity, a.g, nb)) {
                    if (have_box) flush_box<T, NDIM, NC>(tile, a.field_out, box, a.g, ncomp);
                    __syncthreads();
                    int total = ncomp;
#pragma unroll
                    for (int d = 0; d < NDIM; ++d) total *= nb.ex[d];
                    for (int k = threadIdx.x; k < total; k += blockDim.x) tile[k] = T(0);
                    __syncthreads();
                    box = nb;
                    have_box = true;
                    staged = true;
                }
            }
        }
        if (staged) {
            const int sy = NDIM > 2 ? box.ex[2] : 1;
            const int sx = NDIM > 1 ? box.ex[1] * sy : 1;
#pragma unroll
            for (int m = 0; m < MPT; ++m) {
                // this lane's marker: its stencil base in the box (or -1) and weights
                T w[3][S];
                int bofs = -1;
                if (live[m]) {
                    int base[3] = {0, 0, 0};
#pragma unroll
                    for (int d = 0; d < NDIM; ++d)
                        base[d] = axis_stencil<T, KIND, P>(rel[m][d], a.g.num[d], a.g.code[d], w[d]) - box.lo[d];
                    bofs = base[0] * sx + (NDIM > 1 ? base[1] * sy : 0) + (NDIM > 2 ? base[2] : 0);
                } else {
#pragma unroll
                    for (int d = 0; d < 3; ++d)
#pragma unroll
                        for (int s = 0; s < S; ++s) w[d][s] = T(0);
                }
                bidx[lane] = bofs;
                // one component: the contributions, then the runs, group by group
                auto deposit = [&](int c, T v) {
#pragma unroll
                    for (int g = 0; g < GROUPS; ++g) {
                        // contributions of stencil points g * 32 + r, r < ROWS
#pragma unroll
                        for (int r = 0; r < ROWS; ++r) {
                            const int o = g * 32 + r;
                            if (o < SP) {
                                const int ea = NDIM == 3 ? o / (S * S) : (NDIM == 2 ? o / S : o);
                                const int eb = NDIM == 3 ? (o / S) % S : (NDIM == 2 ? o % S : 0);
                                const int ee = NDIM == 3 ? o % S : 0;
                                T wt = w[0][ea];
                                if constexpr (NDIM > 1) wt = wt * w[1][eb];
                                if constexpr (NDIM > 2) wt = wt * w[2][ee];
                                scratch[r * PITCH + lane] = wt * v;
                            }
                        }
                        __syncwarp();
                        const int o = g * 32 + lane;
                        if (lane < ROWS && o < SP) {
                            const int ea = NDIM == 3 ? o / (S * S) : (NDIM == 2 ? o / S : o);
                            const int eb = NDIM == 3 ? (o / S) % S : (NDIM == 2 ? o % S : 0);
                            const int ee = NDIM == 3 ? o % S : 0;
                            const int off = ea * sx + eb * sy + ee;
                            T acc = T(0);
                            int run = bidx[0];
                            for (int j = 0; j < 32; ++j) {
                                const int bj = bidx[j];
                                if (bj != run) {
                                    if (run >= 0) atomicAdd(tile + (run + off) * ncomp + c, acc);
                                    acc = T(0);
                                    run = bj;
                                }
                                acc += scratch[lane * PITCH + j];
                            }
                            if (run >= 0) atomicAdd(tile + (run + off) * ncomp + c, acc);
                        }
                        __syncwarp();
                    }
                };
                if constexpr (NC > 0) {
#pragma unroll
                    for (int c = 0; c < NCC; ++c) deposit(c, live[m] ? val[m][c] : T(0));
                } else {
                    for (int c = 0; c < ncomp; ++c)
                        deposit(c, live[m] ? a.values[c * a.val_stride + first + m * 32 + lane] : T(0));
                }
            }
        } else {
#pragma unroll
            for (int m = 0; m < MPT; ++m) {
                if (!live[m]) continue;
                const int64_t i = first + m * 32 + lane;
                T w[3][S];
                int base[3] = {0, 0, 0};
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    if (d < NDIM) {
                        base[d] = axis_stencil<T, KIND, P>(rel[m][d], a.g.num[d], a.g.code[d], w[d]);
                    } else {
#pragma unroll
                        for (int s = 0; s < S; ++s) w[d][s] = T(s == 0);
                    }
                }
                int64_t off[3][S];
                global_offsets<NDIM, S>(base, a.g.num, a.g.code, a.g.ext, off);
                if constexpr (NC > 0) {
                    stencil_add<T, NDIM, S, NCC, int64_t>(a.field_out, off, w, NC, 0, val[m]);
                } else {
                    for (int c = 0; c < ncomp; ++c) {
                        const T v[1] = {a.values[c * a.val_stride + i]};
                        stencil_add<T, NDIM, S, 1, int64_t>(a.field_out, off, w, ncomp, c, v);
                    }
                }
            }
        }
        if (!a.force_global) __syncthreads();
    }
    if (have_box) {
        __syncthreads();
        flush_box<T, NDIM, NC>(tile, a.field_out, box, a.g, ncomp);
    }
}

// grad(d, i) = sum_c cot(c, i) d/dx_d sum_k W_k(x_i) F(k, c): one thread per marker,
// global memory (the backward pass of a gather with respect to the positions).
template <typename T, int NDIM, int KIND, int P>
__global__ void __launch_bounds__(kMaxBlock) gather_grad_kernel(const NodeArgs<T> a) {
    constexpr int S = P + 1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        T w[3][S], g[3][S];
        int base[3] = {0, 0, 0};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (d < NDIM) {
                base[d] = axis_stencil_derivative<T, KIND, P>(rel_of(a, d, i), a.g.num[d], a.g.code[d],
                                                              w[d], g[d]);
            } else {
#pragma unroll
                for (int s = 0; s < S; ++s) w[d][s] = g[d][s] = T(s == 0);
            }
        }
        int64_t off[3][S];
        global_offsets<NDIM, S>(base, a.g.num, a.g.code, a.g.ext, off);
#pragma unroll
        for (int d = 0; d < NDIM; ++d) {
            T mixed[3][S];
#pragma unroll
            for (int e = 0; e < 3; ++e)
#pragma unroll
                for (int s = 0; s < S; ++s) mixed[e][s] = e == d ? g[e][s] : w[e][s];
            T total = T(0);
            for (int c = 0; c < a.ncomp; ++c) {
                T acc[1];
                stencil_sum<T, NDIM, S, 1, true, int64_t>(a.field_in, off, mixed, a.ncomp, c, acc);
                total += a.values[c * a.val_stride + i] * acc[0];
            }
            a.result[d * a.res_stride + i] = total / a.g.cell[d];
        }
    }
}

}  // namespace mpf

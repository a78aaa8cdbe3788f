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

struct LaunchShape {
    int block;
    int smem;
    unsigned grid;
};

template <typename T>
static LaunchShape node_shape(const NodeArgs<T>& a, const Tuning& t, bool staged_path) {
    LaunchShape s;
    s.block = t.block > 0 ? std::min(t.block, kMaxBlock) : kMaxBlock;
    s.block = std::max(32, s.block / 32 * 32);
    s.smem = staged_path ? (t.smem_bytes > 0 ? t.smem_bytes : 48 * 1024) : 0;
    s.smem = std::min(s.smem, 227 * 1024);
    const int64_t chunk = (int64_t)kMarkersPerThread * s.block;
    const int64_t nchunks = (a.n + chunk - 1) / chunk;
    const int per_sm = t.ctas_per_sm > 0 ? t.ctas_per_sm : (staged_path ? std::max(1, (200 * 1024) / std::max(s.smem, 1)) : 4);
    const int64_t cap = (int64_t)sm_count() * std::min(per_sm, 2048 / s.block);
    s.grid = (unsigned)std::max<int64_t>(1, std::min(nchunks, cap));
    return s;
}

template <typename T, int NDIM, int KIND, int P, int NC>
static int run_gather(NodeArgs<T> a, const Tuning& t, cudaStream_t stream) {
    const bool staged_path = t.path != 1;
    LaunchShape s = node_shape(a, t, staged_path);
    a.force_global = staged_path ? 0 : 1;
    a.capacity = s.smem / (int)sizeof(T);
    auto kernel = gather_kernel<T, NDIM, KIND, P, NC>;
    static int cache[64] = {0};
    if (allow_smem(kernel, s.smem, cache) != MPF_OK) return MPF_ERR_CUDA;
    kernel<<<s.grid, s.block, s.smem, stream>>>(a);
    count_launches(1);
    return launch_status();
}

template <typename T, int NDIM, int KIND, int P, int NC>
static int run_scatter(NodeArgs<T> a, const Tuning& t, cudaStream_t stream) {
    const bool staged_path = t.path != 1;
    LaunchShape s = node_shape(a, t, staged_path);
    a.force_global = staged_path ? 0 : 1;
    a.capacity = s.smem / (int)sizeof(T);
    auto kernel = scatter_kernel<T, NDIM, KIND, P, NC>;
    static int cache[64] = {0};
    if (allow_smem(kernel, s.smem, cache) != MPF_OK) return MPF_ERR_CUDA;
    kernel<<<s.grid, s.block, s.smem, stream>>>(a);
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

// mpf_paths.cu -- launches of the path deposits and edge gathers (mpf_paths.cuh).
#include <algorithm>

#include "mpf_paths.cuh"
#include "mpifield_b200.h"

namespace mpf {

// One thread per path with global atomics (the default: the L2's FP64 adds measured
// faster than shared-memory boxes here, where many lanes add to the same nodes),
// or the tiled kernel (path 2, staged): chunks of 256 x t.block paths (8 when t.block is
// 0), a box of edges in t.smem_bytes (96 KB when 0) of shared memory.
template <typename T, int NDIM, int P, bool WHITNEY>
static int run_deposit(PathArgs<T> a, const Tuning& t, cudaStream_t stream) {
    const int block = 256;
    if (t.path != 2) {
        auto launch = [&](auto kernel, int threads) {
            const int64_t blocks = std::min<int64_t>((a.n + threads - 1) / threads, (int64_t)sm_count() * 32);
            kernel<<<(unsigned)std::max<int64_t>(blocks, 1), threads, 0, stream>>>(a);
        };
        // two CTAs per SM (128 registers a thread) where the path fits them without spills
        // (WHITNEY and spline edges of degree <= 2: QUADRATIC_EDGES 15% faster than one);
        // the cubic edges keep one CTA and their registers. Variant 1: one CTA everywhere;
        // variant 3: spline paths a path at a time instead of piece by piece.
        if constexpr (!WHITNEY && P >= 3) {
            if (t.variant == 3) launch(deposit_paths_kernel<T, NDIM, P, WHITNEY, 256, 1, false>, 256);
            else launch(deposit_paths_kernel<T, NDIM, P, WHITNEY, 256, 1>, 256);
        } else {
            if (t.variant == 1) launch(deposit_paths_kernel<T, NDIM, P, WHITNEY, 256, 1>, 256);
            else if (t.variant == 3) launch(deposit_paths_kernel<T, NDIM, P, WHITNEY, 256, 2, false>, 256);
            else launch(deposit_paths_kernel<T, NDIM, P, WHITNEY, 256, 2>, 256);
        }
        count_launches(1);
        return launch_status();
    }
    const int smem = t.smem_bytes > 0 ? std::min(t.smem_bytes, 227 * 1024) : 96 * 1024;
    a.capacity = smem / (int)sizeof(T);
    a.paths_per_thread = t.block > 0 ? std::max(1, t.block) : 8;
    auto kernel = deposit_paths_tiled_kernel<T, NDIM, P, WHITNEY>;
    static int cache[64] = {0};
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) device = 0;
    if (cache[device] < smem) {
        if (record_cuda_error(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != MPF_OK)
            return MPF_ERR_CUDA;
        cache[device] = smem;
    }
    const int64_t ch = (int64_t)block * a.paths_per_thread;
    const int64_t nchunks = (a.n + ch - 1) / ch;
    const int per_sm = std::max(1, (228 * 1024) / (smem + 2048));
    const int64_t blocks = std::min<int64_t>(nchunks, (int64_t)sm_count() * per_sm);
    kernel<<<(unsigned)std::max<int64_t>(blocks, 1), block, smem, stream>>>(a);
    count_launches(1);
    return launch_status();
}

template <typename T, int NDIM, int P, bool WHITNEY>
static int run_gather_edges(const PathArgs<T>& a, cudaStream_t stream) {
    const int block = 256;
    const int64_t blocks = std::min<int64_t>((a.n + block - 1) / block, (int64_t)sm_count() * 16);
    gather_edges_kernel<T, NDIM, P, WHITNEY><<<(unsigned)std::max<int64_t>(blocks, 1), block, 0, stream>>>(a);
    count_launches(1);
    return launch_status();
}

template <typename T, int NDIM, bool GATHER>
static int paths_by_kind(int kind, int degree, const PathArgs<T>& a, const Tuning& t, cudaStream_t stream) {
    if (kind == LINEAR) return GATHER ? run_gather_edges<T, NDIM, 1, true>(a, stream) : run_deposit<T, NDIM, 1, true>(a, t, stream);
    switch (degree) {
        case 1: return GATHER ? run_gather_edges<T, NDIM, 1, false>(a, stream) : run_deposit<T, NDIM, 1, false>(a, t, stream);
        case 2: return GATHER ? run_gather_edges<T, NDIM, 2, false>(a, stream) : run_deposit<T, NDIM, 2, false>(a, t, stream);
        case 3: return GATHER ? run_gather_edges<T, NDIM, 3, false>(a, stream) : run_deposit<T, NDIM, 3, false>(a, t, stream);
    }
    return MPF_ERR_ARGUMENT;
}

template <typename T>
int launch_deposit_paths(int kind, int degree, int ndim, PathArgs<T> a, const Tuning& t, cudaStream_t stream) {
    switch (ndim) {
        case 1: return paths_by_kind<T, 1, false>(kind, degree, a, t, stream);
        case 2: return paths_by_kind<T, 2, false>(kind, degree, a, t, stream);
        case 3: return paths_by_kind<T, 3, false>(kind, degree, a, t, stream);
    }
    return MPF_ERR_ARGUMENT;
}

template <typename T>
int launch_gather_edges(int kind, int degree, int ndim, const PathArgs<T>& a, cudaStream_t stream) {
    const Tuning t{0, 0, 0, 0, 0};
    switch (ndim) {
        case 1: return paths_by_kind<T, 1, true>(kind, degree, a, t, stream);
        case 2: return paths_by_kind<T, 2, true>(kind, degree, a, t, stream);
        case 3: return paths_by_kind<T, 3, true>(kind, degree, a, t, stream);
    }
    return MPF_ERR_ARGUMENT;
}

template int launch_deposit_paths<double>(int, int, int, PathArgs<double>, const Tuning&, cudaStream_t);
template int launch_deposit_paths<float>(int, int, int, PathArgs<float>, const Tuning&, cudaStream_t);
template int launch_gather_edges<double>(int, int, int, const PathArgs<double>&, cudaStream_t);
template int launch_gather_edges<float>(int, int, int, const PathArgs<float>&, cudaStream_t);

}  // namespace mpf

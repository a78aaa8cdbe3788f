// mpf_paths.cu -- launches of the path deposits and edge gathers (mpf_paths.cuh).
#include <algorithm>

#include "mpf_paths.cuh"
#include "mpifield_b200.h"

namespace mpf {

// One thread per path with global atomics (the default: the L2's FP64 adds measured
// faster than shared-memory boxes here, where many lanes add to the same nodes),
// or the tiled kernel (path 2, staged): chunks of 256 x t.block paths (8 when t.block is
// 0), a box of edges in t.smem_bytes (96 KB when 0) of shared memory.
// Edge fields of at most this many entries are deposited through private copies in shared
// memory when the paths number at least kPrivatePaths per entry (5e6 paths: 1D on 64 or 256
// nodes 0.28-0.36 ms against 1.1-5.1 ms through the L2; 2D 40 x 50 1.1 / 3.5 ms against
// 2.5 / 5.1 ms at degree 2 / 3; 3D 12^3 3.9 against 10.7 ms at degree 2).
constexpr int kPrivateEntries = 8192;
constexpr int kPrivatePaths = 16;

template <typename T, int NDIM, int P, bool WHITNEY>
static int run_deposit_private(const PathArgs<T>& a, int64_t entries, cudaStream_t stream) {
    const int smem = (int)(entries * (int64_t)sizeof(T));
    // the launch shapes of the direct kernel, as many CTAs per SM as the copies also allow
    constexpr bool cubic = !WHITNEY && P >= 3;
    constexpr int threads = cubic ? 128 : 256;
    auto kernel = cubic ? deposit_paths_private_kernel<T, NDIM, P, WHITNEY, 128, 4>
                        : deposit_paths_private_kernel<T, NDIM, P, WHITNEY, 256, 2>;
    const int per_sm = std::max(1, std::min(cubic ? 4 : 2, (228 * 1024) / (smem + 1024)));
    static int cache[64] = {0};
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) device = 0;
    if (cache[device] < smem) {
        if (record_cuda_error(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != MPF_OK)
            return MPF_ERR_CUDA;
        cache[device] = smem;
    }
    const int64_t blocks = std::min<int64_t>((a.n + threads - 1) / threads, (int64_t)sm_count() * per_sm);
    kernel<<<(unsigned)std::max<int64_t>(blocks, 1), threads, smem, stream>>>(a);
    count_launches(1);
    return launch_status();
}

template <typename T, int NDIM, int P, bool WHITNEY>
static int run_deposit(PathArgs<T> a, const Tuning& t, cudaStream_t stream) {
    const int block = 256;
    // (not the 3D cubic edges: their 144 adds a piece collide in shared memory, and the L2
    // spreads them better: 19 against 30 ms for 5e6 paths on 12^3)
    if (t.path == 0 && t.variant != 7 && !(NDIM == 3 && !WHITNEY && P >= 3)) {
        int64_t entries = NDIM;
        for (int d = 0; d < NDIM; ++d) entries *= a.g.ext[d];
        if (entries <= kPrivateEntries && a.n >= kPrivatePaths * entries)
            return run_deposit_private<T, NDIM, P, WHITNEY>(a, entries, stream);
    }
    if (t.path != 2) {
        auto launch = [&](auto kernel, int threads, int smem = 0) {
            const int64_t blocks = std::min<int64_t>((a.n + threads - 1) / threads, (int64_t)sm_count() * 32);
            kernel<<<(unsigned)std::max<int64_t>(blocks, 1), threads, smem, stream>>>(a);
        };
        // WHITNEY: five CTAs of 128 per SM (96 registers; 4% faster than two of 256 on a
        // sorted store). 128 registers a thread: two CTAs of 256 per SM for the spline edges
        // of degree <= 2 (no spills; QUADRATIC_EDGES 15% faster than one CTA; 96 or 80
        // registers spill and measured 15-25% slower), four of 128 for
        // the cubic edges (some spills, but twice the warps of one CTA of 256 at 178
        // registers: CUBIC_EDGES 137 -> 97 ms at 2^25 paths), in 3D with the cross-axis weights
        // of the Gauss points in shared memory, computed once per axis instead of once per edge
        // along it, and the points a rolled loop (97 -> 72 ms; the cache for degree 2 measured
        // slower). Variant 1: one CTA of 256;
        // variant 3: spline paths a path at a time instead of piece by piece; variant 7:
        // never through private copies of a small field.
        if constexpr (!WHITNEY && P >= 3) {
            if (t.variant == 3) launch(deposit_paths_kernel<T, NDIM, P, WHITNEY, 256, 1, false>, 256);
            else if (t.variant == 1) launch(deposit_paths_kernel<T, NDIM, P, WHITNEY, 256, 1>, 256);
            else if constexpr (NDIM == 3)
                launch(deposit_paths_kernel<T, NDIM, P, WHITNEY, 128, 4, true, true>, 128,
                       path_cache_bytes<T, NDIM, P>(128));
            else launch(deposit_paths_kernel<T, NDIM, P, WHITNEY, 128, 4>, 128);
        } else {
            if (t.variant == 1) launch(deposit_paths_kernel<T, NDIM, P, WHITNEY, 256, 1>, 256);
            else if (t.variant == 3) launch(deposit_paths_kernel<T, NDIM, P, WHITNEY, 256, 2, false>, 256);
            else if constexpr (WHITNEY) launch(deposit_paths_kernel<T, NDIM, P, WHITNEY, 128, 5>, 128);
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

// mpf_paths.cu -- launches of the path deposits and edge gathers (mpf_paths.cuh).
#include <algorithm>

#include "mpf_paths.cuh"
#include "mpifield_b200.h"

namespace mpf {

template <typename T, int NDIM, int P, bool WHITNEY>
static int run_deposit(const PathArgs<T>& a, cudaStream_t stream) {
    const int block = 256;
    const int64_t blocks = std::min<int64_t>((a.n + block - 1) / block, (int64_t)sm_count() * 16);
    deposit_paths_kernel<T, NDIM, P, WHITNEY><<<(unsigned)std::max<int64_t>(blocks, 1), block, 0, stream>>>(a);
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
static int paths_by_kind(int kind, int degree, const PathArgs<T>& a, cudaStream_t stream) {
    if (kind == LINEAR) return GATHER ? run_gather_edges<T, NDIM, 1, true>(a, stream) : run_deposit<T, NDIM, 1, true>(a, stream);
    switch (degree) {
        case 1: return GATHER ? run_gather_edges<T, NDIM, 1, false>(a, stream) : run_deposit<T, NDIM, 1, false>(a, stream);
        case 2: return GATHER ? run_gather_edges<T, NDIM, 2, false>(a, stream) : run_deposit<T, NDIM, 2, false>(a, stream);
        case 3: return GATHER ? run_gather_edges<T, NDIM, 3, false>(a, stream) : run_deposit<T, NDIM, 3, false>(a, stream);
    }
    return MPF_ERR_ARGUMENT;
}

template <typename T>
int launch_deposit_paths(int kind, int degree, int ndim, const PathArgs<T>& a, cudaStream_t stream) {
    switch (ndim) {
        case 1: return paths_by_kind<T, 1, false>(kind, degree, a, stream);
        case 2: return paths_by_kind<T, 2, false>(kind, degree, a, stream);
        case 3: return paths_by_kind<T, 3, false>(kind, degree, a, stream);
    }
    return MPF_ERR_ARGUMENT;
}

template <typename T>
int launch_gather_edges(int kind, int degree, int ndim, const PathArgs<T>& a, cudaStream_t stream) {
    switch (ndim) {
        case 1: return paths_by_kind<T, 1, true>(kind, degree, a, stream);
        case 2: return paths_by_kind<T, 2, true>(kind, degree, a, stream);
        case 3: return paths_by_kind<T, 3, true>(kind, degree, a, stream);
    }
    return MPF_ERR_ARGUMENT;
}

template int launch_deposit_paths<double>(int, int, int, const PathArgs<double>&, cudaStream_t);
template int launch_deposit_paths<float>(int, int, int, const PathArgs<float>&, cudaStream_t);
template int launch_gather_edges<double>(int, int, int, const PathArgs<double>&, cudaStream_t);
template int launch_gather_edges<float>(int, int, int, const PathArgs<float>&, cudaStream_t);

}  // namespace mpf

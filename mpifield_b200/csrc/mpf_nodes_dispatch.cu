// mpf_nodes_dispatch.cu -- the node launches by dimension (the kernels live in
// mpf_nodes_<type>_<n>d.cu).
#include "mpf_internal.h"
#include "mpifield_b200.h"

namespace mpf {

template <typename T>
static int by_ndim(int op, int kind, int degree, int ndim, const NodeArgs<T>& a, const Tuning& t, cudaStream_t s) {
    switch (ndim) {
        case 1: return node_launch<T, 1>(op, kind, degree, a, t, s);
        case 2: return node_launch<T, 2>(op, kind, degree, a, t, s);
        case 3: return node_launch<T, 3>(op, kind, degree, a, t, s);
    }
    return MPF_ERR_ARGUMENT;
}

template <typename T>
int launch_gather(int kind, int degree, int ndim, const NodeArgs<T>& a, const Tuning& t, cudaStream_t s) {
    return by_ndim<T>(0, kind, degree, ndim, a, t, s);
}

template <typename T>
int launch_scatter(int kind, int degree, int ndim, const NodeArgs<T>& a, const Tuning& t, cudaStream_t s) {
    return by_ndim<T>(1, kind, degree, ndim, a, t, s);
}

template <typename T>
int launch_gather_grad(int kind, int degree, int ndim, const NodeArgs<T>& a, cudaStream_t s) {
    return by_ndim<T>(2, kind, degree, ndim, a, Tuning{0, 0, 0, 0, 0}, s);
}

template int launch_gather<double>(int, int, int, const NodeArgs<double>&, const Tuning&, cudaStream_t);
template int launch_gather<float>(int, int, int, const NodeArgs<float>&, const Tuning&, cudaStream_t);
template int launch_scatter<double>(int, int, int, const NodeArgs<double>&, const Tuning&, cudaStream_t);
template int launch_scatter<float>(int, int, int, const NodeArgs<float>&, const Tuning&, cudaStream_t);
template int launch_gather_grad<double>(int, int, int, const NodeArgs<double>&, cudaStream_t);
template int launch_gather_grad<float>(int, int, int, const NodeArgs<float>&, cudaStream_t);

}  // namespace mpf

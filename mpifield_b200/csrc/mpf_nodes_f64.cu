// mpf_nodes_f64.cu -- the node kernels instantiated for double.
#include "mpf_nodes_launch.cuh"

namespace mpf {
template int launch_gather<double>(int, int, int, const NodeArgs<double>&, const Tuning&, cudaStream_t);
template int launch_scatter<double>(int, int, int, const NodeArgs<double>&, const Tuning&, cudaStream_t);
template int launch_gather_grad<double>(int, int, int, const NodeArgs<double>&, cudaStream_t);
}  // namespace mpf

// mpf_nodes_f64_2d.cu -- the 2D node kernels instantiated for double.
#include "mpf_nodes_launch.cuh"

namespace mpf {
template int node_launch<double, 2>(int, int, int, const NodeArgs<double>&, const Tuning&, cudaStream_t);
}  // namespace mpf

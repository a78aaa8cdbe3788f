// mpf_nodes_f64_3d.cu -- the 3D node kernels instantiated for double.
#include "mpf_nodes_launch.cuh"

namespace mpf {
template int node_launch<double, 3>(int, int, int, const NodeArgs<double>&, const Tuning&, cudaStream_t);
}  // namespace mpf

// mpf_nodes_f32_1d.cu -- the 1D node kernels instantiated for float.
#include "mpf_nodes_launch.cuh"

namespace mpf {
template int node_launch<float, 1>(int, int, int, const NodeArgs<float>&, const Tuning&, cudaStream_t);
}  // namespace mpf

// mpf_nodes_f32_2d.cu -- the 2D node kernels instantiated for float.
#include "mpf_nodes_launch.cuh"

namespace mpf {
template int node_launch<float, 2>(int, int, int, const NodeArgs<float>&, const Tuning&, cudaStream_t);
}  // namespace mpf

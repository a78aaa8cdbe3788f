// mpf_nodes_f32.cu -- the node kernels instantiated for float.
#include "mpf_nodes_launch.cuh"

namespace mpf {
template int launch_gather<float>(int, int, int, const NodeArgs<float>&, const Tuning&, cudaStream_t);
template int launch_scatter<float>(int, int, int, const NodeArgs<float>&, const Tuning&, cudaStream_t);
template int launch_gather_grad<float>(int, int, int, const NodeArgs<float>&, cudaStream_t);
}  // namespace mpf

// Project-written: CUDA builtins for compiling the reference kernels as serial C++ on the
// host (the scheme of src/mpifield/tests/kernels/test_cuda_emulated.py:30-51). Each
// emulated launch runs one thread per block, blocks one after another.
#pragma once
#include <cmath>
using std::floor;
using std::ceil;
#define __host__
#define __device__
#define __global__
#define __forceinline__ inline
#define __shared__
struct ref_dim3 { unsigned x, y, z; };
static ref_dim3 threadIdx, blockDim, blockIdx, gridDim;
inline void __syncthreads() {}
inline double atomicAdd(double* p, double v) { double o = *p; *p += v; return o; }
inline float atomicAdd(float* p, float v) { float o = *p; *p += v; return o; }

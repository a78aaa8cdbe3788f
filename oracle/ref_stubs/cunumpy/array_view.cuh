// Project-written stand-in for cunumpy's array_view.cuh (cunumpy 0.8.0 is not in this
// image). Test infrastructure only: it lets the mpifield reference kernels compile as
// C++ (or CUDA) in oracle/_ref/. An ArrayND is a data pointer, the shape and the strides
// in elements, brace-initialisable as {data, {shape...}, {strides...}}, the layout the
// reference's own emulation test builds (src/mpifield/tests/kernels/test_cuda_emulated.py:76-83).
#pragma once
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
template <typename T> struct Array1D {
    T* data; long long shape[1]; long long strides[1];
    __host__ __device__ T& operator()(long long i) const { return data[i * strides[0]]; }
};
template <typename T> struct Array2D {
    T* data; long long shape[2]; long long strides[2];
    __host__ __device__ T& operator()(long long i, long long j) const {
        return data[i * strides[0] + j * strides[1]];
    }
};
template <typename T> struct Array3D {
    T* data; long long shape[3]; long long strides[3];
    __host__ __device__ T& operator()(long long i, long long j, long long k) const {
        return data[i * strides[0] + j * strides[1] + k * strides[2]];
    }
};
template <typename T> struct Array4D {
    T* data; long long shape[4]; long long strides[4];
    __host__ __device__ T& operator()(long long i, long long j, long long k, long long l) const {
        return data[i * strides[0] + j * strides[1] + k * strides[2] + l * strides[3]];
    }
};

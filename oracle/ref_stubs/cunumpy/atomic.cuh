// Project-written stand-in for cunumpy's atomic.cuh (not in this image): a plain atomic
// add, as the reference's emulation test assumes (test_cuda_emulated.py:43).
#pragma once
template <typename T> __device__ inline void cunumpy_atomic_add(T* address, T value) {
    atomicAdd(address, value);
}

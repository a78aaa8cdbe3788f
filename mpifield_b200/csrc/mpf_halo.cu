// mpf_halo.cu -- the single-GPU halo work of a block stored with halo layers.
//
// mpifield keeps a field as a block with `h` halo nodes per side (src/mpifield/field.py:
// 150-202). With halos the kernels see a bounded block (field.py:184-186); on one
// process a periodic axis is then closed by mpiarray's update_halos (fill: halos take
// the wrapped interior) and accumulate_halos (fold: halos add onto their wrapped owners
// and are cleared), axis by axis over the whole storage so that corners take two steps
// (the method cards of field.py:601-630). Each axis is one launch, in axis order.
#include <algorithm>
#include <cstdint>

#include "mpf_internal.h"
#include "mpifield_b200.h"

namespace mpf {

// The storage as [outer][axis][inner]: outer spans the axes before `axis`, inner the
// axes after it and the components.
struct AxisView {
    int64_t outer, inner;
    int64_t stored;  // extent along the axis, halos included
    int64_t owned;   // stored - 2 h
    int h;
};

template <typename T>
__global__ void halo_fill_kernel(T* f, AxisView v) {
    const int64_t count = v.outer * v.h * v.inner;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t in = k % v.inner;
        const int64_t l = (k / v.inner) % v.h;
        const int64_t o = k / (v.inner * v.h);
        const int64_t row = o * v.stored;
        // low halo layer l <- owned layer owned - h + l (stored index owned + l);
        // high halo layer l <- owned layer l (stored index h + l)
        f[(row + l) * v.inner + in] = f[(row + v.owned + l) * v.inner + in];
        f[(row + v.owned + v.h + l) * v.inner + in] = f[(row + v.h + l) * v.inner + in];
    }
}

template <typename T>
__global__ void halo_fold_kernel(T* f, AxisView v, int periodic) {
    const int64_t count = v.outer * v.h * v.inner;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t in = k % v.inner;
        const int64_t l = (k / v.inner) % v.h;
        const int64_t o = k / (v.inner * v.h);
        const int64_t row = o * v.stored;
        T* low = f + (row + l) * v.inner + in;
        T* high = f + (row + v.owned + v.h + l) * v.inner + in;
        if (periodic) {
            // two halo layers may add onto one owned node when owned < 2 h
            atomicAdd(f + (row + v.h + l) * v.inner + in, *high);
            atomicAdd(f + (row + v.owned + l) * v.inner + in, *low);
        }
        *low = T(0);
        *high = T(0);
    }
}

// Layers [first, first + h) along the axis of the storage <-> a contiguous buffer
// [outer][h][inner]: the face slabs a rank sends to and takes from its neighbours in the
// halo exchange of a field split over ranks (mpiarray's update_halos and
// accumulate_halos between processes). Unpack writes, or adds with ADD (a fold: every
// buffer entry has its own node, so plain adds).
template <typename T>
__global__ void halo_pack_kernel(const T* f, T* buf, AxisView v, int64_t first) {
    const int64_t count = v.outer * v.h * v.inner;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t in = k % v.inner;
        const int64_t l = (k / v.inner) % v.h;
        const int64_t o = k / (v.inner * v.h);
        buf[k] = f[(o * v.stored + first + l) * v.inner + in];
    }
}

template <typename T, bool ADD>
__global__ void halo_unpack_kernel(T* f, const T* buf, AxisView v, int64_t first) {
    const int64_t count = v.outer * v.h * v.inner;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t in = k % v.inner;
        const int64_t l = (k / v.inner) % v.h;
        const int64_t o = k / (v.inner * v.h);
        T* at = f + (o * v.stored + first + l) * v.inner + in;
        if (ADD) *at += buf[k];
        else *at = buf[k];
    }
}

template <typename T>
__global__ void add_density_kernel(T* dst, const T* dep, int ndim, int num0, int num1, int num2,
                                   int h, int64_t ncomp, T v0, T v1, T v2, int p0, int p1, int p2) {
    const int num[3] = {num0, ndim > 1 ? num1 : 1, ndim > 2 ? num2 : 1};
    const int stored[3] = {num0 + 2 * h, ndim > 1 ? num1 + 2 * h : 1, ndim > 2 ? num2 + 2 * h : 1};
    const T cellv[3] = {v0, v1, v2};
    const int per[3] = {p0, p1, p2};
    const int64_t count = (int64_t)num[0] * num[1] * num[2] * ncomp;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = k % ncomp;
        int64_t node = k / ncomp;
        int idx[3];
        idx[2] = (int)(node % num[2]);
        node /= num[2];
        idx[1] = (int)(node % num[1]);
        idx[0] = (int)(node / num[1]);
        T volume = T(1);
        int64_t s = 0;
        for (int d = 0; d < 3; ++d) {
            if (d < ndim) {
                T factor = cellv[d];
                if (!per[d] && (idx[d] == 0 || idx[d] == num[d] - 1)) factor = factor * T(0.5);
                volume = volume * factor;
            }
            s = s * stored[d] + (d < ndim ? idx[d] + h : 0);
        }
        dst[s * ncomp + c] += dep[s * ncomp + c] / volume;
    }
}

template <typename T>
static int run_halo(T* f, int ndim, const int32_t* stored, int64_t ncomp, int h,
                    const int32_t* periodic, bool fold, cudaStream_t stream) {
    for (int axis = 0; axis < ndim; ++axis) {
        if (!fold && !periodic[axis]) continue;
        AxisView v;
        v.outer = 1;
        for (int d = 0; d < axis; ++d) v.outer *= stored[d];
        v.inner = ncomp;
        for (int d = axis + 1; d < ndim; ++d) v.inner *= stored[d];
        v.stored = stored[axis];
        v.owned = stored[axis] - 2 * (int64_t)h;
        v.h = h;
        const int64_t count = v.outer * h * v.inner;
        if (count == 0) continue;
        const int block = 256;
        const int64_t blocks = std::min<int64_t>((count + block - 1) / block, (int64_t)sm_count() * 16);
        if (fold) halo_fold_kernel<T><<<(unsigned)blocks, block, 0, stream>>>(f, v, periodic[axis]);
        else halo_fill_kernel<T><<<(unsigned)blocks, block, 0, stream>>>(f, v);
        count_launches(1);
        if (launch_status() != MPF_OK) return MPF_ERR_CUDA;
    }
    return MPF_OK;
}

template <typename T>
static int run_density(T* dst, const T* dep, int ndim, const int32_t* num, int h, int64_t ncomp,
                       const double* cell, const int32_t* periodic, cudaStream_t stream) {
    int64_t count = ncomp;
    for (int d = 0; d < ndim; ++d) count *= num[d];
    if (count == 0) return MPF_OK;
    const int block = 256;
    const int64_t blocks = std::min<int64_t>((count + block - 1) / block, (int64_t)sm_count() * 16);
    add_density_kernel<T><<<(unsigned)blocks, block, 0, stream>>>(
        dst, dep, ndim, num[0], ndim > 1 ? num[1] : 1, ndim > 2 ? num[2] : 1, h, ncomp, (T)cell[0],
        (T)(ndim > 1 ? cell[1] : 1.0), (T)(ndim > 2 ? cell[2] : 1.0), periodic[0],
        ndim > 1 ? periodic[1] : 1, ndim > 2 ? periodic[2] : 1);
    count_launches(1);
    return launch_status();
}

// The view of `axis` of a storage (h layers per slab).
static AxisView axis_view(int ndim, const int32_t* stored, int64_t ncomp, int h, int axis) {
    AxisView v;
    v.outer = 1;
    for (int d = 0; d < axis; ++d) v.outer *= stored[d];
    v.inner = ncomp;
    for (int d = axis + 1; d < ndim; ++d) v.inner *= stored[d];
    v.stored = stored[axis];
    v.owned = stored[axis] - 2 * (int64_t)h;
    v.h = h;
    return v;
}

template <typename T>
static int run_slab(T* f, T* buf, int ndim, const int32_t* stored, int64_t ncomp, int h, int axis, int first,
                    int mode, cudaStream_t stream) {
    const AxisView v = axis_view(ndim, stored, ncomp, h, axis);
    const int64_t count = v.outer * h * v.inner;
    if (count == 0) return MPF_OK;
    const int block = 256;
    const int64_t blocks = std::min<int64_t>((count + block - 1) / block, (int64_t)sm_count() * 16);
    if (mode == 0) halo_pack_kernel<T><<<(unsigned)blocks, block, 0, stream>>>(f, buf, v, first);
    else if (mode == 1) halo_unpack_kernel<T, false><<<(unsigned)blocks, block, 0, stream>>>(f, buf, v, first);
    else halo_unpack_kernel<T, true><<<(unsigned)blocks, block, 0, stream>>>(f, buf, v, first);
    count_launches(1);
    return launch_status();
}

int halo_slab(void* f, void* buf, int ndim, const int32_t* stored, int64_t ncomp, int h, int axis, int first,
              int mode, int dtype, cudaStream_t stream) {
    if (dtype == MPF_F64)
        return run_slab<double>((double*)f, (double*)buf, ndim, stored, ncomp, h, axis, first, mode, stream);
    return run_slab<float>((float*)f, (float*)buf, ndim, stored, ncomp, h, axis, first, mode, stream);
}

int halo_fill(void* f, int ndim, const int32_t* stored, int64_t ncomp, int h, const int32_t* periodic,
              int dtype, cudaStream_t stream) {
    if (dtype == MPF_F64) return run_halo<double>((double*)f, ndim, stored, ncomp, h, periodic, false, stream);
    return run_halo<float>((float*)f, ndim, stored, ncomp, h, periodic, false, stream);
}

int halo_fold(void* f, int ndim, const int32_t* stored, int64_t ncomp, int h, const int32_t* periodic,
              int dtype, cudaStream_t stream) {
    if (dtype == MPF_F64) return run_halo<double>((double*)f, ndim, stored, ncomp, h, periodic, true, stream);
    return run_halo<float>((float*)f, ndim, stored, ncomp, h, periodic, true, stream);
}

int add_density(void* dst, const void* dep, int ndim, const int32_t* num, int h, int64_t ncomp,
                const double* cell, const int32_t* periodic, int dtype, cudaStream_t stream) {
    if (dtype == MPF_F64)
        return run_density<double>((double*)dst, (const double*)dep, ndim, num, h, ncomp, cell, periodic, stream);
    return run_density<float>((float*)dst, (const float*)dep, ndim, num, h, ncomp, cell, periodic, stream);
}

}  // namespace mpf

// mpf_nodes.cuh -- node gather, node scatter and the position gradient of a gather.
//
// The arithmetic is that of mpifield's gather_/scatter_{linear,quadratic,spline}_{1,2,3}d
// kernels (e.g. src/mpifield/kernels/gather_spline_3d/gather_spline_3d_cuda.cu:11-53,
// scatter_spline_3d/scatter_spline_3d_cuda.cu:12-61): result(c, i) = sum_k W_k(x_i) F(k, c)
// and F(k, c) += sum_i W_k(x_i) v(c, i), with W_k the tensor product of the per-axis
// stencils of mpf_stencil.cuh, and a marker whose values are all zero skipped before its
// position is read (scatter_quadratic_3d_cuda.cu:32-38).
//
// The B200 organisation is new. A CTA takes a chunk of MPT * blockDim consecutive markers
// (coalesced SoA loads, marker i of a chunk on thread i % blockDim), keeps their
// positions in cells in registers, and reduces the chunk's bounding box of stencil nodes
// (pre-mapping coordinates, so a box may straddle a periodic seam). When the box fits in
// the CTA's shared memory -- markers sorted by cell tile -- the gather stages that box of
// the field once and evaluates every marker from shared memory, and the scatter
// accumulates the chunk into a shared box with shared-memory atomics and flushes it with
// one global atomic add per non-zero node. Otherwise (unsorted markers, a chunk that
// spans the grid) the same chunk reads and adds straight to global memory. The sum over
// the stencil is factored axis by axis (x outermost), which changes the rounding of
// the reference's sum by a few ulps, not the nodes or the weights.
#pragma once
#include <climits>

#include "mpf_internal.h"
#include "mpf_stencil.cuh"

namespace mpf {

extern __shared__ __align__(16) unsigned char mpf_dynamic_smem[];

constexpr int kMarkersPerThread = 4;
constexpr int kMaxBlock = 256;

template <typename T>
__device__ __forceinline__ T rel_of(const NodeArgs<T>& a, int d, int64_t i) {
    return (a.pos[d * a.pos_stride + i] - a.g.lower[d]) / a.g.cell[d];
}

// Block-wide min of lo[] and max of hi[] over NDIM axes, into s_lo / s_hi (which the
// caller set to INT_MAX / INT_MIN and synchronised). Every thread of the block calls it.
template <int NDIM>
__device__ __forceinline__ void block_box(const int* lo, const int* hi, int* s_lo, int* s_hi) {
#pragma unroll
    for (int d = 0; d < NDIM; ++d) {
        const int l = __reduce_min_sync(0xffffffffu, lo[d]);
        const int h = __reduce_max_sync(0xffffffffu, hi[d]);
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&s_lo[d], l);
            atomicMax(&s_hi[d], h);
        }
    }
}

// The node offsets of a stencil: off[d][a] such that node (a, b, e) is at
// (off[0][a] + off[1][b] + off[2][e]) * ncomp. Unused axes hold one zero offset.
template <int NDIM, int S, typename I>
__device__ __forceinline__ void box_offsets(const int* base, const int* lo, const int* ex,
                                            I (&off)[3][S]) {
    const I sy = NDIM > 2 ? (I)ex[2] : (I)1;
    const I sx = NDIM > 1 ? (I)ex[1] * sy : (I)1;
    const I stride[3] = {sx, sy, (I)1};
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int a = 0; a < S; ++a)
            off[d][a] = d < NDIM ? (I)(base[d] - lo[d] + a) * stride[d] : (I)0;
}

template <int NDIM, int S>
__device__ __forceinline__ void global_offsets(const int* base, const int* num, const int* code,
                                               const int* ext, int64_t (&off)[3][S]) {
    const int64_t sy = NDIM > 2 ? (int64_t)ext[2] : 1;
    const int64_t sx = NDIM > 1 ? (int64_t)ext[1] * sy : 1;
    const int64_t stride[3] = {sx, sy, 1};
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int a = 0; a < S; ++a)
            off[d][a] = d < NDIM ? (int64_t)map_node(base[d] + a, num[d], code[d]) * stride[d] : 0;
}

template <typename T, bool LDG> __device__ __forceinline__ T load(const T* p) {
    if constexpr (LDG) return __ldg(p);
    else return *p;
}

// acc[c] = sum_a wx[a] sum_b wy[b] sum_e wz[e] src[(off) * ncomp + c0 + c], c < NCC.
template <typename T, int NDIM, int S, int NCC, bool LDG, typename I>
__device__ __forceinline__ void stencil_sum(const T* __restrict__ src, const I (&off)[3][S],
                                            const T (&w)[3][S], I ncomp, int c0, T* acc) {
    constexpr int SY = NDIM > 1 ? S : 1;
    constexpr int SZ = NDIM > 2 ? S : 1;
#pragma unroll
    for (int c = 0; c < NCC; ++c) acc[c] = T(0);
#pragma unroll
    for (int a = 0; a < S; ++a) {
        T sa[NCC];
#pragma unroll
        for (int c = 0; c < NCC; ++c) sa[c] = T(0);
#pragma unroll
        for (int b = 0; b < SY; ++b) {
            T sb[NCC];
#pragma unroll
            for (int c = 0; c < NCC; ++c) sb[c] = T(0);
#pragma unroll
            for (int e = 0; e < SZ; ++e) {
                const T* p = src + (off[0][a] + off[1][b] + off[2][e]) * ncomp + c0;
#pragma unroll
                for (int c = 0; c < NCC; ++c) {
                    const T v = load<T, LDG>(p + c);
                    if constexpr (NDIM > 2) sb[c] += w[2][e] * v;
                    else sb[c] += v;
                }
            }
#pragma unroll
            for (int c = 0; c < NCC; ++c) {
                if constexpr (NDIM > 1) sa[c] += w[1][b] * sb[c];
                else sa[c] += sb[c];
            }
        }
#pragma unroll
        for (int c = 0; c < NCC; ++c) acc[c] += w[0][a] * sa[c];
    }
}

// dst[(off) * ncomp + c0 + c] += W * v[c] with atomic adds.
template <typename T, int NDIM, int S, int NCC, typename I>
__device__ __forceinline__ void stencil_add(T* dst, const I (&off)[3][S], const T (&w)[3][S],
                                            I ncomp, int c0, const T* v) {
    constexpr int SY = NDIM > 1 ? S : 1;
    constexpr int SZ = NDIM > 2 ? S : 1;
#pragma unroll
    for (int a = 0; a < S; ++a) {
#pragma unroll
        for (int b = 0; b < SY; ++b) {
            const T wab = NDIM > 1 ? w[0][a] * w[1][b] : w[0][a];
#pragma unroll
            for (int e = 0; e < SZ; ++e) {
                const T wt = NDIM > 2 ? wab * w[2][e] : wab;
                T* p = dst + (off[0][a] + off[1][b] + off[2][e]) * ncomp + c0;
#pragma unroll
                for (int c = 0; c < NCC; ++c) atomicAdd(p + c, wt * v[c]);
            }
        }
    }
}

// The pre-mapping node j of a box entry k (node-major, ncomp innermost) and its
// component: k = ((jx * ey + jy) * ez + jz) * ncomp + c.
template <int NDIM>
__device__ __forceinline__ int64_t box_to_global(int64_t k, int ncomp, const int* lo, const int* ex,
                                                 const int* num, const int* code, const int* ext,
                                                 int* comp) {
    *comp = (int)(k % ncomp);
    int64_t node = k / ncomp;
    int j[3] = {0, 0, 0};
#pragma unroll
    for (int d = NDIM - 1; d >= 0; --d) {
        j[d] = (int)(node % ex[d]);
        node /= ex[d];
    }
    int64_t g = 0;
#pragma unroll
    for (int d = 0; d < NDIM; ++d) g = g * ext[d] + map_node(lo[d] + j[d], num[d], code[d]);
    return g;
}

template <typename T, int NDIM, int KIND, int P, int NC>
__global__ void __launch_bounds__(kMaxBlock) gather_kernel(const NodeArgs<T> a) {
    constexpr int S = P + 1;
    constexpr int NCC = NC > 0 ? NC : 1;
    constexpr int MPT = kMarkersPerThread;
    T* tile = reinterpret_cast<T*>(mpf_dynamic_smem);
    __shared__ int s_lo[3], s_hi[3];
    const int ncomp = NC > 0 ? NC : a.ncomp;
    const int64_t chunk = (int64_t)MPT * blockDim.x;
    const int64_t nchunks = (a.n + chunk - 1) / chunk;
    for (int64_t ci = blockIdx.x; ci < nchunks; ci += gridDim.x) {
        const int64_t first = ci * chunk;
        T rel[MPT][NDIM];
        int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
#pragma unroll
        for (int m = 0; m < MPT; ++m) {
            const int64_t i = first + (int64_t)m * blockDim.x + threadIdx.x;
            if (i < a.n) {
#pragma unroll
                for (int d = 0; d < NDIM; ++d) {
                    rel[m][d] = rel_of(a, d, i);
                    T w[S];
                    const int b = axis_stencil<T, KIND, P>(rel[m][d], a.g.num[d], a.g.code[d], w);
                    lo[d] = min(lo[d], b);
                    hi[d] = max(hi[d], b);
                }
            }
        }
        bool staged = false;
        int blo[3] = {0, 0, 0}, bex[3] = {1, 1, 1};
        if (!a.force_global) {
            if (threadIdx.x < 3) {
                s_lo[threadIdx.x] = INT_MAX;
                s_hi[threadIdx.x] = INT_MIN;
            }
            __syncthreads();
            block_box<NDIM>(lo, hi, s_lo, s_hi);
            __syncthreads();
            int64_t vol = 1;
#pragma unroll
            for (int d = 0; d < NDIM; ++d) {
                blo[d] = s_lo[d];
                bex[d] = s_hi[d] - s_lo[d] + S;
                vol *= bex[d];
            }
            staged = vol * ncomp <= (int64_t)a.capacity;
            if (staged) {
                const int64_t total = vol * ncomp;
                for (int64_t k = threadIdx.x; k < total; k += blockDim.x) {
                    int c;
                    const int64_t g = box_to_global<NDIM>(k, ncomp, blo, bex, a.g.num, a.g.code, a.g.ext, &c);
                    tile[k] = __ldg(a.field_in + g * ncomp + c);
                }
                __syncthreads();
            }
        }
#pragma unroll
        for (int m = 0; m < MPT; ++m) {
            const int64_t i = first + (int64_t)m * blockDim.x + threadIdx.x;
            if (i >= a.n) continue;
            T w[3][S];
            int base[3] = {0, 0, 0};
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (d < NDIM) {
                    base[d] = axis_stencil<T, KIND, P>(rel[m][d], a.g.num[d], a.g.code[d], w[d]);
                } else {
#pragma unroll
                    for (int s = 0; s < S; ++s) w[d][s] = T(s == 0);
                }
            }
            if (staged) {
                int off[3][S];
                box_offsets<NDIM, S, int>(base, blo, bex, off);
                if constexpr (NC > 0) {
                    T acc[NCC];
                    stencil_sum<T, NDIM, S, NCC, false, int>(tile, off, w, NC, 0, acc);
#pragma unroll
                    for (int c = 0; c < NCC; ++c) a.result[c * a.res_stride + i] = acc[c];
                } else {
                    for (int c = 0; c < ncomp; ++c) {
                        T acc[1];
                        stencil_sum<T, NDIM, S, 1, false, int>(tile, off, w, ncomp, c, acc);
                        a.result[c * a.res_stride + i] = acc[0];
                    }
                }
            } else {
                int64_t off[3][S];
                global_offsets<NDIM, S>(base, a.g.num, a.g.code, a.g.ext, off);
                if constexpr (NC > 0) {
                    T acc[NCC];
                    stencil_sum<T, NDIM, S, NCC, true, int64_t>(a.field_in, off, w, NC, 0, acc);
#pragma unroll
                    for (int c = 0; c < NCC; ++c) a.result[c * a.res_stride + i] = acc[c];
                } else {
                    for (int c = 0; c < ncomp; ++c) {
                        T acc[1];
                        stencil_sum<T, NDIM, S, 1, true, int64_t>(a.field_in, off, w, ncomp, c, acc);
                        a.result[c * a.res_stride + i] = acc[0];
                    }
                }
            }
        }
        __syncthreads();
    }
}

template <typename T, int NDIM, int KIND, int P, int NC>
__global__ void __launch_bounds__(kMaxBlock) scatter_kernel(const NodeArgs<T> a) {
    constexpr int S = P + 1;
    constexpr int NCC = NC > 0 ? NC : 1;
    constexpr int MPT = kMarkersPerThread;
    T* tile = reinterpret_cast<T*>(mpf_dynamic_smem);
    __shared__ int s_lo[3], s_hi[3];
    const int ncomp = NC > 0 ? NC : a.ncomp;
    const int64_t chunk = (int64_t)MPT * blockDim.x;
    const int64_t nchunks = (a.n + chunk - 1) / chunk;
    for (int64_t ci = blockIdx.x; ci < nchunks; ci += gridDim.x) {
        const int64_t first = ci * chunk;
        T rel[MPT][NDIM];
        T val[MPT][NCC];
        bool live[MPT];
        int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
#pragma unroll
        for (int m = 0; m < MPT; ++m) {
            const int64_t i = first + (int64_t)m * blockDim.x + threadIdx.x;
            live[m] = false;
            if (i < a.n) {
                // a dead marker (all values zero) deposits nothing and its position,
                // which may be non-finite, is not read
                if constexpr (NC > 0) {
#pragma unroll
                    for (int c = 0; c < NCC; ++c) {
                        val[m][c] = a.values[c * a.val_stride + i];
                        live[m] = live[m] || val[m][c] != T(0);
                    }
                } else {
                    for (int c = 0; c < ncomp; ++c) live[m] = live[m] || a.values[c * a.val_stride + i] != T(0);
                }
            }
            if (live[m]) {
#pragma unroll
                for (int d = 0; d < NDIM; ++d) {
                    rel[m][d] = rel_of(a, d, i);
                    T w[S];
                    const int b = axis_stencil<T, KIND, P>(rel[m][d], a.g.num[d], a.g.code[d], w);
                    lo[d] = min(lo[d], b);
                    hi[d] = max(hi[d], b);
                }
            }
        }
        bool staged = false;
        bool empty = false;
        int blo[3] = {0, 0, 0}, bex[3] = {1, 1, 1};
        int64_t total = 0;
        if (!a.force_global) {
            if (threadIdx.x < 3) {
                s_lo[threadIdx.x] = INT_MAX;
                s_hi[threadIdx.x] = INT_MIN;
            }
            __syncthreads();
            block_box<NDIM>(lo, hi, s_lo, s_hi);
            __syncthreads();
            int64_t vol = 1;
#pragma unroll
            for (int d = 0; d < NDIM; ++d) {
                if (s_hi[d] < s_lo[d]) empty = true;
                blo[d] = s_lo[d];
                bex[d] = s_hi[d] - s_lo[d] + S;
                vol *= bex[d];
            }
            if (empty) {
                __syncthreads();
                continue;
            }
            total = vol * ncomp;
            staged = total <= (int64_t)a.capacity;
            if (staged) {
                for (int64_t k = threadIdx.x; k < total; k += blockDim.x) tile[k] = T(0);
                __syncthreads();
            }
        }
        T* dst = staged ? tile : a.field_out;
#pragma unroll
        for (int m = 0; m < MPT; ++m) {
            if (!live[m]) continue;
            const int64_t i = first + (int64_t)m * blockDim.x + threadIdx.x;
            T w[3][S];
            int base[3] = {0, 0, 0};
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (d < NDIM) {
                    base[d] = axis_stencil<T, KIND, P>(rel[m][d], a.g.num[d], a.g.code[d], w[d]);
                } else {
#pragma unroll
                    for (int s = 0; s < S; ++s) w[d][s] = T(s == 0);
                }
            }
            if (staged) {
                int off[3][S];
                box_offsets<NDIM, S, int>(base, blo, bex, off);
                if constexpr (NC > 0) {
                    stencil_add<T, NDIM, S, NCC, int>(dst, off, w, NC, 0, val[m]);
                } else {
                    for (int c = 0; c < ncomp; ++c) {
                        const T v = a.values[c * a.val_stride + i];
                        stencil_add<T, NDIM, S, 1, int>(dst, off, w, ncomp, c, &v);
                    }
                }
            } else {
                int64_t off[3][S];
                global_offsets<NDIM, S>(base, a.g.num, a.g.code, a.g.ext, off);
                if constexpr (NC > 0) {
                    stencil_add<T, NDIM, S, NCC, int64_t>(dst, off, w, NC, 0, val[m]);
                } else {
                    for (int c = 0; c < ncomp; ++c) {
                        const T v = a.values[c * a.val_stride + i];
                        stencil_add<T, NDIM, S, 1, int64_t>(dst, off, w, ncomp, c, &v);
                    }
                }
            }
        }
        if (staged) {
            __syncthreads();
            for (int64_t k = threadIdx.x; k < total; k += blockDim.x) {
                const T v = tile[k];
                if (v != T(0)) {
                    int c;
                    const int64_t g = box_to_global<NDIM>(k, ncomp, blo, bex, a.g.num, a.g.code, a.g.ext, &c);
                    atomicAdd(a.field_out + g * ncomp + c, v);
                }
            }
        }
        __syncthreads();
    }
}

// grad(d, i) = sum_c cot(c, i) d/dx_d sum_k W_k(x_i) F(k, c): one thread per marker,
// global memory (the backward pass of a gather with respect to the positions).
template <typename T, int NDIM, int KIND, int P>
__global__ void __launch_bounds__(kMaxBlock) gather_grad_kernel(const NodeArgs<T> a) {
    constexpr int S = P + 1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        T w[3][S], g[3][S];
        int base[3] = {0, 0, 0};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (d < NDIM) {
                base[d] = axis_stencil_derivative<T, KIND, P>(rel_of(a, d, i), a.g.num[d], a.g.code[d],
                                                              w[d], g[d]);
            } else {
#pragma unroll
                for (int s = 0; s < S; ++s) w[d][s] = g[d][s] = T(s == 0);
            }
        }
        int64_t off[3][S];
        global_offsets<NDIM, S>(base, a.g.num, a.g.code, a.g.ext, off);
#pragma unroll
        for (int d = 0; d < NDIM; ++d) {
            T mixed[3][S];
#pragma unroll
            for (int e = 0; e < 3; ++e)
#pragma unroll
                for (int s = 0; s < S; ++s) mixed[e][s] = e == d ? g[e][s] : w[e][s];
            T total = T(0);
            for (int c = 0; c < a.ncomp; ++c) {
                T acc[1];
                stencil_sum<T, NDIM, S, 1, true, int64_t>(a.field_in, off, mixed, a.ncomp, c, acc);
                total += a.values[c * a.val_stride + i] * acc[0];
            }
            a.result[d * a.res_stride + i] = total / a.g.cell[d];
        }
    }
}

}  // namespace mpf

// mpf_forms.cu -- gather and scatter of the k-forms of B-spline degree 1-3 in 1D-3D.
//
// The spline de Rham sequence of degree P (src/mpifield/kernels/spline_forms.py:1-138,
// gather_forms_spline_{1,2,3}d_cuda.cu): component c of a k-form weighs B_P(r_d - k_d)
// along the axes it is not staggered on and the edge functions B_(P-1)(r_d - k_d - 1/2)
// (existing edges only) along those it is -- an edge (k = 1) along its direction, a face
// of 3D (k = 2) across its normal, the top form (k = ndim) along every axis. Positions
// are clamped to [0, num - 1] on bounded and clamped axes first. The node stencils are
// mpf_stencil.cuh's (the node kernels' fast paths included), the edge stencils
// mpf_paths.cuh's along_stencil: per axis the same indices and weights as the reference.
// One thread per marker, the field read through the read-only cache (gather) or added
// to with global FP64/FP32 atomics (scatter); a marker whose values are all zero is
// skipped before its position is read.
#include <algorithm>

#include "mpf_paths.cuh"
#include "mpifield_b200.h"

namespace mpf {

__host__ __device__ constexpr bool form_staggered(int form, int ndim, int component, int axis) {
    return form == ndim ? true : (form == 1 ? axis == component : (form == 2 && ndim == 3 ? axis != component : false));
}

__host__ __device__ constexpr int form_components(int form, int ndim) {
    return (form == 1 || form == ndim - 1) && form != ndim ? ndim : 1;
}

template <typename T> struct FormArgs {
    Grid<T> g;
    const T* pos;
    int64_t pos_stride;
    const T* values;
    int64_t val_stride;
    const T* field_in;
    T* field_out;
    T* result;
    int64_t res_stride;
    int64_t n;
};

// The stencil of component C of a FORM-form at rel (clamped): per axis its entries'
// array indices, weights and existence, and their count.
template <typename T, int NDIM, int P, int FORM, int C>
__device__ __forceinline__ void form_stencil(const T* rel, const Grid<T>& g, int (&idx)[3][P + 1], T (&wt)[3][P + 1],
                                             bool (&ex)[3][P + 1], int (&cnt)[3]) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        idx[d][0] = 0;
        wt[d][0] = T(1);
        cnt[d] = 1;
#pragma unroll
        for (int s = 0; s <= P; ++s) ex[d][s] = true;
    }
#pragma unroll
    for (int d = 0; d < NDIM; ++d) {
        if (form_staggered(FORM, NDIM, C, d)) {
            along_stencil<T, P>(rel[d], g.num[d], g.code[d], idx[d], wt[d], ex[d]);
            cnt[d] = P;
        } else {
            const int base = axis_stencil<T, SPLINE, P>(rel[d], g.num[d], g.code[d], wt[d]);
#pragma unroll
            for (int s = 0; s <= P; ++s) idx[d][s] = map_node(base + s, g.num[d], g.code[d]);
            cnt[d] = P + 1;
        }
    }
}

template <typename T, int NDIM>
__device__ __forceinline__ void form_positions(const FormArgs<T>& a, int64_t i, T* rel) {
#pragma unroll
    for (int d = 0; d < NDIM; ++d) {
        rel[d] = cells_from(a.pos[d * a.pos_stride + i] - a.g.lower[d], a.g.cell[d], a.g.inv[d], a.g.pow2[d]);
        if (a.g.code[d] != PERIODIC) {
            const T top = T(a.g.num[d] - 1);
            if (rel[d] < T(0)) rel[d] = T(0);
            if (rel[d] > top) rel[d] = top;
        }
    }
}

// Calls fn(node offset, weight) for every existing entry of component C's stencil.
template <typename T, int NDIM, int P, int FORM, int C, typename F>
__device__ __forceinline__ void for_form_stencil(const T* rel, const Grid<T>& g, F&& fn) {
    int idx[3][P + 1];
    T wt[3][P + 1];
    bool ex[3][P + 1];
    int cnt[3];
    form_stencil<T, NDIM, P, FORM, C>(rel, g, idx, wt, ex, cnt);
    constexpr int SX = form_staggered(FORM, NDIM, C, 0) ? P : P + 1;
    constexpr int SY = NDIM > 1 ? (form_staggered(FORM, NDIM, C, 1) ? P : P + 1) : 1;
    constexpr int SZ = NDIM > 2 ? (form_staggered(FORM, NDIM, C, 2) ? P : P + 1) : 1;
#pragma unroll
    for (int x = 0; x < SX; ++x)
#pragma unroll
        for (int y = 0; y < SY; ++y)
#pragma unroll
            for (int z = 0; z < SZ; ++z) {
                if (!(ex[0][x] && ex[1][y] && ex[2][z])) continue;
                T w = wt[0][x];
                if constexpr (NDIM > 1) w = w * wt[1][y];
                if constexpr (NDIM > 2) w = w * wt[2][z];
                int64_t k = idx[0][x];
                if constexpr (NDIM > 1) k = k * g.ext[1] + idx[1][y];
                if constexpr (NDIM > 2) k = k * g.ext[2] + idx[2][z];
                fn(k, w);
            }
}

template <typename T, int NDIM, int P, int FORM, int C>
__device__ __forceinline__ void gather_component(const FormArgs<T>& a, const T* rel, int64_t i) {
    constexpr int NC = form_components(FORM, NDIM);
    if constexpr (C < NC) {
        T total = T(0);
        for_form_stencil<T, NDIM, P, FORM, C>(rel, a.g, [&](int64_t k, T w) { total += w * __ldg(a.field_in + k * NC + C); });
        a.result[C * a.res_stride + i] = total;
        gather_component<T, NDIM, P, FORM, C + 1>(a, rel, i);
    }
}

template <typename T, int NDIM, int P, int FORM, int C>
__device__ __forceinline__ void scatter_component(const FormArgs<T>& a, const T* rel, int64_t i) {
    constexpr int NC = form_components(FORM, NDIM);
    if constexpr (C < NC) {
        const T v = a.values[C * a.val_stride + i];
        if (v != T(0))
            for_form_stencil<T, NDIM, P, FORM, C>(rel, a.g, [&](int64_t k, T w) { atomicAdd(a.field_out + k * NC + C, w * v); });
        scatter_component<T, NDIM, P, FORM, C + 1>(a, rel, i);
    }
}

template <typename T, int NDIM, int P, int FORM>
__global__ void __launch_bounds__(256) gather_forms_kernel(const FormArgs<T> a) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
        T rel[NDIM];
        form_positions<T, NDIM>(a, i, rel);
        gather_component<T, NDIM, P, FORM, 0>(a, rel, i);
    }
}

template <typename T, int NDIM, int P, int FORM>
__global__ void __launch_bounds__(256) scatter_forms_kernel(const FormArgs<T> a) {
    constexpr int NC = form_components(FORM, NDIM);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
        bool live = false;
#pragma unroll
        for (int c = 0; c < NC; ++c) live = live || a.values[c * a.val_stride + i] != T(0);
        if (!live) continue;
        T rel[NDIM];
        form_positions<T, NDIM>(a, i, rel);
        scatter_component<T, NDIM, P, FORM, 0>(a, rel, i);
    }
}

template <typename T, int NDIM, int P, int FORM>
static int run_forms(bool scatter, const FormArgs<T>& a, cudaStream_t stream) {
    const int block = 256;
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((a.n + block - 1) / block, (int64_t)sm_count() * 16));
    if (scatter) scatter_forms_kernel<T, NDIM, P, FORM><<<(unsigned)blocks, block, 0, stream>>>(a);
    else gather_forms_kernel<T, NDIM, P, FORM><<<(unsigned)blocks, block, 0, stream>>>(a);
    count_launches(1);
    return launch_status();
}

template <typename T, int NDIM, int P>
static int forms_by_form(bool scatter, int form, const FormArgs<T>& a, cudaStream_t stream) {
    switch (form) {
        case 1: return run_forms<T, NDIM, P, 1>(scatter, a, stream);
        case 2: if constexpr (NDIM >= 2) return run_forms<T, NDIM, P, 2>(scatter, a, stream); break;
        case 3: if constexpr (NDIM >= 3) return run_forms<T, NDIM, P, 3>(scatter, a, stream); break;
    }
    return MPF_ERR_ARGUMENT;
}

template <typename T, int NDIM>
static int forms_by_degree(bool scatter, int degree, int form, const FormArgs<T>& a, cudaStream_t stream) {
    switch (degree) {
        case 1: return forms_by_form<T, NDIM, 1>(scatter, form, a, stream);
        case 2: return forms_by_form<T, NDIM, 2>(scatter, form, a, stream);
        case 3: return forms_by_form<T, NDIM, 3>(scatter, form, a, stream);
    }
    return MPF_ERR_ARGUMENT;
}

template <typename T>
int launch_forms(bool scatter, int degree, int form, int ndim, const FormArgs<T>& a, cudaStream_t stream) {
    switch (ndim) {
        case 1: return forms_by_degree<T, 1>(scatter, degree, form, a, stream);
        case 2: return forms_by_degree<T, 2>(scatter, degree, form, a, stream);
        case 3: return forms_by_degree<T, 3>(scatter, degree, form, a, stream);
    }
    return MPF_ERR_ARGUMENT;
}

template <typename T>
static Grid<T> forms_grid(int ndim, int degree, const double* lower, const double* cell, const int32_t* num,
                          const int32_t* code) {
    Grid<T> g;
    for (int d = 0; d < 3; ++d) {
        const bool on = d < ndim;
        g.lower[d] = on ? (T)lower[d] : T(0);
        g.cell[d] = on ? (T)cell[d] : T(1);
        g.inv[d] = T(1) / g.cell[d];
        int e = 0;
        const T m = std::frexp(g.cell[d], &e);
        g.pow2[d] = (m == T(0.5) && std::isnormal(g.inv[d]) && std::isnormal(g.cell[d])) ? 1 : 0;
        g.num[d] = on ? num[d] : 1;
        g.code[d] = on ? code[d] : PERIODIC;
        g.ext[d] = on ? axis_extent(num[d], code[d], degree) : 1;
    }
    return g;
}

// The argument checks shared by the two entry points (the grid checks are the node
// kernels' for spline kind; the component count must be that of the form).
static int check_forms(int degree, int form, int ndim, int64_t ncomp, int64_t n, const double* lower,
                       const double* cell, const int32_t* num, const int32_t* code, int dtype) {
    if (degree < 1 || degree > 3 || ndim < 1 || ndim > 3 || form < 1 || form > ndim) return MPF_ERR_ARGUMENT;
    if (ncomp != form_components(form, ndim) || n < 0) return MPF_ERR_ARGUMENT;
    if (dtype != MPF_F64 && dtype != MPF_F32) return MPF_ERR_ARGUMENT;
    if (!lower || !cell || !num || !code) return MPF_ERR_ARGUMENT;
    for (int d = 0; d < ndim; ++d) {
        if (!(cell[d] > 0.0) || !std::isfinite(cell[d]) || !std::isfinite(lower[d])) return MPF_ERR_ARGUMENT;
        if (code[d] < 0 || code[d] > 2 || num[d] < 2) return MPF_ERR_ARGUMENT;
        if (code[d] == PERIODIC && num[d] < 1) return MPF_ERR_ARGUMENT;
    }
    return MPF_OK;
}

static int check_rows_of(const void* p, int64_t& stride, int64_t n, int rows, int dtype) {
    if (stride == 0) stride = n;
    if (stride < n || stride < 0) return MPF_ERR_SHAPE;
    if (n > 0 && rows > 0) {
        if (!p) return MPF_ERR_ARGUMENT;
        const uintptr_t size = dtype == MPF_F64 ? 8 : 4;
        if (reinterpret_cast<uintptr_t>(p) % size) return MPF_ERR_ALIGNMENT;
    }
    return MPF_OK;
}

}  // namespace mpf

using namespace mpf;

extern "C" {

int mpf_gather_forms(int degree, int form, int ndim, const void* positions, int64_t pos_stride, int64_t n,
                     const void* field, int64_t ncomp, void* result, int64_t res_stride, const double* lower,
                     const double* cell, const int32_t* num, const int32_t* code, int dtype, void* stream) {
    int st = check_forms(degree, form, ndim, ncomp, n, lower, cell, num, code, dtype);
    if (st != MPF_OK) return st;
    if ((st = check_rows_of(positions, pos_stride, n, ndim, dtype)) != MPF_OK) return st;
    if ((st = check_rows_of(result, res_stride, n, (int)ncomp, dtype)) != MPF_OK) return st;
    if (n > 0 && !field) return MPF_ERR_ARGUMENT;
    if (n == 0) return MPF_OK;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == MPF_F64) {
        FormArgs<double> a{};
        a.g = forms_grid<double>(ndim, degree, lower, cell, num, code);
        a.pos = (const double*)positions; a.pos_stride = pos_stride; a.n = n;
        a.field_in = (const double*)field; a.result = (double*)result; a.res_stride = res_stride;
        return launch_forms<double>(false, degree, form, ndim, a, s);
    }
    FormArgs<float> a{};
    a.g = forms_grid<float>(ndim, degree, lower, cell, num, code);
    a.pos = (const float*)positions; a.pos_stride = pos_stride; a.n = n;
    a.field_in = (const float*)field; a.result = (float*)result; a.res_stride = res_stride;
    return launch_forms<float>(false, degree, form, ndim, a, s);
}

int mpf_scatter_forms(int degree, int form, int ndim, const void* positions, int64_t pos_stride, const void* values,
                      int64_t val_stride, int64_t n, void* field, int64_t ncomp, const double* lower,
                      const double* cell, const int32_t* num, const int32_t* code, int dtype, void* stream) {
    int st = check_forms(degree, form, ndim, ncomp, n, lower, cell, num, code, dtype);
    if (st != MPF_OK) return st;
    if ((st = check_rows_of(positions, pos_stride, n, ndim, dtype)) != MPF_OK) return st;
    if ((st = check_rows_of(values, val_stride, n, (int)ncomp, dtype)) != MPF_OK) return st;
    if (n > 0 && !field) return MPF_ERR_ARGUMENT;
    if (n == 0) return MPF_OK;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == MPF_F64) {
        FormArgs<double> a{};
        a.g = forms_grid<double>(ndim, degree, lower, cell, num, code);
        a.pos = (const double*)positions; a.pos_stride = pos_stride; a.n = n;
        a.values = (const double*)values; a.val_stride = val_stride; a.field_out = (double*)field;
        return launch_forms<double>(true, degree, form, ndim, a, s);
    }
    FormArgs<float> a{};
    a.g = forms_grid<float>(ndim, degree, lower, cell, num, code);
    a.pos = (const float*)positions; a.pos_stride = pos_stride; a.n = n;
    a.values = (const float*)values; a.val_stride = val_stride; a.field_out = (float*)field;
    return launch_forms<float>(true, degree, form, ndim, a, s);
}

}  // extern "C"

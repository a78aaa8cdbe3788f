// mpf_stencil.cuh -- the per-axis B-spline stencils of the particle-grid kernels.
//
// One axis of a stencil is a `base` node and P + 1 weights: node a of the stencil is
// map(base + a), where map wraps on a periodic axis (code 1), clamps to [0, num - 1]
// on a bounded one (code 0, the fold of a stencil onto the edge node) and is the
// identity on a clamped-knot axis (code 2, whose array holds num + P - 1 entries).
// This reproduces, node for node and operation for operation, the stencils of
// mpifield's src/mpifield/kernels/linear_cell.cuh:12-31 (LINEAR),
// quadratic_cell.cuh:15-37 (QUADRATIC) and spline_cell.cuh:21-105 (degrees 0-3,
// clamped knots by Cox-de Boor), so that cell indices agree bit for bit. The
// conversions saturate and the anchor node is clamped to [0, num], which changes
// nothing for finite positions within about 1e9 cells of the grid and keeps every
// index of every input (NaN, infinities, huge values) inside the arrays.
#pragma once
#include <cstdint>

namespace mpf {

enum Kind : int { LINEAR = 0, QUADRATIC = 1, SPLINE = 2 };
enum Code : int { BOUNDED = 0, PERIODIC = 1, CLAMPED = 2 };

template <typename T> __device__ __forceinline__ int trunc_int(T x);
template <> __device__ __forceinline__ int trunc_int<double>(double x) { return __double2int_rz(x); }
template <> __device__ __forceinline__ int trunc_int<float>(float x) { return __float2int_rz(x); }

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// j modulo num in [0, num): one conditional add or subtract for the pre-mapping nodes of
// a stencil (within a period of the grid), the integer remainder otherwise.
__device__ __forceinline__ int wrap_index(int j, int num) {
    if (j < 0) j += num;
    else if (j >= num) j -= num;
    if ((unsigned)j >= (unsigned)num) {
        j %= num;
        if (j < 0) j += num;
    }
    return j;
}

// Node index of pre-mapping node j on an axis of `num` nodes with boundary `code`.
__device__ __forceinline__ int map_node(int j, int num, int code) {
    if (code == PERIODIC) return wrap_index(j, num);
    if (code == BOUNDED) return clampi(j, 0, num - 1);
    return j;
}

// The number of entries of an array along an axis (num + P - 1 on a clamped axis).
__host__ __device__ __forceinline__ int axis_extent(int num, int code, int degree) {
    return code == CLAMPED ? num + degree - 1 : num;
}

// a / b, correctly rounded, from rb = RN(1 / b): q0 = RN(a rb), one Newton step with the
// exact residual a - q b (an FMA) makes q1 faithful, and Markstein's correction
// q = RN(q1 + (a - q1 b) rb) is then the correctly rounded quotient (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000 processor", IBM J.
// Res. Dev. 34 (1990); Handbook of Floating-Point Arithmetic, ch. 5). Non-finite results
// (infinite or NaN operands, overflow) take the IEEE division.
template <typename T> __device__ __forceinline__ T div_rn(T a, T b, T rb) {
    const T q0 = a * rb;
    const T q1 = fma(fma(-q0, b, a), rb, q0);
    const T q = fma(fma(-q1, b, a), rb, q1);
    return isfinite(q) ? q : a / b;
}

// a / b, correctly rounded: a * rb when b is a power of two (pow2: rb = 1 / b exactly, so
// the product is the quotient, rounding included), else div_rn.
template <typename T> __device__ __forceinline__ T cells_from(T a, T b, T rb, int pow2) {
    return pow2 ? a * rb : div_rn(a, b, rb);
}

// rel - num * floor(rel / num): the periodic wrap of the reference stencils.
template <typename T> __device__ __forceinline__ T wrap_period(T rel, int num) {
    const T n = (T)num;
    return rel - n * floor(rel / n);
}

template <typename T, int P> __device__ __forceinline__ void uniform_weights(T d, T* w) {
    if constexpr (P == 0) {
        w[0] = T(1);
    } else if constexpr (P == 1) {
        w[0] = T(1) - d;
        w[1] = d;
    } else if constexpr (P == 2) {
        w[0] = T(0.5) * (T(0.5) - d) * (T(0.5) - d);
        w[1] = T(0.75) - d * d;
        w[2] = T(0.5) * (T(0.5) + d) * (T(0.5) + d);
    } else {
        const T complement = T(1) - d;
        const T square = d * d;
        const T cube = square * d;
        w[0] = complement * complement * complement / T(6);
        w[1] = (T(3) * cube - T(6) * square + T(4)) / T(6);
        w[2] = (T(-3) * cube + T(3) * square + T(3) * d + T(1)) / T(6);
        w[3] = cube / T(6);
    }
}

// d/dd of uniform_weights.
template <typename T, int P> __device__ __forceinline__ void uniform_derivatives(T d, T* g) {
    if constexpr (P == 0) {
        g[0] = T(0);
    } else if constexpr (P == 1) {
        g[0] = T(-1);
        g[1] = T(1);
    } else if constexpr (P == 2) {
        g[0] = d - T(0.5);
        g[1] = T(-2) * d;
        g[2] = T(0.5) + d;
    } else {
        const T complement = T(1) - d;
        g[0] = T(-0.5) * complement * complement;
        g[1] = T(1.5) * d * d - T(2) * d;
        g[2] = T(-1.5) * d * d + d + T(0.5);
        g[3] = T(0.5) * d * d;
    }
}

// Cox-de Boor on the clamped knots t_k = clip(k - P, 0, num - 1): the P + 1 B-splines
// of degree P that are non-zero in the cell of rel (STAGGERED false), or the P rescaled
// D_i = P / (t_(i+P) - t_i) B_(i,P-1), indexed i - 1 (STAGGERED true). Returns the cell.
template <typename T, int P, bool STAGGERED>
__device__ __forceinline__ int clamped_cell(T rel, int num, T* w) {
    T left[P + 1], right[P + 1];
    T r = rel;
    if (r < T(0)) r = T(0);
    if (r > T(num - 1)) r = T(num - 1);
    const int cell = clampi(trunc_int<T>(r), 0, num - 2);
    const int span = cell + P;
    constexpr int ORDER = STAGGERED ? P - 1 : P;
    w[0] = T(1);
#pragma unroll
    for (int k = 1; k <= ORDER; ++k) {
        const int low = clampi(span + 1 - k - P, 0, num - 1);
        const int high = clampi(span + k - P, 0, num - 1);
        left[k] = r - T(low);
        right[k] = T(high) - r;
        T saved = T(0);
#pragma unroll
        for (int m = 0; m < k; ++m) {
            const T temp = w[m] / (right[m + 1] + left[k - m]);
            w[m] = saved + right[m + 1] * temp;
            saved = left[k - m] * temp;
        }
        w[k] = saved;
    }
    if constexpr (STAGGERED) {
#pragma unroll
        for (int m = 0; m <= ORDER; ++m) {
            const int i = cell + 1 + m;
            const int low = clampi(i - P, 0, num - 1);
            const int high = clampi(i, 0, num - 1);
            w[m] = w[m] * T(P) / T(high - low);
        }
    }
    return cell;
}

// The uniform spline stencil of degree P of rel on a periodic or bounded axis: returns the
// pre-mapping first node and sets t, the offset of rel from the stencil's middle node
// (the weights are uniform_weights<P>(t)).
template <typename T, int P>
__device__ __forceinline__ int spline_frame(T rel, int num, int code, T& t) {
    // the usual case first: a middle node in [1, num - 2] means rel is in [0.5, num - 1.5)
    // (even P) or [1, num - 1) (odd P), where neither the wrap nor the clamps change anything
    {
        const int quick = (P % 2 == 0) ? trunc_int<T>(rel + T(0.5)) : trunc_int<T>(rel);
        if (quick >= 1 && quick <= num - 2) {
            t = rel - T(quick);
            return quick - P / 2;
        }
    }
    if (code == PERIODIC) {
        if (!(rel >= T(0) && rel < T(num))) rel = wrap_period(rel, num);
    } else {
        if (rel < T(0)) rel = T(0);
        if (rel > T(num - 1)) rel = T(num - 1);
    }
    int middle = (P % 2 == 0) ? trunc_int<T>(rel + T(0.5)) : trunc_int<T>(rel);
    middle = clampi(middle, 0, num);
    t = rel - T(middle);
    return middle - P / 2;
}

// The stencil of rel (the position in cells from the first node) along one axis: the
// pre-mapping base node, and the weights w[0..P]. KIND LINEAR needs P == 1, QUADRATIC
// P == 2; SPLINE takes P = 0..3 (clamped axes P >= 1).
template <typename T, int KIND, int P>
__device__ __forceinline__ int axis_stencil(T rel, int num, int code, T* w) {
    if constexpr (KIND == LINEAR) {
        // the usual case first: a left node in [1, num - 2] means 1 <= rel < num - 1, where
        // neither the wrap nor the clamp below changes anything
        {
            const int quick = trunc_int<T>(rel);
            if (quick >= 1 && quick <= num - 2) {
                const T f = rel - T(quick);
                w[0] = T(1) - f;
                w[1] = f;
                return quick;
            }
        }
        int left;
        if (code == PERIODIC) {
            // for 0 < rel < num - 1 the quotient rel / num rounds below 1: the wrap is exact identity
            if (!(rel > T(0) && rel < T(num - 1))) rel = wrap_period(rel, num);
            left = wrap_index(trunc_int<T>(rel), num);
        } else {
            left = rel >= T(0) ? trunc_int<T>(rel) : -1;
            left = clampi(left, 0, num - 2);
        }
        T f = rel - T(left);
        if (f < T(0)) f = T(0);
        if (f > T(1)) f = T(1);
        w[0] = T(1) - f;
        w[1] = f;
        return left;
    } else if constexpr (KIND == QUADRATIC) {
        // the usual case first: a nearest node in [1, num - 2] means 0.5 <= rel < num - 1.5,
        // where neither the wrap nor the clamps below change anything
        {
            const int quick = trunc_int<T>(rel + T(0.5));
            if (quick >= 1 && quick <= num - 2) {
                uniform_weights<T, 2>(rel - T(quick), w);
                return quick - 1;
            }
        }
        int c;
        if (code == PERIODIC) {
            if (!(rel > T(0) && rel < T(num - 1))) rel = wrap_period(rel, num);
            c = clampi(trunc_int<T>(rel + T(0.5)), 0, num);
        } else {
            if (rel < T(0)) rel = T(0);
            if (rel > T(num - 1)) rel = T(num - 1);
            c = clampi(trunc_int<T>(rel + T(0.5)), 0, num - 1);
        }
        uniform_weights<T, 2>(rel - T(c), w);
        return c - 1;
    } else {
        if constexpr (P >= 1) {
            if (code == CLAMPED) return clamped_cell<T, P, false>(rel, num, w);
        }
        T t;
        const int first = spline_frame<T, P>(rel, num, code, t);
        uniform_weights<T, P>(t, w);
        return first;
    }
}

// The stencil and the derivative of its weights with respect to rel; the derivative is
// zero where the stencil clamps the position (beyond a bounded or clamped axis).
template <typename T, int KIND, int P>
__device__ __forceinline__ int axis_stencil_derivative(T rel, int num, int code, T* w, T* g) {
    const int base = axis_stencil<T, KIND, P>(rel, num, code, w);
    const bool outside = code != PERIODIC && (rel < T(0) || rel > T(num - 1));
#pragma unroll
    for (int a = 0; a <= P; ++a) g[a] = T(0);
    if (outside) return base;
    if constexpr (P >= 1) {
        if (KIND == SPLINE && code == CLAMPED) {
            T dw[P > 1 ? P : 1];
            clamped_cell<T, P, true>(rel, num, dw);
#pragma unroll
            for (int m = 0; m <= P; ++m) {
                T v = T(0);
                if (m >= 1) v += dw[m - 1];
                if (m <= P - 1) v -= dw[m];
                g[m] = v;
            }
            return base;
        }
    }
    if constexpr (KIND == LINEAR) {
        g[0] = T(-1);
        g[1] = T(1);
    } else {
        T r = rel;
        if (code == PERIODIC) {
            if (KIND == QUADRATIC || !(r >= T(0) && r < T(num))) r = wrap_period(r, num);
        }
        const int middle = (P % 2 == 0) ? trunc_int<T>(r + T(0.5)) : trunc_int<T>(r);
        uniform_derivatives<T, P>(r - T(middle), g);
    }
    return base;
}

// The anchor node of a stencil (mapped): LINEAR's left node, QUADRATIC's nearest node,
// the middle node of a spline stencil, the cell on a clamped axis. Sort keys use it.
template <typename T, int KIND, int P>
__device__ __forceinline__ int axis_anchor(T rel, int num, int code) {
    T w[P + 1];
    const int base = axis_stencil<T, KIND, P>(rel, num, code, w);
    if constexpr (KIND == LINEAR) return map_node(base, num, code);
    else if constexpr (KIND == QUADRATIC) return map_node(base + 1, num, code);
    else {
        if (code == CLAMPED) return base;
        return map_node(base + P / 2, num, code);
    }
}

}  // namespace mpf

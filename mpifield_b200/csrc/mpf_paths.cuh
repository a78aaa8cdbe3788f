// mpf_paths.cuh -- the charge-conserving path deposits and the edge gathers.
//
// Edge fields are extent + (ndim,): entry (k, a) is the line integral along the edge from
// node k to its neighbour along axis a (src/mpifield/edges.py:1-31).
//
// WHITNEY (degree 1) follows deposit_paths_{1,2,3}d of mpifield
// (src/mpifield/kernels/deposit_paths_3d/deposit_paths_3d_cuda.cu:13-86 with
// whitney_cell.cuh:12-53): a straight path in cells is cut where it crosses a grid plane
// (the next plane of every axis, advanced together on ties), each piece clamped on
// bounded axes; the piece adds q times its length along an axis to the cell's edges
// along that axis, times their weights averaged over the piece (the midpoint's, plus or
// minus delta_u delta_w / 12 in 3D).
//
// The spline-edge deposit of degree P = 1..3 follows deposit_paths_spline_{1,2,3}d
// (deposit_paths_spline_3d_cuda.cu:14-130 with spline_edges.cuh:16-135): stretches of at
// most 4 cells, each cut at its knot planes (half-integers for even P; the nodes on a
// clamped axis) and at the walls of bounded axes, every clamped piece integrated with
// (P - 1 + (ndim - 1) P) / 2 + 1 Gauss-Legendre points; at a point the edges along axis a
// weigh B_{P-1}(r_a - k_a - 1/2) prod_{b != a} B_P(r_b - k_b), and edges past a bounded
// wall do not exist. Where the reference gathers every cut of a stretch into a 32-entry
// array and insertion-sorts it, this kernel merges the per-axis streams of crossing
// times in registers: the same times, each computed by the same formula, taken in the
// same ascending order, so the pieces are the same.
#pragma once
#include "mpf_internal.h"
#include "mpf_nodes.cuh"
#include "mpf_stencil.cuh"

namespace mpf {


// The longest a path may be, in pieces per stretch walk (WHITNEY) or stretches (spline):
// a bound on the work of one thread for absurd inputs; paths of physical length (a few
// cells per step) never reach it.
constexpr int kMaxPathSteps = 1 << 16;

// RN(1 / x), the correctly rounded reciprocal (the divisor table of div_rn).
template <typename T> __device__ __forceinline__ T recip_rn(T x);
template <> __device__ __forceinline__ double recip_rn<double>(double x) { return __drcp_rn(x); }
template <> __device__ __forceinline__ float recip_rn<float>(float x) { return __frcp_rn(x); }

template <typename T> __device__ __forceinline__ T clamp_to_axis(T rel, int num, int code) {
    if (code == PERIODIC) return rel;
    if (rel < T(0)) return T(0);
    if (rel > T(num) - T(1)) return T(num) - T(1);
    return rel;
}

// Adds v to edge (node index per axis, axis) with a global atomic.
template <typename T, int NDIM> struct GlobalEdgeSink {
    T* edges;
    int ext[3];
    __device__ __forceinline__ void add(const int* node, int axis, T v) const {
        int64_t k = node[0];
#pragma unroll
        for (int d = 1; d < NDIM; ++d) k = k * ext[d] + node[d];
        atomicAdd(edges + k * NDIM + axis, v);
    }
};

// The linear (Whitney) cell of a position: left and right nodes, the right weight.
template <typename T>
__device__ __forceinline__ void linear_nodes(T rel, int num, int code, int& left, int& right, T& f) {
    T w[2];
    const int base = axis_stencil<T, LINEAR, 1>(rel, num, code, w);
    left = map_node(base, num, code);
    right = map_node(base + 1, num, code);
    f = w[1];
}

template <typename T, int NDIM, typename Sink>
__device__ void whitney_path(T q, const T* a, const T* b, const Grid<T>& g, const Sink& sink) {
    // the crossing times (plane - a) / dl are correctly rounded quotients from RN(1 / dl)
    // (div_rn): the bits of the division, without a division per cut
    T dl[NDIM], rdl[NDIM], plane[NDIM], step[NDIM], p0[NDIM];
#pragma unroll
    for (int d = 0; d < NDIM; ++d) {
        dl[d] = b[d] - a[d];
        rdl[d] = recip_rn(dl[d]);
        if (dl[d] < T(0)) {
            plane[d] = ceil(a[d]) - T(1);
            step[d] = T(-1);
        } else {
            plane[d] = floor(a[d]) + T(1);
            step[d] = T(1);
        }
        p0[d] = clamp_to_axis(a[d], g.num[d], g.code[d]);
    }
    T time = T(0);
    for (int guard = 0; time < T(1) && guard < kMaxPathSteps; ++guard) {
        T times[NDIM];
        T following = T(1);
#pragma unroll
        for (int d = 0; d < NDIM; ++d) {
            times[d] = dl[d] != T(0) ? div_rn(plane[d] - a[d], dl[d], rdl[d]) : T(2);
            if (times[d] < following) following = times[d];
        }
        T p1[NDIM], f[NDIM], delta[NDIM];
        int lo[NDIM], hi[NDIM];
#pragma unroll
        for (int d = 0; d < NDIM; ++d) {
            p1[d] = clamp_to_axis(following < T(1) ? a[d] + following * dl[d] : b[d], g.num[d], g.code[d]);
            if (times[d] <= following) plane[d] += step[d];
            linear_nodes<T>(T(0.5) * (p0[d] + p1[d]), g.num[d], g.code[d], lo[d], hi[d], f[d]);
            delta[d] = p1[d] - p0[d];
        }
        if constexpr (NDIM == 1) {
            sink.add(lo, 0, q * delta[0]);
        } else if constexpr (NDIM == 2) {
            const T along_x = q * delta[0];
            const T along_y = q * delta[1];
            int n[2];
            n[0] = lo[0]; n[1] = lo[1]; sink.add(n, 0, (T(1) - f[1]) * along_x);
            n[0] = lo[0]; n[1] = hi[1]; sink.add(n, 0, f[1] * along_x);
            n[0] = lo[0]; n[1] = lo[1]; sink.add(n, 1, (T(1) - f[0]) * along_y);
            n[0] = hi[0]; n[1] = lo[1]; sink.add(n, 1, f[0] * along_y);
        } else {
#pragma unroll
            for (int axis = 0; axis < 3; ++axis) {
                // the two axes across this one, in increasing order
                const int ua = axis == 0 ? 1 : 0;
                const int wa = axis == 2 ? 1 : 2;
                const T cross = div_rn(delta[ua] * delta[wa], T(12), T(1) / T(12));
                const T along = q * delta[axis];
#pragma unroll
                for (int u = 0; u < 2; ++u)
#pragma unroll
                    for (int w = 0; w < 2; ++w) {
                        const T eu = u ? f[ua] : T(1) - f[ua];
                        const T ew = w ? f[wa] : T(1) - f[wa];
                        const T weight = eu * ew + (u == w ? cross : -cross);
                        int n[3] = {lo[0], lo[1], lo[2]};
                        n[ua] = u ? hi[ua] : lo[ua];
                        n[wa] = w ? hi[wa] : lo[wa];
                        sink.add(n, axis, along * weight);
                    }
            }
        }
        time = following;
#pragma unroll
        for (int d = 0; d < NDIM; ++d) p0[d] = p1[d];
    }
}

__device__ __forceinline__ int floor_to_int(double x) {
    int whole = trunc_int<double>(x);
    if (x < (double)whole) whole -= 1;
    return whole;
}
__device__ __forceinline__ int floor_to_int(float x) {
    int whole = trunc_int<float>(x);
    if (x < (float)whole) whole -= 1;
    return whole;
}

// The P edges along a periodic or bounded axis around rel: their (mapped) first nodes,
// whether each exists, and the offset t of rel - 1/2 from the middle of the degree P - 1
// stencil (the weights are uniform_weights<P - 1>(t)).
template <typename T, int P>
__device__ __forceinline__ void along_frame(T rel, int num, int code, int* edge, bool* exists, T& t) {
    constexpr int LOWER = P - 1;
    if (code == PERIODIC && !(rel >= T(0) && rel < T(num))) rel = wrap_period(rel, num);
    const T shifted = rel - T(0.5);
    int middle;
    if constexpr (LOWER % 2 == 0) {
        middle = floor_to_int(shifted + T(0.5));
        if (code == BOUNDED && middle > num - 2) middle = num - 2;
    } else {
        middle = floor_to_int(shifted);
    }
    middle = clampi(middle, -2, num + 1);
    t = shifted - T(middle);
    const int first = middle - LOWER / 2;
#pragma unroll
    for (int a = 0; a < P; ++a) {
        const int k = first + a;
        if (code == PERIODIC) {
            edge[a] = map_node(k, num, PERIODIC);
            exists[a] = true;
        } else if (k < 0 || k > num - 2) {
            edge[a] = 0;
            exists[a] = false;
        } else {
            edge[a] = k;
            exists[a] = true;
        }
    }
}

// The P edges along an axis around rel: their (mapped) first nodes, weights
// B_{P-1}(rel - k - 1/2) and whether each exists (spline_edges.cuh:22-65).
template <typename T, int P>
__device__ __forceinline__ void along_stencil(T rel, int num, int code, int* edge, T* weight, bool* exists) {
    if (code == CLAMPED) {
        const int cell = clamped_cell<T, P, true>(rel, num, weight);
#pragma unroll
        for (int a = 0; a < P; ++a) {
            edge[a] = cell + a;
            exists[a] = true;
        }
        return;
    }
    T t;
    along_frame<T, P>(rel, num, code, edge, exists, t);
    uniform_weights<T, P - 1>(t, weight);
}

// Gauss-Legendre points and weights on [0, 1] for COUNT = 1..5 points: the values of
// numpy.polynomial.legendre.leggauss(COUNT) mapped from [-1, 1] (spline_edges.cuh:67-89).
template <typename T, int COUNT> struct Gauss;
template <typename T> struct Gauss<T, 1> {
    static __device__ __forceinline__ T point(int) { return T(0.5); }
    static __device__ __forceinline__ T weight(int) { return T(1.0); }
};
template <typename T> struct Gauss<T, 2> {
    static __device__ __forceinline__ T point(int g) { return g == 0 ? T(0.21132486540518713) : T(0.7886751345948129); }
    static __device__ __forceinline__ T weight(int) { return T(0.5); }
};
template <typename T> struct Gauss<T, 3> {
    static __device__ __forceinline__ T point(int g) {
        return g == 0 ? T(0.1127016653792583) : (g == 1 ? T(0.5) : T(0.8872983346207417));
    }
    static __device__ __forceinline__ T weight(int g) {
        return g == 1 ? T(0.4444444444444444) : T(0.2777777777777778);
    }
};
template <typename T> struct Gauss<T, 4> {
    static __device__ __forceinline__ T point(int g) {
        return g == 0 ? T(0.06943184420297371)
                      : (g == 1 ? T(0.33000947820757187) : (g == 2 ? T(0.6699905217924281) : T(0.9305681557970262)));
    }
    static __device__ __forceinline__ T weight(int g) {
        return (g == 0 || g == 3) ? T(0.17392742256872692) : T(0.3260725774312731);
    }
};
template <typename T> struct Gauss<T, 5> {
    static __device__ __forceinline__ T point(int g) {
        return g == 0 ? T(0.04691007703066802)
                      : (g == 1 ? T(0.23076534494715845)
                                : (g == 2 ? T(0.5) : (g == 3 ? T(0.7692346550528415) : T(0.9530899229693319))));
    }
    static __device__ __forceinline__ T weight(int g) {
        return (g == 0 || g == 4) ? T(0.11846344252809454)
                                  : ((g == 1 || g == 3) ? T(0.2393143352496832) : T(0.28444444444444444));
    }
};

// The ascending crossing times of one axis over a stretch: knot planes first..last
// walked in the direction of increasing time, then merged with the two wall times. The
// times are correctly rounded quotients (div_rn with RN(1 / delta)), the bits of the
// division; the pending walls are a queue of 2-bit codes (1: the wall at 0, 2: the wall
// at num - 1), their times computed when looked at.
template <typename T> struct CutStream {
    T a0, delta, plane;
    int left;   // planes not yet taken
    int walls;  // the pending walls, the next in the low two bits

    __device__ __forceinline__ T wall_time(int code, int num) const {
        return div_rn((code == 1 ? T(0) : T(num) - T(1)) - a0, delta, recip_rn(delta));
    }

    __device__ __forceinline__ void init(T s0, T s1, T shift, int num, int code) {
        a0 = s0;
        delta = s1 - s0;
        left = 0;
        walls = 0;
        plane = T(0);
        if (delta == T(0)) return;
        const T low = delta > T(0) ? s0 : s1;
        const T high = delta > T(0) ? s1 : s0;
        const T offset = code == CLAMPED ? T(0) : shift;
        const T first = T(floor_to_int(low - offset)) + T(1) + offset;
        int count = 0;
        while (first + T(count) < high && count < 64) ++count;
        left = count;
        plane = delta > T(0) ? first : first + T(count - 1);
        if (code != PERIODIC) {
            const T t0 = wall_time(1, num);
            const T t1 = wall_time(2, num);
            const bool in0 = t0 > T(0) && t0 < T(1);
            const bool in1 = t1 > T(0) && t1 < T(1);
            if (in0 && in1) walls = t0 < t1 ? (1 | 2 << 2) : (2 | 1 << 2);
            else if (in0) walls = 1;
            else if (in1) walls = 2;
        }
    }
    // The next plane in the direction of increasing time (delta > 0: up).
    __device__ __forceinline__ void advance() {
        plane += delta > T(0) ? T(1) : T(-1);
        --left;
    }
    // The next plane time inside (0, 1), skipping the ones rounding outside.
    __device__ __forceinline__ T peek_plane() {
        if (left > 0) {
            const T rd = recip_rn(delta);
            while (left > 0) {
                const T t = div_rn(plane - a0, delta, rd);
                if (t > T(0) && t < T(1)) return t;
                advance();
            }
        }
        return T(2);
    }
    __device__ __forceinline__ T peek_wall(int num) const { return walls ? wall_time(walls & 3, num) : T(2); }
    __device__ __forceinline__ void pop_wall() { walls >>= 2; }
};

// One piece of a spline path: q times the line integral of the edge functions from p0
// to p0 + step (cell coordinates, clamped on bounded axes), added to the sink.
//
// CS > 0: `cache` is this thread's column (stride CS) of a shared-memory table that holds,
// for the axis being deposited, the weights of every Gauss point along the two axes across
// it -- computed once per axis instead of once per edge along it.
template <typename T, int NDIM, int P, typename Sink, int CS = 0>
__device__ __forceinline__ void spline_piece(T q, const T* p0, const T* step, const Grid<T>& g, bool clamped,
                                             const Sink& sink, T* cache = nullptr) {
    constexpr int NPTS = (P - 1 + (NDIM - 1) * P) / 2 + 1;
    if (!clamped) {
        // The Gauss points of a piece lie in one knot interval on every axis:
        // the nodes, the edges and their existence are those of the piece's
        // midpoint, and a point's weights are the stencil polynomials at the
        // midpoint's offset plus (point - 1/2) times the step. The contributions
        // of the points are summed in registers, one atomic per edge and axis.
        int sidx[3][P + 1], aidx[3][P > 0 ? P : 1];
        bool aex[3][P > 0 ? P : 1];
        T st[3], at[3];
#pragma unroll
        for (int d = 0; d < NDIM; ++d) {
            const T mid = p0[d] + T(0.5) * step[d];
            const int first = spline_frame<T, P>(mid, g.num[d], g.code[d], st[d]);
#pragma unroll
            for (int s = 0; s <= P; ++s) sidx[d][s] = map_node(first + s, g.num[d], g.code[d]);
            along_frame<T, P>(mid, g.num[d], g.code[d], aidx[d], aex[d], at[d]);
        }
        constexpr int SX = P + 1;
        constexpr int CB = NDIM > 1 ? SX : 1;
        constexpr int CC = NDIM > 2 ? SX : 1;
#pragma unroll
        for (int axis = 0; axis < NDIM; ++axis) {
            if (q * step[axis] == T(0)) continue;
            // the axes across this one, in increasing order
            const int o1 = NDIM > 1 ? (axis == 0 ? 1 : 0) : 0;
            const int o2 = NDIM > 2 ? (axis == 2 ? 1 : 2) : 0;
            if constexpr (CS > 0) {
#pragma unroll 1
                for (int gp = 0; gp < NPTS; ++gp) {
                    const T off = Gauss<T, NPTS>::point(gp) - T(0.5);
                    T wb[SX], wc[SX];
                    uniform_weights<T, P>(st[o1] + off * step[o1], wb);
                    uniform_weights<T, P>(st[o2] + off * step[o2], wc);
#pragma unroll
                    for (int b = 0; b < SX; ++b) {
                        cache[(gp * 2 * SX + b) * CS] = wb[b];
                        cache[(gp * 2 * SX + SX + b) * CS] = wc[b];
                    }
                }
            }
            // one edge along the axis at a time: (P + 1)^(ndim - 1) sums
#pragma unroll
            for (int e = 0; e < P; ++e) {
                if (!aex[axis][e]) continue;
                T acc[CB * CC];
#pragma unroll
                for (int k = 0; k < CB * CC; ++k) acc[k] = T(0);
                // (with the cache the points are a loop, not unrolled: the unrolled cubic
                // body outgrew the instruction cache)
#pragma unroll ((CS > 0 || P >= 2) ? 1 : NPTS)
                for (int gp = 0; gp < NPTS; ++gp) {
                    const T off = Gauss<T, NPTS>::point(gp) - T(0.5);
                    T wa[P > 0 ? P : 1], wb[SX], wc[SX];
                    uniform_weights<T, P - 1>(at[axis] + off * step[axis], wa);
                    if constexpr (CS > 0) {
#pragma unroll
                        for (int b = 0; b < SX; ++b) {
                            wb[b] = cache[(gp * 2 * SX + b) * CS];
                            wc[b] = cache[(gp * 2 * SX + SX + b) * CS];
                        }
                    } else {
                        if constexpr (NDIM > 1) uniform_weights<T, P>(st[o1] + off * step[o1], wb);
                        if constexpr (NDIM > 2) uniform_weights<T, P>(st[o2] + off * step[o2], wc);
                    }
                    const T along = q * Gauss<T, NPTS>::weight(gp) * step[axis] * wa[e];
#pragma unroll
                    for (int b = 0; b < CB; ++b) {
                        const T wab = NDIM > 1 ? along * wb[b] : along;
#pragma unroll
                        for (int c = 0; c < CC; ++c) {
                            T& r = acc[b * CC + c];
                            if constexpr (NDIM > 2) r = fma(wab, wc[c], r);
                            else r = r + wab;
                        }
                    }
                }
#pragma unroll
                for (int b = 0; b < CB; ++b)
#pragma unroll
                    for (int c = 0; c < CC; ++c) {
                        int n[3] = {0, 0, 0};
                        n[axis] = aidx[axis][e];
                        if constexpr (NDIM > 1) n[o1] = sidx[o1][b];
                        if constexpr (NDIM > 2) n[o2] = sidx[o2][c];
                        sink.add(n, axis, acc[b * CC + c]);
                    }
            }
        }
    } else {
        // clamped knots: every Gauss point computes its full stencil (Cox-de Boor
        // near the walls) and adds its own contributions
#pragma unroll
        for (int gp = 0; gp < NPTS; ++gp) {
            const T point = Gauss<T, NPTS>::point(gp);
            const T gw = Gauss<T, NPTS>::weight(gp);
            T rel[NDIM];
#pragma unroll
            for (int d = 0; d < NDIM; ++d) rel[d] = p0[d] + point * step[d];
#pragma unroll 1
            for (int axis = 0; axis < NDIM; ++axis) {
                const T amount = q * gw * step[axis];
                if (amount == T(0)) continue;
                int idx[3][P + 1];
                T wt[3][P + 1];
                bool ex[P > 0 ? P : 1];
#pragma unroll
                for (int d = 0; d < NDIM; ++d) {
                    if (d == axis) {
                        along_stencil<T, P>(rel[d], g.num[d], g.code[d], idx[d], wt[d], ex);
                    } else {
                        const int base = axis_stencil<T, SPLINE, P>(rel[d], g.num[d], g.code[d], wt[d]);
#pragma unroll
                        for (int s2 = 0; s2 <= P; ++s2) idx[d][s2] = map_node(base + s2, g.num[d], g.code[d]);
                    }
                }
                const int cnt0 = axis == 0 ? P : P + 1;
                const int cnt1 = NDIM > 1 ? (axis == 1 ? P : P + 1) : 1;
                const int cnt2 = NDIM > 2 ? (axis == 2 ? P : P + 1) : 1;
                for (int x = 0; x < cnt0; ++x) {
                    if (axis == 0 && !ex[x]) continue;
                    for (int y = 0; y < cnt1; ++y) {
                        if (NDIM > 1 && axis == 1 && !ex[y]) continue;
                        for (int z = 0; z < cnt2; ++z) {
                            if (NDIM > 2 && axis == 2 && !ex[z]) continue;
                            T w = amount * wt[0][x];
                            if constexpr (NDIM > 1) w = w * wt[1][y];
                            if constexpr (NDIM > 2) w = w * wt[2][z];
                            int n[3] = {idx[0][x], NDIM > 1 ? idx[1][y] : 0, NDIM > 2 ? idx[2][z] : 0};
                            sink.add(n, axis, w);
                        }
                    }
                }
            }
        }
    }
}

// The pieces of a spline path, one at a time: stretches of at most 4 cells, each cut at
// its knot planes and walls in ascending time (the merged CutStreams). begin() starts a
// path at its first stretch; piece() takes the next cut and returns true with the piece
// (p0, step) when it has a length, and sets `ended` after the stretch's last cut; then
// more() tells whether another stretch follows, which next() starts (the path's ends
// given again: the walk does not keep them). live turns false after the last stretch.
template <typename T, int NDIM, int P> struct SplineWalk {
    CutStream<T> cs[NDIM];  // cs[d].a0, cs[d].delta: the stretch's start and extent per axis
    T t0;
    int st, stretches, guard;
    bool live, ended;

    __device__ __forceinline__ void start_stretch(const T* r0, const T* r1, const Grid<T>& g) {
        const T shift = (P % 2 == 0) ? T(0.5) : T(0);
#pragma unroll
        for (int d = 0; d < NDIM; ++d) {
            // (x / 1 is x: one stretch, the usual case, divides nothing)
            const T u0 = (r1[d] - r0[d]) * T(st), u1 = (r1[d] - r0[d]) * T(st + 1);
            cs[d].init(r0[d] + (stretches == 1 ? u0 : u0 / T(stretches)),
                       r0[d] + (stretches == 1 ? u1 : u1 / T(stretches)), shift, g.num[d], g.code[d]);
        }
        t0 = T(0);
        guard = 0;
        ended = false;
    }

    __device__ __forceinline__ void begin(const T* r0, const T* r1, const Grid<T>& g) {
        T extent = T(0);
#pragma unroll
        for (int d = 0; d < NDIM; ++d) {
            const T span = r1[d] > r0[d] ? r1[d] - r0[d] : r0[d] - r1[d];
            if (span > extent) extent = span;
        }
        stretches = trunc_int<T>(extent / T(4)) + 1;
        if (stretches > kMaxPathSteps || stretches < 1) stretches = kMaxPathSteps;
        st = 0;
        live = true;
        start_stretch(r0, r1, g);
    }

    __device__ __forceinline__ bool more() const { return st + 1 < stretches; }

    __device__ __forceinline__ void next(const T* r0, const T* r1, const Grid<T>& g) {
        ++st;
        start_stretch(r0, r1, g);
    }

    __device__ __forceinline__ bool piece(const Grid<T>& g, T* p0, T* step) {
        // the next cut: the least pending time of every stream, or the end
        T t1 = T(1);
        int which = -1;
#pragma unroll
        for (int d = 0; d < NDIM; ++d) {
            const T tp = cs[d].peek_plane();
            if (tp < t1) { t1 = tp; which = 2 * d; }
            const T tw = cs[d].peek_wall(g.num[d]);
            if (tw < t1) { t1 = tw; which = 2 * d + 1; }
        }
        if (which >= 0) {
#pragma unroll
            for (int d = 0; d < NDIM; ++d) {
                if (which == 2 * d) cs[d].advance();
                if (which == 2 * d + 1) cs[d].pop_wall();
            }
        }
        const bool length = t1 > t0;
        if (length) {
#pragma unroll
            for (int d = 0; d < NDIM; ++d) {
                T begin_ = cs[d].a0 + t0 * cs[d].delta;
                T finish = cs[d].a0 + t1 * cs[d].delta;
                if (g.code[d] != PERIODIC) {
                    const T top = T(g.num[d] - 1);
                    if (begin_ < T(0)) begin_ = T(0);
                    if (begin_ > top) begin_ = top;
                    if (finish < T(0)) finish = T(0);
                    if (finish > top) finish = top;
                }
                p0[d] = begin_;
                step[d] = finish - begin_;
            }
        }
        t0 = t1;
        if (which < 0 || ++guard >= 64) ended = true;  // the stretch is done
        return length;
    }
};

// Whether any axis has clamped knots.
template <typename T, int NDIM> __device__ __forceinline__ bool any_clamped(const Grid<T>& g) {
    bool clamped = false;
#pragma unroll
    for (int d = 0; d < NDIM; ++d) clamped = clamped || g.code[d] == CLAMPED;
    return clamped;
}

template <typename T, int NDIM, int P, typename Sink>
__device__ void spline_path(T q, const T* r0, const T* r1, const Grid<T>& g, const Sink& sink) {
    const bool clamped = any_clamped<T, NDIM>(g);
    SplineWalk<T, NDIM, P> walk;
    walk.begin(r0, r1, g);
    for (;;) {
        T p0[NDIM], step[NDIM];
        if (walk.piece(g, p0, step)) spline_piece<T, NDIM, P>(q, p0, step, g, clamped, sink);
        if (!walk.ended) continue;
        if (!walk.more()) break;
        walk.next(r0, r1, g);
    }
}



// The cell coordinates r0, r1 of a path's ends s, e; false for a path whose ends are not
// finite (it deposits nothing: src/mpifield/edges.py:87).
template <typename T, int NDIM, bool WHITNEY>
__device__ __forceinline__ bool path_cells_of(const Grid<T>& g, const T* s, const T* e, T* r0, T* r1) {
    bool finite = true;
#pragma unroll
    for (int d = 0; d < NDIM; ++d) {
        r0[d] = cells_from(s[d] - g.lower[d], g.cell[d], g.inv[d], g.pow2[d]);
        r1[d] = cells_from(e[d] - g.lower[d], g.cell[d], g.inv[d], g.pow2[d]);
        if constexpr (WHITNEY) {
            const T big = sizeof(T) == 8 ? T(1e300) : T(3e38);
            if (!(r0[d] > -big && r0[d] < big && r1[d] > -big && r1[d] < big)) finite = false;
        } else {
            if (!(s[d] - s[d] == T(0)) || !(e[d] - e[d] == T(0))) finite = false;
        }
    }
    return finite;
}

// The same for path i of the arguments.
template <typename T, int NDIM, bool WHITNEY>
__device__ __forceinline__ bool path_cells(const PathArgs<T>& a, int64_t i, T* r0, T* r1) {
    T s[NDIM], e[NDIM];
#pragma unroll
    for (int d = 0; d < NDIM; ++d) {
        s[d] = a.start[d * a.start_stride + i];
        e[d] = a.end[d * a.end_stride + i];
    }
    return path_cells_of<T, NDIM, WHITNEY>(a.g, s, e, r0, r1);
}

// edges += the box of a sink (its non-zero entries), with global atomics.
template <typename T, int NDIM, typename Sink, typename G>
__device__ __forceinline__ void flush_edge_box(const T* tile, T* edges, const Sink& sink, const G& g) {
    int vol = NDIM;
#pragma unroll
    for (int d = 0; d < NDIM; ++d) vol *= sink.ex[d];
    for (int k = threadIdx.x; k < vol; k += blockDim.x) {
        const T v = tile[k];
        if (v == T(0)) continue;
        const int axis = k % NDIM;
        int rest = k / NDIM;
        int node[3];
#pragma unroll
        for (int d = NDIM - 1; d >= 0; --d) {
            const int r = rest % sink.ex[d];
            rest /= sink.ex[d];
            int n = sink.lo[d] + r;
            if (sink.periodic[d] && n >= g.num[d]) n -= g.num[d];
            node[d] = n;
        }
        int64_t gi = node[0];
#pragma unroll
        for (int d = 1; d < NDIM; ++d) gi = gi * g.ext[d] + node[d];
        atomicAdd(edges + gi * NDIM + axis, v);
    }
}

// Adds v to edge (node per axis, axis) in the chunk's box of edges in shared memory when
// the node lies in it, else with a global atomic. On a periodic axis the box is an arc of
// the period: the node is inside when (node - lo) mod num < ex.
template <typename T, int NDIM> struct BoxEdgeSink {
    T* tile;
    T* edges;
    int lo[3], ex[3], num[3], ext[3];
    bool periodic[3];
    bool staged;
    __device__ __forceinline__ void add(const int* node, int axis, T v) const {
        if (staged) {
            int k = 0;
            bool inside = true;
#pragma unroll
            for (int d = 0; d < NDIM; ++d) {
                int r = node[d] - lo[d];
                if (periodic[d] && r < 0) r += num[d];
                inside = inside && (unsigned)r < (unsigned)ex[d];
                k = k * ex[d] + r;
            }
            if (inside) {
                atomicAdd(tile + k * NDIM + axis, v);
                return;
            }
        }
        int64_t g = node[0];
#pragma unroll
        for (int d = 1; d < NDIM; ++d) g = g * ext[d] + node[d];
        atomicAdd(edges + g * NDIM + axis, v);
    }
};

// The range of cells whose edges a path can touch along one axis (pre-mapping, with a
// margin for the rounding of the kernel's own cell coordinates).
template <typename T, int P>
__device__ __forceinline__ void path_reach(T r0, T r1, int& first, int& last) {
    constexpr int REACH = P + 1;
    const T lo = r0 < r1 ? r0 : r1;
    const T hi = r0 < r1 ? r1 : r0;
    const T cap = T(1 << 29);
    first = floor_to_int(lo > -cap ? lo : -cap) - REACH;
    last = floor_to_int(hi < cap ? hi : cap) + REACH;
}

// The path deposit on markers sorted by cell tile. A CTA takes a contiguous range of
// chunks of blockDim x paths_per_thread paths. Pass 1 reduces the chunk's reach to a box
// per axis (on a periodic axis in whichever of two frames, the plain one or one shifted
// by half a period, gives the shorter span, so a chunk across the seam stays compact);
// when the box's edges fit the shared memory, pass 2 deposits every path of the chunk
// into it (shared-memory atomic adds) and the box is added to the edge field once, with
// global atomics, when the next chunk needs another box. Otherwise the chunk's paths add
// to global memory as in deposit_paths_kernel. The arithmetic of each path is that of
// whitney_path / spline_path.
template <typename T, int NDIM, int P, bool WHITNEY>
__global__ void __launch_bounds__(256) deposit_paths_tiled_kernel(const PathArgs<T> a) {
    __shared__ int s_lo[3], s_hi[3], s_lo2[3], s_hi2[3];
    T* tile = reinterpret_cast<T*>(mpf_dynamic_smem);
    BoxEdgeSink<T, NDIM> sink;
    sink.tile = tile;
    sink.edges = a.edges_out;
    int half[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        sink.num[d] = a.g.num[d];
        sink.ext[d] = a.g.ext[d];
        sink.periodic[d] = a.g.code[d] == PERIODIC;
        sink.lo[d] = 0;
        sink.ex[d] = 1;
        half[d] = a.g.num[d] / 2;
    }
    sink.staged = false;
    bool have_box = false;
    const int ppt = a.paths_per_thread;
    const int64_t CH = (int64_t)blockDim.x * ppt;
    const int64_t nchunks = (a.n + CH - 1) / CH;
    int64_t c_first, c_last;
    chunk_range(nchunks, c_first, c_last);
    for (int64_t ci = c_first; ci < c_last; ++ci) {
        const int64_t first = ci * CH;
        // pass 1: the reach of the chunk's live paths, in both frames
        int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
        int lo2[3] = {INT_MAX, INT_MAX, INT_MAX}, hi2[3] = {INT_MIN, INT_MIN, INT_MIN};
        for (int m = 0; m < ppt; ++m) {
            const int64_t i = first + (int64_t)m * blockDim.x + threadIdx.x;
            if (i >= a.n) continue;
            const T q = a.charges[i];
            if (q == T(0)) continue;
            T r0[NDIM], r1[NDIM];
            if (!path_cells<T, NDIM, WHITNEY>(a, i, r0, r1)) continue;
#pragma unroll
            for (int d = 0; d < NDIM; ++d) {
                int f, l;
                path_reach<T, P>(r0[d], r1[d], f, l);
                if (a.g.code[d] == PERIODIC) {
                    const int span = l - f;
                    const int s0 = wrap_index(f, a.g.num[d]);
                    const int s1 = wrap_index(f + half[d], a.g.num[d]) + a.g.num[d] - half[d];
                    lo[d] = min(lo[d], s0);
                    hi[d] = max(hi[d], s0 + span);
                    lo2[d] = min(lo2[d], s1);
                    hi2[d] = max(hi2[d], s1 + span);
                } else {
                    lo[d] = min(lo[d], clampi(f, 0, a.g.ext[d] - 1));
                    hi[d] = max(hi[d], clampi(l, 0, a.g.ext[d] - 1));
                }
            }
        }
        bool staged = false;
        if (a.capacity > 0) {
            if (threadIdx.x < 3) {
                s_lo[threadIdx.x] = INT_MAX;
                s_hi[threadIdx.x] = INT_MIN;
                s_lo2[threadIdx.x] = INT_MAX;
                s_hi2[threadIdx.x] = INT_MIN;
            }
            __syncthreads();
            block_box<NDIM>(lo, hi, s_lo, s_hi);
            block_box<NDIM>(lo2, hi2, s_lo2, s_hi2);
            __syncthreads();
            int nlo[3] = {0, 0, 0}, nex[3] = {1, 1, 1};
            bool empty = false;
            int64_t vol = NDIM;
#pragma unroll
            for (int d = 0; d < NDIM; ++d) {
                int l = s_lo[d], h = s_hi[d];
                if (h < l) empty = true;
                if (a.g.code[d] == PERIODIC && s_hi2[d] - s_lo2[d] < h - l) {
                    l = s_lo2[d];
                    h = s_hi2[d];
                }
                if (a.g.code[d] == PERIODIC) {
                    nlo[d] = wrap_index(l, a.g.num[d]);
                    nex[d] = min(h - l + 1, a.g.num[d]);
                } else {
                    nlo[d] = l;
                    nex[d] = h - l + 1;
                }
                vol *= nex[d] > 0 ? nex[d] : 1;
            }
            if (empty) {  // no live path in the chunk
                __syncthreads();
                continue;
            }
            bool holds = have_box;
#pragma unroll
            for (int d = 0; d < NDIM; ++d) {
                int r = nlo[d] - sink.lo[d];
                if (sink.periodic[d] && r < 0) r += a.g.num[d];
                holds = holds && r >= 0 && r + nex[d] <= sink.ex[d];
            }
            if (holds) {
                staged = true;
            } else if (vol <= (int64_t)a.capacity) {
                if (have_box) flush_edge_box<T, NDIM>(tile, a.edges_out, sink, a.g);
                __syncthreads();
                for (int k = threadIdx.x; k < (int)vol; k += blockDim.x) tile[k] = T(0);
#pragma unroll
                for (int d = 0; d < NDIM; ++d) {
                    sink.lo[d] = nlo[d];
                    sink.ex[d] = nex[d];
                }
                __syncthreads();
                have_box = true;
                staged = true;
            }
        }
        sink.staged = staged;
        // pass 2: the paths, into the box where it holds them. Lane l of warp w takes the
        // paths l * (warps * ppt) + w * ppt + m of the chunk: the lanes of a warp are
        // warps * ppt paths apart, in different cells of a sorted store, so that their
        // shared-memory adds of one instruction land on different nodes.
        const int warps = blockDim.x >> 5;
        const int64_t base = first + (int64_t)(threadIdx.x & 31) * warps * ppt + (int64_t)(threadIdx.x >> 5) * ppt;
        for (int m = 0; m < ppt; ++m) {
            const int64_t i = base + m;
            if (i >= a.n) continue;
            const T q = a.charges[i];
            if (q == T(0)) continue;
            T r0[NDIM], r1[NDIM];
            if (!path_cells<T, NDIM, WHITNEY>(a, i, r0, r1)) continue;
            if constexpr (WHITNEY) whitney_path<T, NDIM>(q, r0, r1, a.g, sink);
            else spline_path<T, NDIM, P>(q, r0, r1, a.g, sink);
        }
        __syncthreads();
    }
    if (have_box) flush_edge_box<T, NDIM>(tile, a.edges_out, sink, a.g);
}

// The paths first, first + STRIDE, ... below end deposited into the sink by one thread.
// The spline paths go piece by piece: a lane whose path is done takes its next one while
// the others deposit their next piece, so the lanes of a warp deposit pieces together
// whatever the number of pieces of their paths (a loop over paths would hold every lane
// until the warp's longest path is done). FLAT false: a path at a time.
template <typename T, int NDIM, int P, bool WHITNEY, int STRIDE, bool FLAT, typename Sink, int CS = 0>
__device__ __forceinline__ void deposit_range(const PathArgs<T>& a, int64_t i, int64_t end, const Sink& sink,
                                              T* cache = nullptr) {
    if constexpr (!WHITNEY && FLAT) {
        const bool clamped = any_clamped<T, NDIM>(a.g);
        SplineWalk<T, NDIM, P> walk;
        walk.live = false;
        T q = T(0);
        int64_t ip = 0;  // the walk's path
        for (;;) {
            if (!walk.live) {  // this lane's next path
                if (i >= end) break;
                ip = i;
                i += STRIDE;
                q = a.charges[ip];
                T r0[NDIM], r1[NDIM];
                if (q == T(0) || !path_cells<T, NDIM, false>(a, ip, r0, r1)) continue;
                walk.begin(r0, r1, a.g);
            }
            T p0[NDIM], step[NDIM];
            if (walk.piece(a.g, p0, step)) spline_piece<T, NDIM, P, Sink, CS>(q, p0, step, a.g, clamped, sink, cache);
            if (walk.ended) {
                if (walk.more()) {  // a path of several stretches: its ends again
                    T r0[NDIM], r1[NDIM];
                    path_cells<T, NDIM, false>(a, ip, r0, r1);
                    walk.next(r0, r1, a.g);
                } else {
                    walk.live = false;
                }
            }
        }
    } else {
        for (; i < end; i += STRIDE) {
            const T q = a.charges[i];
            if (q == T(0)) continue;
            T r0[NDIM], r1[NDIM];
            if (!path_cells<T, NDIM, WHITNEY>(a, i, r0, r1)) continue;
            if constexpr (WHITNEY) whitney_path<T, NDIM>(q, r0, r1, a.g, sink);
            else spline_path<T, NDIM, P>(q, r0, r1, a.g, sink);
        }
    }
}

// One thread per path, global atomics; BLOCK threads, at least MINB CTAs per SM. Each CTA
// takes an equal contiguous share of the paths, BLOCK consecutive paths at a time, so that
// in a store sorted by cell the CTAs work in different regions of the grid at once and
// their atomic adds spread over the L2 (a grid-stride walk keeps every CTA in one small
// region of a sorted store). Lane l of warp w takes the path l * (BLOCK / 32) + w of
// the BLOCK: the lanes of a warp are BLOCK / 32 paths apart, in different cells, so the
// adds of one instruction do not pile onto the same edges.
template <typename T, int NDIM, int P, bool WHITNEY, int BLOCK = 256, int MINB = 1, bool FLAT = true,
          bool CACHE = false>
__global__ void __launch_bounds__(BLOCK, MINB) deposit_paths_kernel(const PathArgs<T> a) {
    GlobalEdgeSink<T, NDIM> sink;
    sink.edges = a.edges_out;
#pragma unroll
    for (int d = 0; d < 3; ++d) sink.ext[d] = a.g.ext[d];
    const int slot = (threadIdx.x & 31) * (BLOCK / 32) + (threadIdx.x >> 5);
    const int64_t per = ((a.n + gridDim.x - 1) / gridDim.x + BLOCK - 1) / BLOCK * BLOCK;
    const int64_t mine_end = min(a.n, (int64_t)(blockIdx.x + 1) * per);
    if constexpr (CACHE) {
        T* cache = reinterpret_cast<T*>(mpf_dynamic_smem) + threadIdx.x;
        deposit_range<T, NDIM, P, WHITNEY, BLOCK, FLAT, GlobalEdgeSink<T, NDIM>, BLOCK>(
            a, (int64_t)blockIdx.x * per + slot, mine_end, sink, cache);
    } else {
        deposit_range<T, NDIM, P, WHITNEY, BLOCK, FLAT>(a, (int64_t)blockIdx.x * per + slot, mine_end, sink);
    }
}

// Shared memory of deposit_paths_kernel with CACHE: a column per thread of the cross-axis
// weights of every Gauss point (two axes, P + 1 weights each).
template <typename T, int NDIM, int P>
constexpr int path_cache_bytes(int block) {
    return (P - 1 + (NDIM - 1) * P) / 2 + 1 > 0 ? ((P - 1 + (NDIM - 1) * P) / 2 + 1) * 2 * (P + 1) * block * (int)sizeof(T)
                                                 : 0;
}

// Adds v to edge (node per axis, axis) of a private copy of the whole edge field in
// shared memory (same layout as the field).
template <typename T, int NDIM> struct SharedEdgeSink {
    T* box;
    int ext[3];
    __device__ __forceinline__ void add(const int* node, int axis, T v) const {
        int k = node[0];
#pragma unroll
        for (int d = 1; d < NDIM; ++d) k = k * ext[d] + node[d];
        atomicAdd(box + k * NDIM + axis, v);
    }
};

// The path deposit onto a small edge field (entries in shared memory): each CTA adds its
// share of the paths (as deposit_paths_kernel) into a private copy of the whole field in
// shared memory and then adds the copy's non-zero entries to the field, one global atomic
// each. On a grid of a few hundred edges the global adds of every CTA would pile onto the
// same few L2 lines; here they meet only in the CTA's shared memory.
template <typename T, int NDIM, int P, bool WHITNEY, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) deposit_paths_private_kernel(const PathArgs<T> a) {
    SharedEdgeSink<T, NDIM> sink;
    sink.box = reinterpret_cast<T*>(mpf_dynamic_smem);
    int total = NDIM;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        sink.ext[d] = a.g.ext[d];
        if (d < NDIM) total *= a.g.ext[d];
    }
    for (int q = threadIdx.x; q < total; q += BLOCK) sink.box[q] = T(0);
    __syncthreads();
    const int slot = (threadIdx.x & 31) * (BLOCK / 32) + (threadIdx.x >> 5);
    const int64_t per = ((a.n + gridDim.x - 1) / gridDim.x + BLOCK - 1) / BLOCK * BLOCK;
    const int64_t mine_end = min(a.n, (int64_t)(blockIdx.x + 1) * per);
    deposit_range<T, NDIM, P, WHITNEY, BLOCK, true>(a, (int64_t)blockIdx.x * per + slot, mine_end, sink);
    __syncthreads();
    for (int q = threadIdx.x; q < total; q += BLOCK) {
        const T v = sink.box[q];
        if (v != T(0)) atomicAdd(a.edges_out + q, v);
    }
}

// The field of an edge field at the markers (gather_edges_{1,2,3}d for WHITNEY,
// gather_edges_spline_{1,2,3}d for the spline edges), divided by the cell size.
template <typename T, int NDIM, int P, bool WHITNEY>
__global__ void __launch_bounds__(256) gather_edges_kernel(const PathArgs<T> a) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        T rel[NDIM];
#pragma unroll
        for (int d = 0; d < NDIM; ++d) {
            rel[d] = cells_from(a.pos[d * a.pos_stride + i] - a.g.lower[d], a.g.cell[d], a.g.inv[d], a.g.pow2[d]);
            if (!WHITNEY && a.g.code[d] != PERIODIC) {
                const T top = T(a.g.num[d] - 1);
                if (rel[d] < T(0)) rel[d] = T(0);
                if (rel[d] > top) rel[d] = top;
            }
        }
#pragma unroll
        for (int axis = 0; axis < NDIM; ++axis) {
            constexpr int S = WHITNEY ? 2 : P + 1;
            int idx[3][S];
            T wt[3][S];
            bool ex[S];
            int cnt[3] = {1, 1, 1};
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                idx[d][0] = 0;
                wt[d][0] = T(1);
            }
#pragma unroll
            for (int s = 0; s < S; ++s) ex[s] = true;
#pragma unroll
            for (int d = 0; d < NDIM; ++d) {
                if constexpr (WHITNEY) {
                    int lo, hi;
                    T f;
                    linear_nodes<T>(rel[d], a.g.num[d], a.g.code[d], lo, hi, f);
                    if (d == axis) {
                        idx[d][0] = lo;
                        wt[d][0] = T(1);
                        cnt[d] = 1;
                    } else {
                        idx[d][0] = lo;
                        idx[d][1] = hi;
                        wt[d][0] = T(1) - f;
                        wt[d][1] = f;
                        cnt[d] = 2;
                    }
                } else {
                    if (d == axis) {
                        along_stencil<T, P>(rel[d], a.g.num[d], a.g.code[d], idx[d], wt[d], ex);
                        cnt[d] = P;
                    } else {
                        const int base = axis_stencil<T, SPLINE, P>(rel[d], a.g.num[d], a.g.code[d], wt[d]);
#pragma unroll
                        for (int s = 0; s <= P; ++s) idx[d][s] = map_node(base + s, a.g.num[d], a.g.code[d]);
                        cnt[d] = P + 1;
                    }
                }
            }
            T total = T(0);
            for (int x = 0; x < cnt[0]; ++x) {
                if (axis == 0 && !ex[x]) continue;
                for (int y = 0; y < cnt[1]; ++y) {
                    if (axis == 1 && !ex[y]) continue;
                    for (int z = 0; z < cnt[2]; ++z) {
                        if (axis == 2 && !ex[z]) continue;
                        T w = wt[0][x];
                        if (NDIM > 1) w = w * wt[1][y];
                        if (NDIM > 2) w = w * wt[2][z];
                        int64_t k = idx[0][x];
                        if (NDIM > 1) k = k * a.g.ext[1] + idx[1][y];
                        if (NDIM > 2) k = k * a.g.ext[2] + idx[2][z];
                        total += w * __ldg(a.edges_in + k * NDIM + axis);
                    }
                }
            }
            a.result[axis * a.res_stride + i] = total / a.g.cell[axis];
        }
    }
}

}  // namespace mpf

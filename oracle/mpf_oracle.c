/*
 * mpf_oracle.c -- TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
 *
 * A serial, plain-C restatement of mpifield's particle-grid kernels, used only as the
 * checker by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg.
 * Nothing in mpifield_b200/ links or calls it.
 *
 * What it restates (paths inside the mpifield project):
 *   - the per-axis stencils of src/mpifield/kernels/linear_cell.cuh:12-31,
 *     quadratic_cell.cuh:15-37 and spline_cell.cuh:21-105 (with the clamped
 *     Cox-de Boor cell, spline_cell.cuh:21-59);
 *   - the node gathers and scatters gather_/scatter_{linear,quadratic,spline}_{1,2,3}d
 *     (e.g. gather_spline_3d_cuda.cu:11-53, scatter_spline_3d_cuda.cu:12-61; the dead
 *     marker rule of scatter_quadratic_3d_cuda.cu:32-38);
 *   - the Whitney path deposit deposit_paths_{1,2,3}d_cuda.cu with the helpers of
 *     whitney_cell.cuh:12-53;
 *   - the spline-edge path deposit deposit_paths_spline_{1,2,3}d_cuda.cu with the
 *     edge stencil, cut list and Gauss rules of spline_edges.cuh:16-135;
 *   - the edge gathers gather_edges_{1,2,3}d and gather_edges_spline_{1,2,3}d.
 * The position derivative of a gather (og_gather_grad) has no reference kernel; it
 * follows the B-spline derivative identity B_p' = B_{p-1}(.+1/2) - B_{p-1}(.-1/2)
 * of src/mpifield/splines.py:9,77 and, on clamped axes, B' = D_i - D_{i+1}
 * (spline_cell.cuh:21-28).
 *
 * The arithmetic is the reference's, operation by operation; the file is built with
 * -ffp-contract=off so no multiply-add is fused, like the NumPy kernels. Index
 * arithmetic is followed by clamps that change nothing for finite positions within
 * about 1e9 cells of the grid, so that no input can index outside an array here.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OG_LINEAR 0
#define OG_QUADRATIC 1
#define OG_SPLINE 2

/* (int)x with the saturation of a CUDA conversion, 0 for NaN. */
static int og_to_int(double x) {
    if (x != x) return 0;
    if (x >= 2147483647.0) return 2147483647;
    if (x <= -2147483648.0) return (-2147483647 - 1);
    return (int)x;
}

static int og_clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

static int og_wrap(long long k, int num) {
    long long m = k % num;
    if (m < 0) m += num;
    return (int)m;
}

/* One axis of a stencil: `count` nodes and their weights. */
typedef struct {
    int count;
    int node[4];
    double w[4];
} og_axis;

/* linear_cell.cuh:12-31: the cell of rel and the fraction in it. */
static void og_linear_cell(double rel, int num, int periodic, og_axis* s) {
    int left, right;
    if (periodic) {
        const double n = (double)num;
        rel = rel - n * floor(rel / n);
        left = og_to_int(rel) % num;
        if (left < 0) left += num;
        right = (left + 1) % num;
    } else {
        left = rel >= 0.0 ? og_to_int(rel) : -1;
        left = og_clampi(left, 0, num - 2);
        right = left + 1;
    }
    double f = rel - (double)left;
    if (f < 0.0) f = 0.0;
    if (f > 1.0) f = 1.0;
    s->count = 2;
    s->node[0] = left;
    s->node[1] = right;
    s->w[0] = 1.0 - f;
    s->w[1] = f;
}

/* quadratic_cell.cuh:15-37: the nearest node and its two neighbours. */
static void og_quadratic_cell(double rel, int num, int periodic, og_axis* s) {
    int c;
    if (periodic) {
        const double n = (double)num;
        rel = rel - n * floor(rel / n);
        c = og_clampi(og_to_int(rel + 0.5), 0, num);
        s->node[0] = (c + num - 1) % num;
        s->node[1] = c % num;
        s->node[2] = (c + 1) % num;
    } else {
        if (rel < 0.0) rel = 0.0;
        if (rel > (double)(num - 1)) rel = (double)(num - 1);
        c = og_clampi(og_to_int(rel + 0.5), 0, num - 1);
        s->node[0] = c > 0 ? c - 1 : 0;
        s->node[1] = c;
        s->node[2] = c < num - 1 ? c + 1 : num - 1;
    }
    const double d = rel - (double)c;
    s->count = 3;
    s->w[0] = 0.5 * (0.5 - d) * (0.5 - d);
    s->w[1] = 0.75 - d * d;
    s->w[2] = 0.5 * (0.5 + d) * (0.5 + d);
}

/* spline_cell.cuh:21-59: Cox-de Boor on clamped knots t_k = clip(k - p, 0, num - 1).
 * staggered 0: the p+1 B-splines of degree p of the cell; 1: the p rescaled
 * D_i = p / (t_(i+p) - t_i) B_(i,p-1), indexed i - 1. */
static void og_clamped_cell(double rel, int num, int degree, int staggered, og_axis* s) {
    double left[4], right[4];
    double r = rel;
    if (r < 0.0) r = 0.0;
    if (r > (double)(num - 1)) r = (double)(num - 1);
    int cell = og_to_int(r);
    if (cell > num - 2) cell = num - 2;
    if (cell < 0) cell = 0;
    const int span = cell + degree;
    const int order = degree - staggered;
    double* w = s->w;
    w[0] = 1.0;
    for (int k = 1; k <= order; ++k) {
        const int low = og_clampi(span + 1 - k - degree, 0, num - 1);
        const int high = og_clampi(span + k - degree, 0, num - 1);
        left[k] = r - (double)low;
        right[k] = (double)high - r;
        double saved = 0.0;
        for (int m = 0; m < k; ++m) {
            const double temp = w[m] / (right[m + 1] + left[k - m]);
            w[m] = saved + right[m + 1] * temp;
            saved = left[k - m] * temp;
        }
        w[k] = saved;
    }
    s->count = order + 1;
    for (int m = 0; m <= order; ++m) {
        s->node[m] = cell + m;
        if (staggered) {
            const int i = cell + 1 + m;
            const int low = og_clampi(i - degree, 0, num - 1);
            const int high = og_clampi(i, 0, num - 1);
            w[m] = w[m] * (double)degree / (double)(high - low);
        }
    }
}

/* The uniform B-spline weights of degree p at the offset d from the middle node
 * (spline_cell.cuh:77-94, spline_cell.py:21-41). */
static void og_uniform_weights(int degree, double d, double* w) {
    if (degree == 0) {
        w[0] = 1.0;
    } else if (degree == 1) {
        w[0] = 1.0 - d;
        w[1] = d;
    } else if (degree == 2) {
        w[0] = 0.5 * (0.5 - d) * (0.5 - d);
        w[1] = 0.75 - d * d;
        w[2] = 0.5 * (0.5 + d) * (0.5 + d);
    } else {
        const double complement = 1.0 - d;
        const double square = d * d;
        const double cube = square * d;
        w[0] = complement * complement * complement / 6.0;
        w[1] = (3.0 * cube - 6.0 * square + 4.0) / 6.0;
        w[2] = (-3.0 * cube + 3.0 * square + 3.0 * d + 1.0) / 6.0;
        w[3] = cube / 6.0;
    }
}

/* spline_cell.cuh:61-105: degree 0-3 stencil on a bounded (0), periodic (1) or
 * clamped (2) axis. */
static void og_spline_cell(double rel, int num, int code, int degree, og_axis* s) {
    if (code == 2) {
        og_clamped_cell(rel, num, degree, 0, s);
        return;
    }
    if (code == 1) {
        const double n = (double)num;
        if (!(rel >= 0.0 && rel < n)) rel = rel - n * floor(rel / n);
    } else {
        if (rel < 0.0) rel = 0.0;
        if (rel > (double)(num - 1)) rel = (double)(num - 1);
    }
    int middle = degree % 2 == 0 ? og_to_int(rel + 0.5) : og_to_int(rel);
    middle = og_clampi(middle, 0, num);
    og_uniform_weights(degree, rel - (double)middle, s->w);
    const int first = middle - degree / 2;
    s->count = degree + 1;
    for (int a = 0; a <= degree; ++a) {
        const int k = first + a;
        s->node[a] = code == 1 ? og_wrap(k, num) : og_clampi(k, 0, num - 1);
    }
}

static void og_axis_stencil(int kind, int degree, double rel, int num, int code, og_axis* s) {
    if (kind == OG_LINEAR) og_linear_cell(rel, num, code == 1, s);
    else if (kind == OG_QUADRATIC) og_quadratic_cell(rel, num, code == 1, s);
    else og_spline_cell(rel, num, code, degree, s);
}

/* The extent of the array along an axis: num, or num + p - 1 on a clamped axis
 * (src/mpifield/_types.py:36-40). */
static int og_extent(int num, int code, int degree) { return code == 2 ? num + degree - 1 : num; }

/* ---------------------------------------------------------------- node gathers --- */

/* result(c, i) = sum_k W_k(x_i) field(k, c): the gathers of weighting.py:233-250
 * (gather_spline_3d_cuda.cu:11-53 and its 1D/2D/linear/quadratic twins). The sum runs
 * over the x nodes outermost, as the reference's loops. */
void og_gather(int kind, int degree, int ndim, const double* pos, int64_t pos_stride,
               int64_t n, const double* field, int64_t ncomp, double* result,
               int64_t res_stride, const double* lower, const double* cell,
               const int32_t* num, const int32_t* code) {
    int ext[3] = {1, 1, 1};
    for (int d = 0; d < ndim; ++d) ext[d] = og_extent(num[d], code[d], degree);
    for (int64_t i = 0; i < n; ++i) {
        og_axis s[3];
        for (int d = 0; d < 3; ++d) {
            if (d < ndim) {
                og_axis_stencil(kind, degree, (pos[d * pos_stride + i] - lower[d]) / cell[d],
                                num[d], code[d], &s[d]);
            } else {
                s[d].count = 1;
                s[d].node[0] = 0;
                s[d].w[0] = 1.0;
            }
        }
        for (int64_t c = 0; c < ncomp; ++c) {
            double total = 0.0;
            for (int a = 0; a < s[0].count; ++a)
                for (int b = 0; b < s[1].count; ++b)
                    for (int e = 0; e < s[2].count; ++e) {
                        const int64_t node =
                            ((int64_t)s[0].node[a] * ext[1] + s[1].node[b]) * ext[2] + s[2].node[e];
                        double w = s[0].w[a];
                        if (ndim > 1) w = w * s[1].w[b];
                        if (ndim > 2) w = w * s[2].w[e];
                        total += w * field[node * ncomp + c];
                    }
            result[c * res_stride + i] = total;
        }
    }
}

/* field(k, c) += sum_i W_k(x_i) values(c, i): the scatters of weighting.py:195-213. A
 * marker whose values are all zero is skipped before its position is read
 * (scatter_quadratic_3d_cuda.cu:32-38). */
void og_scatter(int kind, int degree, int ndim, const double* pos, int64_t pos_stride,
                const double* values, int64_t val_stride, int64_t n, double* field,
                int64_t ncomp, const double* lower, const double* cell, const int32_t* num,
                const int32_t* code) {
    int ext[3] = {1, 1, 1};
    for (int d = 0; d < ndim; ++d) ext[d] = og_extent(num[d], code[d], degree);
    for (int64_t i = 0; i < n; ++i) {
        int live = 0;
        for (int64_t c = 0; c < ncomp; ++c)
            if (values[c * val_stride + i] != 0.0) live = 1;
        if (!live) continue;
        og_axis s[3];
        for (int d = 0; d < 3; ++d) {
            if (d < ndim) {
                og_axis_stencil(kind, degree, (pos[d * pos_stride + i] - lower[d]) / cell[d],
                                num[d], code[d], &s[d]);
            } else {
                s[d].count = 1;
                s[d].node[0] = 0;
                s[d].w[0] = 1.0;
            }
        }
        for (int64_t c = 0; c < ncomp; ++c) {
            const double v = values[c * val_stride + i];
            for (int a = 0; a < s[0].count; ++a)
                for (int b = 0; b < s[1].count; ++b)
                    for (int e = 0; e < s[2].count; ++e) {
                        const int64_t node =
                            ((int64_t)s[0].node[a] * ext[1] + s[1].node[b]) * ext[2] + s[2].node[e];
                        double w = s[0].w[a];
                        if (ndim > 1) w = w * s[1].w[b];
                        if (ndim > 2) w = w * s[2].w[e];
                        field[node * ncomp + c] += w * v;
                    }
        }
    }
}

/* ------------------------------------------------------- position derivatives --- */

/* The derivative of the axis weights with respect to rel (in cells), zero where the
 * reference clamps the position (bounded and clamped axes beyond the grid). */
static void og_axis_derivative(int kind, int degree, double rel, int num, int code,
                               og_axis* s, double* dw) {
    og_axis_stencil(kind, degree, rel, num, code, s);
    for (int a = 0; a < 4; ++a) dw[a] = 0.0;
    if (code == 2) {
        if (rel < 0.0 || rel > (double)(num - 1)) return;
        og_axis st;
        og_clamped_cell(rel, num, degree, 1, &st);
        for (int m = 0; m <= degree; ++m) {
            double v = 0.0;
            if (m >= 1) v += st.w[m - 1];
            if (m <= degree - 1) v -= st.w[m];
            dw[m] = v;
        }
        return;
    }
    if (code == 0 && (rel < 0.0 || rel > (double)(num - 1))) return;
    if (kind == OG_LINEAR) {
        /* inside the grid the fraction is rel - left, unclamped */
        dw[0] = -1.0;
        dw[1] = 1.0;
        return;
    }
    double r = rel;
    if (code == 1) {
        const double nn = (double)num;
        if (kind == OG_QUADRATIC || !(r >= 0.0 && r < nn)) r = r - nn * floor(r / nn);
    }
    const int p = kind == OG_QUADRATIC ? 2 : degree;
    int middle = p % 2 == 0 ? og_to_int(r + 0.5) : og_to_int(r);
    const double d = r - (double)middle;
    if (p == 1) {
        dw[0] = -1.0;
        dw[1] = 1.0;
    } else if (p == 2) {
        dw[0] = -(0.5 - d);
        dw[1] = -2.0 * d;
        dw[2] = 0.5 + d;
    } else if (p == 3) {
        const double complement = 1.0 - d;
        dw[0] = -0.5 * complement * complement;
        dw[1] = 1.5 * d * d - 2.0 * d;
        dw[2] = -1.5 * d * d + d + 0.5;
        dw[3] = 0.5 * d * d;
    }
}

/* grad(d, i) = sum_c cotangent(c, i) * d/dx_d sum_k W_k(x_i) field(k, c): the position
 * gradient of a gather contracted with a cotangent (for reverse mode). */
void og_gather_grad(int kind, int degree, int ndim, const double* pos, int64_t pos_stride,
                    int64_t n, const double* field, int64_t ncomp, const double* cot,
                    int64_t cot_stride, double* grad, int64_t grad_stride, const double* lower,
                    const double* cell, const int32_t* num, const int32_t* code) {
    int ext[3] = {1, 1, 1};
    for (int d = 0; d < ndim; ++d) ext[d] = og_extent(num[d], code[d], degree);
    for (int64_t i = 0; i < n; ++i) {
        og_axis s[3];
        double dw[3][4];
        for (int d = 0; d < 3; ++d) {
            if (d < ndim) {
                og_axis_derivative(kind, degree, (pos[d * pos_stride + i] - lower[d]) / cell[d],
                                   num[d], code[d], &s[d], dw[d]);
            } else {
                s[d].count = 1;
                s[d].node[0] = 0;
                s[d].w[0] = 1.0;
                dw[d][0] = 0.0;
            }
        }
        for (int d = 0; d < ndim; ++d) {
            double total = 0.0;
            for (int64_t c = 0; c < ncomp; ++c) {
                double sum = 0.0;
                for (int a = 0; a < s[0].count; ++a)
                    for (int b = 0; b < s[1].count; ++b)
                        for (int e = 0; e < s[2].count; ++e) {
                            const int64_t node = ((int64_t)s[0].node[a] * ext[1] + s[1].node[b]) *
                                                     ext[2] + s[2].node[e];
                            const double wx = d == 0 ? dw[0][a] : s[0].w[a];
                            const double wy = d == 1 ? dw[1][b] : s[1].w[b];
                            const double wz = d == 2 ? dw[2][e] : s[2].w[e];
                            double w = wx;
                            if (ndim > 1) w = w * wy;
                            if (ndim > 2) w = w * wz;
                            sum += w * field[node * ncomp + c];
                        }
                total += cot[c * cot_stride + i] * sum;
            }
            grad[d * grad_stride + i] = total / cell[d];
        }
    }
}

/* ------------------------------------------------------- Whitney path deposit --- */

/* whitney_cell.cuh:34-39 */
static double og_clamp_to_axis(double rel, int num, int periodic) {
    if (periodic) return rel;
    if (rel < 0.0) return 0.0;
    if (rel > num - 1.0) return num - 1.0;
    return rel;
}

/* whitney_cell.cuh:41-53 */
static double og_plane_time(double plane, double rel, double delta) {
    return delta != 0.0 ? (plane - rel) / delta : 2.0;
}

/* The current of straight paths on the edges (deposit_paths_{1,2,3}d_cuda.cu): each
 * path is cut where it crosses a grid plane; a piece adds q times its length along an
 * axis to the cell's edges along that axis, times their weights averaged over the
 * piece (whitney_cell.cuh:19-26 in 3D, the midpoint's in 2D). Edges are num + (ndim,). */
void og_deposit_whitney(int ndim, const double* start, int64_t start_stride,
                        const double* end, int64_t end_stride, const double* charges,
                        int64_t n, double* edges, const double* lower, const double* cell,
                        const int32_t* num, const int32_t* code) {
    int ext[3] = {1, 1, 1};
    for (int d = 0; d < ndim; ++d) ext[d] = num[d];
    for (int64_t i = 0; i < n; ++i) {
        const double q = charges[i];
        if (q == 0.0) continue;
        double a[3], b[3], dl[3], plane[3], step[3], p0[3], p1[3];
        int finite = 1;
        for (int d = 0; d < ndim; ++d) {
            a[d] = (start[d * start_stride + i] - lower[d]) / cell[d];
            b[d] = (end[d * end_stride + i] - lower[d]) / cell[d];
            if (!(a[d] > -1.0e300 && a[d] < 1.0e300 && b[d] > -1.0e300 && b[d] < 1.0e300))
                finite = 0;
        }
        if (!finite) continue;
        for (int d = 0; d < ndim; ++d) {
            dl[d] = b[d] - a[d];
            if (dl[d] < 0.0) {
                plane[d] = ceil(a[d]) - 1.0;
                step[d] = -1.0;
            } else {
                plane[d] = floor(a[d]) + 1.0;
                step[d] = 1.0;
            }
            p0[d] = og_clamp_to_axis(a[d], num[d], code[d] == 1);
        }
        double time = 0.0;
        int guard = 0;
        while (time < 1.0 && guard++ < 100000000) {
            double times[3];
            double following = 1.0;
            for (int d = 0; d < ndim; ++d) {
                times[d] = og_plane_time(plane[d], a[d], dl[d]);
                if (times[d] < following) following = times[d];
            }
            for (int d = 0; d < ndim; ++d) {
                p1[d] = og_clamp_to_axis(following < 1.0 ? a[d] + following * dl[d] : b[d],
                                         num[d], code[d] == 1);
                if (times[d] <= following) plane[d] += step[d];
            }
            int lo[3], hi[3];
            double f[3], delta[3];
            for (int d = 0; d < ndim; ++d) {
                og_axis s;
                og_linear_cell(0.5 * (p0[d] + p1[d]), num[d], code[d] == 1, &s);
                lo[d] = s.node[0];
                hi[d] = s.node[1];
                f[d] = s.w[1];
                delta[d] = p1[d] - p0[d];
            }
            if (ndim == 1) {
                edges[lo[0]] += q * delta[0];
            } else if (ndim == 2) {
                const double along_x = q * delta[0];
                const double along_y = q * delta[1];
                edges[((int64_t)lo[0] * ext[1] + lo[1]) * 2 + 0] += (1.0 - f[1]) * along_x;
                edges[((int64_t)lo[0] * ext[1] + hi[1]) * 2 + 0] += f[1] * along_x;
                edges[((int64_t)lo[0] * ext[1] + lo[1]) * 2 + 1] += (1.0 - f[0]) * along_y;
                edges[((int64_t)hi[0] * ext[1] + lo[1]) * 2 + 1] += f[0] * along_y;
            } else {
                for (int u = 0; u < 2; ++u)
                    for (int w = 0; w < 2; ++w) {
                        for (int axis = 0; axis < 3; ++axis) {
                            /* the two axes across this one, in increasing order */
                            const int ua = axis == 0 ? 1 : 0;
                            const int wa = axis == 2 ? 1 : 2;
                            const double eu = u ? f[ua] : 1.0 - f[ua];
                            const double ew = w ? f[wa] : 1.0 - f[wa];
                            const double cross = delta[ua] * delta[wa] / 12.0;
                            const double weight = eu * ew + (u == w ? cross : -cross);
                            int idx[3] = {lo[0], lo[1], lo[2]};
                            idx[ua] = u ? hi[ua] : lo[ua];
                            idx[wa] = w ? hi[wa] : lo[wa];
                            const int64_t node = ((int64_t)idx[0] * ext[1] + idx[1]) * ext[2] + idx[2];
                            edges[node * 3 + axis] += q * delta[axis] * weight;
                        }
                    }
            }
            time = following;
            for (int d = 0; d < ndim; ++d) p0[d] = p1[d];
        }
    }
}

/* ------------------------------------------------------ spline-edge deposit --- */

#define OG_MAX_CUTS 32

static int og_floor_int(double x) {
    int whole = og_to_int(x);
    if (x < (double)whole) whole -= 1;
    return whole;
}

/* spline_edges.cuh:22-65: the `degree` edges along an axis around rel, their weights
 * B_{p-1}(rel - k - 1/2) and whether each exists (bounded: edges 0 .. num - 2). */
static void og_along_stencil(double rel, int num, int code, int degree, int* edge,
                             double* weight, int* exists) {
    if (code == 2) {
        og_axis s;
        og_clamped_cell(rel, num, degree, 1, &s);
        for (int a = 0; a < degree; ++a) {
            edge[a] = s.node[a];
            weight[a] = s.w[a];
            exists[a] = 1;
        }
        return;
    }
    const int lower = degree - 1;
    if (code == 1 && !(rel >= 0.0 && rel < (double)num))
        rel = rel - (double)num * floor(rel / (double)num);
    const double shifted = rel - 0.5;
    int middle;
    if (lower % 2 == 0) {
        middle = og_floor_int(shifted + 0.5);
        if (code == 0 && middle > num - 2) middle = num - 2;
    } else {
        middle = og_floor_int(shifted);
    }
    og_uniform_weights(lower, shifted - (double)middle, weight);
    const int first = middle - lower / 2;
    for (int a = 0; a < degree; ++a) {
        const int k = first + a;
        if (code == 1) {
            edge[a] = og_wrap(k, num);
            exists[a] = 1;
        } else if (k < 0 || k > num - 2) {
            edge[a] = 0;
            exists[a] = 0;
        } else {
            edge[a] = k;
            exists[a] = 1;
        }
    }
}

/* spline_edges.cuh:67-89: Gauss-Legendre points and weights on [0, 1]. The values are
 * those of numpy.polynomial.legendre.leggauss mapped to [0, 1]. */
static void og_gauss_rule(int count, double* point, double* weight) {
    static const double p1[1] = {0.5}, w1[1] = {1.0};
    static const double p2[2] = {0.21132486540518713, 0.7886751345948129};
    static const double w2[2] = {0.5, 0.5};
    static const double p3[3] = {0.1127016653792583, 0.5, 0.8872983346207417};
    static const double w3[3] = {0.2777777777777778, 0.4444444444444444, 0.2777777777777778};
    static const double p4[4] = {0.06943184420297371, 0.33000947820757187, 0.6699905217924281,
                                 0.9305681557970262};
    static const double w4[4] = {0.17392742256872692, 0.3260725774312731, 0.3260725774312731,
                                 0.17392742256872692};
    static const double p5[5] = {0.04691007703066802, 0.23076534494715845, 0.5,
                                 0.7692346550528415, 0.9530899229693319};
    static const double w5[5] = {0.11846344252809454, 0.2393143352496832, 0.28444444444444444,
                                 0.2393143352496832, 0.11846344252809454};
    const double* ps[5] = {p1, p2, p3, p4, p5};
    const double* ws[5] = {w1, w2, w3, w4, w5};
    const int k = count < 1 ? 0 : (count > 5 ? 4 : count - 1);
    for (int g = 0; g <= k; ++g) {
        point[g] = ps[k][g];
        weight[g] = ws[k][g];
    }
}

/* spline_edges.cuh:91-127: the sorted path parameters where a stretch crosses a knot
 * plane (half-integers for even degree; the nodes on clamped axes) or a wall. */
static int og_path_cuts(const double* r0, const double* r1, int ndim, double shift,
                        const int32_t* num, const int32_t* code, double* cuts) {
    int count = 1;
    cuts[0] = 0.0;
    for (int d = 0; d < ndim; ++d) {
        const double delta = r1[d] - r0[d];
        if (delta == 0.0) continue;
        const double low = delta > 0.0 ? r0[d] : r1[d];
        const double high = delta > 0.0 ? r1[d] : r0[d];
        const double offset = code[d] == 2 ? 0.0 : shift;
        double plane = (double)og_floor_int(low - offset) + 1.0 + offset;
        while (plane < high && count < OG_MAX_CUTS - 3) {
            const double t = (plane - r0[d]) / delta;
            if (t > 0.0 && t < 1.0) cuts[count++] = t;
            plane += 1.0;
        }
        if (code[d] != 1) {
            double t = (0.0 - r0[d]) / delta;
            if (t > 0.0 && t < 1.0 && count < OG_MAX_CUTS - 1) cuts[count++] = t;
            t = ((double)num[d] - 1.0 - r0[d]) / delta;
            if (t > 0.0 && t < 1.0 && count < OG_MAX_CUTS - 1) cuts[count++] = t;
        }
    }
    cuts[count++] = 1.0;
    for (int i = 2; i < count - 1; ++i) {
        const double value = cuts[i];
        int j = i - 1;
        while (j > 0 && cuts[j] > value) {
            cuts[j + 1] = cuts[j];
            --j;
        }
        cuts[j + 1] = value;
    }
    return count;
}

/* The spline-edge current of degree 1-3 (deposit_paths_spline_{1,2,3}d_cuda.cu): the
 * path is split into stretches of at most 4 cells, each cut at knot planes and walls;
 * each clamped piece is integrated with (p - 1 + (ndim - 1) p) / 2 + 1 Gauss points.
 * Edges are ext + (ndim,), ext = num (+ p - 1 on clamped axes). */
void og_deposit_spline(int ndim, int degree, const double* start, int64_t start_stride,
                       const double* end, int64_t end_stride, const double* charges, int64_t n,
                       double* edges, const double* lower, const double* cell,
                       const int32_t* num, const int32_t* code) {
    int ext[3] = {1, 1, 1};
    for (int d = 0; d < ndim; ++d) ext[d] = og_extent(num[d], code[d], degree);
    const double shift = degree % 2 == 0 ? 0.5 : 0.0;
    const int num_points = (degree - 1 + (ndim - 1) * degree) / 2 + 1;
    double point[5], gw[5];
    og_gauss_rule(num_points, point, gw);
    for (int64_t i = 0; i < n; ++i) {
        const double q = charges[i];
        if (q == 0.0) continue;
        double r0[3], r1[3], a0[3], a1[3], p0[3], step[3], cuts[OG_MAX_CUTS];
        double extent = 0.0;
        int finite = 1;
        for (int d = 0; d < ndim; ++d) {
            const double s = start[d * start_stride + i], e = end[d * end_stride + i];
            if (!(s - s == 0.0) || !(e - e == 0.0)) finite = 0;
            r0[d] = (s - lower[d]) / cell[d];
            r1[d] = (e - lower[d]) / cell[d];
            const double span = r1[d] > r0[d] ? r1[d] - r0[d] : r0[d] - r1[d];
            if (span > extent) extent = span;
        }
        if (!finite) continue;
        const int stretches = og_to_int(extent / 4.0) + 1;
        for (int st = 0; st < stretches; ++st) {
            for (int d = 0; d < ndim; ++d) {
                a0[d] = r0[d] + (r1[d] - r0[d]) * st / stretches;
                a1[d] = r0[d] + (r1[d] - r0[d]) * (st + 1) / stretches;
            }
            const int nc = og_path_cuts(a0, a1, ndim, shift, num, code, cuts);
            for (int piece = 0; piece < nc - 1; ++piece) {
                const double t0 = cuts[piece], t1 = cuts[piece + 1];
                if (t1 <= t0) continue;
                for (int d = 0; d < ndim; ++d) {
                    double begin = a0[d] + t0 * (a1[d] - a0[d]);
                    double finish = a0[d] + t1 * (a1[d] - a0[d]);
                    if (code[d] != 1) {
                        const double top = (double)(num[d] - 1);
                        if (begin < 0.0) begin = 0.0;
                        if (begin > top) begin = top;
                        if (finish < 0.0) finish = 0.0;
                        if (finish > top) finish = top;
                    }
                    p0[d] = begin;
                    step[d] = finish - begin;
                }
                for (int g = 0; g < num_points; ++g) {
                    double rel[3];
                    for (int d = 0; d < ndim; ++d) rel[d] = p0[d] + point[g] * step[d];
                    for (int axis = 0; axis < ndim; ++axis) {
                        const double amount = q * gw[g] * step[axis];
                        if (amount == 0.0) continue;
                        int idx_n[3][4], ex[3][4];
                        double wt[3][4];
                        int cnt[3] = {1, 1, 1};
                        for (int d = 0; d < 3; ++d) {
                            idx_n[d][0] = 0;
                            wt[d][0] = 1.0;
                            ex[d][0] = 1;
                        }
                        for (int d = 0; d < ndim; ++d) {
                            if (d == axis) {
                                og_along_stencil(rel[d], num[d], code[d], degree, idx_n[d], wt[d], ex[d]);
                                cnt[d] = degree;
                            } else {
                                og_axis s;
                                og_spline_cell(rel[d], num[d], code[d], degree, &s);
                                for (int a = 0; a <= degree; ++a) {
                                    idx_n[d][a] = s.node[a];
                                    wt[d][a] = s.w[a];
                                    ex[d][a] = 1;
                                }
                                cnt[d] = degree + 1;
                            }
                        }
                        for (int a = 0; a < cnt[0]; ++a)
                            for (int b = 0; b < cnt[1]; ++b)
                                for (int e = 0; e < cnt[2]; ++e) {
                                    if (!(ex[0][a] && ex[1][b] && ex[2][e])) continue;
                                    double w = amount * wt[0][a];
                                    if (ndim > 1) w = w * wt[1][b];
                                    if (ndim > 2) w = w * wt[2][e];
                                    const int64_t node =
                                        ((int64_t)idx_n[0][a] * ext[1] + idx_n[1][b]) * ext[2] +
                                        idx_n[2][e];
                                    edges[node * ndim + axis] += w;
                                }
                    }
                }
            }
        }
    }
}

/* ------------------------------------------------------------- edge gathers --- */

/* The field of an edge field at the markers, E_a = sum W e / h_a, for the Whitney
 * functions (whitney_cell.py:54-71) when degree 0 is passed, else the spline edge
 * functions of that degree (spline_edges.py:110-130, clamped positions). */
void og_gather_edges(int ndim, int degree, const double* pos, int64_t pos_stride, int64_t n,
                     const double* edges, double* result, int64_t res_stride,
                     const double* lower, const double* cell, const int32_t* num,
                     const int32_t* code) {
    const int p = degree == 0 ? 1 : degree;
    int ext[3] = {1, 1, 1};
    for (int d = 0; d < ndim; ++d) ext[d] = og_extent(num[d], code[d], p);
    for (int64_t i = 0; i < n; ++i) {
        double rel[3];
        for (int d = 0; d < ndim; ++d) {
            rel[d] = (pos[d * pos_stride + i] - lower[d]) / cell[d];
            if (degree != 0 && code[d] != 1) {
                const double top = (double)(num[d] - 1);
                if (rel[d] < 0.0) rel[d] = 0.0;
                if (rel[d] > top) rel[d] = top;
            }
        }
        for (int axis = 0; axis < ndim; ++axis) {
            int idx_n[3][4], ex[3][4], cnt[3] = {1, 1, 1};
            double wt[3][4];
            for (int d = 0; d < 3; ++d) {
                idx_n[d][0] = 0;
                wt[d][0] = 1.0;
                ex[d][0] = 1;
            }
            for (int d = 0; d < ndim; ++d) {
                if (degree == 0) {
                    og_axis s;
                    og_linear_cell(rel[d], num[d], code[d] == 1, &s);
                    if (d == axis) {
                        idx_n[d][0] = s.node[0];
                        wt[d][0] = 1.0;
                        ex[d][0] = 1;
                        cnt[d] = 1;
                    } else {
                        for (int a = 0; a < 2; ++a) {
                            idx_n[d][a] = s.node[a];
                            wt[d][a] = s.w[a];
                            ex[d][a] = 1;
                        }
                        cnt[d] = 2;
                    }
                } else if (d == axis) {
                    og_along_stencil(rel[d], num[d], code[d], degree, idx_n[d], wt[d], ex[d]);
                    cnt[d] = degree;
                } else {
                    og_axis s;
                    og_spline_cell(rel[d], num[d], code[d], degree, &s);
                    for (int a = 0; a <= degree; ++a) {
                        idx_n[d][a] = s.node[a];
                        wt[d][a] = s.w[a];
                        ex[d][a] = 1;
                    }
                    cnt[d] = degree + 1;
                }
            }
            double total = 0.0;
            for (int a = 0; a < cnt[0]; ++a)
                for (int b = 0; b < cnt[1]; ++b)
                    for (int e = 0; e < cnt[2]; ++e) {
                        if (!(ex[0][a] && ex[1][b] && ex[2][e])) continue;
                        double w = wt[0][a];
                        if (ndim > 1) w = w * wt[1][b];
                        if (ndim > 2) w = w * wt[2][e];
                        const int64_t node =
                            ((int64_t)idx_n[0][a] * ext[1] + idx_n[1][b]) * ext[2] + idx_n[2][e];
                        total += w * edges[node * ndim + axis];
                    }
            result[axis * res_stride + i] = total / cell[axis];
        }
    }
}

/* ------------------------------------------------------------- k-forms --- */

/* Whether component `component` of a `form`-form in `ndim` dimensions is staggered along
 * `axis` (spline_forms.py:30-40): the top form along every axis, the edges (1-forms) along
 * their direction, the faces of 3D (2-forms) across their normal. */
static int og_staggered(int form, int ndim, int component, int axis) {
    if (form == ndim) return 1;
    if (form == 1) return axis == component;
    if (form == 2 && ndim == 3) return axis != component;
    return 0;
}

/* The stencil of a k-form component at the clamped position rel (spline_forms.py:56-75):
 * the B_(p-1) edges along the staggered axes (with their existence), the B_p nodes along
 * the others; cnt[d] entries per axis. */
static void og_form_stencil(const double* rel, const int32_t* num, const int32_t* code, int ndim, int degree,
                            int form, int component, int idx[3][4], double wt[3][4], int ex[3][4], int cnt[3]) {
    for (int d = 0; d < 3; ++d) {
        idx[d][0] = 0;
        wt[d][0] = 1.0;
        ex[d][0] = 1;
        cnt[d] = 1;
    }
    for (int d = 0; d < ndim; ++d) {
        if (og_staggered(form, ndim, component, d)) {
            og_along_stencil(rel[d], num[d], code[d], degree, idx[d], wt[d], ex[d]);
            cnt[d] = degree;
        } else {
            og_axis s;
            og_spline_cell(rel[d], num[d], code[d], degree, &s);
            for (int a = 0; a <= degree; ++a) {
                idx[d][a] = s.node[a];
                wt[d][a] = s.w[a];
                ex[d][a] = 1;
            }
            cnt[d] = degree + 1;
        }
    }
}

static void og_form_positions(int ndim, const double* pos, int64_t pos_stride, int64_t i, const double* lower,
                              const double* cell, const int32_t* num, const int32_t* code, double* rel) {
    for (int d = 0; d < ndim; ++d) {
        rel[d] = (pos[d * pos_stride + i] - lower[d]) / cell[d];
        if (code[d] != 1) {
            const double top = (double)(num[d] - 1);
            if (rel[d] < 0.0) rel[d] = 0.0;
            if (rel[d] > top) rel[d] = top;
        }
    }
}

/* The gather of a k-form of degree 1..3 (gather_forms_spline, spline_forms.py:85-108):
 * result(c, i) = sum over the stencil of component c of W field(k, c). The field is
 * extent + (ncomp,), the extent num + degree - 1 along a clamped axis. */
void og_gather_forms(int ndim, int degree, int form, const double* pos, int64_t pos_stride, int64_t n,
                     const double* field, int64_t ncomp, double* result, int64_t res_stride, const double* lower,
                     const double* cell, const int32_t* num, const int32_t* code) {
    int ext[3] = {1, 1, 1};
    for (int d = 0; d < ndim; ++d) ext[d] = og_extent(num[d], code[d], degree);
    for (int64_t i = 0; i < n; ++i) {
        double rel[3] = {0.0, 0.0, 0.0};
        og_form_positions(ndim, pos, pos_stride, i, lower, cell, num, code, rel);
        for (int c = 0; c < ncomp; ++c) {
            int idx[3][4], ex[3][4], cnt[3];
            double wt[3][4];
            og_form_stencil(rel, num, code, ndim, degree, form, c, idx, wt, ex, cnt);
            double total = 0.0;
            for (int a = 0; a < cnt[0]; ++a)
                for (int b = 0; b < cnt[1]; ++b)
                    for (int e = 0; e < cnt[2]; ++e) {
                        if (!(ex[0][a] && ex[1][b] && ex[2][e])) continue;
                        double w = wt[0][a];
                        if (ndim > 1) w = w * wt[1][b];
                        if (ndim > 2) w = w * wt[2][e];
                        const int64_t node = ((int64_t)idx[0][a] * ext[1] + idx[1][b]) * ext[2] + idx[2][e];
                        total += w * field[node * ncomp + c];
                    }
            result[c * res_stride + i] = total;
        }
    }
}

/* The scatter of a k-form (scatter_forms_spline, spline_forms.py:111-138): field(k, c) +=
 * W values(c, i); a marker whose values are all zero is skipped before its position is
 * read. */
void og_scatter_forms(int ndim, int degree, int form, const double* pos, int64_t pos_stride, const double* values,
                      int64_t val_stride, int64_t n, double* field, int64_t ncomp, const double* lower,
                      const double* cell, const int32_t* num, const int32_t* code) {
    int ext[3] = {1, 1, 1};
    for (int d = 0; d < ndim; ++d) ext[d] = og_extent(num[d], code[d], degree);
    for (int64_t i = 0; i < n; ++i) {
        int live = 0;
        for (int c = 0; c < ncomp; ++c) live = live || values[c * val_stride + i] != 0.0;
        if (!live) continue;
        double rel[3] = {0.0, 0.0, 0.0};
        og_form_positions(ndim, pos, pos_stride, i, lower, cell, num, code, rel);
        for (int c = 0; c < ncomp; ++c) {
            int idx[3][4], ex[3][4], cnt[3];
            double wt[3][4];
            og_form_stencil(rel, num, code, ndim, degree, form, c, idx, wt, ex, cnt);
            const double v = values[c * val_stride + i];
            for (int a = 0; a < cnt[0]; ++a)
                for (int b = 0; b < cnt[1]; ++b)
                    for (int e = 0; e < cnt[2]; ++e) {
                        if (!(ex[0][a] && ex[1][b] && ex[2][e])) continue;
                        double w = wt[0][a];
                        if (ndim > 1) w = w * wt[1][b];
                        if (ndim > 2) w = w * wt[2][e];
                        const int64_t node = ((int64_t)idx[0][a] * ext[1] + idx[1][b]) * ext[2] + idx[2][e];
                        field[node * ncomp + c] += w * v;
                    }
        }
    }
}

/* ---------------------------------------------------------------- tile keys --- */

/* The cell-tile key of each marker: the anchor node of its stencil along each axis
 * (the left node for LINEAR, the nearest node for QUADRATIC, the spline stencil's
 * middle node; the cell on a clamped axis), divided by the tile size, row-major over
 * the tiles. A marker whose values are all zero gets the key `ntiles` without its
 * position being read. `values` may be NULL (every marker live). This is the key the
 * sort must order stably; it has no counterpart in the reference. */
void og_tile_keys(int kind, int degree, int ndim, const double* pos, int64_t pos_stride,
                  const double* values, int64_t val_stride, int64_t ncomp, int64_t n,
                  const double* lower, const double* cell, const int32_t* num,
                  const int32_t* code, const int32_t* tile, int within, uint32_t* keys) {
    int64_t ntiles[3] = {1, 1, 1};
    int64_t total = 1;
    int64_t cells = 1;
    if (within)
        for (int d = 0; d < ndim; ++d) cells *= tile[d];
    for (int d = 0; d < ndim; ++d) {
        const int e = og_extent(num[d], code[d], degree);
        ntiles[d] = (e + tile[d] - 1) / tile[d];
        total *= ntiles[d];
    }
    for (int64_t i = 0; i < n; ++i) {
        if (values) {
            int live = 0;
            for (int64_t c = 0; c < ncomp; ++c)
                if (values[c * val_stride + i] != 0.0) live = 1;
            if (!live) {
                keys[i] = (uint32_t)(total * cells);
                continue;
            }
        }
        int64_t key = 0, inner = 0;
        for (int d = 0; d < ndim; ++d) {
            og_axis s;
            const double rel = (pos[d * pos_stride + i] - lower[d]) / cell[d];
            og_axis_stencil(kind, degree, rel, num[d], code[d], &s);
            int anchor;
            if (kind == OG_LINEAR) anchor = s.node[0];
            else if (kind == OG_QUADRATIC) anchor = s.node[1];
            else if (code[d] == 2) anchor = s.node[0];
            else anchor = s.node[degree / 2];
            key = key * ntiles[d] + anchor / tile[d];
            inner = inner * tile[d] + anchor % tile[d];
        }
        if (within) key = key * cells + inner;
        keys[i] = (uint32_t)key;
    }
}

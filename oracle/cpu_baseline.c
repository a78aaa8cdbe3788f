/*
 * cpu_baseline.c -- TEST AND BENCHMARK INFRASTRUCTURE, NOT PART OF THE PRODUCT.
 *
 * The reference's CPU kernels, restated in C with OpenMP, for the CPU baseline that
 * bench.py reports beside the GPU numbers. The reference compiles these kernels with
 * Pyccel (src/mpifield/kernels/<name>/<name>_pyccel.py), which is not installed here; this file
 * keeps their structure:
 *   - gathers: contiguous marker chunks per thread when N >= 4096
 *     (gather_quadratic_3d_pyccel.py:19,117-186);
 *   - scatters: per-thread grid copies summed in thread order when N >= 20000,
 *     N >= grid values and threads * grid values <= 16,777,216, else one thread
 *     (scatter_quadratic_3d_pyccel.py:23-25,151-218; scatter_spline_3d_pyccel.py:24-26);
 *   - the Whitney path deposit: per-thread copies of the edges when N >= 20000 and
 *     N >= nodes (deposit_paths_3d_pyccel.py:41,231-262);
 *   - the spline path deposit: serial (deposit_paths_spline_3d_pyccel.py:1-8);
 *   - positions in cells as (x - lower) * (1 / h) (scatter_quadratic_3d_pyccel.py:79-81).
 * It includes the serial oracle for the per-axis stencils and path helpers.
 */
#include "mpf_oracle.c"

#ifdef _OPENMP
#include <omp.h>
#endif

#define CB_MIN_PARALLEL_GATHER 4096
#define CB_MIN_PARALLEL_SCATTER 20000
#define CB_MAX_BUFFER_VALUES 16777216LL

static int cb_threads(int requested) {
#ifdef _OPENMP
    return requested > 0 ? requested : omp_get_max_threads();
#else
    (void)requested;
    return 1;
#endif
}

static int cb_thread_id(void) {
#ifdef _OPENMP
    return omp_get_thread_num();
#else
    return 0;
#endif
}

static void cb_gather_chunk(int kind, int degree, int ndim, const double* pos, int64_t ps,
                            int64_t first, int64_t last, const double* field, int64_t ncomp,
                            double* result, int64_t rs, const double* lower, const double* inv,
                            const int32_t* num, const int32_t* code, const int* ext) {
    for (int64_t i = first; i < last; ++i) {
        og_axis s[3];
        for (int d = 0; d < 3; ++d) {
            if (d < ndim) {
                og_axis_stencil(kind, degree, (pos[d * ps + i] - lower[d]) * inv[d], num[d], code[d], &s[d]);
            } else {
                s[d].count = 1;
                s[d].node[0] = 0;
                s[d].w[0] = 1.0;
            }
        }
        for (int64_t c = 0; c < ncomp; ++c) {
            double total = 0.0;
            for (int a = 0; a < s[0].count; ++a)
                for (int b = 0; b < s[1].count; ++b) {
                    const double wab = ndim > 1 ? s[0].w[a] * s[1].w[b] : s[0].w[a];
                    for (int e = 0; e < s[2].count; ++e) {
                        const int64_t node =
                            ((int64_t)s[0].node[a] * ext[1] + s[1].node[b]) * ext[2] + s[2].node[e];
                        const double w = ndim > 2 ? wab * s[2].w[e] : wab;
                        total += w * field[node * ncomp + c];
                    }
                }
            result[c * rs + i] = total;
        }
    }
}

/* The gather of the Pyccel kernels: OpenMP chunks of markers. */
void cb_gather(int kind, int degree, int ndim, const double* pos, int64_t ps, int64_t n,
               const double* field, int64_t ncomp, double* result, int64_t rs,
               const double* lower, const double* cell, const int32_t* num,
               const int32_t* code, int threads) {
    int ext[3] = {1, 1, 1};
    double inv[3] = {1.0, 1.0, 1.0};
    for (int d = 0; d < ndim; ++d) {
        ext[d] = og_extent(num[d], code[d], degree);
        inv[d] = 1.0 / cell[d];
    }
    const int nt = cb_threads(threads);
    if (nt == 1 || n < CB_MIN_PARALLEL_GATHER) {
        cb_gather_chunk(kind, degree, ndim, pos, ps, 0, n, field, ncomp, result, rs, lower, inv,
                        num, code, ext);
        return;
    }
    const int64_t chunk = (n + nt - 1) / nt;
#pragma omp parallel num_threads(nt)
    {
        const int64_t t = cb_thread_id();
        const int64_t first = t * chunk < n ? t * chunk : n;
        const int64_t last = first + chunk < n ? first + chunk : n;
        cb_gather_chunk(kind, degree, ndim, pos, ps, first, last, field, ncomp, result, rs,
                        lower, inv, num, code, ext);
    }
}

static void cb_scatter_chunk(int kind, int degree, int ndim, const double* pos, int64_t ps,
                             const double* values, int64_t vs, int64_t first, int64_t last,
                             double* buffer, int64_t ncomp, const double* lower,
                             const double* inv, const int32_t* num, const int32_t* code,
                             const int* ext) {
    for (int64_t i = first; i < last; ++i) {
        int live = 0;
        for (int64_t c = 0; c < ncomp; ++c)
            if (values[c * vs + i] != 0.0) live = 1;
        if (!live) continue;
        og_axis s[3];
        for (int d = 0; d < 3; ++d) {
            if (d < ndim) {
                og_axis_stencil(kind, degree, (pos[d * ps + i] - lower[d]) * inv[d], num[d], code[d], &s[d]);
            } else {
                s[d].count = 1;
                s[d].node[0] = 0;
                s[d].w[0] = 1.0;
            }
        }
        for (int a = 0; a < s[0].count; ++a)
            for (int b = 0; b < s[1].count; ++b) {
                const double wab = ndim > 1 ? s[0].w[a] * s[1].w[b] : s[0].w[a];
                for (int e = 0; e < s[2].count; ++e) {
                    const double w = ndim > 2 ? wab * s[2].w[e] : wab;
                    const int64_t node =
                        ((int64_t)s[0].node[a] * ext[1] + s[1].node[b]) * ext[2] + s[2].node[e];
                    for (int64_t c = 0; c < ncomp; ++c) buffer[node * ncomp + c] += w * values[c * vs + i];
                }
            }
    }
}

/* The scatter of the Pyccel kernels: per-thread grid copies when the thresholds allow,
 * else one thread. Returns the number of threads used. */
int cb_scatter(int kind, int degree, int ndim, const double* pos, int64_t ps,
               const double* values, int64_t vs, int64_t n, double* field, int64_t ncomp,
               const double* lower, const double* cell, const int32_t* num, const int32_t* code,
               int threads) {
    int ext[3] = {1, 1, 1};
    double inv[3] = {1.0, 1.0, 1.0};
    int64_t grid_values = ncomp;
    for (int d = 0; d < ndim; ++d) {
        ext[d] = og_extent(num[d], code[d], degree);
        inv[d] = 1.0 / cell[d];
        grid_values *= ext[d];
    }
    const int nt = cb_threads(threads);
    if (nt == 1 || n < CB_MIN_PARALLEL_SCATTER || n < grid_values ||
        (int64_t)nt * grid_values > CB_MAX_BUFFER_VALUES) {
        cb_scatter_chunk(kind, degree, ndim, pos, ps, values, vs, 0, n, field, ncomp, lower, inv,
                         num, code, ext);
        return 1;
    }
    double* buffer = (double*)calloc((size_t)nt * (size_t)grid_values, sizeof(double));
    if (!buffer) {
        cb_scatter_chunk(kind, degree, ndim, pos, ps, values, vs, 0, n, field, ncomp, lower, inv,
                         num, code, ext);
        return 1;
    }
    const int64_t chunk = (n + nt - 1) / nt;
#pragma omp parallel num_threads(nt)
    {
        const int64_t t = cb_thread_id();
        const int64_t first = t * chunk < n ? t * chunk : n;
        const int64_t last = first + chunk < n ? first + chunk : n;
        cb_scatter_chunk(kind, degree, ndim, pos, ps, values, vs, first, last,
                         buffer + t * grid_values, ncomp, lower, inv, num, code, ext);
#pragma omp barrier
#pragma omp for schedule(static)
        for (int64_t k = 0; k < grid_values; ++k) {
            double total = 0.0;
            for (int u = 0; u < nt; ++u) total += buffer[(int64_t)u * grid_values + k];
            field[k] += total;
        }
    }
    free(buffer);
    return nt;
}

/* The Whitney path deposit of the Pyccel kernels: per-thread copies of the edges when
 * there are enough paths. Returns the number of threads used. */
int cb_deposit_whitney(int ndim, const double* start, int64_t ss, const double* end,
                       int64_t es, const double* charges, int64_t n, double* edges,
                       const double* lower, const double* cell, const int32_t* num,
                       const int32_t* code, int threads) {
    int64_t nodes = 1;
    for (int d = 0; d < ndim; ++d) nodes *= num[d];
    int nt = cb_threads(threads);
    if (n < CB_MIN_PARALLEL_SCATTER || n < nodes) nt = 1;
    if (nt == 1) {
        og_deposit_whitney(ndim, start, ss, end, es, charges, n, edges, lower, cell, num, code);
        return 1;
    }
    const int64_t values = nodes * ndim;
    double* buffer = (double*)calloc((size_t)nt * (size_t)values, sizeof(double));
    if (!buffer) {
        og_deposit_whitney(ndim, start, ss, end, es, charges, n, edges, lower, cell, num, code);
        return 1;
    }
    const int64_t chunk = (n + nt - 1) / nt;
#pragma omp parallel num_threads(nt)
    {
        const int64_t t = cb_thread_id();
        const int64_t first = t * chunk < n ? t * chunk : n;
        const int64_t last = first + chunk < n ? first + chunk : n;
        if (last > first)
            og_deposit_whitney(ndim, start + first, ss, end + first, es, charges + first,
                               last - first, buffer + t * values, lower, cell, num, code);
#pragma omp barrier
#pragma omp for schedule(static)
        for (int64_t k = 0; k < values; ++k) {
            double total = 0.0;
            for (int u = 0; u < nt; ++u) total += buffer[(int64_t)u * values + k];
            edges[k] += total;
        }
    }
    free(buffer);
    return nt;
}

/* The spline path deposit of the Pyccel kernels: serial. */
int cb_deposit_spline(int ndim, int degree, const double* start, int64_t ss, const double* end,
                      int64_t es, const double* charges, int64_t n, double* edges,
                      const double* lower, const double* cell, const int32_t* num,
                      const int32_t* code) {
    og_deposit_spline(ndim, degree, start, ss, end, es, charges, n, edges, lower, cell, num, code);
    return 1;
}

// mpf_batch.cu -- the serving batch: many small FP64 gathers, scatters and path deposits in
// one launch.
//
// The requests of a batch sit in a device table (mpf_batch_request); request r owns the
// tiles first_tile .. first_tile + ceil(n / tile_markers) - 1. Persistent CTAs take tiles
// from the header's counter; a tile is a range of one request's markers, one marker per
// thread (a path per thread for a deposit), with the arithmetic of the single-request
// kernels (the same stencils and path walks, global loads, FP64 atomic adds for the
// scatter and the deposit). The last CTA to finish resets the counter, so
// the launch replays from a CUDA graph with nothing but the table rewritten.
#include <algorithm>

#include "mpf_paths.cuh"
#include "mpifield_b200.h"

namespace mpf {

__device__ __forceinline__ Grid<double> grid_of(const mpf_batch_request& r) {
    Grid<double> g;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        g.lower[d] = r.lower[d];
        g.cell[d] = r.cell[d];
        g.inv[d] = r.inv[d];
        g.pow2[d] = 0;
        g.num[d] = r.num[d];
        g.code[d] = r.code[d];
        g.ext[d] = r.ext[d];
    }
    return g;
}

// The stencil of marker i of a request: weights and global node offsets per axis.
template <int NDIM, int KIND, int P>
__device__ __forceinline__ void batch_stencil(const mpf_batch_request& r, const Grid<double>& g, int64_t i,
                                              double (&w)[3][P + 1], int64_t (&off)[3][P + 1]) {
    constexpr int S = P + 1;
    int base[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (d < NDIM) {
            base[d] = axis_stencil<double, KIND, P>(rel_from(r.positions[d * r.pos_stride + i], g, d), g.num[d],
                                                    g.code[d], w[d]);
        } else {
#pragma unroll
            for (int s = 0; s < S; ++s) w[d][s] = double(s == 0);
        }
    }
    global_offsets<NDIM, S>(base, g.num, g.code, g.ext, off);
}

template <int NDIM, int KIND, int P>
__device__ __noinline__ void batch_gather(const mpf_batch_request& r, int64_t first, int64_t last) {
    constexpr int S = P + 1;
    const Grid<double> g = grid_of(r);
    const int64_t ncomp = r.ncomp;
    for (int64_t i = first + threadIdx.x; i < last; i += blockDim.x) {
        double w[3][S];
        int64_t off[3][S];
        batch_stencil<NDIM, KIND, P>(r, g, i, w, off);
        for (int c = 0; c < (int)ncomp; ++c) {
            double acc[1];
            stencil_sum<double, NDIM, S, 1, true, int64_t>(r.field, off, w, ncomp, c, acc);
            r.out[c * r.out_stride + i] = acc[0];
        }
    }
}

template <int NDIM, int KIND, int P>
__device__ __noinline__ void batch_scatter(const mpf_batch_request& r, int64_t first, int64_t last) {
    constexpr int S = P + 1;
    const Grid<double> g = grid_of(r);
    const int64_t ncomp = r.ncomp;
    for (int64_t i = first + threadIdx.x; i < last; i += blockDim.x) {
        // a dead marker (all values zero) deposits nothing and its position is not read
        bool live = false;
        for (int c = 0; c < (int)ncomp; ++c) live = live || r.values[c * r.val_stride + i] != 0.0;
        if (!live) continue;
        double w[3][S];
        int64_t off[3][S];
        batch_stencil<NDIM, KIND, P>(r, g, i, w, off);
        for (int c = 0; c < (int)ncomp; ++c) {
            const double v[1] = {r.values[c * r.val_stride + i]};
            stencil_add<double, NDIM, S, 1, int64_t>(r.out, off, w, ncomp, c, v);
        }
    }
}

// Paths first .. last - 1 of a deposit request (WHITNEY or spline edges of degree P).
template <int NDIM, int P, bool WHITNEY>
__device__ __noinline__ void batch_paths(const mpf_batch_request& r, int64_t first, int64_t last) {
    PathArgs<double> a{};
    a.g = grid_of(r);
    a.start = r.positions;
    a.start_stride = r.pos_stride;
    a.end = r.field;
    a.end_stride = r.out_stride;
    a.charges = r.values;
    a.edges_out = r.out;
    a.n = r.n;
    GlobalEdgeSink<double, NDIM> sink;
    sink.edges = r.out;
#pragma unroll
    for (int d = 0; d < 3; ++d) sink.ext[d] = a.g.ext[d];
    for (int64_t i = first + threadIdx.x; i < last; i += blockDim.x) {
        const double q = r.values[i];
        if (q == 0.0) continue;
        double r0[NDIM], r1[NDIM];
        if (!path_cells<double, NDIM, WHITNEY>(a, i, r0, r1)) continue;
        if constexpr (WHITNEY) whitney_path<double, NDIM>(q, r0, r1, a.g, sink);
        else spline_path<double, NDIM, P>(q, r0, r1, a.g, sink);
    }
}

template <int NDIM, int KIND, int P>
__device__ __forceinline__ void batch_op(const mpf_batch_request& r, int64_t first, int64_t last) {
    if (r.op == MPF_OP_PATHS) {
        if constexpr (KIND == LINEAR) batch_paths<NDIM, 1, true>(r, first, last);
        else if constexpr (KIND == SPLINE && P >= 1) batch_paths<NDIM, P, false>(r, first, last);
        return;
    }
    if (r.op == MPF_OP_GATHER) batch_gather<NDIM, KIND, P>(r, first, last);
    else batch_scatter<NDIM, KIND, P>(r, first, last);
}

template <int NDIM>
__device__ __forceinline__ void batch_by_kind(const mpf_batch_request& r, int64_t first, int64_t last) {
    if (r.kind == LINEAR) return batch_op<NDIM, LINEAR, 1>(r, first, last);
    if (r.kind == QUADRATIC) return batch_op<NDIM, QUADRATIC, 2>(r, first, last);
    switch (r.degree) {
        case 0: return batch_op<NDIM, SPLINE, 0>(r, first, last);
        case 1: return batch_op<NDIM, SPLINE, 1>(r, first, last);
        case 2: return batch_op<NDIM, SPLINE, 2>(r, first, last);
        default: return batch_op<NDIM, SPLINE, 3>(r, first, last);
    }
}

__global__ void __launch_bounds__(256, 2) batch_kernel(const mpf_batch_request* __restrict__ table,
                                                    mpf_batch_header* header) {
    __shared__ long long s_tile;
    __shared__ long long s_request;
    const long long requests = header->requests;
    const long long tiles = header->tiles;
    const long long markers = header->tile_markers;
    while (true) {
        if (threadIdx.x == 0) {
            const long long t = (long long)atomicAdd(reinterpret_cast<unsigned long long*>(&header->next_tile), 1ull);
            s_tile = t;
            // the request of tile t: the last entry whose first_tile <= t
            long long lo = 0, hi = requests - 1;
            while (lo < hi) {
                const long long mid = (lo + hi + 1) / 2;
                if (table[mid].first_tile <= t) lo = mid;
                else hi = mid - 1;
            }
            s_request = lo;
        }
        __syncthreads();
        const long long t = s_tile;
        const long long ri = s_request;
        __syncthreads();
        if (t >= tiles || requests <= 0 || markers <= 0) break;
        const mpf_batch_request& r = table[ri];
        const int64_t first = (t - r.first_tile) * markers;
        const int64_t last = min((int64_t)r.n, first + (int64_t)markers);
        if (first < 0 || first >= last) continue;
        switch (r.ndim) {
            case 1: batch_by_kind<1>(r, first, last); break;
            case 2: batch_by_kind<2>(r, first, last); break;
            default: batch_by_kind<3>(r, first, last); break;
        }
    }
    // the last CTA out sets the counters back to zero for the next launch
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned long long done =
            atomicAdd(reinterpret_cast<unsigned long long*>(&header->finished), 1ull);
        if (done == (unsigned long long)gridDim.x - 1) {
            atomicExch(reinterpret_cast<unsigned long long*>(&header->next_tile), 0ull);
            atomicExch(reinterpret_cast<unsigned long long*>(&header->finished), 0ull);
        }
    }
}

int launch_batch(const mpf_batch_request* table, mpf_batch_header* header, int grid, int block,
                 cudaStream_t stream) {
    if (block <= 0) block = 256;
    block = std::max(32, std::min(256, block / 32 * 32));
    if (grid <= 0) grid = sm_count() * 2;
    batch_kernel<<<grid, block, 0, stream>>>(table, header);
    count_launches(1);
    return launch_status();
}

}  // namespace mpf

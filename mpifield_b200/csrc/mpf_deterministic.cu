// mpf_deterministic.cu -- the bit-reproducible scatter (FP64).
//
// Every contribution c = W_k(x) v of the scatter is written as an exact pair of 64-bit
// fixed-point integers: hi = rint(c 2^f) and lo = rint((c 2^f - hi) 2^L), both summed per
// node with integer atomics. Integer addition is associative, so the sums -- and the
// field += hi 2^-f + lo 2^-(f + L) written at the end in a fixed order -- are the same
// bits for any order of the adds, any launch shape and any order of the markers. The
// scale f comes from a bound that does not depend on any order either: every node sum is
// at most N max |v| (the weights of a marker are at most 1 and sum to 1), so
// f = 61 - ceil(log2(N max |v|)) keeps |sum hi| below 2^62; |lo| <= 2^(L-1) per
// contribution keeps sum lo below 2^63 for up to 2^34 contributions to a node. The
// truncation is at most 2^-(f + L + 1) per contribution (L = 28): about 1e-19 of the bound.
// The values must be finite (a non-finite value has no fixed-point image).
#include <cmath>

#include "mpf_nodes_launch.cuh"
#include "mpifield_b200.h"

namespace mpf {

constexpr int kLowBits = 28;

// The header of the workspace: the bit pattern of max |v| (ordered as an integer), then
// the node accumulators hi[entries], lo[entries].
struct DetHeader {
    unsigned long long max_bits;
    unsigned long long pad[31];
};

__global__ void det_clear_kernel(long long* acc, int64_t count, DetHeader* h) {
    if (blockIdx.x == 0 && threadIdx.x == 0) h->max_bits = 0ull;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        acc[i] = 0;
}

__global__ void det_max_kernel(const double* values, int64_t val_stride, int64_t n, int ncomp, DetHeader* h) {
    unsigned long long best = 0ull;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        for (int c = 0; c < ncomp; ++c) {
            // the bit patterns of non-negative doubles order as the values
            const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(values[c * val_stride + i]));
            best = b > best ? b : best;
        }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_down_sync(0xffffffffu, best, o);
        best = other > best ? other : best;
    }
    if ((threadIdx.x & 31) == 0 && best) atomicMax(&h->max_bits, best);
}

// The scale exponent f for n markers whose |values| are at most the header's max: with
// max < 2^ev and n <= 2^en, every node sum is below 2^(ev + en).
__device__ __forceinline__ int det_scale(const DetHeader* h, int64_t n) {
    const double vmax = __longlong_as_double((long long)h->max_bits);
    if (!(vmax > 0.0)) return 0;
    int ev = 0;
    frexp(vmax, &ev);
    const int en = 64 - __clzll((long long)(n > 1 ? n - 1 : 1));
    return 61 - ev - en;
}

template <int NDIM, int KIND, int P>
__global__ void __launch_bounds__(256) det_scatter_kernel(const NodeArgs<double> a, long long* hi, long long* lo,
                                                          int64_t entries, const DetHeader* h) {
    constexpr int S = P + 1;
    const int f = det_scale(h, a.n);
    const double low = ldexp(1.0, kLowBits);
    const int ncomp = a.ncomp;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
        bool live = false;
        for (int c = 0; c < ncomp; ++c) live = live || a.values[c * a.val_stride + i] != 0.0;
        if (!live) continue;  // a dead marker deposits nothing and its position is not read
        double w[3][S];
        int base[3] = {0, 0, 0};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (d < NDIM) {
                base[d] = axis_stencil<double, KIND, P>(rel_of(a, d, i), a.g.num[d], a.g.code[d], w[d]);
            } else {
#pragma unroll
                for (int s = 0; s < S; ++s) w[d][s] = double(s == 0);
            }
        }
        int64_t off[3][S];
        global_offsets<NDIM, S>(base, a.g.num, a.g.code, a.g.ext, off);
        constexpr int SY = NDIM > 1 ? S : 1;
        constexpr int SZ = NDIM > 2 ? S : 1;
        for (int c = 0; c < ncomp; ++c) {
            const double v = a.values[c * a.val_stride + i];
#pragma unroll
            for (int x = 0; x < S; ++x)
#pragma unroll
                for (int y = 0; y < SY; ++y)
#pragma unroll
                    for (int z = 0; z < SZ; ++z) {
                        double wt = w[0][x];
                        if (NDIM > 1) wt *= w[1][y];
                        if (NDIM > 2) wt *= w[2][z];
                        const double scaled = ldexp(wt * v, f);  // exact scaling by a power of two
                        const double whole = rint(scaled);
                        const long long part = (long long)whole;
                        const long long rest = (long long)rint((scaled - whole) * low);
                        const int64_t k = (off[0][x] + off[1][y] + off[2][z]) * ncomp + c;
                        atomicAdd(reinterpret_cast<unsigned long long*>(hi + k), (unsigned long long)part);
                        atomicAdd(reinterpret_cast<unsigned long long*>(lo + k), (unsigned long long)rest);
                    }
        }
    }
}

// The bit-reproducible scatter for markers sorted by cell tile (mpf_sort_by_tile), one
// component, every axis periodic: the same fixed-point contributions as det_scatter_kernel,
// summed per tile in a shared-memory box of integer pairs (shared-memory integer atomics)
// and added to the node accumulators once per tile piece, instead of two global atomics per
// contribution. Integer sums are exact, so the accumulators -- and the field -- have the
// same bits as with det_scatter_kernel. The CTA's share of the ranks is cut at tile
// boundaries as in the tile scatter; markers go to threads in stride; a marker whose anchor
// is not in its rank's tile adds to the node accumulators directly.
template <int NDIM, int KIND, int P, int TX = 0, int TY = 0, int TZ = 0>
__global__ void __launch_bounds__(kMaxBlock, 3) det_scatter_tiles_kernel(const NodeArgs<double> a, long long* hi,
                                                                        long long* lo, const DetHeader* h) {
    constexpr int S = P + 1;
    constexpr int H = P / 2;
    constexpr int SY = NDIM > 1 ? S : 1;
    constexpr int SZ = NDIM > 2 ? S : 1;
    __shared__ TileLoop s_loop;
    __shared__ TileStep s_step;
    const int t = threadIdx.x;
    const int tl[3] = {TX > 0 ? TX : a.tile[0], TY > 0 ? TY : a.tile[1], TZ > 0 ? TZ : a.tile[2]};
    int ex[3] = {1, 1, 1};
    tile_box_extents<NDIM, P>(tl, ex);
    const int total = ex[0] * ex[1] * ex[2];
    unsigned long long* bhi = reinterpret_cast<unsigned long long*>(mpf_dynamic_smem);
    unsigned long long* blo = bhi + total;
    for (int q = t; q < 2 * total; q += kMaxBlock) bhi[q] = 0ull;
    const int se = NDIM > 2 ? 1 : 0;
    const int sb = NDIM > 2 ? ex[2] : (NDIM > 1 ? 1 : 0);
    const int sa = NDIM > 2 ? ex[1] * ex[2] : (NDIM > 1 ? ex[1] : 1);
    const int st[3] = {sa, NDIM > 1 ? sb : 0, NDIM > 2 ? se : 0};
    if (t == 0) {
        const int64_t live = min(max(__ldg(a.tile_start + a.ntiles), (int64_t)0), a.n);
        const int64_t per = (live + gridDim.x - 1) / gridDim.x;
        s_loop.m = min((int64_t)blockIdx.x * per, live);
        s_loop.m_end = min(s_loop.m + per, live);
        s_loop.e = s_loop.m;
        s_loop.cur = -1;
        s_loop.sub = s_loop.nsub = 0;
        s_loop.part = s_loop.extra = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) s_step.blo[d] = s_step.old_lo[d] = 0;
    }
    const int f = det_scale(h, a.n);
    const double low = ldexp(1.0, kLowBits);
#pragma unroll 1
    for (;;) {
        if (t == 0) plan_tile_step<NDIM, H>(s_loop, s_step, a.tile_start, a.ntiles, a.tiles, tl, 1 << 28);
        // the plan is visible and the previous piece's adds are complete
        __syncthreads();
        const int64_t first = s_step.first;
        const int count = s_step.count;
        if (s_step.retire) {
            const int olo[3] = {s_step.old_lo[0], s_step.old_lo[1], s_step.old_lo[2]};
            for_box_entries<NDIM>(olo, ex, a.g.num, a.g.ext, [&](int e, auto node) {
                const unsigned long long vh = bhi[e], vl = blo[e];
                if (vh != 0ull || vl != 0ull) {
                    const int64_t at = node();
                    atomicAdd(reinterpret_cast<unsigned long long*>(hi + at), vh);
                    atomicAdd(reinterpret_cast<unsigned long long*>(lo + at), vl);
                    bhi[e] = 0ull;
                    blo[e] = 0ull;
                }
            });
            __syncthreads();
        }
        if (count == 0) break;
        const int blo_[3] = {s_step.blo[0], s_step.blo[1], s_step.blo[2]};
        // thread t takes the t-th of kMaxBlock contiguous ranges of the piece, so that the
        // lanes of a warp add to different cells at a time (same-address integer atomics of
        // one instruction serialise)
        const int per = count / kMaxBlock, rem = count % kMaxBlock;
        const int j0 = t * per + min(t, rem), j1 = j0 + per + (t < rem ? 1 : 0);
#pragma unroll 1
        for (int j = j0; j < j1; ++j) {
            const int64_t i = first + j;
            const double v = a.values[i];
            if (v == 0.0) continue;  // a dead marker deposits nothing and its position is not read
            double w[3][S];
            int base[3] = {0, 0, 0};
            int k = 0;
            bool inside = true;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (d < NDIM) {
                    base[d] = axis_stencil<double, KIND, P>(rel_of(a, d, i), a.g.num[d], PERIODIC, w[d]);
                    const int off = wrap_index(base[d] + H - blo_[d], a.g.num[d]);
                    inside = inside && (unsigned)off < (unsigned)tl[d];
                    k += off * st[d];
                } else {
#pragma unroll
                    for (int s = 0; s < S; ++s) w[d][s] = double(s == 0);
                }
            }
            int64_t goff[3][S];
            if (!inside) global_offsets<NDIM, S>(base, a.g.num, a.g.code, a.g.ext, goff);
#pragma unroll
            for (int x = 0; x < S; ++x)
#pragma unroll
                for (int y = 0; y < SY; ++y)
#pragma unroll
                    for (int z = 0; z < SZ; ++z) {
                        double wt = w[0][x];
                        if (NDIM > 1) wt *= w[1][y];
                        if (NDIM > 2) wt *= w[2][z];
                        const double scaled = ldexp(wt * v, f);  // exact scaling by a power of two
                        const double whole = rint(scaled);
                        const long long part = (long long)whole;
                        const long long rest = (long long)rint((scaled - whole) * low);
                        if (inside) {
                            const int e = k + x * sa + y * sb + z * se;
                            atomicAdd(bhi + e, (unsigned long long)part);
                            atomicAdd(blo + e, (unsigned long long)rest);
                        } else {
                            const int64_t at = goff[0][x] + goff[1][y] + goff[2][z];
                            atomicAdd(reinterpret_cast<unsigned long long*>(hi + at), (unsigned long long)part);
                            atomicAdd(reinterpret_cast<unsigned long long*>(lo + at), (unsigned long long)rest);
                        }
                    }
        }
    }
}

// The tile form when it applies (tile starts given, one component, periodic axes, the box
// of integer pairs within a third of an SM's shared memory); MPF_ERR_ARGUMENT otherwise.
template <int NDIM, int KIND, int P>
static int det_tiles_launch(const NodeArgs<double>& a, long long* hi, long long* lo, const DetHeader* h,
                            cudaStream_t s) {
    if (!a.tile_start || a.ncomp != 1 || !all_periodic<double, NDIM>(a)) return MPF_ERR_ARGUMENT;
    int64_t total = 1;
    for (int d = 0; d < NDIM; ++d) {
        int64_t e = (int64_t)a.tile[d] + P;
        if (d == NDIM - 1 && (e & 1) == 0) ++e;
        total *= e;
    }
    const int64_t box_bytes = 2 * total * (int64_t)sizeof(long long);
    if (box_bytes > (228 * 1024) / 3 - 2048) return MPF_ERR_ARGUMENT;
    const int smem = (int)box_bytes;
    auto kernel = det_scatter_tiles_kernel<NDIM, KIND, P>;
    int shape = 0;
    if constexpr (NDIM == 3 && P == 2) {
        if (a.tile[0] == 4 && a.tile[1] == 4 && a.tile[2] == 64) {
            kernel = det_scatter_tiles_kernel<NDIM, KIND, P, 4, 4, 64>;
            shape = 1;
        } else if (a.tile[0] == 8 && a.tile[1] == 8 && a.tile[2] == 8) {
            kernel = det_scatter_tiles_kernel<NDIM, KIND, P, 8, 8, 8>;
            shape = 2;
        }
    }
    static int cache[3][64] = {{0}};
    if (allow_smem(kernel, smem, cache[shape]) != MPF_OK) return MPF_ERR_CUDA;
    const int64_t units = (a.n + kMaxBlock - 1) / kMaxBlock;
    kernel<<<grid_for(units, smem, kMaxBlock, 3), kMaxBlock, smem, s>>>(a, hi, lo, h);
    return MPF_OK;
}

__global__ void det_finish_kernel(double* field, const long long* hi, const long long* lo, int64_t entries,
                                  const DetHeader* h, int64_t n) {
    const int f = det_scale(h, n);
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < entries; k += (int64_t)gridDim.x * blockDim.x) {
        if (hi[k] == 0 && lo[k] == 0) continue;
        field[k] += ldexp((double)hi[k], -f) + ldexp((double)lo[k], -f - kLowBits);
    }
}

size_t det_workspace_bytes(int64_t entries) { return sizeof(DetHeader) + 2 * (size_t)entries * sizeof(long long); }

template <int NDIM, int KIND, int P>
static void det_launch(const NodeArgs<double>& a, long long* hi, long long* lo, int64_t entries, const DetHeader* h,
                       cudaStream_t s) {
    if (det_tiles_launch<NDIM, KIND, P>(a, hi, lo, h, s) != MPF_ERR_ARGUMENT) return;  // launched, or a CUDA error
    const int64_t blocks = std::min<int64_t>((a.n + 255) / 256, (int64_t)sm_count() * 8);
    det_scatter_kernel<NDIM, KIND, P><<<(unsigned)std::max<int64_t>(blocks, 1), 256, 0, s>>>(a, hi, lo, entries, h);
}

template <int NDIM>
static int det_by_kind(int kind, int degree, const NodeArgs<double>& a, long long* hi, long long* lo,
                       int64_t entries, const DetHeader* h, cudaStream_t s) {
    if (kind == LINEAR) det_launch<NDIM, LINEAR, 1>(a, hi, lo, entries, h, s);
    else if (kind == QUADRATIC) det_launch<NDIM, QUADRATIC, 2>(a, hi, lo, entries, h, s);
    else if (degree == 0) det_launch<NDIM, SPLINE, 0>(a, hi, lo, entries, h, s);
    else if (degree == 1) det_launch<NDIM, SPLINE, 1>(a, hi, lo, entries, h, s);
    else if (degree == 2) det_launch<NDIM, SPLINE, 2>(a, hi, lo, entries, h, s);
    else if (degree == 3) det_launch<NDIM, SPLINE, 3>(a, hi, lo, entries, h, s);
    else return MPF_ERR_ARGUMENT;
    return MPF_OK;
}

int launch_scatter_deterministic(int kind, int degree, int ndim, const NodeArgs<double>& a, int64_t entries,
                                 void* workspace, cudaStream_t s) {
    DetHeader* h = static_cast<DetHeader*>(workspace);
    long long* hi = reinterpret_cast<long long*>(h + 1);
    long long* lo = hi + entries;
    const unsigned grid = (unsigned)std::max(1, sm_count() * 4);
    det_clear_kernel<<<grid, 256, 0, s>>>(hi, 2 * entries, h);
    det_max_kernel<<<grid, 256, 0, s>>>(a.values, a.val_stride, a.n, a.ncomp, h);
    int st = MPF_ERR_ARGUMENT;
    switch (ndim) {
        case 1: st = det_by_kind<1>(kind, degree, a, hi, lo, entries, h, s); break;
        case 2: st = det_by_kind<2>(kind, degree, a, hi, lo, entries, h, s); break;
        case 3: st = det_by_kind<3>(kind, degree, a, hi, lo, entries, h, s); break;
    }
    if (st != MPF_OK) return st;
    det_finish_kernel<<<grid, 256, 0, s>>>(a.field_out, hi, lo, entries, h, a.n);
    count_launches(4);
    return launch_status();
}

}  // namespace mpf

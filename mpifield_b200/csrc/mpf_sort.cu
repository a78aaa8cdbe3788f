// mpf_sort.cu -- the cell-tile keys of the markers and their stable sort.
//
// The key of a marker is the tile of the anchor node of its stencil (mpf_stencil.cuh,
// axis_anchor), row-major over the tiles; a marker whose values are all zero gets the
// sentinel key num_tiles without its position being read. The sort is a least-
// significant-digit radix sort of (key, marker) pairs with 8- to 10-bit digits, as few
// passes as the key's bits allow. Each pass: a per-CTA digit histogram, an exclusive scan of the
// histograms in digit-major order, and a stable scatter in which every warp ranks its
// 32 keys of a round with __match_any_sync against a per-warp digit count, so the rank
// of a key follows the marker order inside the warp, the warps of a CTA and the CTAs:
// the result is the stable order (numpy.argsort(keys, kind="stable")), bit for bit.
#include <algorithm>
#include <cstdint>
#include <mutex>

#include "mpf_internal.h"
#include "mpf_stencil.cuh"
#include "mpifield_b200.h"

namespace mpf {

constexpr int kSortBlock = 256;
constexpr int kSortItems = 16;  // keys per thread per tile
constexpr int kSortTile = kSortBlock * kSortItems;
constexpr int kWarps = kSortBlock / 32;


// The rare cases of the key, out of line so that the key kernel's unrolled body keeps only
// the usual case (inlined at every marker and axis, the wraps, clamps and divisions of the
// rare ones outgrew the instruction cache).
template <typename T, int KIND, int P>
__device__ __noinline__ int axis_anchor_rare(T rel, int num, int code) {
    return axis_anchor<T, KIND, P>(rel, num, code);
}

__device__ __noinline__ int quotient_rare(int a, int b) { return a / b; }

// The anchor node of rel (axis_anchor). Usually the stencil's middle node `quick` lies in
// [1, num - 2]: there every stencil takes it unchanged (no wrap, no clamp, no mapping), as
// their own quick paths do, so it is the anchor; clamped spline axes of degree >= 1 and
// everything else take the full computation.
template <typename T, int KIND, int P>
__device__ __forceinline__ int key_anchor(T rel, int num, int code) {
    constexpr bool half = KIND == QUADRATIC || (KIND == SPLINE && P % 2 == 0);
    const int quick = trunc_int<T>(half ? rel + T(0.5) : rel);
    const bool clamped_spline = KIND == SPLINE && P >= 1 && code == CLAMPED;
    if (quick >= 1 && quick <= num - 2 && !clamped_spline) return quick;
    return axis_anchor_rare<T, KIND, P>(rel, num, code);
}

// The key of marker i at position x: its anchor node's tile, then (within) its cell. A
// tile extent that is a power of two (shift[d] >= 0) divides a non-negative anchor by a
// shift, the same quotient as the division.
template <typename T, int NDIM, int KIND, int P>
__device__ __forceinline__ void tile_key_of(const KeyArgs<T>& a, const T* x, int64_t i, const int* shift) {
    int64_t key = 0, inner = 0;
#pragma unroll
    for (int d = 0; d < NDIM; ++d) {
        const T rel = cells_from(x[d] - a.g.lower[d], a.g.cell[d], a.g.inv[d], a.g.pow2[d]);
        const int anchor = key_anchor<T, KIND, P>(rel, a.g.num[d], a.g.code[d]);
        const int t = shift[d] >= 0 && anchor >= 0 ? anchor >> shift[d] : quotient_rare(anchor, a.tile[d]);
        key = key * a.ntiles[d] + t;
        inner = inner * a.tile[d] + (anchor - t * a.tile[d]);
    }
    if (a.within) {
        int64_t cells = 1;
#pragma unroll
        for (int d = 0; d < NDIM; ++d) cells *= a.tile[d];
        key = key * cells + inner;
    }
    a.keys[i] = (uint32_t)key;
}

// Four markers a thread per round (i, i + stride, ...), their positions loaded before any
// key is formed, so a thread keeps 4 x NDIM loads in flight; four CTAs an SM, one wave.
constexpr int kKeyUnroll = 4;
constexpr int kKeyBlocksPerSm = 4;

template <typename T, int NDIM, int KIND, int P>
__global__ void __launch_bounds__(kSortBlock, kKeyBlocksPerSm) tile_keys_kernel(const KeyArgs<T> a) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int shift[NDIM];
#pragma unroll
    for (int d = 0; d < NDIM; ++d) shift[d] = (a.tile[d] & (a.tile[d] - 1)) == 0 ? __ffs(a.tile[d]) - 1 : -1;
    for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < a.n; i0 += stride * kKeyUnroll) {
        bool live[kKeyUnroll];
#pragma unroll
        for (int u = 0; u < kKeyUnroll; ++u) {
            const int64_t i = i0 + u * stride;
            live[u] = i < a.n;
            if (a.values && live[u]) {
                bool any = false;
                for (int64_t c = 0; c < a.ncomp; ++c) any = any || a.values[c * a.val_stride + i] != T(0);
                if (!any) a.keys[i] = a.sentinel;
                live[u] = any;
            }
        }
        T x[kKeyUnroll][NDIM];
#pragma unroll
        for (int u = 0; u < kKeyUnroll; ++u)
#pragma unroll
            for (int d = 0; d < NDIM; ++d) x[u][d] = live[u] ? a.pos[d * a.pos_stride + i0 + u * stride] : T(0);
#pragma unroll
        for (int u = 0; u < kKeyUnroll; ++u)
            if (live[u]) tile_key_of<T, NDIM, KIND, P>(a, x[u], i0 + u * stride, shift);
    }
}

template <int BITS>
__global__ void digit_histogram_kernel(const uint32_t* keys, int64_t n, const int64_t* n_dev, int shift,
                                       uint32_t* counts, int64_t nblocks) {
    constexpr int DIGITS = 1 << BITS;
    if (n_dev) n = min(n, *n_dev);  // the count known on the device only (a mover sort)
    __shared__ uint32_t hist[DIGITS];
    for (int d = threadIdx.x; d < DIGITS; d += blockDim.x) hist[d] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    uint32_t key[kSortItems];  // the thread's keys loaded first, then counted
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const int64_t i = base + (int64_t)r * kSortBlock + threadIdx.x;
        key[r] = i < n ? keys[i] : 0u;
    }
#pragma unroll
    for (int r = 0; r < kSortItems; ++r)
        if (base + (int64_t)r * kSortBlock + threadIdx.x < n) atomicAdd(&hist[(key[r] >> shift) & (DIGITS - 1)], 1u);
    __syncthreads();
    for (int d = threadIdx.x; d < DIGITS; d += blockDim.x) counts[(int64_t)d * nblocks + blockIdx.x] = hist[d];
}

// Exclusive scan of `count` u32 values in place, in three kernels: chunk sums, a scan of
// the sums in one CTA, and the chunks rescanned with their offsets.
constexpr int kScanChunk = 2048;

__global__ void scan_sums_kernel(const uint32_t* data, int64_t count, uint32_t* sums) {
    __shared__ uint32_t part[kSortBlock / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanChunk;
    uint32_t s = 0;
    for (int k = threadIdx.x; k < kScanChunk; k += blockDim.x) {
        const int64_t i = base + k;
        if (i < count) s += data[i];
    }
    s = __reduce_add_sync(0xffffffffu, s);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
        sums[blockIdx.x] = t;
    }
}

__global__ void scan_single_kernel(uint32_t* sums, int64_t count) {
    // one CTA: sequential over chunks of blockDim, scan within each
    __shared__ uint32_t buf[kSortBlock];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < count; base += blockDim.x) {
        const int64_t i = base + threadIdx.x;
        const uint32_t v = i < count ? sums[i] : 0;
        buf[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < (int)blockDim.x; off <<= 1) {
            const uint32_t add = threadIdx.x >= (unsigned)off ? buf[threadIdx.x - off] : 0;
            __syncthreads();
            buf[threadIdx.x] += add;
            __syncthreads();
        }
        if (i < count) sums[i] = carry + buf[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += buf[threadIdx.x];
        __syncthreads();
    }
}

__global__ void scan_chunks_kernel(uint32_t* data, int64_t count, const uint32_t* offsets) {
    __shared__ uint32_t buf[kSortBlock];
    __shared__ uint32_t carry;
    const int64_t base = (int64_t)blockIdx.x * kScanChunk;
    if (threadIdx.x == 0) carry = offsets[blockIdx.x];
    __syncthreads();
    for (int sub = 0; sub < kScanChunk; sub += blockDim.x) {
        const int64_t i = base + sub + threadIdx.x;
        const uint32_t v = i < count ? data[i] : 0;
        buf[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < (int)blockDim.x; off <<= 1) {
            const uint32_t add = threadIdx.x >= (unsigned)off ? buf[threadIdx.x - off] : 0;
            __syncthreads();
            buf[threadIdx.x] += add;
            __syncthreads();
        }
        if (i < count) data[i] = carry + buf[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += buf[threadIdx.x];
        __syncthreads();
    }
}

// The stable scatter of one pass. Warp w of a CTA owns the contiguous segment
// [w * 32 * kSortItems, (w + 1) * 32 * kSortItems) of the CTA's tile and walks it in
// rounds of 32 consecutive keys, ranking each key among the warp's keys of its digit
// (__match_any_sync) against per-warp digit counts in shared memory. The tile's pairs are
// then placed in shared memory in digit order (a CTA-wide scan of the digit counts) and
// written out in that order: consecutive threads write consecutive ranks of one digit's
// run, so the writes of a warp cover a few runs instead of 32 scattered words. The CTA's
// output offsets of its digits are read once, at the start (two per thread), and folded
// into the digit starts; a value is read where it is placed, not held through the ranking,
// and the ranks are kept two to a register (64 registers: four CTAs an SM for digits of up
// to 9 bits, against two when the values and ranks were held whole); a CTA past the
// device-side count (a mover sort, its grid sized for every marker) returns at once.
template <int BITS>
__global__ void __launch_bounds__(kSortBlock, BITS <= 9 ? 4 : 3)
    digit_scatter_kernel(const uint32_t* keys_in, const int32_t* vals_in, int64_t n, const int64_t* n_dev,
                         int shift, const uint32_t* offsets, int64_t nblocks, uint32_t* keys_out,
                         int32_t* vals_out) {
    constexpr int DIGITS = 1 << BITS;
    constexpr int PER = DIGITS / kSortBlock;  // digits a thread scans (DIGITS >= kSortBlock)
    static_assert(DIGITS % kSortBlock == 0, "a whole number of digits per thread");
    if (n_dev) n = min(n, *n_dev);
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    if (base >= n) return;  // the whole CTA: nothing of it is in the sort
    extern __shared__ uint32_t smem_words[];
    uint32_t* warp_count = smem_words;                 // [kWarps][DIGITS]
    uint32_t* digit_start = warp_count + kWarps * DIGITS;  // [DIGITS]: the tile's first place of a digit
    uint32_t* tile_keys = digit_start + DIGITS;        // [kSortTile]
    int32_t* tile_vals = reinterpret_cast<int32_t*>(tile_keys + kSortTile);  // [kSortTile]
    __shared__ uint32_t warp_sums[kWarps];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    uint32_t out_at[PER];  // this CTA's first output rank of each of the thread's digits
#pragma unroll
    for (int q = 0; q < PER; ++q) out_at[q] = offsets[(int64_t)(threadIdx.x * PER + q) * nblocks + blockIdx.x];
    for (int d = threadIdx.x; d < kWarps * DIGITS; d += blockDim.x) warp_count[d] = 0;
    __syncthreads();
    uint32_t* mine = warp_count + warp * DIGITS;
    const int64_t seg = base + (int64_t)warp * 32 * kSortItems;
    uint32_t key[kSortItems];
    uint32_t rank[kSortItems / 2];  // two ranks (< kSortTile) per word
    static_assert(kSortTile <= 65536 && kSortItems % 2 == 0, "ranks packed in halves");
    const unsigned below = (1u << lane) - 1u;
    // all the segment's keys in flight at once, before the ranking's warp barriers
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const int64_t i = seg + (int64_t)r * 32 + lane;
        key[r] = i < n ? keys_in[i] : 0xffffffffu;
    }
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const int64_t i = seg + (int64_t)r * 32 + lane;
        const bool have = i < n;
        const uint32_t digit = (key[r] >> shift) & (DIGITS - 1);
        // lanes holding the same digit this round, and those of them before this lane
        const unsigned same = __match_any_sync(0xffffffffu, have ? (int)digit : -1 - lane);
        const unsigned before = __popc(same & below);
        const uint32_t count = have ? mine[digit] : 0;
        const uint32_t rk = count + before;
        rank[r / 2] = (r & 1) ? (rank[r / 2] | (rk << 16)) : rk;
        __syncwarp();
        if (have && before == 0) mine[digit] = count + __popc(same);
        __syncwarp();
    }
    __syncthreads();
    // per digit: the warps' counts become their first places within the digit's run, and
    // the digit's run in the tile starts after the smaller digits' runs (a CTA-wide scan)
    uint32_t total[PER];
    uint32_t run = 0;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int d = threadIdx.x * PER + q;
        uint32_t s = 0;
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t c = warp_count[w * DIGITS + d];
            warp_count[w * DIGITS + d] = s;
            s += c;
        }
        total[q] = s;
        run += s;
    }
    uint32_t incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t x = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += x;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    uint32_t before_warps = 0;
    for (int w = 0; w < warp; ++w) before_warps += warp_sums[w];
    uint32_t at = before_warps + incl - run;
    uint32_t start[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        start[q] = at;
        digit_start[threadIdx.x * PER + q] = at;
        at += total[q];
    }
    __syncthreads();
    // the tile's pairs in digit order in shared memory
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const int64_t i = seg + (int64_t)r * 32 + lane;
        if (i < n) {
            const uint32_t digit = (key[r] >> shift) & (DIGITS - 1);
            const uint32_t place = digit_start[digit] + mine[digit] + ((rank[r / 2] >> (16 * (r & 1))) & 0xffffu);
            tile_keys[place] = key[r];
            tile_vals[place] = vals_in ? vals_in[i] : (int32_t)i;
        }
    }
    __syncthreads();
    // place p of digit d goes to rank out_at[d] + p - start[d] of the output
#pragma unroll
    for (int q = 0; q < PER; ++q) digit_start[threadIdx.x * PER + q] = out_at[q] - start[q];
    __syncthreads();
    const int count = (int)min((int64_t)kSortTile, n - base);
    for (int p = threadIdx.x; p < count; p += blockDim.x) {
        const uint32_t k = tile_keys[p];
        const uint32_t dst = digit_start[(k >> shift) & (DIGITS - 1)] + (uint32_t)p;
        keys_out[dst] = k;
        vals_out[dst] = tile_vals[p];
    }
}

// tile_start[t] = the first rank whose tile is >= t, t = 0 .. num_tiles (the sentinel tile
// of dead markers); tile_start[num_tiles + 1] = n. A key's tile is key / cells.
__global__ void tile_starts_kernel(const uint32_t* sorted, int64_t n, int64_t num_tiles, int64_t cells,
                                   int64_t* start) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j <= n;
         j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t prev = j == 0 ? -1 : (int64_t)sorted[j - 1] / cells;
        const int64_t cur = j == n ? num_tiles + 1 : (int64_t)sorted[j] / cells;
        for (int64_t k = prev + 1; k <= cur && k <= num_tiles + 1; ++k) start[k] = (k == num_tiles + 1) ? n : j;
    }
}

template <typename T>
__global__ void permute_rows_kernel(T* dst, int64_t ds, const T* src, int64_t ss, int64_t rows,
                                    const int32_t* order, int64_t n) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t from = order[j];
        // an order entry outside [0, n) reads nothing: the row gets NaN
        const bool inside = from >= 0 && from < n;
        for (int64_t r = 0; r < rows; ++r) dst[r * ds + j] = inside ? __ldg(src + r * ss + from) : T(NAN);
    }
}

template <typename T>
__global__ void unpermute_rows_kernel(T* dst, int64_t ds, const T* src, int64_t ss, int64_t rows,
                                      const int32_t* order, int64_t n) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t to = order[j];
        if (to < 0 || to >= n) continue;  // an entry outside [0, n) writes nothing
        for (int64_t r = 0; r < rows; ++r) dst[r * ds + to] = src[r * ss + j];
    }
}

// ------------------------------------------------------------------ host side --

constexpr int64_t sort_blocks(int64_t n) { return n > 0 ? (n + kSortTile - 1) / kSortTile : 1; }
constexpr int64_t scan_chunks(int64_t count) { return count > 0 ? (count + kScanChunk - 1) / kScanChunk : 1; }
constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }

struct SortLayout {
    size_t keys_a, keys_b, vals_a, vals_b, counts, sums, total;
};

constexpr SortLayout sort_layout(int64_t n) {
    const int64_t nb = sort_blocks(n);
    const int64_t count = nb * (1 << 10);
    const size_t items = align256(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    SortLayout L{0, 0, 0, 0, 0, 0, 0};
    size_t off = 0;
    L.keys_a = off; off += items;
    L.keys_b = off; off += items;
    L.vals_a = off; off += items;
    L.vals_b = off; off += items;
    L.counts = off; off += align256(sizeof(uint32_t) * (size_t)count);
    L.sums = off; off += align256(sizeof(uint32_t) * (size_t)scan_chunks(count));
    L.total = off;
    return L;
}

size_t sort_workspace_bytes(int64_t n) { return sort_layout(n).total; }

static int scan_exclusive(uint32_t* data, int64_t count, uint32_t* sums, cudaStream_t stream) {
    const int64_t chunks = scan_chunks(count);
    scan_sums_kernel<<<(unsigned)chunks, kSortBlock, 0, stream>>>(data, count, sums);
    count_launches(1);
    scan_single_kernel<<<1, kSortBlock, 0, stream>>>(sums, chunks);
    count_launches(1);
    scan_chunks_kernel<<<(unsigned)chunks, kSortBlock, 0, stream>>>(data, count, sums);
    count_launches(1);
    return launch_status();
}

template <typename T, int NDIM, int KIND, int P>
static int run_keys(const KeyArgs<T>& a, cudaStream_t stream) {
    const int block = kSortBlock;
    const int64_t blocks = std::min<int64_t>((a.n + block * kKeyUnroll - 1) / (block * kKeyUnroll),
                                             (int64_t)sm_count() * kKeyBlocksPerSm);
    tile_keys_kernel<T, NDIM, KIND, P><<<(unsigned)std::max<int64_t>(blocks, 1), block, 0, stream>>>(a);
    count_launches(1);
    return launch_status();
}

template <typename T, int NDIM>
static int keys_by_kind(int kind, int degree, const KeyArgs<T>& a, cudaStream_t stream) {
    if (kind == LINEAR) return run_keys<T, NDIM, LINEAR, 1>(a, stream);
    if (kind == QUADRATIC) return run_keys<T, NDIM, QUADRATIC, 2>(a, stream);
    switch (degree) {
        case 0: return run_keys<T, NDIM, SPLINE, 0>(a, stream);
        case 1: return run_keys<T, NDIM, SPLINE, 1>(a, stream);
        case 2: return run_keys<T, NDIM, SPLINE, 2>(a, stream);
        case 3: return run_keys<T, NDIM, SPLINE, 3>(a, stream);
    }
    return MPF_ERR_ARGUMENT;
}

template <typename T>
int tile_keys(int kind, int degree, int ndim, const KeyArgs<T>& a, cudaStream_t stream) {
    switch (ndim) {
        case 1: return keys_by_kind<T, 1>(kind, degree, a, stream);
        case 2: return keys_by_kind<T, 2>(kind, degree, a, stream);
        case 3: return keys_by_kind<T, 3>(kind, degree, a, stream);
    }
    return MPF_ERR_ARGUMENT;
}

template <int BITS>
static int radix_pass(const uint32_t* kin, const int32_t* vin, int64_t n, const int64_t* n_dev, int shift,
                      uint32_t* counts, uint32_t* sums, int64_t nb, uint32_t* kout, int32_t* vout,
                      cudaStream_t stream) {
    digit_histogram_kernel<BITS><<<(unsigned)nb, kSortBlock, 0, stream>>>(kin, n, n_dev, shift, counts, nb);
    count_launches(1);
    if (launch_status() != MPF_OK) return MPF_ERR_CUDA;
    const int st = scan_exclusive(counts, nb << BITS, sums, stream);
    if (st != MPF_OK) return st;
    const int smem = (kWarps * (1 << BITS) + (1 << BITS) + 2 * kSortTile) * (int)sizeof(uint32_t);
    static int configured = 0;
    if (configured < smem) {
        if (record_cuda_error(cudaFuncSetAttribute(digit_scatter_kernel<BITS>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != MPF_OK)
            return MPF_ERR_CUDA;
        configured = smem;
    }
    digit_scatter_kernel<BITS><<<(unsigned)nb, kSortBlock, smem, stream>>>(kin, vin, n, n_dev, shift, counts, nb,
                                                                          kout, vout);
    count_launches(1);
    return launch_status();
}

// Sorts (key, value) pairs stably by key: the n keys (at most n_dev[0] of them when
// n_dev is not null, a count known on the device only) with values vals_in (null: the
// indices 0, 1, ...); the values in key order land in vals_out, the keys in keys_out
// (null: a workspace buffer, returned). Keys are at most max_key; the passes take 8 to
// 10 bits each, as few passes as 10-bit digits allow.
static uint32_t* radix_sort(const uint32_t* keys, const int32_t* vals_in, int64_t n, const int64_t* n_dev,
                            uint64_t max_key, int32_t* vals_out, uint32_t* keys_out, void* workspace, int& status,
                            cudaStream_t stream) {
    const SortLayout L = sort_layout(n);
    char* ws = static_cast<char*>(workspace);
    uint32_t* ka = reinterpret_cast<uint32_t*>(ws + L.keys_a);
    uint32_t* kb = reinterpret_cast<uint32_t*>(ws + L.keys_b);
    int32_t* va = reinterpret_cast<int32_t*>(ws + L.vals_a);
    int32_t* vb = reinterpret_cast<int32_t*>(ws + L.vals_b);
    uint32_t* counts = reinterpret_cast<uint32_t*>(ws + L.counts);
    uint32_t* sums = reinterpret_cast<uint32_t*>(ws + L.sums);
    int bits = 1;
    while (bits < 32 && (max_key >> bits) != 0) ++bits;
    const int passes = std::max(1, (bits + 9) / 10);
    const int digit_bits = std::max(8, (bits + passes - 1) / passes);
    const int64_t nb = sort_blocks(n);
    const uint32_t* kin = keys;
    const int32_t* vin = vals_in;
    uint32_t* kout_buf[2] = {ka, kb};
    int32_t* vout_buf[2] = {va, vb};
    uint32_t* kout = ka;
    status = MPF_OK;
    for (int p = 0; p < passes; ++p) {
        const int shift = digit_bits * p;
        const bool last = p == passes - 1;
        kout = (last && keys_out) ? keys_out : kout_buf[p & 1];
        int32_t* vout = last ? vals_out : vout_buf[p & 1];
        if (digit_bits <= 8) status = radix_pass<8>(kin, vin, n, n_dev, shift, counts, sums, nb, kout, vout, stream);
        else if (digit_bits == 9) status = radix_pass<9>(kin, vin, n, n_dev, shift, counts, sums, nb, kout, vout, stream);
        else status = radix_pass<10>(kin, vin, n, n_dev, shift, counts, sums, nb, kout, vout, stream);
        if (status != MPF_OK) return kout;
        kin = kout;
        vin = vout;
    }
    return kout;
}

static int tile_starts(const uint32_t* sorted, int64_t n, int64_t num_tiles, int64_t cells, int64_t* tile_start,
                       cudaStream_t stream) {
    const int block = 256;
    const int64_t blocks = std::min<int64_t>((n + 1 + block - 1) / block, (int64_t)sm_count() * 16);
    tile_starts_kernel<<<(unsigned)std::max<int64_t>(blocks, 1), block, 0, stream>>>(sorted, n, num_tiles, cells,
                                                                                   tile_start);
    count_launches(1);
    return launch_status();
}

// Sort (keys, marker) pairs stably; the marker order lands in `order`, the tile starts
// in `tile_start`; keys are at most num_tiles * cells (the sentinel).
int sort_keys(const uint32_t* keys, int64_t n, int64_t num_tiles, int64_t cells, int32_t* order,
              int64_t* tile_start, void* workspace, cudaStream_t stream) {
    if (n == 0) return tile_starts(nullptr, 0, num_tiles, cells, tile_start, stream);
    int st = MPF_OK;
    const uint32_t* sorted = radix_sort(keys, nullptr, n, nullptr, (uint64_t)num_tiles * (uint64_t)cells, order,
                                        nullptr, workspace, st, stream);
    if (st != MPF_OK) return st;
    return tile_starts(sorted, n, num_tiles, cells, tile_start, stream);
}

// ------------------------------------------------------ the incremental re-sort --
//
// A store sorted by key whose markers then moved a little: the new stable order is the
// order of (new key, store rank). A marker whose key did not change (a stayer) keeps its
// place among the other stayers -- their keys are the old ones, already ascending in
// store order -- so only the markers whose key changed (the movers) need sorting. The
// re-sort splits the ranks into stayers and movers (stable compaction), radix-sorts the
// movers alone by (key, rank) (their count is known on the device only: the passes read
// it there), and merges the two lists: the output rank of a stayer is its index among
// the stayers plus the number of movers before it in (key, rank) order, found from the
// first mover of every key and a binary search among the movers of its own key, and
// likewise for a mover. The result is the order a full stable sort of the new keys gives,
// bit for bit; its cost is a pass over the store plus a sort of the movers only.

// Movers of every block of kSortTile ranks.
__global__ void mover_count_kernel(const uint32_t* knew, const uint32_t* kprev, int64_t n, uint32_t* counts) {
    __shared__ uint32_t part[kWarps];
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    uint32_t c = 0;
    for (int k = threadIdx.x; k < kSortTile; k += blockDim.x) {
        const int64_t i = base + k;
        if (i < n && knew[i] != kprev[i]) ++c;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kWarps; ++w) t += part[w];
        counts[blockIdx.x] = t;
    }
}

// Stable compaction of the ranks into stayers and movers (key and rank each), the block's
// movers starting at offsets[block] (an exclusive scan of mover_count_kernel's counts).
// The last block writes the totals: totals[0] movers, totals[1] stayers.
__global__ void split_kernel(const uint32_t* knew, const uint32_t* kprev, int64_t n, const uint32_t* offsets,
                             int64_t nblocks, uint32_t* s_keys, int32_t* s_ranks, uint32_t* m_keys,
                             int32_t* m_ranks, int64_t* totals) {
    __shared__ uint32_t warp_movers[kWarps];
    __shared__ uint32_t carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    if (threadIdx.x == 0) carry = 0;
    const uint32_t first_mover = offsets[blockIdx.x];
    // the thread's keys of every round, new and previous, loaded before the rounds' barriers
    uint32_t knew_r[kSortItems], kprev_r[kSortItems];
#pragma unroll
    for (int round = 0; round < kSortItems; ++round) {
        const int64_t i = base + (int64_t)round * kSortBlock + threadIdx.x;
        knew_r[round] = i < n ? knew[i] : 0;
        kprev_r[round] = i < n ? kprev[i] : 0;
    }
    __syncthreads();
#pragma unroll
    for (int round = 0; round < kSortItems; ++round) {
        const int64_t i = base + (int64_t)round * kSortBlock + threadIdx.x;
        const bool have = i < n;
        const uint32_t key = knew_r[round];
        const bool mover = have && key != kprev_r[round];
        const unsigned ballot = __ballot_sync(0xffffffffu, mover);
        if (lane == 0) warp_movers[warp] = __popc(ballot);
        __syncthreads();
        uint32_t before = carry;
        for (int w = 0; w < warp; ++w) before += warp_movers[w];
        before += __popc(ballot & ((1u << lane) - 1u));  // movers of this round before this rank
        if (have) {
            const int64_t movers_before = (int64_t)first_mover + before;
            if (mover) {
                m_keys[movers_before] = key;
                m_ranks[movers_before] = (int32_t)i;
            } else {
                const int64_t stayers_before = i - movers_before;
                s_keys[stayers_before] = key;
                s_ranks[stayers_before] = (int32_t)i;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t t = 0;
            for (int w = 0; w < kWarps; ++w) t += warp_movers[w];
            carry += t;
        }
        __syncthreads();
    }
    if (blockIdx.x == nblocks - 1 && threadIdx.x == 0) {
        totals[0] = (int64_t)first_mover + carry;
        totals[1] = n - totals[0];
    }
}

// starts[k] = the first index of a sorted key array at or above key k, k = 0 .. nkeys;
// the array holds *count keys (count known on the device).
__global__ void key_starts_kernel(const uint32_t* sorted, int64_t n_max, const int64_t* count, int64_t nkeys,
                                  int32_t* starts) {
    const int64_t n = min(n_max, *count);
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j <= n;
         j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t prev = j == 0 ? -1 : (int64_t)sorted[j - 1];
        const int64_t cur = j == n ? nkeys : min((int64_t)sorted[j], nkeys);
        for (int64_t k = prev + 1; k <= cur; ++k) starts[k] = (int32_t)j;
    }
}

// The number of ranks[lo .. hi) below r (ranks ascending).
__device__ __forceinline__ int32_t ranks_below(const int32_t* ranks, int32_t lo, int32_t hi, int32_t r) {
    while (lo < hi) {
        const int32_t mid = lo + (hi - lo) / 2;
        if (ranks[mid] < r) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// The merge: every stayer and every mover to its output rank; order[rank] = its store
// rank, keys_out[rank] = its key.
__global__ void merge_place_kernel(const uint32_t* s_keys, const int32_t* s_ranks, const int32_t* s_starts,
                                   const uint32_t* m_keys, const int32_t* m_ranks, const int32_t* m_starts,
                                   const int64_t* totals, int64_t n, int64_t nkeys, int32_t* order,
                                   uint32_t* keys_out) {
    const int64_t movers = totals[0], stayers = totals[1];
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const bool stayer = j < stayers;
        const int64_t idx = stayer ? j : j - stayers;
        if (!stayer && idx >= movers) continue;
        const uint32_t key = stayer ? s_keys[idx] : m_keys[idx];
        const int32_t rank = stayer ? s_ranks[idx] : m_ranks[idx];
        const int64_t k = min((int64_t)key, nkeys - 1);
        // the other list's elements before this one: all of smaller keys, and those of the
        // same key with smaller store ranks
        const int32_t* other_starts = stayer ? m_starts : s_starts;
        const int32_t* other_ranks = stayer ? m_ranks : s_ranks;
        const int32_t before = ranks_below(other_ranks, other_starts[k], other_starts[k + 1], rank);
        const int64_t at = idx + before;
        if (at >= 0 && at < n) {
            order[at] = rank;
            keys_out[at] = key;
        }
    }
}

struct ResortLayout {
    size_t keys_new, s_keys, s_ranks, m_keys, m_ranks, m_sorted_keys, m_sorted_ranks, counts, sums, totals,
        s_starts, m_starts, radix, total;
};

static ResortLayout resort_layout(int64_t n, int64_t nkeys) {
    const size_t items = align256(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    const int64_t nb = sort_blocks(n);
    const size_t starts = align256(sizeof(int32_t) * (size_t)(nkeys + 1));
    ResortLayout L{};
    size_t off = 0;
    L.keys_new = off; off += items;
    L.s_keys = off; off += items;
    L.s_ranks = off; off += items;
    L.m_keys = off; off += items;
    L.m_ranks = off; off += items;
    L.m_sorted_keys = off; off += items;
    L.m_sorted_ranks = off; off += items;
    L.counts = off; off += align256(sizeof(uint32_t) * (size_t)nb);
    L.sums = off; off += align256(sizeof(uint32_t) * (size_t)scan_chunks(nb));
    L.totals = off; off += 256;
    L.s_starts = off; off += starts;
    L.m_starts = off; off += starts;
    L.radix = off; off += sort_layout(n).total;
    L.total = off;
    return L;
}

size_t resort_workspace_bytes(int64_t n, int64_t nkeys) { return resort_layout(n, nkeys).total; }

// The keys of the store's markers are in the workspace (resort_keys_buffer); with
// prev_sorted null a full sort, else the re-sort against the store's previous sorted keys.
uint32_t* resort_keys_buffer(void* workspace, int64_t n) {
    return reinterpret_cast<uint32_t*>(static_cast<char*>(workspace) + resort_layout(n, 1).keys_new);
}

int resort_keys(int64_t n, int64_t num_tiles, int64_t cells, const uint32_t* prev_sorted, uint32_t* sorted_out,
                int32_t* order, int64_t* tile_start, void* workspace, cudaStream_t stream) {
    const int64_t nkeys = num_tiles * cells + 1;  // keys 0 .. the sentinel
    const ResortLayout L = resort_layout(n, nkeys);
    char* ws = static_cast<char*>(workspace);
    auto at = [&](size_t off) { return reinterpret_cast<void*>(ws + off); };
    const uint32_t* knew = static_cast<const uint32_t*>(at(L.keys_new));
    if (n == 0) return tile_starts(nullptr, 0, num_tiles, cells, tile_start, stream);
    const uint64_t max_key = (uint64_t)num_tiles * (uint64_t)cells;
    int st = MPF_OK;
    if (!prev_sorted) {
        radix_sort(knew, nullptr, n, nullptr, max_key, order, sorted_out, at(L.radix), st, stream);
        if (st != MPF_OK) return st;
        return tile_starts(sorted_out, n, num_tiles, cells, tile_start, stream);
    }
    uint32_t* counts = static_cast<uint32_t*>(at(L.counts));
    uint32_t* sums = static_cast<uint32_t*>(at(L.sums));
    int64_t* totals = static_cast<int64_t*>(at(L.totals));
    uint32_t* s_keys = static_cast<uint32_t*>(at(L.s_keys));
    int32_t* s_ranks = static_cast<int32_t*>(at(L.s_ranks));
    uint32_t* m_keys = static_cast<uint32_t*>(at(L.m_keys));
    int32_t* m_ranks = static_cast<int32_t*>(at(L.m_ranks));
    uint32_t* m_sorted_keys = static_cast<uint32_t*>(at(L.m_sorted_keys));
    int32_t* m_sorted_ranks = static_cast<int32_t*>(at(L.m_sorted_ranks));
    int32_t* s_starts = static_cast<int32_t*>(at(L.s_starts));
    int32_t* m_starts = static_cast<int32_t*>(at(L.m_starts));
    const int64_t nb = sort_blocks(n);
    mover_count_kernel<<<(unsigned)nb, kSortBlock, 0, stream>>>(knew, prev_sorted, n, counts);
    count_launches(1);
    if ((st = launch_status()) != MPF_OK) return st;
    if ((st = scan_exclusive(counts, nb, sums, stream)) != MPF_OK) return st;
    split_kernel<<<(unsigned)nb, kSortBlock, 0, stream>>>(knew, prev_sorted, n, counts, nb, s_keys, s_ranks, m_keys,
                                                          m_ranks, totals);
    count_launches(1);
    if ((st = launch_status()) != MPF_OK) return st;
    // the movers by (key, rank): a stable sort of their keys carrying their ranks
    radix_sort(m_keys, m_ranks, n, totals, max_key, m_sorted_ranks, m_sorted_keys, at(L.radix), st, stream);
    if (st != MPF_OK) return st;
    const int block = 256;
    const int64_t blocks = std::min<int64_t>((n + 1 + block - 1) / block, (int64_t)sm_count() * 16);
    key_starts_kernel<<<(unsigned)blocks, block, 0, stream>>>(s_keys, n, totals + 1, nkeys, s_starts);
    key_starts_kernel<<<(unsigned)blocks, block, 0, stream>>>(m_sorted_keys, n, totals, nkeys, m_starts);
    merge_place_kernel<<<(unsigned)blocks, block, 0, stream>>>(s_keys, s_ranks, s_starts, m_sorted_keys,
                                                              m_sorted_ranks, m_starts, totals, n, nkeys, order,
                                                              sorted_out);
    count_launches(3);
    if ((st = launch_status()) != MPF_OK) return st;
    return tile_starts(sorted_out, n, num_tiles, cells, tile_start, stream);
}

int permute_rows(void* dst, int64_t ds, const void* src, int64_t ss, int64_t rows, const int32_t* order,
                 int64_t n, int dtype, cudaStream_t stream) {
    const int block = 256;
    const int64_t blocks = std::min<int64_t>((n + block - 1) / block, (int64_t)sm_count() * 16);
    if (dtype == MPF_F64)
        permute_rows_kernel<double><<<(unsigned)std::max<int64_t>(blocks, 1), block, 0, stream>>>(
            (double*)dst, ds, (const double*)src, ss, rows, order, n);
    else
        permute_rows_kernel<float><<<(unsigned)std::max<int64_t>(blocks, 1), block, 0, stream>>>(
            (float*)dst, ds, (const float*)src, ss, rows, order, n);
    count_launches(1);
    return launch_status();
}

int unpermute_rows(void* dst, int64_t ds, const void* src, int64_t ss, int64_t rows, const int32_t* order,
                   int64_t n, int dtype, cudaStream_t stream) {
    const int block = 256;
    const int64_t blocks = std::min<int64_t>((n + block - 1) / block, (int64_t)sm_count() * 16);
    if (dtype == MPF_F64)
        unpermute_rows_kernel<double><<<(unsigned)std::max<int64_t>(blocks, 1), block, 0, stream>>>(
            (double*)dst, ds, (const double*)src, ss, rows, order, n);
    else
        unpermute_rows_kernel<float><<<(unsigned)std::max<int64_t>(blocks, 1), block, 0, stream>>>(
            (float*)dst, ds, (const float*)src, ss, rows, order, n);
    count_launches(1);
    return launch_status();
}

// ------------------------------------------------- the sort without allocation --
//
// Some callers of the sort cannot call cudaMalloc: a host application that hands every
// byte of device memory to its own pool or arena at start-up and allows no allocation
// afterwards, or a real-time loop (a control or streaming step) that cannot take the
// implicit device synchronisation an allocation may bring. They sort through
// mpf_sort_by_tile_noalloc, whose workspace is this file-scope array instead of a buffer
// of theirs: every GPU that loads the library holds it (sort_layout(2^20).total, about
// 18 MB) until the process exits; it keeps the last call's contents (no part of the sort
// needs a starting value in it: every pass writes what it later reads); and calls that
// overlap on the GPU (on two streams, or from two host threads at once) race on it.

constexpr int64_t kNoAllocMaxMarkers = MPF_NOALLOC_MAX_MARKERS;
constexpr size_t kNoAllocBytes = sort_layout(kNoAllocMaxMarkers).total;

static __device__ __align__(256) unsigned char g_noalloc_sort_scratch[kNoAllocBytes];

// The device address of the array on the current device. In host code the array's name
// stands for a host-side shadow, not device memory, so kernels get this address instead:
// cudaGetSymbolAddress with the device current, once per device and context (kept with
// the context's identity, looked up again in a new context, e.g. after cudaDeviceReset),
// under a lock so that host threads may call concurrently. Null on a CUDA error.
static void* noalloc_scratch() {
    int device = 0;
    if (record_cuda_error(cudaGetDevice(&device)) != MPF_OK || device < 0 || device >= 64) return nullptr;
    static std::mutex lock;
    static unsigned long long owner[64] = {0};
    static void* address[64] = {nullptr};
    std::lock_guard<std::mutex> guard(lock);
    const unsigned long long ctx = current_context_id();
    if (!address[device] || ctx == 0 || owner[device] != ctx) {
        void* p = nullptr;
        if (record_cuda_error(cudaGetSymbolAddress(&p, g_noalloc_sort_scratch)) != MPF_OK) return nullptr;
        address[device] = p;
        owner[device] = current_context_id();
    }
    return address[device];
}

template int tile_keys<double>(int, int, int, const KeyArgs<double>&, cudaStream_t);
template int tile_keys<float>(int, int, int, const KeyArgs<float>&, cudaStream_t);

}  // namespace mpf

extern "C" int mpf_sort_by_tile_noalloc(int kind, int degree, int ndim, const void* positions, int64_t pos_stride,
                                        const void* values, int64_t val_stride, int64_t ncomp, int64_t n,
                                        const double* lower, const double* cell, const int32_t* num,
                                        const int32_t* code, const int32_t* tile, int within, uint32_t* keys,
                                        int32_t* order, int64_t* tile_start, int dtype, void* stream) {
    // every argument is checked before any CUDA call: a bad one returns its status and
    // touches neither the device nor the array
    if (n < 0) return MPF_ERR_ARGUMENT;
    if (n > mpf::kNoAllocMaxMarkers) return MPF_ERR_WORKSPACE;
    int64_t ntiles = 0, cells = 1;
    const int checked = mpf::check_sort_arguments(kind, degree, ndim, positions, pos_stride, values, val_stride,
                                                  ncomp, n, lower, cell, num, code, tile, within, keys, order,
                                                  tile_start, dtype, &ntiles, &cells);
    if (checked != MPF_OK) return checked;
    void* scratch = mpf::noalloc_scratch();
    if (!scratch) return MPF_ERR_CUDA;
    return mpf_sort_by_tile(kind, degree, ndim, positions, pos_stride, values, val_stride, ncomp, n, lower, cell,
                            num, code, tile, within, keys, order, tile_start, scratch, mpf::kNoAllocBytes, dtype,
                            stream);
}

// mpf_runs.cuh -- the lean tile-order gather and scatter.
//
// Both take a marker store sorted by cell tile (mpf_sort_by_tile, cells of a tile in
// row-major order) with its tile_start, periodic axes. A CTA takes an equal share of the
// live ranks and walks it piece by piece, a piece being the CTA's ranks of one tile;
// every thread plans the pieces itself (the same few broadcast reads of tile_start), so
// no thread waits for another's plan. Markers go to threads in stride (lane l of a warp,
// rank l of 32 consecutive ones): position and value reads and result writes are
// coalesced, and in a sorted store the lanes of a warp sit in a few neighbouring cells,
// so that the warp's instructions stay convergent. (A thread owning a contiguous range of
// ranks can reuse the stencil of consecutive markers of one cell from its registers, but
// the lanes of a warp change cell at different markers, and every such change is then
// issued for the whole warp: measured slower for the gather, and no faster for the
// scatter than the run scatter of mpf_nodes.cuh.)
//
// The ranks of the sentinel tile -- markers whose values were all zero when the store was
// sorted -- are gathered too, and deposited if their values are not zero, through global
// memory: the results never depend on the order or the values the store was sorted with.
#pragma once

namespace mpf {

// The pieces of a CTA's share of the live ranks: ranks [m, e) of tile `tile`, the tile's
// first anchor node blo[d] per axis; and the CTA's share [tail, tail_end) of the
// sentinel tile's ranks. Every thread of the CTA holds its own copy and advances it
// identically.
struct PieceWalk {
    int64_t m, m_end, e, tile;
    int blo[3];
    int64_t tail, tail_end;

    __device__ __forceinline__ void start(const int64_t* ts, int64_t ntiles, int64_t n) {
        const int64_t live = min(max(__ldg(ts + ntiles), (int64_t)0), n);
        const int64_t per = (live + gridDim.x - 1) / gridDim.x;
        m = min((int64_t)blockIdx.x * per, live);
        m_end = min(m + per, live);
        e = m;
        tile = -1;
        const int64_t dead = (n - live + gridDim.x - 1) / gridDim.x;
        tail = min(live + (int64_t)blockIdx.x * dead, n);
        tail_end = min(tail + dead, n);
    }

    // The next piece; false when the share is done.
    template <int NDIM>
    __device__ __forceinline__ bool next(const int64_t* ts, int64_t ntiles, const int* tiles, const int* tl) {
        m = e;
        if (m >= m_end) return false;
        tile = tile_of(ts, ntiles, tile, m);
        e = min(min(m_end, m + ((int64_t)1 << 30)), max(m + 1, __ldg(ts + tile + 1)));
        int rest = (int)tile;  // tiles number fewer than 2^31
#pragma unroll
        for (int d = NDIM - 1; d >= 0; --d) {
            const int c = rest % tiles[d];
            rest /= tiles[d];
            blo[d] = c * tl[d];
        }
        return true;
    }
};

// The ranks [first, end) of the sentinel tile deposited straight to global memory, a
// thread every `block` ranks: normally they add nothing (their values were zero).
template <typename T, int NDIM, int KIND, int P>
__device__ __forceinline__ void scatter_tail(const NodeArgs<T>& a, int64_t first, int64_t end, int block) {
    constexpr int S = P + 1;
#pragma unroll 1
    for (int64_t i = first + threadIdx.x; i < end; i += block) {
        const T v = a.values[i];
        if (v == T(0)) continue;
        T w[3][S];
        int base[3] = {0, 0, 0};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (d < NDIM) {
                base[d] = axis_stencil<T, KIND, P>(rel_from(a.pos[d * a.pos_stride + i], a.g, d), a.g.num[d],
                                                   PERIODIC, w[d]);
            } else {
#pragma unroll
                for (int z = 0; z < S; ++z) w[d][z] = T(z == 0);
            }
        }
        int64_t goff[3][S];
        global_offsets<NDIM, S>(base, a.g.num, a.g.code, a.g.ext, goff);
        const T vv[1] = {v};
        stencil_add<T, NDIM, S, 1, int64_t>(a.field_out, goff, w, 1, 0, vv);
    }
}

// ------------------------------------------------------------- the lean gather --
//
// The tile gather with the fewest instructions a marker: the tile's node box sits in
// shared memory with compile-time strides (TX, TY, TZ > 0), so the S^NDIM x NC reads of a
// marker are shared-memory loads at constant offsets from one base, and the stencil
// takes its fast path (no wrap, no clamp) for all but the markers next to a seam. With
// BUFFERS == 2 the box of the next piece is copied in (cp.async) while the current one
// is worked on, two boxes alternating; with one box the CTA waits for each copy, and the
// other CTAs of the SM keep it busy meanwhile.
template <typename T, int NDIM, int KIND, int P, int NC, int TX, int TY, int TZ, int BLOCK, int MINB,
          int BUFFERS>
__global__ void __launch_bounds__(BLOCK, MINB) gather_lean_kernel(const NodeArgs<T> a) {
    constexpr int S = P + 1;
    constexpr int H = P / 2;
    constexpr int L = NDIM - 1;
    const int t = threadIdx.x;
    const int tl[3] = {TX > 0 ? TX : a.tile[0], TY > 0 ? TY : a.tile[1], TZ > 0 ? TZ : a.tile[2]};
    // box extents and strides in nodes (compile-time constants for a fixed tile shape)
    const int ex0 = tl[0] + P, ex1 = NDIM > 1 ? tl[1] + P : 1, ex2 = NDIM > 2 ? tl[2] + P : 1;
    const int ex[3] = {ex0, ex1, ex2};
    const int st[3] = {NDIM == 3 ? ex1 * ex2 : (NDIM == 2 ? ex1 : 1), NDIM == 3 ? ex2 : (NDIM == 2 ? 1 : 0),
                       NDIM == 3 ? 1 : 0};
    const int box_nodes = ex0 * ex1 * ex2;
    T* boxes = reinterpret_cast<T*>(mpf_dynamic_smem);  // [BUFFERS][box_nodes * NC]
    int rows = 1;
#pragma unroll
    for (int d = 0; d < L; ++d) rows *= ex[d];
    const int rowlen = ex[L] * NC;
    const int sy = NDIM > 2 ? a.g.ext[2] : 1;
    const int sx = NDIM > 1 ? a.g.ext[1] * sy : 1;
    const int gstride[3] = {NDIM == 1 ? 1 : sx, NDIM == 2 ? 1 : sy, 1};
    // copies the box of the tile whose first anchor is blo into `box` (cp.async, one group):
    // rows along the last axis, a warp a row, entries (node, component)
    auto stage = [&](T* box, const int* blo) {
        const int lane = t & 31;
        for (int r = t >> 5; r < rows; r += BLOCK / 32) {
            int rest = r, prefix = 0;
#pragma unroll
            for (int d = L - 1; d >= 0; --d) {
                const int j = rest % ex[d];
                rest /= ex[d];
                prefix += map_node(blo[d] - H + j, a.g.num[d], PERIODIC) * gstride[d];
            }
            const int z0 = blo[L] - H;
            for (int e = lane; e < rowlen; e += 32) {
                const int j = e / NC;
                const int c = e - j * NC;
                const int node = prefix + map_node(z0 + j, a.g.num[L], PERIODIC) * gstride[L];
                cp_async<sizeof(T)>(box + r * rowlen + e, a.field_in + (int64_t)node * NC + c);
            }
        }
        cp_async_commit();
    };
    PieceWalk walk, ahead;
    walk.start(a.tile_start, a.ntiles, a.n);
    ahead = walk;
    bool have_next = ahead.next<NDIM>(a.tile_start, a.ntiles, a.tiles, tl);
    if (BUFFERS == 2 && have_next) stage(boxes, ahead.blo);
    int slot = 0;
#pragma unroll 1
    while (have_next) {
        walk = ahead;
        have_next = ahead.next<NDIM>(a.tile_start, a.ntiles, a.tiles, tl);
        const T* box = boxes + slot * box_nodes * NC;
        if constexpr (BUFFERS == 2) {
            // this piece's box has landed (the only group in flight) and every thread is
            // done with the other box: the next piece's box may go there
            cp_async_wait_all();
            __syncthreads();
            if (have_next) stage(boxes + (slot ^ 1) * box_nodes * NC, ahead.blo);
        } else {
            __syncthreads();  // every thread is done with the box
            stage(boxes, walk.blo);
            cp_async_wait_all();
            __syncthreads();  // everyone's copies have landed
        }
        const int64_t first = walk.m;
        const int count = (int)(walk.e - walk.m);
        T next[3] = {T(0), T(0), T(0)};
        if (t < count) {
#pragma unroll
            for (int d = 0; d < NDIM; ++d) next[d] = __ldg(a.pos + d * a.pos_stride + first + t);
        }
#pragma unroll 1
        for (int j = t; j < count; j += BLOCK) {
            const int64_t i = first + j;
            T x[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) x[d] = next[d];
            if (j + BLOCK < count) {
#pragma unroll
                for (int d = 0; d < NDIM; ++d) next[d] = __ldg(a.pos + d * a.pos_stride + i + BLOCK);
            }
            T w[3][S];
            int base[3] = {0, 0, 0};
            int at = 0;
            bool inside = true;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (d < NDIM) {
                    base[d] = axis_stencil<T, KIND, P>(rel_from(x[d], a.g, d), a.g.num[d], PERIODIC, w[d]);
                    const int off = wrap_index(base[d] + H - walk.blo[d], a.g.num[d]);
                    inside = inside && (unsigned)off < (unsigned)tl[d];
                    at += off * st[d];
                } else {
#pragma unroll
                    for (int z = 0; z < S; ++z) w[d][z] = T(z == 0);
                }
            }
            T acc[NC];
            if (inside) {
                // the sum in the order of stencil_sum: x outermost, the last axis innermost
                const T* p = box + at * NC;
                constexpr int SY = NDIM > 1 ? S : 1, SZ = NDIM > 2 ? S : 1;
#pragma unroll
                for (int c = 0; c < NC; ++c) acc[c] = T(0);
#pragma unroll
                for (int xa = 0; xa < S; ++xa) {
                    T sa[NC];
#pragma unroll
                    for (int c = 0; c < NC; ++c) sa[c] = T(0);
#pragma unroll
                    for (int yb = 0; yb < SY; ++yb) {
                        T sb[NC];
#pragma unroll
                        for (int c = 0; c < NC; ++c) sb[c] = T(0);
#pragma unroll
                        for (int ze = 0; ze < SZ; ++ze) {
                            const int node = xa * st[0] + (NDIM > 1 ? yb * st[1] : 0) + (NDIM > 2 ? ze : 0);
#pragma unroll
                            for (int c = 0; c < NC; ++c) {
                                const T v = p[node * NC + c];
                                if constexpr (NDIM > 2) sb[c] += w[2][ze] * v;
                                else sb[c] += v;
                            }
                        }
#pragma unroll
                        for (int c = 0; c < NC; ++c) {
                            if constexpr (NDIM > 1) sa[c] += w[1][yb] * sb[c];
                            else sa[c] += sb[c];
                        }
                    }
#pragma unroll
                    for (int c = 0; c < NC; ++c) acc[c] += w[0][xa] * sa[c];
                }
            } else {  // not this tile's marker: the field in global memory
                int off[3][S];
#pragma unroll
                for (int d = 0; d < 3; ++d)
#pragma unroll
                    for (int q = 0; q < S; ++q)
                        off[d][q] = d < NDIM ? map_node(base[d] + q, a.g.num[d], PERIODIC) * gstride[d] : 0;
                stencil_sum<T, NDIM, S, NC, true, int>(a.field_in, off, w, NC, 0, acc);
            }
#pragma unroll
            for (int c = 0; c < NC; ++c) a.result[c * a.res_stride + i] = acc[c];
        }
        if constexpr (BUFFERS == 2) slot ^= 1;
    }
    cp_async_wait_all();
    // the sentinel tile's ranks, from the field in global memory
#pragma unroll 1
    for (int64_t i = walk.tail + t; i < walk.tail_end; i += BLOCK) {
        T w[3][S];
        int off[3][S];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (d < NDIM) {
                const int b0 = axis_stencil<T, KIND, P>(rel_from(__ldg(a.pos + d * a.pos_stride + i), a.g, d),
                                                        a.g.num[d], PERIODIC, w[d]);
#pragma unroll
                for (int q = 0; q < S; ++q) off[d][q] = map_node(b0 + q, a.g.num[d], PERIODIC) * gstride[d];
            } else {
#pragma unroll
                for (int q = 0; q < S; ++q) {
                    w[d][q] = T(q == 0);
                    off[d][q] = 0;
                }
            }
        }
        T acc[NC];
        stencil_sum<T, NDIM, S, NC, true, int>(a.field_in, off, w, NC, 0, acc);
#pragma unroll
        for (int c = 0; c < NC; ++c) a.result[c * a.res_stride + i] = acc[c];
    }
}

// ------------------------------------------------------------ the lean scatter --
//
// The tile scatter with coherent lanes: every warp takes 32 consecutive ranks of a piece
// (read one step ahead), and each lane writes the SP stencil contributions of its marker
// into the warp's table in shared memory (row = lane). Then lane k < SP walks down column
// k, summing stencil point k of consecutive markers while their anchor stays the same,
// and adds each sum to the tile's box at a run end. Run ends are the same for every lane
// (a ballot of anchor changes), so the walk has no divergent branch, and one atomic
// instruction adds SP distinct nodes. A marker whose value is zero adds nothing; one whose
// anchor is not in the piece's tile adds to global memory directly. The box goes to the
// field with one global atomic per non-zero node at the end of the piece.
template <typename T, int NDIM, int KIND, int P, int TX, int TY, int TZ, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) scatter_lean_kernel(const NodeArgs<T> a) {
    constexpr int S = P + 1;
    constexpr int SY = NDIM > 1 ? S : 1;
    constexpr int SZ = NDIM > 2 ? S : 1;
    constexpr int SP = S * SY * SZ;
    static_assert(SP <= 32, "a stencil point per lane");
    constexpr int H = P / 2;
    constexpr int PITCH = SP + 2;  // rows an odd number of 8-byte pairs apart: a column spreads over the banks
    constexpr unsigned FULL = 0xffffffffu;
    const int t = threadIdx.x;
    const int lane = t & 31;
    const int tl[3] = {TX > 0 ? TX : a.tile[0], TY > 0 ? TY : a.tile[1], TZ > 0 ? TZ : a.tile[2]};
    int ex[3] = {1, 1, 1};
    tile_box_extents<NDIM, P>(tl, ex);
    const int box_entries = ex[0] * ex[1] * ex[2];
    T* box = reinterpret_cast<T*>(mpf_dynamic_smem);
    T* table = box + ((box_entries + 1) & ~1) + (t >> 5) * (32 * PITCH);
    for (int q = t; q < box_entries; q += BLOCK) box[q] = T(0);
    // box strides; stencil point k = (x SY + y) SZ + z of an anchor at box entry key is at key + off
    const int se = NDIM > 2 ? 1 : 0;
    const int sb = NDIM > 2 ? ex[2] : (NDIM > 1 ? 1 : 0);
    const int sa = NDIM > 2 ? ex[1] * ex[2] : (NDIM > 1 ? ex[1] : 1);
    const int st[3] = {sa, NDIM > 1 ? sb : 0, NDIM > 2 ? se : 0};
    const int kx = lane / (SY * SZ), ky = (lane / SZ) % SY, kz = lane % SZ;
    const int off = kx * sa + ky * sb + kz * se;
    PieceWalk walk;
    walk.start(a.tile_start, a.ntiles, a.n);
    __syncthreads();  // the box is zero
    // a lane's marker of a step (value and position), read one step ahead
    auto fetch = [&](int64_t m, int64_t end, T& v, T (&x)[3]) {
        v = T(0);
#pragma unroll
        for (int d = 0; d < 3; ++d) x[d] = T(0);
        if (m < end) {
            v = __ldg(a.values + m);
#pragma unroll
            for (int d = 0; d < NDIM; ++d) x[d] = __ldg(a.pos + d * a.pos_stride + m);
        }
    };
#pragma unroll 1
    while (walk.next<NDIM>(a.tile_start, a.ntiles, a.tiles, tl)) {
        T nv, nx[3];
        fetch(walk.m + (t & ~31) + lane, walk.e, nv, nx);
#pragma unroll 1
        for (int64_t first = walk.m + (t & ~31); first < walk.e; first += BLOCK) {
            const T v = nv;
            T x[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) x[d] = nx[d];
            fetch(first + BLOCK + lane, walk.e, nv, nx);
            int key = -1;  // the box anchor of the marker's stencil, -1: adds nothing here
            T contrib[SP];
#pragma unroll
            for (int q = 0; q < SP; ++q) contrib[q] = T(0);
            if (v != T(0)) {
                T w[3][S];
                int base[3] = {0, 0, 0};
                int k = 0;
                bool inside = true;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    if (d < NDIM) {
                        base[d] = axis_stencil<T, KIND, P>(rel_from(x[d], a.g, d), a.g.num[d], PERIODIC, w[d]);
                        const int o = wrap_index(base[d] + H - walk.blo[d], a.g.num[d]);
                        inside = inside && (unsigned)o < (unsigned)tl[d];
                        k += o * st[d];
                    } else {
#pragma unroll
                        for (int z = 0; z < S; ++z) w[d][z] = T(z == 0);
                    }
                }
                if (inside) {
                    key = k;
                    T wz[SZ];
#pragma unroll
                    for (int z = 0; z < SZ; ++z) wz[z] = NDIM > 2 ? w[2][z] * v : v;
#pragma unroll
                    for (int xa = 0; xa < S; ++xa)
#pragma unroll
                        for (int y = 0; y < SY; ++y) {
                            const T wxy = NDIM > 1 ? w[0][xa] * w[1][y] : w[0][xa];
#pragma unroll
                            for (int z = 0; z < SZ; ++z) contrib[(xa * SY + y) * SZ + z] = wxy * wz[z];
                        }
                } else {  // not this tile's marker: straight to global memory
                    int64_t goff[3][S];
                    global_offsets<NDIM, S>(base, a.g.num, a.g.code, a.g.ext, goff);
                    const T vv[1] = {v};
                    stencil_add<T, NDIM, S, 1, int64_t>(a.field_out, goff, w, 1, 0, vv);
                }
            }
            T* row = table + lane * PITCH;
#pragma unroll
            for (int q = 0; q < SP; ++q) row[q] = contrib[q];
            // a run ends at a lane whose next lane has another anchor (and at the last lane)
            const int following = __shfl_down_sync(FULL, key, 1);
            const unsigned ends = __ballot_sync(FULL, lane == 31 || following != key);
            __syncwarp();
            // four partial sums (rows r mod 4) keep the adds of a long run independent
            T acc[4] = {T(0), T(0), T(0), T(0)};
            const T* col = table + (lane < SP ? lane : 0);
#pragma unroll
            for (int r = 0; r < 32; ++r) {
                acc[r & 3] += col[r * PITCH];
                if (ends & (1u << r)) {
                    const int at = __shfl_sync(FULL, key, r);
                    if (lane < SP && at >= 0) atomicAdd(box + at + off, (acc[0] + acc[1]) + (acc[2] + acc[3]));
#pragma unroll
                    for (int q = 0; q < 4; ++q) acc[q] = T(0);
                }
            }
            __syncwarp();  // the table is read before the next step writes it
        }
        __syncthreads();  // every add of the piece is in the box
        int lo[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) lo[d] = walk.blo[d] - H;
        flush_clear_box<T, NDIM>(box, a.field_out, lo, ex, a.g);
        __syncthreads();  // the box is zero again
    }
    scatter_tail<T, NDIM, KIND, P>(a, walk.tail, walk.tail_end, BLOCK);
}

}  // namespace mpf

/*
 * mpifield_b200.h -- the C ABI of the B200 particle-grid backend (libmpifield_b200.so).
 *
 * One entry point per operation of mpifield's kernel convention (src/mpifield/weighting.py:
 * 22-38, src/mpifield/edges.py:23-31), with plain pointers and sizes. Every array lives
 * in device memory of the current CUDA device; every call is asynchronous on `stream`
 * (a cudaStream_t, NULL for the legacy default stream) and returns a status code
 * (MPF_OK or one of the MPF_ERR_* below); no call traps, synchronises or allocates.
 *
 * Conventions shared by the calls:
 *   - `ndim` is 1, 2 or 3. The grid is mpifield's BlockGrid.geometry
 *     (src/mpifield/_types.py:27-44) split into four arrays of `ndim` entries:
 *     `lower` (node 0), `cell` (node spacing), `num` (node count) and `code`
 *     (0 bounded, 1 periodic, 2 clamped knots). On a clamped axis an array of degree p
 *     holds num + p - 1 entries along it.
 *   - Marker arrays are row-major rows of `n` elements, `stride` elements apart (the
 *     (ndim, N) positions and (ncomp, N) values of the reference, which may have gaps
 *     between rows). A stride of 0 means n.
 *   - Grid arrays (fields, edge fields) are C-contiguous, components innermost:
 *     extent + (ncomp,).
 *   - `dtype` is MPF_F64 (double) or MPF_F32 (float); all the floating-point arrays of
 *     a call have that type.
 *   - `kind` picks the stencil arithmetic of the reference's weightings: MPF_LINEAR
 *     (linear_cell.cuh, degree 1, LINEAR), MPF_QUADRATIC (quadratic_cell.cuh, degree 2,
 *     QUADRATIC) or MPF_SPLINE (spline_cell.cuh, degree 0-3; CUBIC is degree 3).
 *   - `tuning` may be NULL (the autotuned defaults).
 */
#ifndef MPIFIELD_B200_H
#define MPIFIELD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Exported from the shared library, whatever the default visibility of the build. */
#if defined(__GNUC__)
#define MPF_API __attribute__((visibility("default")))
#else
#define MPF_API
#endif

/* Status codes. */
#define MPF_OK 0
#define MPF_ERR_ARGUMENT 1     /* a dimension, kind, degree, code or count out of range */
#define MPF_ERR_SHAPE 2        /* a stride or extent inconsistent with the sizes */
#define MPF_ERR_ALIGNMENT 3    /* a pointer not aligned to its element type */
#define MPF_ERR_WORKSPACE 4    /* a workspace smaller than the call needs */
#define MPF_ERR_CUDA 5         /* a CUDA launch or attribute call failed */
#define MPF_ERR_UNSUPPORTED 6  /* a combination this build does not provide */
#define MPF_ERR_TIMEOUT 7      /* a bounded wait gave up (serving queue) */

/* Stencil kinds. */
#define MPF_LINEAR 0
#define MPF_QUADRATIC 1
#define MPF_SPLINE 2

/* Element types. */
#define MPF_F64 0
#define MPF_F32 1

/* Paths (mpf_tuning.path). */
#define MPF_PATH_AUTO 0
#define MPF_PATH_DIRECT 1 /* global memory only, one marker per thread */
#define MPF_PATH_STAGED 2 /* shared-memory boxes per chunk of markers, else global */

typedef struct mpf_tuning {
    int32_t path;        /* MPF_PATH_* */
    int32_t block;       /* threads per CTA (multiple of 32, <= 256); 0: default */
    int32_t smem_bytes;  /* dynamic shared memory per CTA for a box; 0: default */
    int32_t ctas_per_sm; /* resident CTAs per SM the grid is sized for; 0: default */
    int32_t variant;     /* kernel variant; 0: the default for the shape (see mpf_gather, mpf_scatter) */
    int32_t wait_limit;  /* tries of a bounded wait on a bulk copy before the CTA gives up and raises
                            MPF_DEVICE_ERROR_WAIT; 0: the default (far beyond any copy of a working
                            device), < 0: none (gives up at once: a test of the give-up path) */
} mpf_tuning;

/* The library version, e.g. 10000 for 1.0.0. */
MPF_API int mpf_version(void);

/* The number of kernels this library has launched in the process (a diagnostic). */
MPF_API int64_t mpf_launch_count(void);

/* The name of the last CUDA error behind an MPF_ERR_CUDA status ("none" if there was none). */
MPF_API const char* mpf_last_error(void);

/*
 * The error bits the kernels of the current device raised since the last clear
 * (MPF_DEVICE_ERROR_WAIT: a bounded wait on a bulk copy gave up and the CTA left early,
 * so results of that launch are incomplete). Synchronous; clears them when `clear`.
 */
#define MPF_DEVICE_ERROR_WAIT 1u
MPF_API int mpf_device_errors(int clear, uint32_t* flags);

/* A static, human-readable name of a status code. */
MPF_API const char* mpf_status_string(int status);

/*
 * Node gather: result(c, i) = sum_k W_k(x_i) field(k, c), overwriting result.
 * Replaces the `gather(positions, field, result, *geometry)` kernels of mpifield's
 * weightings: gather_{linear,quadratic,spline}_{1,2,3}d (src/mpifield/weighting.py:
 * 233-250; e.g. src/mpifield/kernels/gather_spline_3d/gather_spline_3d_cuda.cu:11-53).
 * positions (ndim, n), field extent + (ncomp,), result (ncomp, n).
 */
MPF_API int mpf_gather(int kind, int degree, int ndim, const void* positions, int64_t pos_stride,
               int64_t n, const void* field, int64_t ncomp, void* result, int64_t res_stride,
               const double* lower, const double* cell, const int32_t* num, const int32_t* code,
               int dtype, const mpf_tuning* tuning, void* stream);

/*
 * mpf_scatter_deterministic for markers sorted by cell tile (tile and tile_start as for
 * mpf_scatter_tiles): the same bits as mpf_scatter_deterministic on the same arguments,
 * whatever the order of the markers. With one component and every axis periodic, each
 * tile's fixed-point sums are gathered in shared memory and added to the workspace once per
 * tile; otherwise mpf_scatter_deterministic's kernel runs. No counterpart in the reference.
 */
MPF_API int mpf_scatter_deterministic_tiles(int kind, int degree, int ndim, const void* positions,
                                            int64_t pos_stride, const void* values, int64_t val_stride,
                                            int64_t n, void* field, int64_t ncomp, const double* lower,
                                            const double* cell, const int32_t* num, const int32_t* code,
                                            const int32_t* tile, const int64_t* tile_start, void* workspace,
                                            size_t workspace_bytes, void* stream);

/*
 * mpf_gather for markers sorted by cell tile: positions in the rank order of
 * mpf_sort_by_tile (keys of the same kind, degree, geometry and `tile`), tile_start its
 * num_tiles + 2 starts (8-byte aligned device memory). The result is mpf_gather's, bit for
 * bit, whatever the order of the markers: a marker outside its rank's tile reads the field
 * in global memory. With every axis periodic, 1-3 components and the tile's node box within
 * a third of an SM's shared memory, each CTA copies a tile's box into shared memory once
 * and its markers read it there; other shapes, and tuning->variant != 0, run mpf_gather's
 * kernels. No counterpart in the reference (src/mpifield/weighting.py:233-250).
 */
MPF_API int mpf_gather_tiles(int kind, int degree, int ndim, const void* positions, int64_t pos_stride,
                             int64_t n, const void* field, int64_t ncomp, void* result, int64_t res_stride,
                             const double* lower, const double* cell, const int32_t* num,
                             const int32_t* code, const int32_t* tile, const int64_t* tile_start,
                             int dtype, const mpf_tuning* tuning, void* stream);

/*
 * Node scatter (deposit): field(k, c) += sum_i W_k(x_i) values(c, i). A marker whose
 * values are all zero deposits nothing and its position is not read.
 * Replaces `scatter(positions, values, field, *geometry)`: scatter_{linear,quadratic,
 * spline}_{1,2,3}d (src/mpifield/weighting.py:195-213; e.g.
 * src/mpifield/kernels/scatter_quadratic_3d/scatter_quadratic_3d_cuda.cu:12-60).
 */
MPF_API int mpf_scatter(int kind, int degree, int ndim, const void* positions, int64_t pos_stride,
                const void* values, int64_t val_stride, int64_t n, void* field, int64_t ncomp,
                const double* lower, const double* cell, const int32_t* num, const int32_t* code,
                int dtype, const mpf_tuning* tuning, void* stream);

/*
 * mpf_scatter for markers sorted by cell tile: positions and values in the rank order of
 * mpf_sort_by_tile (keys of the same kind, degree, geometry and `tile`, `within` either
 * way), tile_start its num_tiles + 2 starts (8-byte aligned device memory). The result
 * is mpf_scatter's on the same arguments up to the order of the floating-point adds,
 * whatever the order of the markers: a marker outside its rank's tile adds to global
 * memory directly. With one component, every axis periodic and a stencil of at most 27
 * points, each tile's share of the markers is summed in a shared-memory box known from
 * the tile (no per-chunk box search); other shapes, and tuning->variant != 0, run
 * mpf_scatter's kernels. No counterpart in the reference, which scatters in marker
 * order (src/mpifield/weighting.py:195-213).
 */
MPF_API int mpf_scatter_tiles(int kind, int degree, int ndim, const void* positions, int64_t pos_stride,
                              const void* values, int64_t val_stride, int64_t n, void* field, int64_t ncomp,
                              const double* lower, const double* cell, const int32_t* num,
                              const int32_t* code, const int32_t* tile, const int64_t* tile_start,
                              int dtype, const mpf_tuning* tuning, void* stream);

/* Bytes of the workspace of mpf_scatter_deterministic for a field of `entries` values
 * (the product of its extent and ncomp). */
MPF_API int mpf_scatter_deterministic_workspace_bytes(int64_t entries, size_t* bytes);

/*
 * The bit-reproducible scatter (FP64 only): field(k, c) += sum_i W_k(x_i) values(c, i)
 * as mpf_scatter computes it, every contribution summed as a pair of 64-bit fixed-point
 * integers (integer adds are associative), so the result has the same bits for every run,
 * launch shape and order of the markers; it differs from the FP64 atomic scatter by
 * rounding only (the fixed-point quantum is about 1e-19 of N max |values|). The values
 * must be finite. workspace: mpf_scatter_deterministic_workspace_bytes bytes, 16-byte
 * aligned, owned by the caller. No counterpart in the reference, whose scatters add
 * floating-point atomics in arrival order.
 */
MPF_API int mpf_scatter_deterministic(int kind, int degree, int ndim, const void* positions, int64_t pos_stride,
                                      const void* values, int64_t val_stride, int64_t n, void* field,
                                      int64_t ncomp, const double* lower, const double* cell, const int32_t* num,
                                      const int32_t* code, void* workspace, size_t workspace_bytes, void* stream);

/*
 * Position gradient of a gather contracted with a cotangent, for reverse mode:
 * grad(d, i) = sum_c cot(c, i) d/dx_d sum_k W_k(x_i) field(k, c), overwriting grad
 * (ndim, n). The weight derivatives follow B_p' = B_{p-1}(.+1/2) - B_{p-1}(.-1/2)
 * (src/mpifield/splines.py:9,77); zero where a bounded axis clamps the position. No
 * kernel of the reference computes it.
 */
MPF_API int mpf_gather_grad(int kind, int degree, int ndim, const void* positions, int64_t pos_stride,
                    int64_t n, const void* field, int64_t ncomp, const void* cotangent,
                    int64_t cot_stride, void* grad, int64_t grad_stride, const double* lower,
                    const double* cell, const int32_t* num, const int32_t* code, int dtype,
                    void* stream);

/*
 * Path deposit: edges += the current of `charges` (n,) moving from start to end
 * (ndim, n), edges extent + (ndim,). kind MPF_LINEAR with degree 1 is WHITNEY
 * (deposit_paths_{1,2,3}d, src/mpifield/kernels/deposit_paths_3d/deposit_paths_3d_cuda.cu:
 * 13-86); kind MPF_SPLINE with degree 1-3 is the spline-edge deposit of
 * QUADRATIC_EDGES / CUBIC_EDGES (deposit_paths_spline_{1,2,3}d,
 * deposit_paths_spline_3d_cuda.cu:14-130), replacing `deposit_paths(start, end, charges,
 * edges, *geometry)` (src/mpifield/edges.py:187-215). A path with zero charge or a
 * non-finite end deposits nothing.
 */
MPF_API int mpf_deposit_paths(int kind, int degree, int ndim, const void* start, int64_t start_stride,
                      const void* end, int64_t end_stride, const void* charges, int64_t n,
                      void* edges, const double* lower, const double* cell, const int32_t* num,
                      const int32_t* code, int dtype, const mpf_tuning* tuning, void* stream);

/*
 * Edge gather: result(a, i) = sum W_{k,a}(x_i) edges(k, a) / cell[a], overwriting
 * result (ndim, n). kind MPF_LINEAR (degree 1) is WHITNEY's gather_edges_{1,2,3}d,
 * MPF_SPLINE with degree 1-3 gather_edges_spline_{1,2,3}d (src/mpifield/edges.py:
 * 169-185).
 */
MPF_API int mpf_gather_edges(int kind, int degree, int ndim, const void* positions, int64_t pos_stride,
                     int64_t n, const void* edges, void* result, int64_t res_stride,
                     const double* lower, const double* cell, const int32_t* num,
                     const int32_t* code, int dtype, void* stream);

/*
 * Halo fill of one block: on every periodic axis the `halo` low halo layers take the
 * last `halo` owned layers and the high halo layers the first ones, axis by axis over
 * the whole stored extent (corners included); other axes are left alone. `stored` is
 * the extent with halos (owned + 2 halo per axis). Replaces Field.fill_halos on one
 * process (src/mpifield/field.py:601-613, mpiarray's update_halos).
 */
MPF_API int mpf_halo_fill(void* field, int ndim, const int32_t* stored, int64_t ncomp, int32_t halo,
                  const int32_t* periodic, int dtype, void* stream);

/*
 * Halo fold-back of one block after a deposit: on a periodic axis the high halo layers
 * are added onto the first owned layers and the low ones onto the last, then every
 * halo layer is zeroed (at a wall its values are dropped), axis by axis. Replaces
 * Field.exchange_halos on one process (src/mpifield/field.py:615-630, mpiarray's
 * accumulate_halos).
 */
MPF_API int mpf_halo_fold(void* field, int ndim, const int32_t* stored, int64_t ncomp, int32_t halo,
                  const int32_t* periodic, int dtype, void* stream);

/*
 * The face slabs of a halo exchange between ranks that each hold a block of a split field
 * (mpiarray's update_halos / accumulate_halos across processes, behind Field.fill_halos /
 * Field.exchange_halos, src/mpifield/field.py:601-630). pack copies the `halo` layers
 * [first, first + halo) along `axis` of the storage (all of the other axes, halos
 * included, and every component) into `buffer`, contiguous as [outer][halo][inner];
 * unpack writes the buffer into those layers, or adds it with `accumulate`.
 */
MPF_API int mpf_halo_pack(const void* field, int ndim, const int32_t* stored, int64_t ncomp, int32_t halo,
                  int axis, int32_t first, void* buffer, int dtype, void* stream);
MPF_API int mpf_halo_unpack(void* field, int ndim, const int32_t* stored, int64_t ncomp, int32_t halo,
                    int axis, int32_t first, const void* buffer, int accumulate, int dtype, void* stream);

/*
 * dst += deposit / node volume over a block of `num` owned nodes stored with `halo`
 * halo layers per axis (both arrays with the same storage), the volume being
 * prod(cell), halved on the first and last node of a bounded axis. Halo nodes of dst
 * are left unchanged. The last step of Field.deposit_density (src/mpifield/field.py:
 * 1182-1218, node_volumes :563-588).
 */
MPF_API int mpf_add_density(void* dst, const void* deposit, int ndim, const int32_t* num, int32_t halo,
                    int64_t ncomp, const double* cell, const int32_t* periodic, int dtype,
                    void* stream);

/*
 * Cell-tile sort. The tile of marker i is the anchor node of its stencil per axis
 * (LINEAR's left node, QUADRATIC's nearest node, the middle node of a spline stencil,
 * the cell on a clamped axis) divided by tile[d], row-major over the ceil(extent / tile)
 * tiles; keys[i] is that tile, or with `within` = 1 the tile followed by the anchor's
 * cell inside the tile (row-major): tile * prod(tile) + cell. With `values` non-NULL
 * ((ncomp, n) rows) a marker whose values are all zero gets the largest key (num_tiles,
 * times prod(tile) with `within`) without its position being read. order[j] is the
 * marker of rank j in the stable ascending order of the keys (equal to
 * numpy.argsort(keys, kind="stable")); tile_start (num_tiles + 2 entries) the first rank
 * of every tile, of the dead markers, and n at the end. `workspace` holds
 * `mpf_sort_workspace_bytes` bytes of device memory, 256-byte aligned. No reference
 * kernel sorts (picnic's sort_by_cell is external,
 * src/mpifield/kernels/scatter_linear_3d/scatter_linear_3d_pyccel.py:11-12).
 */
MPF_API int mpf_sort_workspace_bytes(int64_t n, int64_t num_tiles, size_t* bytes);
MPF_API int mpf_sort_by_tile(int kind, int degree, int ndim, const void* positions, int64_t pos_stride,
                     const void* values, int64_t val_stride, int64_t ncomp, int64_t n,
                     const double* lower, const double* cell, const int32_t* num,
                     const int32_t* code, const int32_t* tile, int within, uint32_t* keys,
                     int32_t* order, int64_t* tile_start, void* workspace, size_t workspace_bytes,
                     int dtype, void* stream);

/*
 * k-forms of B-spline degree 1-3 (form 1 .. ndim): component c of a `form`-form weighs
 * the degree-`degree` B-spline along the axes it is not staggered on and the edge
 * functions B_(degree-1)(r - k - 1/2) (existing edges only) along those it is -- an edge
 * (form 1) along its direction, a face of 3D (form 2) across its normal, the top form
 * (form ndim) along every axis; positions are clamped on bounded and clamped axes. The
 * field is extent + (ncomp,) with ncomp = ndim choose form (extent num + degree - 1 on a
 * clamped axis). mpf_gather_forms overwrites result (ncomp, n); mpf_scatter_forms adds
 * values (ncomp, n) into the field, skipping markers whose values are all zero before
 * reading their positions. Replace gather_forms_spline_{1,2,3}d and
 * scatter_forms_spline_{1,2,3}d (src/mpifield/kernels/spline_forms.py:85-138, used by
 * the faces and cells of src/mpifield/splines.py:185-205).
 */
MPF_API int mpf_gather_forms(int degree, int form, int ndim, const void* positions, int64_t pos_stride, int64_t n,
                             const void* field, int64_t ncomp, void* result, int64_t res_stride,
                             const double* lower, const double* cell, const int32_t* num, const int32_t* code,
                             int dtype, void* stream);
MPF_API int mpf_scatter_forms(int degree, int form, int ndim, const void* positions, int64_t pos_stride,
                              const void* values, int64_t val_stride, int64_t n, void* field, int64_t ncomp,
                              const double* lower, const double* cell, const int32_t* num,
                              const int32_t* code, int dtype, void* stream);

/*
 * The cell-tile sort of a store that is kept sorted: the markers' keys as in
 * mpf_sort_by_tile, computed from the positions (and values) in the store's current
 * order; order[j] is the current rank of the marker of new rank j in the stable
 * ascending order of the keys (numpy.argsort(keys, kind="stable"), bit for bit), tile_start
 * as in mpf_sort_by_tile, and sorted_keys[j] the key of rank j -- what the next call takes
 * as prev_sorted_keys once the store's arrays have been permuted by order
 * (mpf_permute_rows). With prev_sorted_keys NULL it is a full sort; with the sorted keys
 * this call returned for the store before its markers moved, only the markers whose key
 * changed are sorted and merged with the others (the order is the same): after a step
 * in which markers move less than a cell, a fraction of the full sort's cost.
 * prev_sorted_keys must be exactly those keys, and must not be sorted_keys. `workspace`
 * holds `mpf_resort_workspace_bytes` bytes of device memory, 256-byte aligned. No
 * reference kernel sorts (picnic's sort_by_cell keeps the reference's stores sorted,
 * src/mpifield/kernels/scatter_linear_3d/scatter_linear_3d_pyccel.py:11-12).
 */
MPF_API int mpf_resort_workspace_bytes(int kind, int degree, int ndim, const int32_t* num, const int32_t* code,
                                       const int32_t* tile, int within, int64_t n, size_t* bytes);
MPF_API int mpf_resort_by_tile(int kind, int degree, int ndim, const void* positions, int64_t pos_stride,
                               const void* values, int64_t val_stride, int64_t ncomp, int64_t n,
                               const double* lower, const double* cell, const int32_t* num,
                               const int32_t* code, const int32_t* tile, int within,
                               const uint32_t* prev_sorted_keys, uint32_t* sorted_keys, int32_t* order,
                               int64_t* tile_start, void* workspace, size_t workspace_bytes, int dtype,
                               void* stream);

/*
 * mpf_sort_by_tile without a workspace argument and without any allocation. No
 * counterpart in the reference. It is for callers that cannot call cudaMalloc: a host
 * application that gives all device memory to its own pool or arena at start-up and
 * allows no allocation afterwards, or a real-time loop that cannot take the implicit
 * device synchronisation an allocation may bring. The workspace is a fixed array inside
 * the library (about 18 MB on every GPU that loads it, held until the process exits), so
 * n is at most MPF_NOALLOC_MAX_MARKERS; a larger n returns MPF_ERR_WORKSPACE and a bad
 * argument its status, both before any CUDA call. The array's device address is looked
 * up with cudaGetSymbolAddress on the first call on a device (with that device current,
 * again in a new context); that first call may also load the library's device code, so
 * make it before any stream capture on that device. Safe to call from several host
 * threads, but all calls share the array: calls that overlap on the GPU race, so order
 * them on one stream or with events. The array keeps the last call's contents; no part
 * of the sort needs a starting value in it.
 */
#define MPF_NOALLOC_MAX_MARKERS (1 << 20)
MPF_API int mpf_sort_by_tile_noalloc(int kind, int degree, int ndim, const void* positions,
                                     int64_t pos_stride, const void* values, int64_t val_stride,
                                     int64_t ncomp, int64_t n, const double* lower,
                                     const double* cell, const int32_t* num, const int32_t* code,
                                     const int32_t* tile, int within, uint32_t* keys,
                                     int32_t* order, int64_t* tile_start, int dtype, void* stream);

/* The number of tiles of a grid for mpf_sort_by_tile, into *num_tiles. */
MPF_API int mpf_num_tiles(int kind, int degree, int ndim, const int32_t* num, const int32_t* code,
                  const int32_t* tile, int64_t* num_tiles);

/*
 * dst(r, j) = src(r, order[j]) for r < rows, j < n: a marker array permuted into sorted
 * order (rows of n elements, strides in elements). dst and src must not overlap. An
 * order entry outside [0, n) reads nothing and gives NaN.
 */
MPF_API int mpf_permute_rows(void* dst, int64_t dst_stride, const void* src, int64_t src_stride,
                     int64_t rows, const int32_t* order, int64_t n, int dtype, void* stream);

/*
 * dst(r, order[j]) = src(r, j): the inverse of mpf_permute_rows, returning results computed
 * in sorted order to the markers' own order. An order entry outside [0, n) writes nothing.
 */
MPF_API int mpf_unpermute_rows(void* dst, int64_t dst_stride, const void* src, int64_t src_stride,
                               int64_t rows, const int32_t* order, int64_t n, int dtype, void* stream);

/* ------------------------------------------------------------------ serving batches --
 *
 * One launch runs many small FP64 gather and scatter requests. The requests sit in a
 * device table of mpf_batch_request entries; each is cut into tiles of
 * header->tile_markers markers, and persistent CTAs take tiles from the counter
 * header->next_tile until header->tiles are done. The last CTA to finish sets the
 * counter back to zero, so a launch captured once in a CUDA graph replays with new table
 * contents (the table, the header and their sizes live in device memory the caller
 * owns). No counterpart in the reference, whose kernels run one call per launch; each
 * request's arithmetic is that of mpf_gather / mpf_scatter on the same arguments (global
 * memory, one marker per thread, scatter adds as FP64 atomics).
 */
#define MPF_OP_GATHER 0
#define MPF_OP_SCATTER 1
#define MPF_OP_PATHS 2 /* path deposit: positions = start, field = end (rows out_stride apart),
                          values = charges (n,), out = the edge field added into */

typedef struct mpf_batch_request {
    int32_t op, kind, degree, ndim;
    int32_t ncomp, reserved;
    int64_t n;
    int64_t first_tile;          /* tiles of the requests before this one in the table */
    const double* positions;     /* (ndim, n), rows pos_stride apart */
    int64_t pos_stride;
    const double* values;        /* scatter: (ncomp, n), rows val_stride apart */
    int64_t val_stride;
    const double* field;         /* gather: extent + (ncomp,) */
    double* out;                 /* gather: result (ncomp, n) rows out_stride apart; scatter: the field */
    int64_t out_stride;
    double lower[3], cell[3], inv[3];
    int32_t num[3], code[3], ext[3];
    int32_t pad;
} mpf_batch_request;

typedef struct mpf_batch_header {
    int64_t requests;      /* entries of the table */
    int64_t tiles;         /* tiles of all requests (the last entry's first_tile + its tiles) */
    int64_t tile_markers;  /* markers per tile */
    int64_t next_tile;     /* the work counter: zero before a launch, zero again after it */
    int64_t finished;      /* CTAs done (the last one resets both counters) */
    int64_t pad[3];
} mpf_batch_header;

/* sizeof(mpf_batch_request), for bindings that lay the table out themselves. */
MPF_API int64_t mpf_batch_request_size(void);

/*
 * Checks one request as mpf_gather / mpf_scatter / mpf_deposit_paths would and fills *r
 * (host memory) for the table; first_tile is left for the caller. op MPF_OP_GATHER: values
 * ignored, out is the result; MPF_OP_SCATTER: field ignored, out is the field added into;
 * MPF_OP_PATHS (kind MPF_LINEAR degree 1 WHITNEY, MPF_SPLINE degree 1-3 spline edges):
 * positions the starts, field the ends (rows out_stride apart), values the n charges, out
 * the edge field extent + (ndim,) added into, ncomp ignored.
 */
MPF_API int mpf_batch_request_init(mpf_batch_request* r, int op, int kind, int degree, int ndim,
                                   const void* positions, int64_t pos_stride, const void* values,
                                   int64_t val_stride, int64_t n, const void* field, void* out,
                                   int64_t out_stride, int ncomp, const double* lower, const double* cell,
                                   const int32_t* num, const int32_t* code);

/*
 * The batch launch: table and header in device memory; grid CTAs of block threads
 * (0: 2 CTAs per SM of 256 threads). Reads the sizes from the header when it runs.
 */
MPF_API int mpf_batch_launch(const mpf_batch_request* table, mpf_batch_header* header, int grid, int block,
                             void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MPIFIELD_B200_H */

// mpf_internal.h -- argument blocks and launch entry points shared by the .cu files.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace mpf {

// The grid of a block, as the kernels see it (src/mpifield/_types.py:27-44): the
// position of node 0, the node spacing, the node count and the boundary code per axis,
// and the array extent (num, or num + P - 1 on a clamped axis).
template <typename T> struct Grid {
    T lower[3];
    T cell[3];
    T inv[3];  // RN(1 / cell), for the correctly rounded (x - lower) / cell
    int num[3];
    int code[3];
    int ext[3];
    int pow2[3];  // 1: cell is a power of two, so (x - lower) * inv is the quotient exactly
};

// A node gather, scatter or position-gradient gather.
template <typename T> struct NodeArgs {
    Grid<T> g;
    const T* pos;        // (ndim, n), rows pos_stride apart
    int64_t pos_stride;
    const T* values;     // scatter: (ncomp, n); gradient: the cotangent (ncomp, n)
    int64_t val_stride;
    const T* field_in;   // gather / gradient: ext + (ncomp,), C-contiguous
    T* field_out;        // scatter
    T* result;           // gather: (ncomp, n); gradient: (ndim, n)
    int64_t res_stride;
    int64_t n;
    int ncomp;
    int capacity;        // shared-memory box capacity, in elements of T
    int force_global;    // 1: never stage (the direct path), for tests and unsorted input
    int bulk;            // 1: positions are 16-byte aligned rows, prefetched by bulk copies
    unsigned* error;     // device word of MPF_DEVICE_ERROR_* bits
    int wait_limit;      // tries of a bounded wait before it gives up (0: gives up at once)
    // a scatter of markers sorted by cell tile (mpf_sort_by_tile); tile_start null otherwise
    const int64_t* tile_start;  // first rank of every tile, then of the sentinel tile
    int64_t ntiles;
    int tile[3];         // anchor nodes per tile, per axis
    int tiles[3];        // tiles per axis
};

// The tries of a bounded wait on a bulk copy before a CTA gives up (about 0.1 s of
// polling): far beyond any copy of a working device.
constexpr int kDefaultWaitLimit = 1 << 22;

// The tuning of one launch (the autotuned table supplies it; zero fields take defaults).
struct Tuning {
    int path;        // 0 auto, 1 direct (global memory only), 2 staged boxes
    int block;       // threads per CTA
    int smem_bytes;  // dynamic shared memory per CTA for the box
    int ctas_per_sm; // resident CTAs per SM the grid is sized for
    int variant;     // kernel variant, 0 the default for the shape
    int wait_limit;  // tries of a bounded wait: 0 the default, < 0 none (gives up at once)
};

template <typename T, int NDIM>
int node_launch(int op, int kind, int degree, const NodeArgs<T>& a, const Tuning& t, cudaStream_t stream);
template <typename T>
int launch_gather(int kind, int degree, int ndim, const NodeArgs<T>& a, const Tuning& t,
                  cudaStream_t stream);
template <typename T>
int launch_scatter(int kind, int degree, int ndim, const NodeArgs<T>& a, const Tuning& t,
                   cudaStream_t stream);
template <typename T>
int launch_gather_grad(int kind, int degree, int ndim, const NodeArgs<T>& a, cudaStream_t stream);

// A path deposit or an edge gather.
template <typename T> struct PathArgs {
    Grid<T> g;
    const T* start;
    int64_t start_stride;
    const T* end;
    int64_t end_stride;
    const T* charges;
    const T* pos;  // edge gather
    int64_t pos_stride;
    const T* edges_in;
    T* edges_out;
    T* result;
    int64_t res_stride;
    int64_t n;
    int capacity;          // deposit: shared-memory edge box, elements of T (0: global atomics only)
    int paths_per_thread;  // deposit: paths a thread takes per chunk
};

// The cell-tile keys of the markers.
template <typename T> struct KeyArgs {
    Grid<T> g;
    const T* pos;
    int64_t pos_stride;
    const T* values;
    int64_t val_stride;
    int64_t ncomp;
    int64_t n;
    int tile[3];
    int64_t ntiles[3];
    int within;  // 1: the key continues with the cell inside the tile
    uint32_t sentinel;
    uint32_t* keys;
};

template <typename T>
int launch_deposit_paths(int kind, int degree, int ndim, PathArgs<T> a, const Tuning& t, cudaStream_t stream);
template <typename T>
int launch_gather_edges(int kind, int degree, int ndim, const PathArgs<T>& a, cudaStream_t stream);

// Pack (mode 0) the layers [first, first + h) along `axis` into buf, unpack buf into them
// (mode 1) or add buf onto them (mode 2).
int halo_slab(void* f, void* buf, int ndim, const int32_t* stored, int64_t ncomp, int h, int axis, int first,
              int mode, int dtype, cudaStream_t stream);
int halo_fill(void* f, int ndim, const int32_t* stored, int64_t ncomp, int h, const int32_t* periodic,
              int dtype, cudaStream_t stream);
int halo_fold(void* f, int ndim, const int32_t* stored, int64_t ncomp, int h, const int32_t* periodic,
              int dtype, cudaStream_t stream);
int add_density(void* dst, const void* dep, int ndim, const int32_t* num, int h, int64_t ncomp,
                const double* cell, const int32_t* periodic, int dtype, cudaStream_t stream);

template <typename T>
int tile_keys(int kind, int degree, int ndim, const KeyArgs<T>& a, cudaStream_t stream);
size_t sort_workspace_bytes(int64_t n);
int sort_keys(const uint32_t* keys, int64_t n, int64_t num_tiles, int64_t cells, int32_t* order,
              int64_t* tile_start, void* workspace, cudaStream_t stream);
int permute_rows(void* dst, int64_t ds, const void* src, int64_t ss, int64_t rows, const int32_t* order,
                 int64_t n, int dtype, cudaStream_t stream);
size_t resort_workspace_bytes(int64_t n, int64_t nkeys);
uint32_t* resort_keys_buffer(void* workspace, int64_t n);
int resort_keys(int64_t n, int64_t num_tiles, int64_t cells, const uint32_t* prev_sorted, uint32_t* sorted_out,
                int32_t* order, int64_t* tile_start, void* workspace, cudaStream_t stream);

int unpermute_rows(void* dst, int64_t ds, const void* src, int64_t ss, int64_t rows, const int32_t* order,
                   int64_t n, int dtype, cudaStream_t stream);

int sm_count();

int compute_keys(int kind, int degree, int ndim, const void* positions, int64_t pos_stride, const void* values,
                 int64_t val_stride, int64_t ncomp, int64_t n, const double* lower, const double* cell,
                 const int32_t* num, const int32_t* code, const int32_t* tile, int within, int64_t ntiles,
                 int64_t cells, uint32_t* keys, int dtype, cudaStream_t s);

int check_sort_arguments(int kind, int degree, int ndim, const void* positions, int64_t& pos_stride,
                         const void* values, int64_t& val_stride, int64_t ncomp, int64_t n, const double* lower,
                         const double* cell, const int32_t* num, const int32_t* code, const int32_t* tile,
                         int within, const uint32_t* keys, const int32_t* order, const int64_t* tile_start,
                         int dtype, int64_t* ntiles_out, int64_t* cells_out);
}  // namespace mpf
struct mpf_batch_request;
struct mpf_batch_header;
namespace mpf {
// The bit-reproducible scatter (mpf_deterministic.cu).
size_t det_workspace_bytes(int64_t entries);
int launch_scatter_deterministic(int kind, int degree, int ndim, const NodeArgs<double>& a, int64_t entries,
                                 void* workspace, cudaStream_t s);
// The serving batch launch (mpf_batch.cu).
int launch_batch(const mpf_batch_request* table, mpf_batch_header* header, int grid, int block,
                 cudaStream_t stream);

// Counts kernel launches of this library (read by mpf_launch_count).
void count_launches(int k);

// The device word the kernels report MPF_DEVICE_ERROR_* bits in (per device), or NULL.
unsigned* device_error_word();

// A number that identifies the CUDA context current on the calling thread (the driver's
// cuCtxGetId), or 0 when there is none or the driver does not tell. Addresses of
// __device__ variables are cached per device and per this identity, so that a cache
// never outlives its context (cudaDeviceReset makes a new one).
unsigned long long current_context_id();

// MPF_OK after a launch, or MPF_ERR_CUDA with the CUDA error recorded for mpf_last_error.
int launch_status();
int record_cuda_error(cudaError_t e);

}  // namespace mpf

// mpf_capi.cu -- the extern "C" entry points of include/mpifield_b200.h: argument checks
// (the ValueErrors the reference raises in Python before a kernel, src/mpifield/
// weighting.py:91-97,156-164 and edges.py:145-167,210-213, become status codes here) and
// the dispatch to the typed launchers.
#include <atomic>
#include <mutex>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "mpf_internal.h"
#include "mpf_stencil.cuh"
#include "mpifield_b200.h"

namespace mpf {

static std::atomic<long long> g_launches{0};

void count_launches(int k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

static std::atomic<int> g_last_error{0};

int record_cuda_error(cudaError_t e) {
    if (e == cudaSuccess) return MPF_OK;
    g_last_error.store((int)e, std::memory_order_relaxed);
    return MPF_ERR_CUDA;
}

int launch_status() { return record_cuda_error(cudaGetLastError()); }

// The driver's cuCtxGetCurrent and cuCtxGetId, reached through the runtime (the library
// does not link the driver library itself); null where the driver lacks them.
using CtxGetCurrentFn = int (*)(void** ctx);
using CtxGetIdFn = int (*)(void* ctx, unsigned long long* id);
static std::once_flag g_ctx_once;
static CtxGetCurrentFn g_ctx_get_current = nullptr;
static CtxGetIdFn g_ctx_get_id = nullptr;

unsigned long long current_context_id() {
    std::call_once(g_ctx_once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult found;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &found) == cudaSuccess &&
            found == cudaDriverEntryPointSuccess)
            g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
        fn = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &found) == cudaSuccess &&
            found == cudaDriverEntryPointSuccess)
            g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(fn);
        cudaGetLastError();  // a failed query leaves no error behind for the next launch
    });
    if (!g_ctx_get_current || !g_ctx_get_id) return 0;
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (g_ctx_get_current(&ctx) != 0 || !ctx || g_ctx_get_id(ctx, &id) != 0) return 0;
    return id;
}

// Bits the kernels raise when a bounded wait gives up (one word per device).
static __device__ unsigned g_device_errors;

// The word's device address, looked up with cudaGetSymbolAddress once per device and
// context (with that device current) and kept with the context's identity; a new context
// (after cudaDeviceReset) or an unknown identity looks it up again. Safe to call from
// several host threads.
unsigned* device_error_word() {
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) return nullptr;
    static std::mutex lock;
    static unsigned long long owner[64] = {0};
    static unsigned* words[64] = {nullptr};
    std::lock_guard<std::mutex> guard(lock);
    const unsigned long long ctx = current_context_id();
    if (!words[device] || ctx == 0 || owner[device] != ctx) {
        void* p = nullptr;
        if (record_cuda_error(cudaGetSymbolAddress(&p, g_device_errors)) != MPF_OK) return nullptr;
        words[device] = static_cast<unsigned*>(p);
        owner[device] = current_context_id();
    }
    return words[device];
}

int sm_count() {
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return 148;
    static int cached[64] = {0};
    if (device < 0 || device >= 64) return 148;
    if (cached[device] == 0) {
        int count = 0;
        if (cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || count <= 0)
            count = 148;
        cached[device] = count;
    }
    return cached[device];
}

static bool valid_kind(int kind, int degree) {
    if (kind == MPF_LINEAR) return degree == 1;
    if (kind == MPF_QUADRATIC) return degree == 2;
    if (kind == MPF_SPLINE) return degree >= 0 && degree <= 3;
    return false;
}

// The checks of a grid: dimensions, positive finite spacing, node counts (two at least
// on bounded and clamped axes, whose stencils take the last cell), codes, and clamped
// axes only for spline stencils of degree >= 1 (src/mpifield/weighting.py:91-97).
static int check_grid(int kind, int degree, int ndim, const double* lower, const double* cell,
                      const int32_t* num, const int32_t* code) {
    if (ndim < 1 || ndim > 3) return MPF_ERR_ARGUMENT;
    if (!lower || !cell || !num || !code) return MPF_ERR_ARGUMENT;
    for (int d = 0; d < ndim; ++d) {
        if (!std::isfinite(lower[d]) || !std::isfinite(cell[d]) || cell[d] == 0.0) return MPF_ERR_ARGUMENT;
        if (code[d] < 0 || code[d] > 2) return MPF_ERR_ARGUMENT;
        if (num[d] < 1 || num[d] > (1 << 28)) return MPF_ERR_ARGUMENT;
        if (code[d] != PERIODIC && num[d] < 2) return MPF_ERR_ARGUMENT;
        if (code[d] == CLAMPED && (kind != MPF_SPLINE || degree < 1)) return MPF_ERR_UNSUPPORTED;
    }
    return MPF_OK;
}

// Whether c is a power of two whose reciprocal is a normal number of T: then RN(1 / c) is
// exact and a / c = a * (1 / c) for every a, rounding included.
template <typename T> static bool exact_reciprocal(T c) {
    int e = 0;
    const T m = std::frexp(c, &e);
    const T r = T(1) / c;
    return m == T(0.5) && std::isnormal(r) && std::isnormal(c);
}

template <typename T>
static Grid<T> make_grid(int ndim, int degree, const double* lower, const double* cell, const int32_t* num,
                         const int32_t* code) {
    Grid<T> g;
    for (int d = 0; d < 3; ++d) {
        const bool on = d < ndim;
        g.lower[d] = on ? (T)lower[d] : T(0);
        g.cell[d] = on ? (T)cell[d] : T(1);
        g.inv[d] = T(1) / g.cell[d];  // host IEEE division in T: RN(1 / cell)
        g.pow2[d] = exact_reciprocal<T>(g.cell[d]) ? 1 : 0;
        g.num[d] = on ? num[d] : 1;
        g.code[d] = on ? code[d] : PERIODIC;
        g.ext[d] = on ? axis_extent(num[d], code[d], degree) : 1;
    }
    return g;
}

static bool aligned(const void* p, int dtype) {
    const uintptr_t size = dtype == MPF_F64 ? 8 : 4;
    return (reinterpret_cast<uintptr_t>(p) % size) == 0;
}

static int check_rows(const void* p, int64_t& stride, int64_t n, int rows, int dtype) {
    if (stride == 0) stride = n;
    if (stride < n || stride < 0) return MPF_ERR_SHAPE;
    if (n > 0 && rows > 0) {
        if (!p) return MPF_ERR_ARGUMENT;
        if (!aligned(p, dtype)) return MPF_ERR_ALIGNMENT;
    }
    return MPF_OK;
}

static Tuning tuning_of(const mpf_tuning* t) {
    Tuning u{0, 0, 0, 0, 0, 0};
    if (t) {
        u.variant = t->variant;
        u.path = t->path;
        u.block = t->block;
        u.smem_bytes = t->smem_bytes;
        u.ctas_per_sm = t->ctas_per_sm;
        u.wait_limit = t->wait_limit;
    }
    return u;
}

template <typename T>
static NodeArgs<T> node_args(int ndim, int degree, const double* lower, const double* cell, const int32_t* num,
                             const int32_t* code) {
    NodeArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    a.g = make_grid<T>(ndim, degree, lower, cell, num, code);
    return a;
}

// The tile-order fields of a launch (mpf_gather_tiles, mpf_scatter_tiles).
template <typename T>
static void set_tiles(NodeArgs<T>& a, int ndim, int degree, const int32_t* num, const int32_t* code,
                      const int32_t* tile, const int64_t* tile_start, int64_t ntiles) {
    a.tile_start = tile_start;
    a.ntiles = ntiles;
    for (int d = 0; d < ndim; ++d) {
        a.tile[d] = tile[d];
        a.tiles[d] = (int)((axis_extent(num[d], code[d], degree) + tile[d] - 1) / tile[d]);
    }
}

}  // namespace mpf

using namespace mpf;

#define MPF_TRY(expr)                     \
    do {                                  \
        const int status_ = (expr);       \
        if (status_ != MPF_OK) return status_; \
    } while (0)

extern "C" {

int mpf_version(void) { return 10000; }

int64_t mpf_launch_count(void) { return (int64_t)g_launches.load(std::memory_order_relaxed); }

int mpf_device_errors(int clear, uint32_t* flags) {
    if (!flags) return MPF_ERR_ARGUMENT;
    unsigned value = 0;
    if (record_cuda_error(cudaMemcpyFromSymbol(&value, g_device_errors, sizeof(value))) != MPF_OK) return MPF_ERR_CUDA;
    *flags = value;
    if (clear && value) {
        const unsigned zero = 0;
        if (record_cuda_error(cudaMemcpyToSymbol(g_device_errors, &zero, sizeof(zero))) != MPF_OK) return MPF_ERR_CUDA;
    }
    return MPF_OK;
}

const char* mpf_last_error(void) {
    const int e = g_last_error.load(std::memory_order_relaxed);
    return e == 0 ? "none" : cudaGetErrorName((cudaError_t)e);
}

const char* mpf_status_string(int status) {
    switch (status) {
        case MPF_OK: return "ok";
        case MPF_ERR_ARGUMENT: return "invalid argument";
        case MPF_ERR_SHAPE: return "inconsistent shape or stride";
        case MPF_ERR_ALIGNMENT: return "misaligned pointer";
        case MPF_ERR_WORKSPACE: return "workspace too small";
        case MPF_ERR_CUDA: return "CUDA error";
        case MPF_ERR_UNSUPPORTED: return "unsupported combination";
        case MPF_ERR_TIMEOUT: return "timed out";
    }
    return "unknown status";
}

int mpf_gather(int kind, int degree, int ndim, const void* positions, int64_t pos_stride, int64_t n,
               const void* field, int64_t ncomp, void* result, int64_t res_stride, const double* lower,
               const double* cell, const int32_t* num, const int32_t* code, int dtype,
               const mpf_tuning* tuning, void* stream) {
    if (!valid_kind(kind, degree) || (dtype != MPF_F64 && dtype != MPF_F32)) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_grid(kind, degree, ndim, lower, cell, num, code));
    if (n < 0 || ncomp < 1 || ncomp > (1 << 20)) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_rows(positions, pos_stride, n, ndim, dtype));
    MPF_TRY(check_rows(result, res_stride, n, (int)ncomp, dtype));
    if (n == 0) return MPF_OK;
    if (!field) return MPF_ERR_ARGUMENT;
    if (!aligned(field, dtype)) return MPF_ERR_ALIGNMENT;
    const Tuning t = tuning_of(tuning);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == MPF_F64) {
        NodeArgs<double> a = node_args<double>(ndim, degree, lower, cell, num, code);
        a.pos = (const double*)positions; a.pos_stride = pos_stride;
        a.field_in = (const double*)field; a.result = (double*)result; a.res_stride = res_stride;
        a.n = n; a.ncomp = (int)ncomp;
        return launch_gather<double>(kind, degree, ndim, a, t, s);
    }
    NodeArgs<float> a = node_args<float>(ndim, degree, lower, cell, num, code);
    a.pos = (const float*)positions; a.pos_stride = pos_stride;
    a.field_in = (const float*)field; a.result = (float*)result; a.res_stride = res_stride;
    a.n = n; a.ncomp = (int)ncomp;
    return launch_gather<float>(kind, degree, ndim, a, t, s);
}

int mpf_gather_tiles(int kind, int degree, int ndim, const void* positions, int64_t pos_stride, int64_t n,
                     const void* field, int64_t ncomp, void* result, int64_t res_stride, const double* lower,
                     const double* cell, const int32_t* num, const int32_t* code, const int32_t* tile,
                     const int64_t* tile_start, int dtype, const mpf_tuning* tuning, void* stream) {
    if (!valid_kind(kind, degree) || (dtype != MPF_F64 && dtype != MPF_F32)) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_grid(kind, degree, ndim, lower, cell, num, code));
    if (n < 0 || ncomp < 1 || ncomp > (1 << 20)) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_rows(positions, pos_stride, n, ndim, dtype));
    MPF_TRY(check_rows(result, res_stride, n, (int)ncomp, dtype));
    int64_t ntiles = 0;
    MPF_TRY(mpf_num_tiles(kind, degree, ndim, num, code, tile, &ntiles));
    if (!tile_start) return MPF_ERR_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(tile_start) % alignof(int64_t) != 0) return MPF_ERR_ALIGNMENT;
    if (n == 0) return MPF_OK;
    if (!field) return MPF_ERR_ARGUMENT;
    if (!aligned(field, dtype)) return MPF_ERR_ALIGNMENT;
    const Tuning t = tuning_of(tuning);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == MPF_F64) {
        NodeArgs<double> a = node_args<double>(ndim, degree, lower, cell, num, code);
        a.pos = (const double*)positions; a.pos_stride = pos_stride;
        a.field_in = (const double*)field; a.result = (double*)result; a.res_stride = res_stride;
        a.n = n; a.ncomp = (int)ncomp;
        set_tiles(a, ndim, degree, num, code, tile, tile_start, ntiles);
        return launch_gather<double>(kind, degree, ndim, a, t, s);
    }
    NodeArgs<float> a = node_args<float>(ndim, degree, lower, cell, num, code);
    a.pos = (const float*)positions; a.pos_stride = pos_stride;
    a.field_in = (const float*)field; a.result = (float*)result; a.res_stride = res_stride;
    a.n = n; a.ncomp = (int)ncomp;
    set_tiles(a, ndim, degree, num, code, tile, tile_start, ntiles);
    return launch_gather<float>(kind, degree, ndim, a, t, s);
}

int mpf_scatter(int kind, int degree, int ndim, const void* positions, int64_t pos_stride, const void* values,
                int64_t val_stride, int64_t n, void* field, int64_t ncomp, const double* lower,
                const double* cell, const int32_t* num, const int32_t* code, int dtype,
                const mpf_tuning* tuning, void* stream) {
    if (!valid_kind(kind, degree) || (dtype != MPF_F64 && dtype != MPF_F32)) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_grid(kind, degree, ndim, lower, cell, num, code));
    if (n < 0 || ncomp < 1 || ncomp > (1 << 20)) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_rows(positions, pos_stride, n, ndim, dtype));
    MPF_TRY(check_rows(values, val_stride, n, (int)ncomp, dtype));
    if (n == 0) return MPF_OK;
    if (!field) return MPF_ERR_ARGUMENT;
    if (!aligned(field, dtype)) return MPF_ERR_ALIGNMENT;
    const Tuning t = tuning_of(tuning);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == MPF_F64) {
        NodeArgs<double> a = node_args<double>(ndim, degree, lower, cell, num, code);
        a.pos = (const double*)positions; a.pos_stride = pos_stride;
        a.values = (const double*)values; a.val_stride = val_stride;
        a.field_out = (double*)field; a.n = n; a.ncomp = (int)ncomp;
        return launch_scatter<double>(kind, degree, ndim, a, t, s);
    }
    NodeArgs<float> a = node_args<float>(ndim, degree, lower, cell, num, code);
    a.pos = (const float*)positions; a.pos_stride = pos_stride;
    a.values = (const float*)values; a.val_stride = val_stride;
    a.field_out = (float*)field; a.n = n; a.ncomp = (int)ncomp;
    return launch_scatter<float>(kind, degree, ndim, a, t, s);
}

int mpf_scatter_tiles(int kind, int degree, int ndim, const void* positions, int64_t pos_stride, const void* values,
                      int64_t val_stride, int64_t n, void* field, int64_t ncomp, const double* lower,
                      const double* cell, const int32_t* num, const int32_t* code, const int32_t* tile,
                      const int64_t* tile_start, int dtype, const mpf_tuning* tuning, void* stream) {
    if (!valid_kind(kind, degree) || (dtype != MPF_F64 && dtype != MPF_F32)) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_grid(kind, degree, ndim, lower, cell, num, code));
    if (n < 0 || ncomp < 1 || ncomp > (1 << 20)) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_rows(positions, pos_stride, n, ndim, dtype));
    MPF_TRY(check_rows(values, val_stride, n, (int)ncomp, dtype));
    int64_t ntiles = 0;
    MPF_TRY(mpf_num_tiles(kind, degree, ndim, num, code, tile, &ntiles));
    if (!tile_start) return MPF_ERR_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(tile_start) % alignof(int64_t) != 0) return MPF_ERR_ALIGNMENT;
    if (n == 0) return MPF_OK;
    if (!field) return MPF_ERR_ARGUMENT;
    if (!aligned(field, dtype)) return MPF_ERR_ALIGNMENT;
    const Tuning t = tuning_of(tuning);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == MPF_F64) {
        NodeArgs<double> a = node_args<double>(ndim, degree, lower, cell, num, code);
        a.pos = (const double*)positions; a.pos_stride = pos_stride;
        a.values = (const double*)values; a.val_stride = val_stride;
        a.field_out = (double*)field; a.n = n; a.ncomp = (int)ncomp;
        set_tiles(a, ndim, degree, num, code, tile, tile_start, ntiles);
        return launch_scatter<double>(kind, degree, ndim, a, t, s);
    }
    NodeArgs<float> a = node_args<float>(ndim, degree, lower, cell, num, code);
    a.pos = (const float*)positions; a.pos_stride = pos_stride;
    a.values = (const float*)values; a.val_stride = val_stride;
    a.field_out = (float*)field; a.n = n; a.ncomp = (int)ncomp;
    set_tiles(a, ndim, degree, num, code, tile, tile_start, ntiles);
    return launch_scatter<float>(kind, degree, ndim, a, t, s);
}

int mpf_scatter_deterministic_workspace_bytes(int64_t entries, size_t* bytes) {
    if (entries < 0 || !bytes) return MPF_ERR_ARGUMENT;
    *bytes = det_workspace_bytes(entries);
    return MPF_OK;
}

// mpf_scatter_deterministic and its tile-sorted form (tile null: markers in any order).
static int scatter_deterministic(int kind, int degree, int ndim, const void* positions, int64_t pos_stride,
                                 const void* values, int64_t val_stride, int64_t n, void* field, int64_t ncomp,
                                 const double* lower, const double* cell, const int32_t* num, const int32_t* code,
                                 const int32_t* tile, const int64_t* tile_start, void* workspace,
                                 size_t workspace_bytes, void* stream) {
    if (!valid_kind(kind, degree)) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_grid(kind, degree, ndim, lower, cell, num, code));
    if (n < 0 || ncomp < 1 || ncomp > (1 << 20)) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_rows(positions, pos_stride, n, ndim, MPF_F64));
    MPF_TRY(check_rows(values, val_stride, n, (int)ncomp, MPF_F64));
    int64_t ntiles = 0;
    if (tile) {
        MPF_TRY(mpf_num_tiles(kind, degree, ndim, num, code, tile, &ntiles));
        if (!tile_start) return MPF_ERR_ARGUMENT;
        if (reinterpret_cast<uintptr_t>(tile_start) % alignof(int64_t) != 0) return MPF_ERR_ALIGNMENT;
    }
    if (n == 0) return MPF_OK;
    if (!field) return MPF_ERR_ARGUMENT;
    if (!aligned(field, MPF_F64)) return MPF_ERR_ALIGNMENT;
    const Grid<double> g = make_grid<double>(ndim, degree, lower, cell, num, code);
    int64_t entries = ncomp;
    for (int d = 0; d < ndim; ++d) entries *= g.ext[d];
    if (!workspace) return MPF_ERR_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(workspace) % 16 != 0) return MPF_ERR_ALIGNMENT;
    if (workspace_bytes < det_workspace_bytes(entries)) return MPF_ERR_WORKSPACE;
    NodeArgs<double> a = node_args<double>(ndim, degree, lower, cell, num, code);
    a.pos = (const double*)positions; a.pos_stride = pos_stride;
    a.values = (const double*)values; a.val_stride = val_stride;
    a.field_out = (double*)field; a.n = n; a.ncomp = (int)ncomp;
    if (tile) set_tiles(a, ndim, degree, num, code, tile, tile_start, ntiles);
    return launch_scatter_deterministic(kind, degree, ndim, a, entries, workspace, static_cast<cudaStream_t>(stream));
}

int mpf_scatter_deterministic(int kind, int degree, int ndim, const void* positions, int64_t pos_stride,
                              const void* values, int64_t val_stride, int64_t n, void* field, int64_t ncomp,
                              const double* lower, const double* cell, const int32_t* num, const int32_t* code,
                              void* workspace, size_t workspace_bytes, void* stream) {
    return scatter_deterministic(kind, degree, ndim, positions, pos_stride, values, val_stride, n, field, ncomp,
                                 lower, cell, num, code, nullptr, nullptr, workspace, workspace_bytes, stream);
}

int mpf_scatter_deterministic_tiles(int kind, int degree, int ndim, const void* positions, int64_t pos_stride,
                                    const void* values, int64_t val_stride, int64_t n, void* field, int64_t ncomp,
                                    const double* lower, const double* cell, const int32_t* num,
                                    const int32_t* code, const int32_t* tile, const int64_t* tile_start,
                                    void* workspace, size_t workspace_bytes, void* stream) {
    if (!tile) return MPF_ERR_ARGUMENT;
    return scatter_deterministic(kind, degree, ndim, positions, pos_stride, values, val_stride, n, field, ncomp,
                                 lower, cell, num, code, tile, tile_start, workspace, workspace_bytes, stream);
}

int mpf_gather_grad(int kind, int degree, int ndim, const void* positions, int64_t pos_stride, int64_t n,
                    const void* field, int64_t ncomp, const void* cotangent, int64_t cot_stride, void* grad,
                    int64_t grad_stride, const double* lower, const double* cell, const int32_t* num,
                    const int32_t* code, int dtype, void* stream) {
    if (!valid_kind(kind, degree) || (dtype != MPF_F64 && dtype != MPF_F32)) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_grid(kind, degree, ndim, lower, cell, num, code));
    if (n < 0 || ncomp < 1 || ncomp > (1 << 20)) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_rows(positions, pos_stride, n, ndim, dtype));
    MPF_TRY(check_rows(cotangent, cot_stride, n, (int)ncomp, dtype));
    MPF_TRY(check_rows(grad, grad_stride, n, ndim, dtype));
    if (n == 0) return MPF_OK;
    if (!field) return MPF_ERR_ARGUMENT;
    if (!aligned(field, dtype)) return MPF_ERR_ALIGNMENT;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == MPF_F64) {
        NodeArgs<double> a = node_args<double>(ndim, degree, lower, cell, num, code);
        a.pos = (const double*)positions; a.pos_stride = pos_stride;
        a.field_in = (const double*)field; a.values = (const double*)cotangent; a.val_stride = cot_stride;
        a.result = (double*)grad; a.res_stride = grad_stride; a.n = n; a.ncomp = (int)ncomp;
        return launch_gather_grad<double>(kind, degree, ndim, a, s);
    }
    NodeArgs<float> a = node_args<float>(ndim, degree, lower, cell, num, code);
    a.pos = (const float*)positions; a.pos_stride = pos_stride;
    a.field_in = (const float*)field; a.values = (const float*)cotangent; a.val_stride = cot_stride;
    a.result = (float*)grad; a.res_stride = grad_stride; a.n = n; a.ncomp = (int)ncomp;
    return launch_gather_grad<float>(kind, degree, ndim, a, s);
}

static bool valid_edge_kind(int kind, int degree) {
    if (kind == MPF_LINEAR) return degree == 1;
    if (kind == MPF_SPLINE) return degree >= 1 && degree <= 3;
    return false;
}

// The arguments of a path deposit: kind and degree, grid, and the rows of starts, ends and
// charges (strides of 0 taken as n).
static int check_paths(int kind, int degree, int ndim, const void* start, int64_t& start_stride, const void* end,
                       int64_t& end_stride, const void* charges, int64_t n, const double* lower, const double* cell,
                       const int32_t* num, const int32_t* code, int dtype) {
    if (!valid_edge_kind(kind, degree) || (dtype != MPF_F64 && dtype != MPF_F32)) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_grid(kind == MPF_LINEAR ? MPF_LINEAR : MPF_SPLINE, degree, ndim, lower, cell, num, code));
    if (n < 0) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_rows(start, start_stride, n, ndim, dtype));
    MPF_TRY(check_rows(end, end_stride, n, ndim, dtype));
    int64_t one = n;
    return check_rows(charges, one, n, 1, dtype);
}

int mpf_deposit_paths(int kind, int degree, int ndim, const void* start, int64_t start_stride, const void* end,
                      int64_t end_stride, const void* charges, int64_t n, void* edges, const double* lower,
                      const double* cell, const int32_t* num, const int32_t* code, int dtype,
                      const mpf_tuning* tuning, void* stream) {
    const Tuning t = tuning_of(tuning);
    MPF_TRY(check_paths(kind, degree, ndim, start, start_stride, end, end_stride, charges, n, lower, cell, num, code,
                        dtype));
    if (n == 0) return MPF_OK;
    if (!edges) return MPF_ERR_ARGUMENT;
    if (!aligned(edges, dtype)) return MPF_ERR_ALIGNMENT;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == MPF_F64) {
        PathArgs<double> a;
        std::memset(&a, 0, sizeof(a));
        a.g = make_grid<double>(ndim, degree, lower, cell, num, code);
        a.start = (const double*)start; a.start_stride = start_stride;
        a.end = (const double*)end; a.end_stride = end_stride;
        a.charges = (const double*)charges; a.edges_out = (double*)edges; a.n = n;
        return launch_deposit_paths<double>(kind, degree, ndim, a, t, s);
    }
    PathArgs<float> a;
    std::memset(&a, 0, sizeof(a));
    a.g = make_grid<float>(ndim, degree, lower, cell, num, code);
    a.start = (const float*)start; a.start_stride = start_stride;
    a.end = (const float*)end; a.end_stride = end_stride;
    a.charges = (const float*)charges; a.edges_out = (float*)edges; a.n = n;
    return launch_deposit_paths<float>(kind, degree, ndim, a, t, s);
}

int mpf_gather_edges(int kind, int degree, int ndim, const void* positions, int64_t pos_stride, int64_t n,
                     const void* edges, void* result, int64_t res_stride, const double* lower,
                     const double* cell, const int32_t* num, const int32_t* code, int dtype, void* stream) {
    if (!valid_edge_kind(kind, degree) || (dtype != MPF_F64 && dtype != MPF_F32)) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_grid(kind == MPF_LINEAR ? MPF_LINEAR : MPF_SPLINE, degree, ndim, lower, cell, num, code));
    if (n < 0) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_rows(positions, pos_stride, n, ndim, dtype));
    MPF_TRY(check_rows(result, res_stride, n, ndim, dtype));
    if (n == 0) return MPF_OK;
    if (!edges) return MPF_ERR_ARGUMENT;
    if (!aligned(edges, dtype)) return MPF_ERR_ALIGNMENT;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == MPF_F64) {
        PathArgs<double> a;
        std::memset(&a, 0, sizeof(a));
        a.g = make_grid<double>(ndim, degree, lower, cell, num, code);
        a.pos = (const double*)positions; a.pos_stride = pos_stride;
        a.edges_in = (const double*)edges; a.result = (double*)result; a.res_stride = res_stride; a.n = n;
        return launch_gather_edges<double>(kind, degree, ndim, a, s);
    }
    PathArgs<float> a;
    std::memset(&a, 0, sizeof(a));
    a.g = make_grid<float>(ndim, degree, lower, cell, num, code);
    a.pos = (const float*)positions; a.pos_stride = pos_stride;
    a.edges_in = (const float*)edges; a.result = (float*)result; a.res_stride = res_stride; a.n = n;
    return launch_gather_edges<float>(kind, degree, ndim, a, s);
}

static int check_block(void* field, int ndim, const int32_t* extent, int64_t ncomp, int32_t halo,
                       const int32_t* periodic, int dtype, bool stored) {
    if (ndim < 1 || ndim > 3 || !extent || !periodic || ncomp < 1 || halo < 0) return MPF_ERR_ARGUMENT;
    if (dtype != MPF_F64 && dtype != MPF_F32) return MPF_ERR_ARGUMENT;
    for (int d = 0; d < ndim; ++d) {
        const int64_t owned = stored ? (int64_t)extent[d] - 2 * (int64_t)halo : extent[d];
        if (owned < 1 || owned < halo) return MPF_ERR_SHAPE;
    }
    if (!field) return MPF_ERR_ARGUMENT;
    if (!aligned(field, dtype)) return MPF_ERR_ALIGNMENT;
    return MPF_OK;
}

int mpf_halo_fill(void* field, int ndim, const int32_t* stored, int64_t ncomp, int32_t halo,
                  const int32_t* periodic, int dtype, void* stream) {
    MPF_TRY(check_block(field, ndim, stored, ncomp, halo, periodic, dtype, true));
    if (halo == 0) return MPF_OK;
    return halo_fill(field, ndim, stored, ncomp, halo, periodic, dtype, static_cast<cudaStream_t>(stream));
}

int mpf_halo_fold(void* field, int ndim, const int32_t* stored, int64_t ncomp, int32_t halo,
                  const int32_t* periodic, int dtype, void* stream) {
    MPF_TRY(check_block(field, ndim, stored, ncomp, halo, periodic, dtype, true));
    if (halo == 0) return MPF_OK;
    return halo_fold(field, ndim, stored, ncomp, halo, periodic, dtype, static_cast<cudaStream_t>(stream));
}

// The storage, axis and slab [first, first + halo) of a halo pack or unpack, checked.
static int check_slab(const void* field, const void* buffer, int ndim, const int32_t* stored, int64_t ncomp,
                      int32_t halo, int axis, int32_t first, int dtype) {
    if (ndim < 1 || ndim > 3 || !stored || ncomp < 1 || halo < 1) return MPF_ERR_ARGUMENT;
    if (dtype != MPF_F64 && dtype != MPF_F32) return MPF_ERR_ARGUMENT;
    if (axis < 0 || axis >= ndim) return MPF_ERR_ARGUMENT;
    for (int d = 0; d < ndim; ++d)
        if (stored[d] < 1) return MPF_ERR_SHAPE;
    if (first < 0 || (int64_t)first + halo > stored[axis]) return MPF_ERR_SHAPE;
    if (!field || !buffer) return MPF_ERR_ARGUMENT;
    if (!aligned(field, dtype) || !aligned(buffer, dtype)) return MPF_ERR_ALIGNMENT;
    return MPF_OK;
}

int mpf_halo_pack(const void* field, int ndim, const int32_t* stored, int64_t ncomp, int32_t halo, int axis,
                  int32_t first, void* buffer, int dtype, void* stream) {
    MPF_TRY(check_slab(field, buffer, ndim, stored, ncomp, halo, axis, first, dtype));
    return halo_slab(const_cast<void*>(field), buffer, ndim, stored, ncomp, halo, axis, first, 0, dtype,
                     static_cast<cudaStream_t>(stream));
}

int mpf_halo_unpack(void* field, int ndim, const int32_t* stored, int64_t ncomp, int32_t halo, int axis,
                    int32_t first, const void* buffer, int accumulate, int dtype, void* stream) {
    MPF_TRY(check_slab(field, buffer, ndim, stored, ncomp, halo, axis, first, dtype));
    return halo_slab(field, const_cast<void*>(buffer), ndim, stored, ncomp, halo, axis, first, accumulate ? 2 : 1,
                     dtype, static_cast<cudaStream_t>(stream));
}

int mpf_add_density(void* dst, const void* deposit, int ndim, const int32_t* num, int32_t halo, int64_t ncomp,
                    const double* cell, const int32_t* periodic, int dtype, void* stream) {
    MPF_TRY(check_block(dst, ndim, num, ncomp, halo, periodic, dtype, false));
    if (!deposit || !cell) return MPF_ERR_ARGUMENT;
    if (!aligned(deposit, dtype)) return MPF_ERR_ALIGNMENT;
    for (int d = 0; d < ndim; ++d)
        if (!std::isfinite(cell[d]) || cell[d] == 0.0) return MPF_ERR_ARGUMENT;
    return add_density(dst, deposit, ndim, num, halo, ncomp, cell, periodic, dtype, static_cast<cudaStream_t>(stream));
}

int mpf_num_tiles(int kind, int degree, int ndim, const int32_t* num, const int32_t* code, const int32_t* tile,
                  int64_t* num_tiles) {
    if (!valid_kind(kind, degree) || ndim < 1 || ndim > 3 || !num || !code || !tile || !num_tiles)
        return MPF_ERR_ARGUMENT;
    int64_t total = 1;
    for (int d = 0; d < ndim; ++d) {
        if (tile[d] < 1 || num[d] < 1 || code[d] < 0 || code[d] > 2) return MPF_ERR_ARGUMENT;
        const int64_t e = axis_extent(num[d], code[d], degree);
        total *= (e + tile[d] - 1) / tile[d];
        if (total >= (int64_t)1 << 31) return MPF_ERR_ARGUMENT;
    }
    *num_tiles = total;
    return MPF_OK;
}

int mpf_sort_workspace_bytes(int64_t n, int64_t num_tiles, size_t* bytes) {
    if (n < 0 || n > INT32_MAX || num_tiles < 1 || !bytes) return MPF_ERR_ARGUMENT;
    *bytes = sort_workspace_bytes(n);
    return MPF_OK;
}

}  // extern "C"
namespace mpf {
// The argument checks of mpf_sort_by_tile apart from its workspace (shared with
// mpf_sort_by_tile_noalloc, which checks them before any CUDA call); a row stride of 0
// becomes n, and the number of tiles and the cells per tile key unit are set.
int check_sort_arguments(int kind, int degree, int ndim, const void* positions, int64_t& pos_stride,
                         const void* values, int64_t& val_stride, int64_t ncomp, int64_t n, const double* lower,
                         const double* cell, const int32_t* num, const int32_t* code, const int32_t* tile,
                         int within, const uint32_t* keys, const int32_t* order, const int64_t* tile_start,
                         int dtype, int64_t* ntiles_out, int64_t* cells_out) {
    if (!valid_kind(kind, degree) || (dtype != MPF_F64 && dtype != MPF_F32)) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_grid(kind, degree, ndim, lower, cell, num, code));
    if (n < 0 || n > INT32_MAX) return MPF_ERR_ARGUMENT;
    int64_t ntiles = 0;
    MPF_TRY(mpf_num_tiles(kind, degree, ndim, num, code, tile, &ntiles));
    if (within != 0 && within != 1) return MPF_ERR_ARGUMENT;
    int64_t cells = 1;
    if (within)
        for (int d = 0; d < ndim; ++d) cells *= tile[d];
    if ((uint64_t)ntiles * (uint64_t)cells >= ((uint64_t)1 << 32)) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_rows(positions, pos_stride, n, ndim, dtype));
    if (values) {
        if (ncomp < 1) return MPF_ERR_ARGUMENT;
        MPF_TRY(check_rows(values, val_stride, n, (int)ncomp, dtype));
    }
    if (!tile_start || (n > 0 && (!keys || !order))) return MPF_ERR_ARGUMENT;
    *ntiles_out = ntiles;
    *cells_out = cells;
    return MPF_OK;
}

// The cell-tile keys of the markers (tile_keys_kernel), arguments already checked.
int compute_keys(int kind, int degree, int ndim, const void* positions, int64_t pos_stride, const void* values,
                 int64_t val_stride, int64_t ncomp, int64_t n, const double* lower, const double* cell,
                 const int32_t* num, const int32_t* code, const int32_t* tile, int within, int64_t ntiles,
                 int64_t cells, uint32_t* keys, int dtype, cudaStream_t s) {
    if (n == 0) return MPF_OK;
    if (dtype == MPF_F64) {
        KeyArgs<double> a;
        std::memset(&a, 0, sizeof(a));
        a.g = make_grid<double>(ndim, degree, lower, cell, num, code);
        a.pos = (const double*)positions; a.pos_stride = pos_stride;
        a.values = (const double*)values; a.val_stride = val_stride; a.ncomp = ncomp; a.n = n;
        for (int d = 0; d < 3; ++d) {
            a.tile[d] = d < ndim ? tile[d] : 1;
            a.ntiles[d] = d < ndim ? (a.g.ext[d] + a.tile[d] - 1) / a.tile[d] : 1;
        }
        a.sentinel = (uint32_t)(ntiles * cells); a.within = within; a.keys = keys;
        return tile_keys<double>(kind, degree, ndim, a, s);
    }
    KeyArgs<float> a;
    std::memset(&a, 0, sizeof(a));
    a.g = make_grid<float>(ndim, degree, lower, cell, num, code);
    a.pos = (const float*)positions; a.pos_stride = pos_stride;
    a.values = (const float*)values; a.val_stride = val_stride; a.ncomp = ncomp; a.n = n;
    for (int d = 0; d < 3; ++d) {
        a.tile[d] = d < ndim ? tile[d] : 1;
        a.ntiles[d] = d < ndim ? (a.g.ext[d] + a.tile[d] - 1) / a.tile[d] : 1;
    }
    a.sentinel = (uint32_t)(ntiles * cells); a.within = within; a.keys = keys;
    return tile_keys<float>(kind, degree, ndim, a, s);
}

}  // namespace mpf
extern "C" {

int mpf_sort_by_tile(int kind, int degree, int ndim, const void* positions, int64_t pos_stride, const void* values,
                     int64_t val_stride, int64_t ncomp, int64_t n, const double* lower, const double* cell,
                     const int32_t* num, const int32_t* code, const int32_t* tile, int within, uint32_t* keys,
                     int32_t* order, int64_t* tile_start, void* workspace, size_t workspace_bytes, int dtype,
                     void* stream) {
    int64_t ntiles = 0, cells = 1;
    MPF_TRY(check_sort_arguments(kind, degree, ndim, positions, pos_stride, values, val_stride, ncomp, n, lower,
                                 cell, num, code, tile, within, keys, order, tile_start, dtype, &ntiles, &cells));
    if (workspace_bytes < sort_workspace_bytes(n) || (!workspace && n > 0)) return MPF_ERR_WORKSPACE;
    if ((reinterpret_cast<uintptr_t>(workspace) % 256) != 0) return MPF_ERR_ALIGNMENT;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    MPF_TRY(compute_keys(kind, degree, ndim, positions, pos_stride, values, val_stride, ncomp, n, lower, cell, num,
                         code, tile, within, ntiles, cells, keys, dtype, s));
    return sort_keys(keys, n, ntiles, cells, order, tile_start, workspace, s);
}

int mpf_resort_workspace_bytes(int kind, int degree, int ndim, const int32_t* num, const int32_t* code,
                               const int32_t* tile, int within, int64_t n, size_t* bytes) {
    if (!bytes || n < 0 || n > INT32_MAX || (within != 0 && within != 1)) return MPF_ERR_ARGUMENT;
    int64_t ntiles = 0;
    MPF_TRY(mpf_num_tiles(kind, degree, ndim, num, code, tile, &ntiles));
    int64_t cells = 1;
    if (within)
        for (int d = 0; d < ndim; ++d) cells *= tile[d];
    *bytes = resort_workspace_bytes(n, ntiles * cells + 1);
    return MPF_OK;
}

int mpf_resort_by_tile(int kind, int degree, int ndim, const void* positions, int64_t pos_stride,
                       const void* values, int64_t val_stride, int64_t ncomp, int64_t n, const double* lower,
                       const double* cell, const int32_t* num, const int32_t* code, const int32_t* tile, int within,
                       const uint32_t* prev_sorted_keys, uint32_t* sorted_keys, int32_t* order, int64_t* tile_start,
                       void* workspace, size_t workspace_bytes, int dtype, void* stream) {
    int64_t ntiles = 0, cells = 1;
    MPF_TRY(check_sort_arguments(kind, degree, ndim, positions, pos_stride, values, val_stride, ncomp, n, lower,
                                 cell, num, code, tile, within, sorted_keys, order, tile_start, dtype, &ntiles,
                                 &cells));
    if (workspace_bytes < resort_workspace_bytes(n, ntiles * cells + 1) || (!workspace && n > 0))
        return MPF_ERR_WORKSPACE;
    if ((reinterpret_cast<uintptr_t>(workspace) % 256) != 0) return MPF_ERR_ALIGNMENT;
    if (prev_sorted_keys && prev_sorted_keys == sorted_keys) return MPF_ERR_ARGUMENT;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t* keys = n > 0 ? resort_keys_buffer(workspace, n) : nullptr;
    MPF_TRY(compute_keys(kind, degree, ndim, positions, pos_stride, values, val_stride, ncomp, n, lower, cell, num,
                         code, tile, within, ntiles, cells, keys, dtype, s));
    return resort_keys(n, ntiles, cells, prev_sorted_keys, sorted_keys, order, tile_start, workspace, s);
}

int mpf_permute_rows(void* dst, int64_t dst_stride, const void* src, int64_t src_stride, int64_t rows,
                     const int32_t* order, int64_t n, int dtype, void* stream) {
    if (dtype != MPF_F64 && dtype != MPF_F32) return MPF_ERR_ARGUMENT;
    if (n < 0 || rows < 0) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_rows(dst, dst_stride, n, (int)rows, dtype));
    MPF_TRY(check_rows(src, src_stride, n, (int)rows, dtype));
    if (n == 0 || rows == 0) return MPF_OK;
    if (!order) return MPF_ERR_ARGUMENT;
    return permute_rows(dst, dst_stride, src, src_stride, rows, order, n, dtype, static_cast<cudaStream_t>(stream));
}

int mpf_unpermute_rows(void* dst, int64_t dst_stride, const void* src, int64_t src_stride, int64_t rows,
                       const int32_t* order, int64_t n, int dtype, void* stream) {
    if (dtype != MPF_F64 && dtype != MPF_F32) return MPF_ERR_ARGUMENT;
    if (n < 0 || rows < 0) return MPF_ERR_ARGUMENT;
    MPF_TRY(check_rows(dst, dst_stride, n, (int)rows, dtype));
    MPF_TRY(check_rows(src, src_stride, n, (int)rows, dtype));
    if (n == 0 || rows == 0) return MPF_OK;
    if (!order) return MPF_ERR_ARGUMENT;
    return unpermute_rows(dst, dst_stride, src, src_stride, rows, order, n, dtype, static_cast<cudaStream_t>(stream));
}

int64_t mpf_batch_request_size(void) { return (int64_t)sizeof(mpf_batch_request); }

int mpf_batch_request_init(mpf_batch_request* r, int op, int kind, int degree, int ndim, const void* positions,
                           int64_t pos_stride, const void* values, int64_t val_stride, int64_t n, const void* field,
                           void* out, int64_t out_stride, int ncomp, const double* lower, const double* cell,
                           const int32_t* num, const int32_t* code) {
    if (!r) return MPF_ERR_ARGUMENT;
    if (op != MPF_OP_GATHER && op != MPF_OP_SCATTER && op != MPF_OP_PATHS) return MPF_ERR_ARGUMENT;
    if (op == MPF_OP_PATHS) {
        MPF_TRY(check_paths(kind, degree, ndim, positions, pos_stride, field, out_stride, values, n, lower, cell, num,
                            code, MPF_F64));
        ncomp = ndim;
    } else {
        if (!valid_kind(kind, degree)) return MPF_ERR_ARGUMENT;
        MPF_TRY(check_grid(kind, degree, ndim, lower, cell, num, code));
        if (n < 0 || ncomp < 1) return MPF_ERR_ARGUMENT;
        MPF_TRY(check_rows(positions, pos_stride, n, ndim, MPF_F64));
    }
    if (!out || !aligned(out, MPF_F64)) return out ? MPF_ERR_ALIGNMENT : MPF_ERR_ARGUMENT;
    if (op == MPF_OP_PATHS) {
        // (checked above)
    } else if (op == MPF_OP_GATHER) {
        if (!field) return MPF_ERR_ARGUMENT;
        if (!aligned(field, MPF_F64)) return MPF_ERR_ALIGNMENT;
        MPF_TRY(check_rows(out, out_stride, n, ncomp, MPF_F64));
    } else {
        MPF_TRY(check_rows(values, val_stride, n, ncomp, MPF_F64));
    }
    std::memset(r, 0, sizeof(*r));
    r->op = op;
    r->kind = kind;
    r->degree = degree;
    r->ndim = ndim;
    r->ncomp = ncomp;
    r->n = n;
    r->positions = static_cast<const double*>(positions);
    r->pos_stride = pos_stride;
    r->values = static_cast<const double*>(values);
    r->val_stride = val_stride;
    r->field = static_cast<const double*>(field);
    r->out = static_cast<double*>(out);
    r->out_stride = out_stride;
    const Grid<double> g = make_grid<double>(ndim, degree, lower, cell, num, code);
    for (int d = 0; d < 3; ++d) {
        r->lower[d] = g.lower[d];
        r->cell[d] = g.cell[d];
        r->inv[d] = g.inv[d];
        r->num[d] = g.num[d];
        r->code[d] = g.code[d];
        r->ext[d] = g.ext[d];
    }
    return MPF_OK;
}

int mpf_batch_launch(const mpf_batch_request* table, mpf_batch_header* header, int grid, int block, void* stream) {
    if (!table || !header || grid < 0 || block < 0) return MPF_ERR_ARGUMENT;
    return launch_batch(table, header, grid, block, static_cast<cudaStream_t>(stream));
}

}  // extern "C"

// api.cu -- the exported C ABI of libcuSZp (include/cuSZp.h) and the 36 per-mode
// C++ entry points (include/cuSZp/cuSZp_entry_*.h).  Thin: validate, obtain
// workspace, enqueue the fused kernel, and (for the reference-compatible calls)
// wait for the result.
#include "../../include/cuSZp.h"
#include "codec_launch.cuh"

#include <cstddef>
#include <cstdio>
#include <cstring>
#include <mutex>

using namespace cuszp;

namespace {

const char* status_text(int st)
{
    switch (st) {
        case OK: return "success";
        case E_ARG: return "invalid argument";
        case E_UNSUPPORTED: return "unsupported shape (2D/3D need dims.x % 4 == 0)";
        case E_CUDA: return "CUDA runtime error";
        case E_TIMEOUT: return "device-side wait timed out";
        case E_WORKSPACE: return "workspace missing or too small";
        case E_CAPACITY: return "output capacity too small";
        default: return "unknown error";
    }
}

// Keep freed stream-ordered allocations in the device pool between calls so the
// per-call workspace costs no driver allocation after the first call.
void keep_pool_warm()
{
    static std::once_flag once[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev >= 64) return;
    std::call_once(once[dev], [dev]() {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t thr = 256ull << 20;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
    });
}

int check_ptrs(const Problem& p, const void* data, const void* cmp)
{
    if (p.g.ntiles == 0) return OK;
    if (!data || !cmp) return E_ARG;
    const uintptr_t es = p.type == 0 ? 4 : 8;
    if ((uintptr_t)data % es) return E_ARG;
    if (p.mode != MODE_OUTLIER && (uintptr_t)cmp % 4) return E_ARG;   // word-aligned payloads
    return OK;
}

// Status of a launch's error word: a timed-out wait, else a stream that did not fit
// its buffer (or, decompressing, rate bytes no valid stream holds).
int status_of(uint32_t err)
{
    if (err & kTimeoutErrs) return E_TIMEOUT;
    if (err & ERR_CAPACITY) return E_CAPACITY;
    return OK;
}

// Synchronous call with a pool-allocated workspace.  Returns a Status; for
// compress, *S receives the stream length (also when the stream did not fit
// `capacity`, E_CAPACITY: then it is the capacity needed).
int run_sync(bool comp, const void* data_in, void* data_out, const uint8_t* cmp_in, uint8_t* cmp_out,
             size_t nbEle, double eb, int dim, uint3 dims, int type, int mode, cudaStream_t stream, size_t* S,
             size_t capacity = ~(size_t)0)
{
    Problem p;
    int st = make_problem(p, type, mode, dim, nbEle, dims.x, dims.y, dims.z);
    if (st) return st;
    st = comp ? check_ptrs(p, data_in, cmp_out) : check_ptrs(p, data_out, cmp_in);
    if (st) return st;
    if (p.g.ntiles == 0) { if (S) *S = (size_t)p.g.rate_bytes; return OK; }
    if (comp) {
        if (capacity < p.g.rate_bytes) return E_CAPACITY;   // the rate region alone does not fit
        p.g.cap = capacity;
    }
    keep_pool_warm();
    const size_t wsb = workspace_bytes(p);
    void* ws = nullptr;
    if (cudaMallocAsync(&ws, wsb, stream) != cudaSuccess) return E_CUDA;
    cudaMemsetAsync(ws, 0, wsb, stream);
    st = comp ? launch_compress(p, data_in, cmp_out, eb, ws, stream)
              : launch_decompress(p, data_out, cmp_in, eb, ws, stream);
    WsHeader h;
    std::memset(&h, 0, sizeof(h));
    cudaMemcpyAsync(&h, ws, sizeof(h), cudaMemcpyDeviceToHost, stream);
    cudaFreeAsync(ws, stream);
    const cudaError_t e = cudaStreamSynchronize(stream);
    if (st) return st;
    if (e != cudaSuccess) return E_CUDA;
    st = status_of(h.err);
    if (S && (st == OK || st == E_CAPACITY)) *S = (size_t)h.total;
    return st;
}

void report(const char* what, int st)
{
    if (st == E_ARG || st == E_UNSUPPORTED || st == E_CUDA || st == E_TIMEOUT || st == E_CAPACITY)
        std::fprintf(stderr, "cuSZp: %s failed: %s\n", what, status_text(st));
}

// Reference dispatcher messages for bad enums (src/cuSZp.cu:18,41,82).
bool enums_ok(cuszp_dim_t dim, cuszp_type_t type, cuszp_mode_t mode)
{
    if (type != CUSZP_TYPE_FLOAT && type != CUSZP_TYPE_DOUBLE) { std::printf("Unsupported type in cuSZp.\n"); return false; }
    if (mode < CUSZP_MODE_FIXED || mode > CUSZP_MODE_OUTLIER) { std::printf("Unsupported mode in cuSZp.\n"); return false; }
    if (dim < CUSZP_DIM_1D || dim > CUSZP_DIM_3D) { std::printf("Unsupported dimension in cuSZp.\n"); return false; }
    return true;
}

void compress_legacy(const void* d_in, unsigned char* d_cmp, size_t nbEle, size_t* cmpSize, double eb,
                     int dim, uint3 dims, int type, int mode, cudaStream_t stream)
{
    size_t S = 0;
    const int st = run_sync(true, d_in, nullptr, nullptr, d_cmp, nbEle, eb, dim, dims, type, mode, stream, &S);
    report("compression", st);
    if (cmpSize) *cmpSize = st ? 0 : S;
}

void decompress_legacy(void* d_out, const unsigned char* d_cmp, size_t nbEle, double eb,
                       int dim, uint3 dims, int type, int mode, cudaStream_t stream)
{
    const int st = run_sync(false, nullptr, d_out, d_cmp, nullptr, nbEle, eb, dim, dims, type, mode, stream, nullptr);
    report("decompression", st);
}

}  // namespace

// ------------------------------------------------------------------ reference C entry points

extern "C" void cuSZp_compress(void* d_oriData, unsigned char* d_cmpBytes, size_t nbEle, size_t* cmpSize,
                               float errorBound, cuszp_dim_t dim, uint3 dims, cuszp_type_t type,
                               cuszp_mode_t mode, cudaStream_t stream)
{
    if (!enums_ok(dim, type, mode)) return;
    // f64 data: the generic API widens the float bound (src/cuSZp.cu:45)
    compress_legacy(d_oriData, d_cmpBytes, nbEle, cmpSize, (double)errorBound, dim, dims, type, mode, stream);
}

extern "C" void cuSZp_decompress(void* d_decData, unsigned char* d_cmpBytes, size_t nbEle, size_t cmpSize,
                                 float errorBound, cuszp_dim_t dim, uint3 dims, cuszp_type_t type,
                                 cuszp_mode_t mode, cudaStream_t stream)
{
    (void)cmpSize;   // offsets are re-derived from the rate bytes, as in the reference
    if (!enums_ok(dim, type, mode)) return;
    decompress_legacy(d_decData, d_cmpBytes, nbEle, (double)errorBound, dim, dims, type, mode, stream);
}

// ------------------------------------------------------------------ extensions

extern "C" size_t cuSZp_max_compressed_size(size_t nbEle, cuszp_dim_t dim, uint3 dims, cuszp_type_t type,
                                            cuszp_mode_t mode)
{
    Problem p;
    if (make_problem(p, type, mode, dim, nbEle, dims.x, dims.y, dims.z)) return 0;
    return max_stream_bytes(p);
}

extern "C" size_t cuSZp_workspace_size(size_t nbEle, cuszp_dim_t dim, uint3 dims, cuszp_type_t type,
                                       cuszp_mode_t mode)
{
    Problem p;
    if (make_problem(p, type, mode, dim, nbEle, dims.x, dims.y, dims.z)) return 0;
    return workspace_bytes(p);
}

extern "C" int cuSZp_compress_async(const void* d_oriData, unsigned char* d_cmpBytes, size_t cmpCapacity,
                                    size_t nbEle, float errorBound, cuszp_dim_t dim, uint3 dims,
                                    cuszp_type_t type, cuszp_mode_t mode, void* d_workspace,
                                    size_t workspaceBytes, unsigned long long* d_cmpSize, cudaStream_t stream)
{
    Problem p;
    int st = make_problem(p, type, mode, dim, nbEle, dims.x, dims.y, dims.z);
    if (st) return st;
    if ((st = check_ptrs(p, d_oriData, d_cmpBytes))) return st;
    if (p.g.ntiles == 0) {
        if (d_cmpSize) {
            if (cudaMemsetAsync(d_cmpSize, 0, sizeof(unsigned long long), stream) != cudaSuccess) return E_CUDA;
        }
        return OK;
    }
    if (cmpCapacity < p.g.rate_bytes) return E_CAPACITY;   // the rate region alone does not fit
    p.g.cap = cmpCapacity;
    if (!d_workspace || workspaceBytes < workspace_bytes(p) || (uintptr_t)d_workspace % 16) return E_WORKSPACE;
    // the kernel's last CTA writes the length into d_cmpSize (no copy after the kernel)
    return launch_compress(p, d_oriData, d_cmpBytes, (double)errorBound, d_workspace, stream, d_cmpSize);
}

extern "C" int cuSZp_decompress_async(void* d_decData, const unsigned char* d_cmpBytes, size_t nbEle,
                                      float errorBound, cuszp_dim_t dim, uint3 dims, cuszp_type_t type,
                                      cuszp_mode_t mode, void* d_workspace, size_t workspaceBytes,
                                      cudaStream_t stream)
{
    Problem p;
    int st = make_problem(p, type, mode, dim, nbEle, dims.x, dims.y, dims.z);
    if (st) return st;
    if ((st = check_ptrs(p, d_decData, d_cmpBytes))) return st;
    if (p.g.ntiles == 0) return OK;
    if (!d_workspace || workspaceBytes < workspace_bytes(p) || (uintptr_t)d_workspace % 16) return E_WORKSPACE;
    return launch_decompress(p, d_decData, d_cmpBytes, (double)errorBound, d_workspace, stream);
}

extern "C" int cuSZp_workspace_check(void* d_workspace, size_t workspaceBytes, cudaStream_t stream)
{
    if (!d_workspace || workspaceBytes < sizeof(WsHeader)) return E_WORKSPACE;
    WsHeader h;
    if (cudaMemcpyAsync(&h, d_workspace, sizeof(h), cudaMemcpyDeviceToHost, stream) != cudaSuccess) return E_CUDA;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return E_CUDA;
    const int st = status_of(h.err);
    if (st == E_TIMEOUT) {
        // an aborted call may leave tickets and tile status behind: start clean
        if (cudaMemsetAsync(d_workspace, 0, workspaceBytes, stream) != cudaSuccess) return E_CUDA;
    } else if (st == E_CAPACITY) {
        // the launch completed (the workspace is clean again): clear the error word only
        if (cudaMemsetAsync(&reinterpret_cast<WsHeader*>(d_workspace)->err, 0, sizeof(uint32_t), stream) != cudaSuccess)
            return E_CUDA;
    }
    if (st && cudaStreamSynchronize(stream) != cudaSuccess) return E_CUDA;
    return st;
}

extern "C" int cuSZp_workspace_error_async(void* d_workspace, unsigned int* h_err, cudaStream_t stream)
{
    if (!d_workspace || !h_err) return E_ARG;
    const char* w = static_cast<const char*>(d_workspace) + offsetof(WsHeader, err);
    return cudaMemcpyAsync(h_err, w, sizeof(unsigned int), cudaMemcpyDeviceToHost, stream) == cudaSuccess ? OK : E_CUDA;
}

extern "C" int cuSZp_serve_submit_async(int compress, const void* d_in, void* d_out, size_t outCapacity,
                                        size_t nbEle, float errorBound, cuszp_dim_t dim, uint3 dims,
                                        cuszp_type_t type, cuszp_mode_t mode, void* d_workspace,
                                        size_t workspaceBytes, void* h_words, cudaStream_t producer,
                                        cudaEvent_t order, cudaEvent_t done, cudaStream_t stream)
{
    if (!h_words) return E_ARG;
    Problem p;
    int st = make_problem(p, type, mode, dim, nbEle, dims.x, dims.y, dims.z);
    if (st) return st;
    // the lane's previous request is complete (its slot is free): no copy into these
    // words is in flight, so an empty array's zero length can be written from the host
    memset(h_words, 0, 16);
    if (order && producer != stream) {
        if (cudaEventRecord(order, producer) != cudaSuccess) return E_CUDA;
        if (cudaStreamWaitEvent(stream, order, 0) != cudaSuccess) return E_CUDA;
    }
    st = compress ? cuSZp_compress_async(d_in, static_cast<unsigned char*>(d_out), outCapacity, nbEle, errorBound,
                                         dim, dims, type, mode, d_workspace, workspaceBytes, nullptr, stream)
                  : cuSZp_decompress_async(d_out, static_cast<const unsigned char*>(d_in), nbEle, errorBound, dim,
                                           dims, type, mode, d_workspace, workspaceBytes, stream);
    if (st) return st;
    if (p.g.ntiles) {
        // error word, wait cap and stream length: header bytes 8..23 in one copy
        static_assert(offsetof(WsHeader, total) == offsetof(WsHeader, err) + 8, "err, wait_cap, total adjacent");
        const char* w = static_cast<const char*>(d_workspace) + offsetof(WsHeader, err);
        if (cudaMemcpyAsync(h_words, w, 16, cudaMemcpyDeviceToHost, stream) != cudaSuccess) return E_CUDA;
    }
    if (done && cudaEventRecord(done, stream) != cudaSuccess) return E_CUDA;
    return OK;
}

extern "C" int cuSZp_compress_ex(const void* d_oriData, unsigned char* d_cmpBytes, size_t cmpCapacity,
                                 size_t nbEle, size_t* cmpSize, float errorBound, cuszp_dim_t dim, uint3 dims,
                                 cuszp_type_t type, cuszp_mode_t mode, cudaStream_t stream)
{
    size_t S = 0;
    const int st = run_sync(true, d_oriData, nullptr, nullptr, d_cmpBytes, nbEle, (double)errorBound, dim, dims,
                            type, mode, stream, &S, cmpCapacity);
    if (cmpSize) *cmpSize = (st == OK || st == E_CAPACITY) ? S : 0;
    return st;
}

extern "C" int cuSZp_decompress_ex(void* d_decData, const unsigned char* d_cmpBytes, size_t nbEle, size_t cmpSize,
                                   float errorBound, cuszp_dim_t dim, uint3 dims, cuszp_type_t type,
                                   cuszp_mode_t mode, cudaStream_t stream)
{
    (void)cmpSize;
    return run_sync(false, nullptr, d_decData, d_cmpBytes, nullptr, nbEle, (double)errorBound, dim, dims, type, mode,
                    stream, nullptr);
}

extern "C" size_t cuSZp_reference_cmpsize(size_t streamBytes, size_t nbEle, cuszp_dim_t dim, uint3 dims,
                                          cuszp_type_t type, cuszp_mode_t mode)
{
    Problem p;
    if (make_problem(p, type, mode, dim, nbEle, dims.x, dims.y, dims.z)) return 0;
    const uint64_t payload = streamBytes - p.g.rate_bytes;
    uint64_t grid;
    if (dim == 1) grid = ((uint64_t)nbEle + 32767) / 32768;             // entry_1D_f32.cu:21
    else {
        const uint64_t per = 32ull * (type == CUSZP_TYPE_FLOAT ? 16 : 32);  // kernels_2D_f32.h:5 / _f64.h:5
        grid = (p.g.nblocks + per - 1) / per;
    }
    // only CTAs other than the first publish the total (kernels_1D_f32.cu:702-708)
    const uint64_t glob = grid > 1 ? (uint32_t)payload : 0;
    return (size_t)(glob + (dim == 1 ? p.g.rate_bytes : p.g.nblocks));
}

extern "C" int cuSZp_value_range(const void* d_data, size_t nbEle, cuszp_type_t type, double* minValue,
                                 double* maxValue, cudaStream_t stream)
{
    if (!d_data || nbEle == 0 || (type != CUSZP_TYPE_FLOAT && type != CUSZP_TYPE_DOUBLE)) return E_ARG;
    keep_pool_warm();
    const size_t wsb = range_ws_bytes(nbEle) + 16;
    void* ws = nullptr;
    if (cudaMallocAsync(&ws, wsb, stream) != cudaSuccess) return E_CUDA;
    cudaMemsetAsync(ws, 0, wsb, stream);
    char* res = reinterpret_cast<char*>(ws) + range_ws_bytes(nbEle);
    int st = launch_range(d_data, nbEle, type, res, ws, stream);
    double out[2] = {0, 0};
    unsigned char raw[16];
    cudaMemcpyAsync(raw, res, 16, cudaMemcpyDeviceToHost, stream);
    cudaFreeAsync(ws, stream);
    if (cudaStreamSynchronize(stream) != cudaSuccess) return E_CUDA;
    if (st) return st;
    if (type == CUSZP_TYPE_FLOAT) {
        float f[2];
        std::memcpy(f, raw, 8);
        out[0] = f[0]; out[1] = f[1];
    } else {
        std::memcpy(out, raw, 16);
    }
    if (minValue) *minValue = out[0];
    if (maxValue) *maxValue = out[1];
    return OK;
}

extern "C" int cuSZp_rel_error_bound(const void* d_data, size_t nbEle, cuszp_type_t type, float rel,
                                     float* errorBound, cudaStream_t stream)
{
    double mn = 0, mx = 0;
    const int st = cuSZp_value_range(d_data, nbEle, type, &mn, &mx, stream);
    if (st) return st;
    if (errorBound) {
        if (type == CUSZP_TYPE_FLOAT) *errorBound = rel * ((float)mx - (float)mn);
        else *errorBound = rel * (float)(mx - mn);
    }
    return OK;
}

extern "C" const char* cuSZp_version(void) { return "cuSZp-B200 1.0 (sm_100a)"; }

// ------------------------------------------------------------------ per-mode C++ entry points

#define CUSZP_ENTRY_1D(MODE_NAME, MODE_ID, T, TYPE_ID, SUFFIX)                                                   \
    void cuSZp_compress_1D_##MODE_NAME##_##SUFFIX(T* d_oriData, unsigned char* d_cmpBytes, size_t nbEle,         \
                                                  size_t* cmpSize, T errorBound, cudaStream_t stream)            \
    {                                                                                                            \
        compress_legacy(d_oriData, d_cmpBytes, nbEle, cmpSize, (double)errorBound, 1, make_uint3(0, 0, 0),      \
                        TYPE_ID, MODE_ID, stream);                                                               \
    }                                                                                                            \
    void cuSZp_decompress_1D_##MODE_NAME##_##SUFFIX(T* d_decData, unsigned char* d_cmpBytes, size_t nbEle,       \
                                                    size_t cmpSize, T errorBound, cudaStream_t stream)           \
    {                                                                                                            \
        (void)cmpSize;                                                                                           \
        decompress_legacy(d_decData, d_cmpBytes, nbEle, (double)errorBound, 1, make_uint3(0, 0, 0), TYPE_ID,    \
                          MODE_ID, stream);                                                                      \
    }

#define CUSZP_ENTRY_ND(DIM, MODE_NAME, MODE_ID, T, TYPE_ID, SUFFIX)                                              \
    void cuSZp_compress_##DIM##D_##MODE_NAME##_##SUFFIX(T* d_oriData, unsigned char* d_cmpBytes, size_t nbEle,   \
                                                        size_t* cmpSize, uint3 dims, T errorBound,               \
                                                        cudaStream_t stream)                                     \
    {                                                                                                            \
        compress_legacy(d_oriData, d_cmpBytes, nbEle, cmpSize, (double)errorBound, DIM, dims, TYPE_ID, MODE_ID, \
                        stream);                                                                                 \
    }                                                                                                            \
    void cuSZp_decompress_##DIM##D_##MODE_NAME##_##SUFFIX(T* d_decData, unsigned char* d_cmpBytes, size_t nbEle, \
                                                          size_t cmpSize, uint3 dims, T errorBound,              \
                                                          cudaStream_t stream)                                   \
    {                                                                                                            \
        (void)cmpSize;                                                                                           \
        decompress_legacy(d_decData, d_cmpBytes, nbEle, (double)errorBound, DIM, dims, TYPE_ID, MODE_ID, stream); \
    }

CUSZP_ENTRY_1D(fixed, 0, float, 0, f32)
CUSZP_ENTRY_1D(plain, 1, float, 0, f32)
CUSZP_ENTRY_1D(outlier, 2, float, 0, f32)
CUSZP_ENTRY_1D(fixed, 0, double, 1, f64)
CUSZP_ENTRY_1D(plain, 1, double, 1, f64)
CUSZP_ENTRY_1D(outlier, 2, double, 1, f64)
CUSZP_ENTRY_ND(2, fixed, 0, float, 0, f32)
CUSZP_ENTRY_ND(2, plain, 1, float, 0, f32)
CUSZP_ENTRY_ND(2, outlier, 2, float, 0, f32)
CUSZP_ENTRY_ND(2, fixed, 0, double, 1, f64)
CUSZP_ENTRY_ND(2, plain, 1, double, 1, f64)
CUSZP_ENTRY_ND(2, outlier, 2, double, 1, f64)
CUSZP_ENTRY_ND(3, fixed, 0, float, 0, f32)
CUSZP_ENTRY_ND(3, plain, 1, float, 0, f32)
CUSZP_ENTRY_ND(3, outlier, 2, float, 0, f32)
CUSZP_ENTRY_ND(3, fixed, 0, double, 1, f64)
CUSZP_ENTRY_ND(3, plain, 1, double, 1, f64)
CUSZP_ENTRY_ND(3, outlier, 2, double, 1, f64)

// ref_kernels.cu -- kernel-only timing harness for the reference's own CUDA kernels.
//
// Test and measurement infrastructure, not part of the product: `make -C oracle ref`
// links this file with the reference's kernel sources, compiled where they lie, into
// oracle/_ref/libcuszp_refk.so.  It launches a reference kernel the way the reference's
// per-mode entry points do (src/cuSZp_entry_1D_f32.cu:20-39, src/cuSZp_entry_2D_f64.cu:21-43,
// src/cuSZp_entry_3D_f32.cu:21-41: 32-thread CTAs, grid = ceil(work units / (32 x per-thread
// units)), three zeroed u32 scratch arrays of grid + 1 words, 8 bytes of dynamic shared
// memory), but allocates the scratch once per call of this harness, zeroes it outside the
// timed region and brackets only the kernel launch with CUDA events.  The time therefore
// excludes the entry points' per-call cudaMalloc / cudaMemset / cudaFree and their blocking
// size read-back, which the reference's own CLI timing includes.
//
// The kernel prototypes restate the reference's declarations
// (include/cuSZp/cuSZp_kernels_{1,2,3}D_f{32,64}.h) so that the linker finds them.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdio>

typedef volatile unsigned int vu32;
typedef volatile int vi32;

#define REF_1D(DIR, MODE, SUF, T, IN_T, OUT_T)                                                              \
    __global__ void cuSZp_##DIR##_kernel_1D_##MODE##_##SUF(IN_T* const __restrict__, OUT_T* const __restrict__, \
                                                           vu32* const __restrict__, vu32* const __restrict__,   \
                                                           vi32* const __restrict__, const T, const size_t);
#define REF_ND(DIR, D, MODE, SUF, T, IN_T, OUT_T)                                                                 \
    __global__ void cuSZp_##DIR##_kernel_##D##_##MODE##_vec4_##SUF(IN_T* const __restrict__, OUT_T* const __restrict__, \
                                                                   vu32* const __restrict__, vu32* const __restrict__,   \
                                                                   vi32* const __restrict__, unsigned int, const uint3, \
                                                                   const T);
#define REF_ALL(MODE, SUF, T)                                                  \
    REF_1D(compress, MODE, SUF, T, const T, unsigned char)                     \
    REF_1D(decompress, MODE, SUF, T, T, const unsigned char)                   \
    REF_ND(compress, 2D, MODE, SUF, T, const T, unsigned char)                 \
    REF_ND(decompress, 2D, MODE, SUF, T, T, const unsigned char)               \
    REF_ND(compress, 3D, MODE, SUF, T, const T, unsigned char)                 \
    REF_ND(decompress, 3D, MODE, SUF, T, T, const unsigned char)

REF_ALL(fixed, f32, float)
REF_ALL(plain, f32, float)
REF_ALL(outlier, f32, float)
REF_ALL(fixed, f64, double)
REF_ALL(plain, f64, double)
REF_ALL(outlier, f64, double)

namespace {

// Work units per thread of the reference's launch configuration: elements per thread in
// 1D (its thread_chunk), data blocks per thread in 2D/3D (its block_per_thread).
unsigned int per_thread(int dim, int type) { return dim == 1 ? 1024u : (type == 0 ? 16u : 32u); }

unsigned int block_count(int dim, uint3 d)
{
    if (dim == 2) return d.z * ((d.y + 7) / 8) * ((d.x + 7) / 8);
    return ((d.z + 3) / 4) * ((d.y + 3) / 4) * ((d.x + 3) / 4);
}

template <typename T>
cudaError_t launch(int dir, int dim, int mode, void* data, unsigned char* cmp, size_t n, uint3 dims, double eb,
                   unsigned int grid, unsigned int blocks, vu32* a, vu32* b, vi32* c, cudaStream_t s);

#define CASE_1D(MODE_ID, MODE, SUF)                                                                              \
    if (mode == MODE_ID) {                                                                                       \
        if (dir == 0)                                                                                            \
            cuSZp_compress_kernel_1D_##MODE##_##SUF<<<grid, 32, 8, s>>>((const T*)data, cmp, a, b, c, (T)eb, n); \
        else                                                                                                     \
            cuSZp_decompress_kernel_1D_##MODE##_##SUF<<<grid, 32, 8, s>>>((T*)data, cmp, a, b, c, (T)eb, n);     \
    }
#define CASE_ND(D, MODE_ID, MODE, SUF)                                                                            \
    if (mode == MODE_ID) {                                                                                        \
        if (dir == 0)                                                                                             \
            cuSZp_compress_kernel_##D##_##MODE##_vec4_##SUF<<<grid, 32, 8, s>>>((const T*)data, cmp, a, b, c,     \
                                                                                blocks, dims, (T)eb);             \
        else                                                                                                      \
            cuSZp_decompress_kernel_##D##_##MODE##_vec4_##SUF<<<grid, 32, 8, s>>>((T*)data, cmp, a, b, c, blocks, \
                                                                                  dims, (T)eb);                   \
    }

template <>
cudaError_t launch<float>(int dir, int dim, int mode, void* data, unsigned char* cmp, size_t n, uint3 dims, double eb,
                          unsigned int grid, unsigned int blocks, vu32* a, vu32* b, vi32* c, cudaStream_t s)
{
    using T = float;
    if (dim == 1) { CASE_1D(0, fixed, f32) CASE_1D(1, plain, f32) CASE_1D(2, outlier, f32) }
    else if (dim == 2) { CASE_ND(2D, 0, fixed, f32) CASE_ND(2D, 1, plain, f32) CASE_ND(2D, 2, outlier, f32) }
    else { CASE_ND(3D, 0, fixed, f32) CASE_ND(3D, 1, plain, f32) CASE_ND(3D, 2, outlier, f32) }
    return cudaGetLastError();
}
template <>
cudaError_t launch<double>(int dir, int dim, int mode, void* data, unsigned char* cmp, size_t n, uint3 dims, double eb,
                           unsigned int grid, unsigned int blocks, vu32* a, vu32* b, vi32* c, cudaStream_t s)
{
    using T = double;
    if (dim == 1) { CASE_1D(0, fixed, f64) CASE_1D(1, plain, f64) CASE_1D(2, outlier, f64) }
    else if (dim == 2) { CASE_ND(2D, 0, fixed, f64) CASE_ND(2D, 1, plain, f64) CASE_ND(2D, 2, outlier, f64) }
    else { CASE_ND(3D, 0, fixed, f64) CASE_ND(3D, 1, plain, f64) CASE_ND(3D, 2, outlier, f64) }
    return cudaGetLastError();
}

}  // namespace

// Times `reps` launches (after `warmup` untimed ones) of one reference kernel.
//   dir: 0 compress, 1 decompress; type: 0 f32, 1 f64; dim 1/2/3; mode 0 fixed, 1 plain,
//   2 outlier.  `eb` is passed to the kernel as T (the generic entry point's f64 path
//   gives the kernels (double)(float)eb; the caller passes that value).
// Writes the mean and minimum kernel time (ms) and the payload byte count the last
// compress launch left in the scratch (the value the entry points add the rate region
// to).  Returns a cudaError_t value (0 on success).
extern "C" int cuszp_refk_time(int dir, int type, int dim, int mode, void* data, unsigned char* cmp, size_t nbEle,
                               uint3 dims, double eb, int warmup, int reps, float* ms_mean, float* ms_min,
                               unsigned long long* payload, cudaStream_t stream)
{
    if (dir < 0 || dir > 1 || type < 0 || type > 1 || dim < 1 || dim > 3 || mode < 0 || mode > 2 || reps < 1)
        return (int)cudaErrorInvalidValue;
    const unsigned int blocks = dim == 1 ? 0u : block_count(dim, dims);
    const size_t units = dim == 1 ? nbEle : blocks;
    const size_t chunk = 32ull * per_thread(dim, type);
    const unsigned int grid = (unsigned int)((units + chunk - 1) / chunk);
    if (grid == 0) return (int)cudaErrorInvalidValue;
    const size_t words = (size_t)grid + 1;
    unsigned int* scratch = nullptr;
    cudaError_t e = cudaMalloc((void**)&scratch, 3 * words * sizeof(unsigned int));
    if (e != cudaSuccess) return (int)e;
    vu32* a = scratch;
    vu32* b = scratch + words;
    vi32* c = reinterpret_cast<vi32*>(scratch + 2 * words);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double sum = 0.0;
    float best = 1e30f;
    for (int i = 0; i < warmup + reps && e == cudaSuccess; i++) {
        e = cudaMemsetAsync(scratch, 0, 3 * words * sizeof(unsigned int), stream);
        if (e != cudaSuccess) break;
        cudaEventRecord(e0, stream);
        e = type == 0 ? launch<float>(dir, dim, mode, data, cmp, nbEle, dims, eb, grid, blocks, a, b, c, stream)
                      : launch<double>(dir, dim, mode, data, cmp, nbEle, dims, eb, grid, blocks, a, b, c, stream);
        cudaEventRecord(e1, stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e == cudaSuccess && i >= warmup) {
            sum += ms;
            best = ms < best ? ms : best;
        }
    }
    if (e == cudaSuccess) {
        unsigned int last = 0;
        e = cudaMemcpy(&last, scratch + grid, sizeof(last), cudaMemcpyDeviceToHost);
        if (payload) *payload = last;
        if (ms_mean) *ms_mean = (float)(sum / reps);
        if (ms_min) *ms_min = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(scratch);
    return (int)e;
}

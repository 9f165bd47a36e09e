// noalloc.cu -- a compression entry point that allocates nothing.
//
// Every other entry point needs device scratch for the look-back (a small header and
// one status word per tile), either from the caller (cuSZp_*_async) or from the
// stream-ordered pool (cuSZp_compress / _ex).  Some callers cannot provide either:
// code running where allocation is forbidden or would stall -- inside a region whose
// owner reserved all device memory up front, a real-time loop that must never hit an
// allocator, a plugin hosted by a framework that owns the device heap.  For them,
// cuSZp_compress_noalloc takes its scratch from one fixed array compiled into this
// library (kNoAllocScratchBytes per device; every GPU that loads the library holds it
// until the process exits).  The caller still passes the input, the output buffer and
// a device word for the stream length.
//
// The array is shared by every call on a device: calls whose kernels overlap on the
// GPU (different streams, no ordering) race on it and must not be issued.  It keeps
// the last call's contents, so each call clears the part it uses before launching.
#include "../../include/cuSZp.h"
#include "codec_kernels.cuh"
#include "codec_launch.cuh"

#include <cstdio>
#include <mutex>

namespace cuszp {

// 1 MiB: a 48-byte header plus 131,066 tile-status words.  In 1D a tile is 128 blocks of
// 32 elements and the tile count is rounded up to whole 1,024-block rate granules (8
// tiles), so 1D arrays of up to 16,383 x 32,768 = 536,838,144 elements fit; in 2D/3D a
// tile is 64 data blocks, so up to 8,388,224 blocks fit (536,846,336 elements when every
// block is whole).
constexpr size_t kNoAllocScratchBytes = 1u << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Same tile pipeline as compress_kernel, on scratch at `ws`; the stream length goes to
// *size_out, or ~0 when a bounded look-back wait gave up.
template <typename T, int DIM, int MODE, typename Tl = Tiling<DIM>>
__global__ void __launch_bounds__(Tl::THREADS, 2)
compress_noalloc_kernel(const T* __restrict__ in, uint8_t* __restrict__ cmp, Geom g, T recip, unsigned char* ws,
                        unsigned long long* __restrict__ size_out)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WsHeader* hdr = reinterpret_cast<WsHeader*>(ws);
    unsigned long long* status = reinterpret_cast<unsigned long long*>(ws + sizeof(WsHeader));
    SingleSource<T, DIM, MODE, Tl> src{in, cmp, g, recip, hdr, status, size_out};
    compress_pipeline<T, DIM, Tl>(src, smem_raw, &hdr->err);
    __shared__ int s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(&hdr->done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (s_last && threadIdx.x == 0) {
        __threadfence();
        if (hdr->err) *size_out = ~0ull;
    }
}

namespace {

template <typename T, int DIM>
const void* pick_noalloc(int mode, size_t* smem)
{
    *smem = compress_smem_bytes<T, DIM, Tiling<DIM>>();
    if (mode == 0) return (const void*)compress_noalloc_kernel<T, DIM, 0>;
    if (mode == 1) return (const void*)compress_noalloc_kernel<T, DIM, 1>;
    return (const void*)compress_noalloc_kernel<T, DIM, 2>;
}

const void* noalloc_kernel(const Problem& p, size_t* smem)
{
    if (p.type == 0) {
        if (p.dim == 1) return pick_noalloc<float, 1>(p.mode, smem);
        if (p.dim == 2) return pick_noalloc<float, 2>(p.mode, smem);
        return pick_noalloc<float, 3>(p.mode, smem);
    }
    if (p.dim == 1) return pick_noalloc<double, 1>(p.mode, smem);
    if (p.dim == 2) return pick_noalloc<double, 2>(p.mode, smem);
    return pick_noalloc<double, 3>(p.mode, smem);
}

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_scratch_addr[kMaxDevices] = {};
int g_sms[kMaxDevices] = {};
// per device and kernel (type x dim x mode): CTAs per SM, 0 until the kernel's shared
// memory limit is set and its occupancy known
int g_occ[kMaxDevices][2][3][3] = {};

// Once per device, with that device current: the array's device address (in host
// code the symbol itself is only a host-side stand-in) and the SM count; once per device
// and kernel: the kernel's shared-memory limit and occupancy.
int device_setup(int dev, const Problem& p, const void* fn, size_t smem, unsigned char** addr, int* sms, int* occ)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void* a = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&a, g_noalloc_scratch);
        if (e != cudaSuccess || !a) {
            std::fprintf(stderr, "cuSZp_compress_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev,
                         cudaGetErrorString(e));
            return E_CUDA;
        }
        if (cudaDeviceGetAttribute(&g_sms[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return E_CUDA;
        g_scratch_addr[dev] = static_cast<unsigned char*>(a);
    }
    int& o = g_occ[dev][p.type][p.dim - 1][p.mode];
    if (o == 0) {
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return E_CUDA;
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kThreads, smem) != cudaSuccess) return E_CUDA;
        o = n < 1 ? 1 : n;
    }
    *addr = g_scratch_addr[dev];
    *sms = g_sms[dev];
    *occ = o;
    return OK;
}

}  // namespace
}  // namespace cuszp

using namespace cuszp;

extern "C" int cuSZp_compress_noalloc(const void* d_oriData, unsigned char* d_cmpBytes, size_t nbEle,
                                      float errorBound, cuszp_dim_t dim, uint3 dims, cuszp_type_t type,
                                      cuszp_mode_t mode, unsigned long long* d_cmpSize, cudaStream_t stream)
{
    if (!d_cmpSize) return E_ARG;
    Problem p;
    int st = make_problem(p, type, mode, dim, nbEle, dims.x, dims.y, dims.z);
    if (st) return st;
    if (p.g.ntiles == 0) {   // empty stream: length 0, nothing to launch
        return cudaMemsetAsync(d_cmpSize, 0, sizeof(unsigned long long), stream) == cudaSuccess ? OK : E_CUDA;
    }
    if (!d_oriData || !d_cmpBytes) return E_ARG;
    if ((uintptr_t)d_oriData % (type == CUSZP_TYPE_FLOAT ? 4 : 8)) return E_ARG;
    if (mode != CUSZP_MODE_OUTLIER && (uintptr_t)d_cmpBytes % 4) return E_ARG;
    const size_t need = workspace_bytes(p);
    if (need > kNoAllocScratchBytes) {
        std::fprintf(stderr,
                     "cuSZp_compress_noalloc: this array needs %llu tiles of look-back state (%zu bytes); the "
                     "built-in scratch holds %llu tiles (%zu bytes). Use cuSZp_compress_async with a workspace.\n",
                     (unsigned long long)p.g.ntiles, need,
                     (unsigned long long)((kNoAllocScratchBytes - sizeof(WsHeader)) / 8), kNoAllocScratchBytes);
        return E_WORKSPACE;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return E_CUDA;
    size_t smem = 0;
    const void* fn = noalloc_kernel(p, &smem);
    unsigned char* ws = nullptr;
    int sms = 0, occ = 0;
    if ((st = device_setup(dev, p, fn, smem, &ws, &sms, &occ))) return st;
    // a previous call may have been aborted mid-way: start from zero
    if (cudaMemsetAsync(ws, 0, need, stream) != cudaSuccess) return E_CUDA;
    const uint64_t want = (uint64_t)sms * occ;
    const unsigned grid = (unsigned)(p.g.ntiles < want ? p.g.ntiles : want);
    Geom g = p.g;
    float rf = 0.5f / errorBound;
    double rd = 0.5 / (double)errorBound;
    void* args[6];
    args[0] = (void*)&d_oriData;
    args[1] = (void*)&d_cmpBytes;
    args[2] = (void*)&g;
    args[3] = type == CUSZP_TYPE_FLOAT ? (void*)&rf : (void*)&rd;
    args[4] = (void*)&ws;
    args[5] = (void*)&d_cmpSize;
    return cudaLaunchKernel(fn, dim3(grid), dim3(kThreads), args, smem, stream) == cudaSuccess ? OK : E_CUDA;
}

// codec_launch.cu -- geometry, grid sizing and dispatch of the 36 fused kernels
// (f32/f64 x fixed/plain/outlier x 1D/2D/3D, compress and decompress), plus the
// value-range reduction used for relative error bounds.
#include "codec_launch.cuh"
#include "codec_kernels.cuh"
#include "compress_tma.cuh"
#include "decompress_tma.cuh"

#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <vector>

namespace cuszp {

int make_problem(Problem& p, int type, int mode, int dim, size_t nbEle, unsigned dx, unsigned dy, unsigned dz)
{
    p = Problem{};
    if (type != 0 && type != 1) return E_ARG;
    if (mode < 0 || mode > 2) return E_ARG;
    p.type = type; p.mode = mode; p.dim = dim;
    Geom& g = p.g;
    g.nbEle = nbEle;
    g.dx = dx; g.dy = dy; g.dz = dz;
    g.cap = ~0ull;
    if (dim == 1) {
        g.nblocks = (nbEle + 31) / 32;
        g.rate_bytes = ((uint64_t)nbEle + 32767) / 32768 * 32768 / 32;
        g.ntiles = g.rate_bytes / Tiling<1>::TB;
        if (g.nblocks > 0xffffffffull) return E_ARG;
    } else if (dim == 2 || dim == 3) {
        if (dx == 0 || dy == 0 || dz == 0) return E_ARG;
        if (dx % 4 != 0) return E_UNSUPPORTED;   // src/cuSZp_kernels_2D_f32.cu:94 float4 rows
        const uint64_t bs = dim == 2 ? 8 : 4;
        g.bxn = (uint32_t)((dx + bs - 1) / bs);
        g.byn = (uint32_t)((dy + bs - 1) / bs);
        const uint64_t nbz = dim == 2 ? dz : (dz + 3) / 4;
        g.nblocks = nbz * g.byn * g.bxn;
        if ((uint64_t)g.bxn * g.byn > 0xffffffffull) return E_ARG;
        g.div_bx = FastDiv::make(g.bxn);
        g.div_plane = FastDiv::make(g.bxn * g.byn);
        if (g.nblocks > 0xffffffffull) return E_ARG;
        g.rate_bytes = (g.nblocks + 3) / 4 * 4;
        g.ntiles = (g.nblocks + Tiling<2>::TB - 1) / Tiling<2>::TB;
        g.nbEle = (uint64_t)dx * dy * dz;
    } else {
        return E_ARG;
    }
    return OK;
}

size_t workspace_bytes(const Problem& p)
{
    return sizeof(WsHeader) + sizeof(unsigned long long) * (size_t)(p.g.ntiles ? p.g.ntiles : 1);
}

size_t max_stream_bytes(const Problem& p)
{
    const uint64_t W = p.dim == 1 ? 4 : 8;
    return (size_t)(p.g.rate_bytes + p.g.nblocks * (W + 4 + 32 * W));
}

// ------------------------------------------------------------------ per-device set-up

namespace {
std::mutex g_setup_mu;
struct SetupEnt {
    const void* fn;
    int dev;
    int threads;
    size_t smem;
    int occ;   // -1: dynamic shared memory enabled (no occupancy entry)
};
std::vector<SetupEnt> g_setup;
int g_sms[64] = {};
}  // namespace

bool enable_dynamic_smem(const void* fn, size_t bytes)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    std::lock_guard<std::mutex> lk(g_setup_mu);
    for (const SetupEnt& e : g_setup)
        if (e.fn == fn && e.dev == dev && e.occ < 0 && e.smem >= bytes) return true;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess) {
        cudaGetLastError();   // not sticky: leave no error for the caller's next check
        return false;
    }
    g_setup.push_back(SetupEnt{fn, dev, 0, bytes, -1});
    return true;
}

int resident_ctas(const void* fn, int threads, size_t smem)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    std::lock_guard<std::mutex> lk(g_setup_mu);
    for (const SetupEnt& e : g_setup)
        if (e.fn == fn && e.dev == dev && e.occ >= 0 && e.threads == threads && e.smem == smem) return e.occ;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    g_setup.push_back(SetupEnt{fn, dev, threads, smem, occ});
    return occ;
}

int sm_count()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 0;
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (dev < 64 && g_sms[dev]) return g_sms[dev];
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (dev < 64) g_sms[dev] = n;
    return n;
}

// ------------------------------------------------------------------ dispatch tables

struct KernelRef {
    const void* fn;
    size_t smem;       // dynamic shared memory (compress: prefetch + staging buffers)
    unsigned threads;  // threads per CTA
};

template <typename T, int DIM, int MODE>
static KernelRef ckernel()
{
    using Tl = Tiling<DIM>;
    const void* fn = (const void*)compress_kernel<T, DIM, MODE, Tl>;
    constexpr size_t bytes = compress_smem_bytes<T, DIM, Tl>();
    enable_dynamic_smem(fn, bytes);   // a refusal surfaces as the launch's error
    return {fn, bytes, kThreads};
}
template <typename T, int DIM, int MODE>
static KernelRef dkernel() { return {(const void*)decompress_kernel<T, DIM, MODE>, 0, kThreads}; }

template <typename T, int DIM>
static KernelRef pick(bool comp, int mode)
{
    if (comp) {
        switch (mode) {
            case 0: return ckernel<T, DIM, 0>();
            case 1: return ckernel<T, DIM, 1>();
            default: return ckernel<T, DIM, 2>();
        }
    }
    switch (mode) {
        case 0: return dkernel<T, DIM, 0>();
        case 1: return dkernel<T, DIM, 1>();
        default: return dkernel<T, DIM, 2>();
    }
}

static KernelRef kernel_for(const Problem& p, bool comp)
{
    if (p.type == 0) {
        if (p.dim == 1) return pick<float, 1>(comp, p.mode);
        if (p.dim == 2) return pick<float, 2>(comp, p.mode);
        return pick<float, 3>(comp, p.mode);
    }
    if (p.dim == 1) return pick<double, 1>(comp, p.mode);
    if (p.dim == 2) return pick<double, 2>(comp, p.mode);
    return pick<double, 3>(comp, p.mode);
}

// Persistent grid: every SM filled to the kernel's occupancy, never more CTAs than tiles.
static unsigned grid_for(const KernelRef& k, uint64_t ntiles)
{
    const int occ = std::max(1, resident_ctas(k.fn, (int)k.threads, k.smem));
    const int sms = sm_count();
    const uint64_t want = (uint64_t)(sms > 0 ? sms : 148) * (uint64_t)occ;
    return (unsigned)(ntiles < want ? ntiles : want);
}

// ------------------------------------------------------------------ TMA compress path

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The driver's tensor-map encoder, looked up once through the runtime (no libcuda link).
static EncodeTiledFn encode_tiled()
{
    static EncodeTiledFn fn = []() -> EncodeTiledFn {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<EncodeTiledFn>(f);
    }();
    return fn;
}

// CUSZP_NO_ROW_BOXES=1 in the environment keeps 3D arrays on one box per block.
static bool row_boxes_allowed()
{
    static const bool ok = [] {
        const char* e = std::getenv("CUSZP_NO_ROW_BOXES");
        return !(e && e[0] == '1');
    }();
    return ok;
}

// 2D/3D tensor map of an array for the TMA kernels.  2D arrays whose blocks are all
// whole and whose block rows hold whole groups get a grouped map: the array as the 5D
// tensor (column in block, row in block, block column, block row, slice), so that one
// box of kGroup whole blocks lands in shared memory in block order (k = 8r + c per
// block); *grouped is set then.  3D arrays whose rows hold whole row boxes (dx a
// multiple of 32 f32 / 16 f64 elements) get a row-box map, *grouped set too: one box of
// 128-byte rows x 4 x 4 holds 8 f32 / 4 f64 whole blocks, stored 128-byte swizzled (so
// the kernels' reads and writes of it are free of bank conflicts), one load or store per
// 8 / 4 blocks instead of one per block.  Otherwise the array as a 3D tensor (x fastest) with one data block per box.
// Out-of-array elements are zero-filled on loads and clipped on stores.
bool make_block_map(CUtensorMap* m, const Problem& p, const void* in, bool* grouped)
{
    EncodeTiledFn enc = encode_tiled();
    *grouped = false;
    if (!enc) return false;
    const cuuint64_t esz = p.type == 0 ? 4 : 8;
    const CUtensorMapDataType dt = p.type == 0 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    if (p.dim == 2 && p.g.dx % 8 == 0 && p.g.dy % 8 == 0 && p.g.bxn % kGroup == 0) {
        const cuuint64_t dims5[5] = {8, 8, p.g.bxn, p.g.byn, p.g.dz};
        const cuuint64_t strides5[4] = {p.g.dx * esz, 8 * esz, 8ull * p.g.dx * esz, (cuuint64_t)p.g.dx * p.g.dy * esz};
        const cuuint32_t box5[5] = {8, 8, kGroup, 1, 1};
        const cuuint32_t estr5[5] = {1, 1, 1, 1, 1};
        if (enc(m, dt, 5, const_cast<void*>(in), dims5, strides5, box5, estr5, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS) {
            *grouped = true;
            return true;
        }
    }
    const cuuint64_t dims[3] = {p.g.dx, p.g.dy, p.g.dz};
    const cuuint64_t strides[2] = {p.g.dx * esz, (cuuint64_t)p.g.dx * p.g.dy * esz};
    // row boxes: 128-byte rows of 32 f32 / 16 f64 elements (8 / 4 blocks)
    const cuuint32_t rx = p.type == 0 ? 32u : 16u;
    if (p.dim == 3 && p.g.dx % rx == 0 && row_boxes_allowed()) {
        const cuuint32_t rbox[3] = {rx, 4, 4};
        const cuuint32_t restr[3] = {1, 1, 1};
        if (enc(m, dt, 3, const_cast<void*>(in), dims, strides, rbox, restr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS) {
            *grouped = true;
            return true;
        }
    }
    const cuuint32_t box[3] = {p.dim == 2 ? 8u : 4u, p.dim == 2 ? 8u : 4u, p.dim == 2 ? 1u : 4u};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(m, p.type == 0 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
               const_cast<void*>(in), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename T, int DIM, int MODE>
static KernelRef tma_kernel()
{
    const void* fn = (const void*)compress_tma_kernel<T, DIM, MODE>;
    constexpr size_t bytes = TmaCfg<T, DIM>::smem_bytes();
    enable_dynamic_smem(fn, bytes);
    return {fn, bytes, TmaCfg<T, DIM>::THREADS};
}

template <typename T, int DIM>
static KernelRef tma_pick(int mode)
{
    switch (mode) {
        case 0: return tma_kernel<T, DIM, 0>();
        case 1: return tma_kernel<T, DIM, 1>();
        default: return tma_kernel<T, DIM, 2>();
    }
}

static KernelRef tma_kernel_for(const Problem& p)
{
    if (p.type == 0) {
        if (p.dim == 1) return tma_pick<float, 1>(p.mode);
        if (p.dim == 2) return tma_pick<float, 2>(p.mode);
        return tma_pick<float, 3>(p.mode);
    }
    if (p.dim == 1) return tma_pick<double, 1>(p.mode);
    if (p.dim == 2) return tma_pick<double, 2>(p.mode);
    return tma_pick<double, 3>(p.mode);
}

// CUSZP_NO_TMA=1 in the environment selects the cp.async kernels for every input.
bool tma_allowed()
{
    static const bool ok = [] {
        const char* e = std::getenv("CUSZP_NO_TMA");
        return !(e && e[0] == '1');
    }();
    return ok;
}

// Compress through the TMA kernel when the input starts on a 16-byte boundary (and the
// tensor map encodes); returns -1 when the caller should use the cp.async kernel.
static int launch_tma(const Problem& p, const void* in, void* cmp, double eb, void* ws, cudaStream_t s)
{
    if (!tma_allowed() || (reinterpret_cast<uintptr_t>(in) & 15u)) return -1;
    alignas(64) CUtensorMap map;
    std::memset(&map, 0, sizeof(map));
    bool grouped = false;
    if (p.dim != 1 && !make_block_map(&map, p, in, &grouped)) return -1;
    const KernelRef k = tma_kernel_for(p);
    const unsigned grid = grid_for(k, p.g.ntiles);
    WsHeader* hdr = reinterpret_cast<WsHeader*>(ws);
    unsigned long long* status = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(ws) + sizeof(WsHeader));
    Geom g = p.g;
    g.grouped = grouped ? 1u : 0u;
    float rf = 0.5f / (float)eb;
    double rd = 0.5 / eb;
    const void* src = in;
    void* dst = cmp;
    void* args[] = {(void*)&map, (void*)&src, (void*)&dst, (void*)&g, p.type == 0 ? (void*)&rf : (void*)&rd,
                    (void*)&hdr, (void*)&status};
    return cudaLaunchKernel(k.fn, dim3(grid), dim3(k.threads), args, k.smem, s) == cudaSuccess ? OK : E_CUDA;
}

template <typename T, int DIM, int MODE, bool DIRECT = false>
static KernelRef dtma_kernel()
{
    const void* fn = (const void*)decompress_tma_kernel<T, DIM, MODE, DIRECT>;
    constexpr size_t bytes = DecCfg<T, DIM, DIRECT>::smem_bytes();
    enable_dynamic_smem(fn, bytes);
    return {fn, bytes, DecCfg<T, DIM, DIRECT>::THREADS};
}

template <typename T, int DIM, bool DIRECT = false>
static KernelRef dtma_pick(int mode)
{
    switch (mode) {
        case 0: return dtma_kernel<T, DIM, 0, DIRECT>();
        case 1: return dtma_kernel<T, DIM, 1, DIRECT>();
        default: return dtma_kernel<T, DIM, 2, DIRECT>();
    }
}

// grouped: a grouped 2D map (the direct-store kernel)
static KernelRef dtma_kernel_for(const Problem& p, bool grouped)
{
    if (p.type == 0) {
        if (p.dim == 1) return dtma_pick<float, 1>(p.mode);
        if (p.dim == 2) return grouped ? dtma_pick<float, 2, true>(p.mode) : dtma_pick<float, 2>(p.mode);
        return dtma_pick<float, 3>(p.mode);
    }
    if (p.dim == 1) return dtma_pick<double, 1>(p.mode);
    if (p.dim == 2) return grouped ? dtma_pick<double, 2, true>(p.mode) : dtma_pick<double, 2>(p.mode);
    return dtma_pick<double, 3>(p.mode);
}

// Tiles per decompress ticket chosen for large arrays.
constexpr int kTicketTiles = 4;

// CUSZP_TICKET_TILES=1..16 in the environment fixes the TMA decompress kernel's tiles per
// ticket (0: the size-based choice) -- for tests of both ticket forms on small arrays.
static int ticket_tiles_override()
{
    static const int v = [] {
        const char* e = std::getenv("CUSZP_TICKET_TILES");
        const int x = e ? std::atoi(e) : 0;
        return x >= 1 && x <= kMaxTicketTiles ? x : 0;
    }();
    return v;
}

// Decompress through the TMA kernel when the stream and the output start on 16-byte
// boundaries; returns -1 when the caller should use the other decompress kernel.
static int launch_dtma(const Problem& p, const void* cmp, void* out, double eb, void* ws, cudaStream_t s)
{
    if (!tma_allowed() || ((reinterpret_cast<uintptr_t>(cmp) | reinterpret_cast<uintptr_t>(out)) & 15u)) return -1;
    alignas(64) CUtensorMap map;
    std::memset(&map, 0, sizeof(map));
    bool grouped = false;
    if (p.dim != 1 && !make_block_map(&map, p, out, &grouped)) return -1;
    const KernelRef k = dtma_kernel_for(p, grouped);
    const unsigned threads = k.threads;
    const unsigned grid = grid_for(k, p.g.ntiles);
    WsHeader* hdr = reinterpret_cast<WsHeader*>(ws);
    unsigned long long* status = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(ws) + sizeof(WsHeader));
    Geom g = p.g;
    g.grouped = grouped ? 1u : 0u;
    float ebf = (float)eb;
    void* dst = out;
    const void* src = cmp;
    // the look-back chain limits once decoding is fast: tickets of kTicketTiles tiles
    // when every front warp still gets two of them (measured on 512^3 f32 3D and 8192^2 f64
    // 2D: 4 tiles beat 1, 2, 3, 8 and 16), two tiles while there are more tiles than front
    // warps (2^23 and 2^24 f32 1D: 2 beat 1, 3 and 4 by 2-11 %; a group may end short at
    // the array's last tile), single tiles below that: a front warp loads a group's tiles
    // one after another into its one slot, and with fewer tiles than front warps that
    // serialisation costs more than the shorter chain saves (2^16-2^20 f32: 1 tile 4 us faster)
    const uint64_t front = (uint64_t)grid * (k.threads / 32 - DecCfg<double, 1>::WARPS);   // front warps
    int tickets = p.g.ntiles >= 2ull * kTicketTiles * front ? kTicketTiles : p.g.ntiles >= front ? 2 : 1;
    if (const int forced = ticket_tiles_override()) tickets = forced;
    void* args[] = {(void*)&map, (void*)&dst, (void*)&src, (void*)&g, p.type == 0 ? (void*)&ebf : (void*)&eb,
                    (void*)&hdr, (void*)&status, (void*)&tickets};
    return cudaLaunchKernel(k.fn, dim3(grid), dim3(threads), args, k.smem, s) == cudaSuccess ? OK : E_CUDA;
}

static int launch(const Problem& p, bool comp, const void* a0, void* a1, double eb, void* ws, cudaStream_t s)
{
    if (p.g.ntiles == 0) return OK;
    {
        const int st = comp ? launch_tma(p, a0, a1, eb, ws, s) : launch_dtma(p, a0, a1, eb, ws, s);
        if (st >= 0) return st;
    }
    const KernelRef k = kernel_for(p, comp);
    const unsigned grid = grid_for(k, p.g.ntiles);
    WsHeader* hdr = reinterpret_cast<WsHeader*>(ws);
    unsigned long long* status = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(ws) + sizeof(WsHeader));
    Geom g = p.g;
    float ebf = (float)eb, rf = 0.5f / (float)eb;
    double rd = 0.5 / eb;
    // compress(in, cmp, g, recip, hdr, status) / decompress(out, cmp, g, eb, hdr, status)
    const void* src = a0;
    void* dst = a1;
    void* args[6];
    args[0] = comp ? (void*)&src : (void*)&dst;
    args[1] = comp ? (void*)&dst : (void*)&src;
    args[2] = &g;
    if (p.type == 0) args[3] = comp ? (void*)&rf : (void*)&ebf;
    else             args[3] = comp ? (void*)&rd : (void*)&eb;
    args[4] = &hdr;
    args[5] = &status;
    const cudaError_t e = cudaLaunchKernel(k.fn, dim3(grid), dim3(kThreads), args, k.smem, s);
    return e == cudaSuccess ? OK : E_CUDA;
}

int launch_compress(const Problem& p, const void* d_in, uint8_t* d_cmp, double eb, void* ws, cudaStream_t s,
                    unsigned long long* d_size)
{
    if (!d_size) return launch(p, true, d_in, d_cmp, eb, ws, s);
    Problem q = p;
    q.g.size_out = d_size;
    return launch(q, true, d_in, d_cmp, eb, ws, s);
}

int launch_decompress(const Problem& p, void* d_out, const uint8_t* d_cmp, double eb, void* ws, cudaStream_t s)
{
    return launch(p, false, d_cmp, d_out, eb, ws, s);
}

// ------------------------------------------------------------------ value range

constexpr int kRangeThreads = 256;
constexpr int kRangeBlocks = 148 * 4;

size_t range_ws_bytes(size_t) { return sizeof(double) * 2 * (kRangeBlocks + 1) + 16; }

template <typename T>
__global__ void __launch_bounds__(kRangeThreads)
range_kernel(const T* __restrict__ in, size_t n, T* __restrict__ partial, unsigned* __restrict__ counter,
             T* __restrict__ result)
{
    T mx = -INFINITY, mn = INFINITY;   // NaN-skipping running extrema
    range_accumulate(in, 0, n, (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, (uint64_t)gridDim.x * blockDim.x, mx,
                     mn);
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(FULL, mx, o));
        mn = fmin(mn, __shfl_xor_sync(FULL, mn, o));
    }
    __shared__ T smx[kRangeThreads / 32], smn[kRangeThreads / 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { smx[warp] = mx; smn[warp] = mn; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kRangeThreads / 32; w++) { mx = fmax(mx, smx[w]); mn = fmin(mn, smn[w]); }
        partial[2 * blockIdx.x] = mx;
        partial[2 * blockIdx.x + 1] = mn;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        T gmx = -INFINITY, gmn = INFINITY;
        for (unsigned b = 0; b < gridDim.x; b++) {
            gmx = fmax(gmx, ((volatile T*)partial)[2 * b]);
            gmn = fmin(gmn, ((volatile T*)partial)[2 * b + 1]);
        }
        const T first = in[0];
        if (first != first) { gmx = first; gmn = first; }   // CLI loop starts from element 0
        result[0] = gmn;
        result[1] = gmx;
        *counter = 0u;
    }
}

int launch_range(const void* d_in, size_t n, int type, void* d_minmax, void* ws, cudaStream_t s)
{
    if (n == 0) return E_ARG;
    unsigned* counter = reinterpret_cast<unsigned*>(ws);
    char* part = reinterpret_cast<char*>(ws) + 16;
    const size_t per_block = 4096;
    unsigned grid = (unsigned)((n + per_block - 1) / per_block);
    if (grid > (unsigned)kRangeBlocks) grid = kRangeBlocks;
    if (grid == 0) grid = 1;
    if (type == 0)
        range_kernel<float><<<grid, kRangeThreads, 0, s>>>((const float*)d_in, n, (float*)part, counter, (float*)d_minmax);
    else
        range_kernel<double><<<grid, kRangeThreads, 0, s>>>((const double*)d_in, n, (double*)part, counter, (double*)d_minmax);
    return cudaGetLastError() == cudaSuccess ? OK : E_CUDA;
}

}  // namespace cuszp

// batch.cu -- batched compression/decompression of many arrays in one persistent
// launch, behind a plan object (include/cuSZp.h: cuSZp_batch_*):
//   plan_create  -> device item table, tile map and value-range chunk map (once)
//   plan_tune    -> autotuner: tile shape (warps x blocks per warp) and CTAs per SM
//   plan_execute -> [value-range pass -> eb per array] -> one codec launch;
//                   only kernel launches on the stream, so it can be captured in
//                   a CUDA graph and replayed.
// Per array the output is byte-identical to the single-array path: the tile body
// is the same pipelined compress/decompress phases, with each array's own look-back chain.
#include "../../include/cuSZp.h"
#include "batch.cuh"
#include "codec_kernels.cuh"
#include "codec_launch.cuh"
#include "decompress_tma.cuh"

#include <algorithm>
#include <cstddef>
#include <type_traits>
#include <cstring>
#include <vector>

namespace cuszp {

// ------------------------------------------------------------------ maps and value ranges

__global__ void fill_maps_kernel(const BatchItem* __restrict__ items, int n, uint32_t* __restrict__ tile_map,
                                 uint32_t* __restrict__ chunk_map)
{
    for (int a = blockIdx.x; a < n; a += gridDim.x) {
        const BatchItem& it = items[a];
        for (uint64_t t = threadIdx.x; t < it.g.ntiles; t += blockDim.x) tile_map[it.tile_start + t] = (uint32_t)a;
        if (chunk_map)
            for (uint64_t c = threadIdx.x; c < it.nchunks; c += blockDim.x) chunk_map[it.chunk_start + c] = (uint32_t)a;
    }
}

template <typename T>
__global__ void __launch_bounds__(256)
range_partial_kernel(const BatchItem* __restrict__ items, const uint32_t* __restrict__ chunk_map,
                     uint64_t total_chunks, double* __restrict__ partial)
{
    __shared__ double smx[8], smn[8];
    for (uint64_t c = blockIdx.x; c < total_chunks; c += gridDim.x) {
        const BatchItem& it = items[chunk_map[c]];
        const T* in = static_cast<const T*>(it.in);
        const uint64_t n = it.g.nbEle;
        const uint64_t lo = (c - it.chunk_start) * kRangeChunk;
        const uint64_t hi = min(n, lo + kRangeChunk);
        T mx = -INFINITY, mn = INFINITY;   // NaN-skipping
        range_accumulate(in, lo, hi, threadIdx.x, blockDim.x, mx, mn);
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            mx = fmax(mx, __shfl_xor_sync(FULL, mx, o));
            mn = fmin(mn, __shfl_xor_sync(FULL, mn, o));
        }
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (lane == 0) { smx[warp] = (double)mx; smn[warp] = (double)mn; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = smx[0], b = smn[0];
            for (int w = 1; w < (int)(blockDim.x / 32); w++) { a = fmax(a, smx[w]); b = fmin(b, smn[w]); }
            partial[2 * c] = b;
            partial[2 * c + 1] = a;
        }
        __syncthreads();
    }
}

// eb = rel * (max - min) with the reference CLI's float arithmetic
// (examples/cuSZp.cpp:186 f32, :209 f64); NaN-first arrays give NaN.
template <typename T>
__global__ void range_finalize_kernel(BatchItem* __restrict__ items, int n, const double* __restrict__ partial)
{
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
        BatchItem& it = items[a];
        if (it.rel < 0.0f || it.nchunks == 0) continue;   // absolute bound given
        double mn = INFINITY, mx = -INFINITY;
        for (uint64_t c = it.chunk_start; c < it.chunk_start + it.nchunks; c++) {
            mn = fmin(mn, partial[2 * c]);
            mx = fmax(mx, partial[2 * c + 1]);
        }
        const T first = static_cast<const T*>(it.in)[0];
        if (first != first) { mn = (double)first; mx = (double)first; }
        if (sizeof(T) == 4) it.eb = it.rel * ((float)mx - (float)mn);
        else it.eb = it.rel * (float)(mx - mn);
    }
}

// ------------------------------------------------------------------ batched codec

template <typename T> __device__ __forceinline__ T recip_of(float eb);
template <> __device__ __forceinline__ float recip_of<float>(float eb) { return __fdiv_rn(0.5f, eb); }
template <> __device__ __forceinline__ double recip_of<double>(float eb) { return __ddiv_rn(0.5, (double)eb); }

// Calls f(integral_constant<int, mode>) so per-array modes reach template code.
template <typename F>
__device__ __forceinline__ void with_mode(int mode, F&& f)
{
    switch (mode) {
        case 0: f(std::integral_constant<int, 0>{}); break;
        case 1: f(std::integral_constant<int, 1>{}); break;
        default: f(std::integral_constant<int, 2>{}); break;
    }
}

// Thread 0 takes a ticket and looks up its array (tile_map) into slot `k`.
template <int WARPS>
__device__ __forceinline__ void take_ticket(TileShared<WARPS>& sh, uint32_t* s_item, int k, WsHeader* hdr,
                                            const uint32_t* __restrict__ tile_map, uint64_t total_tiles)
{
    const int64_t t = (int64_t)atomicAdd(&hdr->ticket, 1u);
    sh.ticket[k] = t;
    s_item[k] = (uint64_t)t < total_tiles ? tile_map[t] : 0u;
}

// Tile source over the arrays of a batch: tickets index the global tile sequence,
// the tile map names the array, each array has its own status words and bound.
template <typename T, int DIM, typename Tl>
struct BatchSource {
    const BatchItem* items;
    const uint32_t* tile_map;
    uint64_t total_tiles;
    WsHeader* hdr;
    unsigned long long* status;
    unsigned long long* sizes;
    __device__ __forceinline__ void take(PipeShared<Tl::WARPS>& sp, int k)
    {
        const int64_t t = (int64_t)atomicAdd(&hdr->ticket, 1u);
        sp.ticket[k] = t;
        sp.item[k] = (uint64_t)t < total_tiles ? tile_map[t] : 0u;
    }
    __device__ __forceinline__ bool ctx(const PipeShared<Tl::WARPS>& sp, int k, TileCtx& c) const
    {
        const int64_t t = sp.ticket[k];
        if ((uint64_t)t >= total_tiles) return false;
        const uint32_t a = sp.item[k];
        const BatchItem& it = items[a];
        c.in = it.in;
        c.cmp = static_cast<uint8_t*>(it.out);
        c.g = it.g;
        c.status = status + it.tile_start;
        c.total_out = sizes + a;
        c.local = t - (int64_t)it.tile_start;
        c.mode = it.mode;
        c.eb = it.eb;
        return true;
    }
    __device__ __forceinline__ unsigned long long encode(const T* buf, uint32_t ok0, uint32_t ok1, const TileCtx& c,
                                                         uint8_t* sb, PipeShared<Tl::WARPS>& sp) const
    {
        const T recip = recip_of<T>(c.eb);
        unsigned long long agg = 0;
        with_mode(c.mode, [&](auto m) { agg = encode_tile<T, DIM, decltype(m)::value, Tl>(buf, ok0, ok1, c, recip, sb, sp); });
        return agg;
    }
};

template <typename T, int DIM, typename Tl>
__global__ void __launch_bounds__(Tl::THREADS, 512 / Tl::THREADS > 0 ? 512 / Tl::THREADS : 1)
compress_batch_kernel(const BatchItem* __restrict__ items, const uint32_t* __restrict__ tile_map,
                      uint64_t total_tiles, WsHeader* __restrict__ hdr, unsigned long long* __restrict__ status,
                      unsigned long long* __restrict__ sizes)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BatchSource<T, DIM, Tl> src{items, tile_map, total_tiles, hdr, status, sizes};
    compress_pipeline<T, DIM, Tl>(src, smem_raw, &hdr->err);
    finish_cta(hdr, status, total_tiles);
}

template <typename T, int DIM, typename Tl>
__global__ void __launch_bounds__(Tl::THREADS, 512 / Tl::THREADS > 0 ? 512 / Tl::THREADS : 1)
decompress_batch_kernel(const BatchItem* __restrict__ items, const uint32_t* __restrict__ tile_map,
                        uint64_t total_tiles, WsHeader* __restrict__ hdr, unsigned long long* __restrict__ status,
                        unsigned long long* __restrict__ sizes)
{
    __shared__ TileShared<Tl::WARPS> sh;
    __shared__ uint32_t s_item[2];
    if (threadIdx.x == 0) take_ticket<Tl::WARPS>(sh, s_item, 0, hdr, tile_map, total_tiles);
    __syncthreads();
    int64_t tile = sh.ticket[0];
    uint32_t a = s_item[0];
    int slot = 0;
    DecompRates<Tl> R;
    if ((uint64_t)tile < total_tiles) {
        const BatchItem& it = items[a];
        const int64_t local = tile - (int64_t)it.tile_start;
        with_mode(it.mode, [&](auto m) {
            decompress_rates<DIM, decltype(m)::value, Tl>(R, static_cast<const uint8_t*>(it.in), it.g, local);
        });
        post_aggregate<Tl::WARPS>(R.wtot, local, status + it.tile_start, sh.dwarp[0], &sh.dagg[0]);
    }
    for (int k = 1; (uint64_t)tile < total_tiles; k++) {
        if (threadIdx.x == 0) take_ticket<Tl::WARPS>(sh, s_item, k & 1, hdr, tile_map, total_tiles);
        __syncthreads();
        const int64_t next = sh.ticket[k & 1];
        const uint32_t an = s_item[k & 1];
        DecompRates<Tl> Rn = R;
        if ((uint64_t)next < total_tiles) {
            const BatchItem& itn = items[an];
            const int64_t ln = next - (int64_t)itn.tile_start;
            with_mode(itn.mode, [&](auto m) {
                decompress_rates<DIM, decltype(m)::value, Tl>(Rn, static_cast<const uint8_t*>(itn.in), itn.g, ln);
            });
            post_aggregate<Tl::WARPS>(Rn.wtot, ln, status + itn.tile_start, sh.dwarp[slot ^ 1], &sh.dagg[slot ^ 1]);
        }
        const BatchItem& it = items[a];
        const Geom g = it.g;
        const int64_t local = tile - (int64_t)it.tile_start;
        const uint8_t* cmp = static_cast<const uint8_t*>(it.in);
        const uint64_t excl = resolve_tile<Tl::WARPS>(local, g.ntiles, status + it.tile_start, &hdr->err, sizes + a,
                                                      g.rate_bytes, sh.dagg[slot], sh.lb);
        const uint8_t* pbase = cmp + g.rate_bytes + excl + sh.dwarp[slot][threadIdx.x >> 5];
        const T eb = (T)it.eb;
        T* out = static_cast<T*>(it.out);
        DecompPayload<DIM, Tl> P;
        with_mode(it.mode, [&](auto m) {
            decompress_load<DIM, decltype(m)::value, Tl>(P, R, pbase);
            decompress_store<T, DIM, decltype(m)::value, Tl>(P, R, out, g, eb, local);
        });
        tile = next;
        a = an;
        R = Rn;
        slot ^= 1;
    }
    finish_cta(hdr, status, total_tiles);
}

// ------------------------------------------------------------------ batched TMA codec

// Tile source of the warp-specialised TMA kernels over the arrays of a batch: the tile
// map names a global tile's array; each array has its own stream, status words, bound,
// encoding mode and (2D/3D) tensor map.  COMP: items hold (data, stream), else
// (stream, data).
template <typename T, bool COMP>
struct BatchTiles {
    const BatchItem* items;
    const uint32_t* tile_map;
    const CUtensorMap* tmaps;   // one per array (2D/3D); written by the host before the launch
    uint64_t total_tiles;
    unsigned long long* status;
    unsigned long long* sizes;
    __device__ __forceinline__ uint64_t total() const { return total_tiles; }
    __device__ __forceinline__ unsigned long long* size_out() const { return nullptr; }   // per array: `sizes`
    // one tile per ticket: a group of tiles could straddle two arrays
    __device__ __forceinline__ int ticket_tiles() const { return 1; }
    __device__ __forceinline__ void locate(int64_t t, int32_t& a, int64_t& local) const
    {
        a = (int32_t)__ldg(tile_map + t);
        local = t - (int64_t)items[a].tile_start;
    }
    __device__ __forceinline__ TileArray array(int32_t a) const
    {
        const BatchItem& it = items[a];
        void* data = COMP ? const_cast<void*>(it.in) : it.out;
        uint8_t* cmp = static_cast<uint8_t*>(COMP ? it.out : const_cast<void*>(it.in));
        return TileArray{data, cmp, &it.g, status + it.tile_start, sizes + a, tmaps + a, it.eb, it.mode};
    }
    __device__ __forceinline__ T recip_of(const TileArray& A) const { return cuszp::recip_of<T>(A.eb); }
    __device__ __forceinline__ T eb_of(const TileArray& A) const { return (T)A.eb; }
    // The map was copied into global memory by the host: order that write before the
    // tensor-map proxy reads it.
    __device__ __forceinline__ void acquire_map(const CUtensorMap* m) const
    {
        asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;" ::"l"(m) : "memory");
    }
    template <typename F>
    __device__ __forceinline__ void with_mode(int mode, F&& f) const { cuszp::with_mode(mode, static_cast<F&&>(f)); }
};

template <typename T, int DIM>
__global__ void __launch_bounds__(TmaCfg<T, DIM>::THREADS, 2)
compress_tma_batch_kernel(const BatchItem* __restrict__ items, const uint32_t* __restrict__ tile_map,
                          const CUtensorMap* __restrict__ tmaps, uint64_t total_tiles, WsHeader* __restrict__ hdr,
                          unsigned long long* __restrict__ status, unsigned long long* __restrict__ sizes)
{
    const BatchTiles<T, true> src{items, tile_map, tmaps, total_tiles, status, sizes};
    compress_tma_body<T, DIM>(src, hdr, status);
}

template <typename T, int DIM>
__global__ void __launch_bounds__(DecCfg<T, DIM>::THREADS, DecCfg<T, DIM>::MIN_CTAS)
decompress_tma_batch_kernel(const BatchItem* __restrict__ items, const uint32_t* __restrict__ tile_map,
                            const CUtensorMap* __restrict__ tmaps, uint64_t total_tiles, WsHeader* __restrict__ hdr,
                            unsigned long long* __restrict__ status, unsigned long long* __restrict__ sizes)
{
    const BatchTiles<T, false> src{items, tile_map, tmaps, total_tiles, status, sizes};
    decompress_tma_body<T, DIM, false>(src, hdr, status);
}

// ------------------------------------------------------------------ tile-shape variants

struct Variant {
    int warps, bpw1, bpwn;   // codec warps per CTA; data blocks per codec warp in 1D and in 2D/3D
    int (*threads)(int type, int dim, bool comp);   // threads per CTA
    bool tma;                // warp-specialised TMA kernels: arrays on 16-byte boundaries only
    const void* (*kernel)(int type, int dim, bool comp);
    size_t (*smem)(int type, int dim, bool comp);   // dynamic shared memory (set on first use)
};

template <int DIM, int WARPS, int BPW>
static const void* kernel_for_variant(int type, bool comp)
{
    using Tl = Tiling<DIM, WARPS, BPW>;
    if (type == 0) return comp ? (const void*)compress_batch_kernel<float, DIM, Tl> : (const void*)decompress_batch_kernel<float, DIM, Tl>;
    return comp ? (const void*)compress_batch_kernel<double, DIM, Tl> : (const void*)decompress_batch_kernel<double, DIM, Tl>;
}

// Enables (once per device) the dynamic shared memory a kernel needs and returns it
// (a refusal surfaces as the launch's error).
static size_t enable_smem(const void* fn, size_t bytes)
{
    enable_dynamic_smem(fn, bytes);
    return bytes;
}

template <typename T, int DIM, typename Tl>
static size_t smem_for_variant(bool comp)
{
    if (!comp) return 0;
    return enable_smem((const void*)compress_batch_kernel<T, DIM, Tl>, compress_smem_bytes<T, DIM, Tl>());
}

template <int WARPS, int BPW1D, int BPWND>
static const void* kv(int type, int dim, bool comp)
{
    if (dim == 1) return kernel_for_variant<1, WARPS, BPW1D>(type, comp);
    if (dim == 2) return kernel_for_variant<2, WARPS, BPWND>(type, comp);
    return kernel_for_variant<3, WARPS, BPWND>(type, comp);
}

template <int WARPS, int BPW1D, int BPWND>
static size_t ks(int type, int dim, bool comp)
{
    if (type == 0) {
        if (dim == 1) return smem_for_variant<float, 1, Tiling<1, WARPS, BPW1D>>(comp);
        if (dim == 2) return smem_for_variant<float, 2, Tiling<2, WARPS, BPWND>>(comp);
        return smem_for_variant<float, 3, Tiling<3, WARPS, BPWND>>(comp);
    }
    if (dim == 1) return smem_for_variant<double, 1, Tiling<1, WARPS, BPW1D>>(comp);
    if (dim == 2) return smem_for_variant<double, 2, Tiling<2, WARPS, BPWND>>(comp);
    return smem_for_variant<double, 3, Tiling<3, WARPS, BPWND>>(comp);
}

template <typename T, int DIM>
static const void* tma_batch_kernel(bool comp)
{
    return comp ? (const void*)compress_tma_batch_kernel<T, DIM> : (const void*)decompress_tma_batch_kernel<T, DIM>;
}

template <typename T, int DIM>
static size_t tma_batch_smem(bool comp)
{
    return comp ? enable_smem(tma_batch_kernel<T, DIM>(true), TmaCfg<T, DIM>::smem_bytes())
                : enable_smem(tma_batch_kernel<T, DIM>(false), DecCfg<T, DIM>::smem_bytes());
}

template <int N>
static int fixed_threads(int, int, bool) { return N; }

template <typename T>
static int tma_threads_of(int dim, bool comp)
{
    if (comp) return dim == 1 ? TmaCfg<T, 1>::THREADS : dim == 2 ? TmaCfg<T, 2>::THREADS : TmaCfg<T, 3>::THREADS;
    return dim == 1 ? DecCfg<T, 1>::THREADS : dim == 2 ? DecCfg<T, 2>::THREADS : DecCfg<T, 3>::THREADS;
}

static int tma_threads(int type, int dim, bool comp)
{
    return type == 0 ? tma_threads_of<float>(dim, comp) : tma_threads_of<double>(dim, comp);
}

static const void* tk(int type, int dim, bool comp)
{
    if (type == 0) return dim == 1 ? tma_batch_kernel<float, 1>(comp) : dim == 2 ? tma_batch_kernel<float, 2>(comp) : tma_batch_kernel<float, 3>(comp);
    return dim == 1 ? tma_batch_kernel<double, 1>(comp) : dim == 2 ? tma_batch_kernel<double, 2>(comp) : tma_batch_kernel<double, 3>(comp);
}

static size_t tks(int type, int dim, bool comp)
{
    if (type == 0) return dim == 1 ? tma_batch_smem<float, 1>(comp) : dim == 2 ? tma_batch_smem<float, 2>(comp) : tma_batch_smem<float, 3>(comp);
    return dim == 1 ? tma_batch_smem<double, 1>(comp) : dim == 2 ? tma_batch_smem<double, 2>(comp) : tma_batch_smem<double, 3>(comp);
}

// Variant 0 is the TMA kernel pair (8 codec warps; the same tiles as variant 1);
// then the cp.async kernels as (warps per CTA, blocks per warp in 1D, in 2D/3D).
static const Variant kVariants[] = {
    {8, 16, 8, tma_threads, true, tk, tks},
    {8, 16, 8, fixed_threads<256>, false, kv<8, 16, 8>, ks<8, 16, 8>},
    {4, 16, 8, fixed_threads<128>, false, kv<4, 16, 8>, ks<4, 16, 8>},
    {8, 8, 4, fixed_threads<256>, false, kv<8, 8, 4>, ks<8, 8, 4>},
    {16, 8, 4, fixed_threads<512>, false, kv<16, 8, 4>, ks<16, 8, 4>},
};
static_assert(TmaCfg<float, 1>::TB == 8 * 16 && TmaCfg<float, 2>::TB == 8 * 8 && TmaCfg<double, 2>::TB == 8 * 8,
              "TMA tiles as in variant 1");
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

}  // namespace cuszp

using namespace cuszp;

extern "C" void cuSZp_batch_plan_destroy_async(cuszp_batch_plan_t p, cudaStream_t stream);

struct cuszp_batch_plan {
    int count = 0;
    int dim = 1, type = 0;
    bool compress = true;
    bool any_rel = false;
    int variant = 1;
    int ctas_per_sm = 0;       // 0: occupancy limit
    bool configured = false;   // variant chosen by the autotuner or set_config
    bool tma_ok = false;       // every array suits the TMA kernels (variant 0)
    CUtensorMap* d_maps = nullptr;   // per-array tensor maps of the TMA kernels (2D/3D)
    int cap_items = 0, cap_maps = 0; // device capacity of d_items / d_maps (arrays)
    // pinned staging of the uploads (items, maps): the copies are truly asynchronous and
    // never wait on the stream; `staged` marks when the last upload has read them
    BatchItem* h_items = nullptr;
    CUtensorMap* h_maps = nullptr;
    int hcap_items = 0, hcap_maps = 0;
    std::vector<void*> h_old;        // outgrown staging buffers, freed with the plan
    cudaEvent_t staged = nullptr;
    std::vector<uint8_t> grouped;    // per array: its map is a grouped 2D map
    int sms = 148;
    std::vector<cuszp_batch_item_t> host_items;
    std::vector<BatchItem> items;
    BatchItem* d_items = nullptr;
    void* d_ws = nullptr;      // header + status + tile map + chunk map + partials
    size_t ws_bytes = 0;
    uint64_t total_tiles = 0, total_chunks = 0;
    size_t status_off = 0, map_off = 0, cmap_off = 0, part_off = 0;
};

// Pinned host memory of at least `n` elements of T for a staging buffer (grown by
// doubling; an outgrown buffer is kept until the plan is destroyed, as freeing pinned
// memory would synchronize the device).
template <typename T>
static int grow_pinned(cuszp_batch_plan* p, T** buf, int* cap, int n)
{
    if (n <= *cap) return OK;
    const int want = std::max(n, 2 * *cap);
    void* q = nullptr;
    if (cudaHostAlloc(&q, sizeof(T) * (size_t)want, cudaHostAllocDefault) != cudaSuccess) return E_CUDA;
    if (*buf) p->h_old.push_back(*buf);
    *buf = static_cast<T*>(q);
    *cap = want;
    return OK;
}

// Device memory of at least `n` elements of T (grown by doubling, stream-ordered on s).
template <typename T>
static int grow_device(T** buf, int* cap, int n, cudaStream_t s)
{
    if (n <= *cap && *buf) return OK;
    const int want = std::max(std::max(n, 1), 2 * *cap);
    if (*buf) cudaFreeAsync(*buf, s);
    *buf = nullptr;
    *cap = 0;
    if (cudaMallocAsync((void**)buf, sizeof(T) * (size_t)want, s) != cudaSuccess) return E_CUDA;
    *cap = want;
    return OK;
}

// The staging buffers are free once the previous upload has read them.
static int stage_wait(cuszp_batch_plan* p)
{
    return p->staged && cudaEventSynchronize(p->staged) != cudaSuccess ? E_CUDA : OK;
}

// Uploads the item table through the pinned staging buffer.
static int stage_items(cuszp_batch_plan* p, cudaStream_t s)
{
    int st = stage_wait(p);
    if (!st) st = grow_pinned(p, &p->h_items, &p->hcap_items, p->count);
    if (st) return st;
    std::memcpy(p->h_items, p->items.data(), sizeof(BatchItem) * p->count);
    if (cudaMemcpyAsync(p->d_items, p->h_items, sizeof(BatchItem) * p->count, cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaEventRecord(p->staged, s) != cudaSuccess)
        return E_CUDA;
    return OK;
}

// (Re)builds the device item table, workspace and maps for a tile shape.  All
// device work is stream-ordered on `s`; nothing here synchronizes the device.
static int plan_layout(cuszp_batch_plan* p, int variant, cudaStream_t s)
{
    const Variant& v = kVariants[variant];
    const int tb = v.warps * (p->dim == 1 ? v.bpw1 : v.bpwn);
    uint64_t tiles = 0, chunks = 0;
    for (int a = 0; a < p->count; a++) {
        const cuszp_batch_item_t& h = p->host_items[a];
        Problem pr;
        int st = make_problem(pr, p->type, h.mode, p->dim, h.nbEle, h.dims.x, h.dims.y, h.dims.z);
        if (st) return st;
        Geom g = pr.g;
        if (p->dim == 1) g.ntiles = g.rate_bytes / (uint64_t)tb;
        else g.ntiles = (g.nblocks + tb - 1) / tb;
        BatchItem& it = p->items[a];
        std::memset(&it, 0, sizeof(it));
        it.in = h.d_in;
        it.out = h.d_out;
        it.g = g;
        it.g.grouped = (size_t)a < p->grouped.size() ? p->grouped[a] : 0u;   // read by the TMA kernels only
        it.tile_start = tiles;
        it.mode = h.mode;
        it.eb = h.rel ? 0.0f : h.errorBound;
        it.rel = h.rel ? h.errorBound : -1.0f;
        it.chunk_start = chunks;
        it.nchunks = (h.rel && p->compress) ? (g.nbEle + kRangeChunk - 1) / kRangeChunk : 0;
        tiles += g.ntiles;
        chunks += it.nchunks;
    }
    p->total_tiles = tiles;
    p->total_chunks = chunks;
    p->status_off = sizeof(WsHeader);
    p->map_off = p->status_off + 8 * (tiles ? tiles : 1);
    p->cmap_off = (p->map_off + 4 * (tiles ? tiles : 1) + 15) / 16 * 16;
    p->part_off = (p->cmap_off + 4 * (chunks ? chunks : 1) + 15) / 16 * 16;
    const size_t need = p->part_off + 16 * (chunks ? chunks : 1);
    if (need > p->ws_bytes) {
        if (p->d_ws) cudaFreeAsync(p->d_ws, s);
        p->d_ws = nullptr;
        if (cudaMallocAsync(&p->d_ws, need, s) != cudaSuccess) return E_CUDA;
        p->ws_bytes = need;
    }
    if (cudaMemsetAsync(p->d_ws, 0, p->ws_bytes, s) != cudaSuccess) return E_CUDA;
    if (p->count) {
        int st = stage_items(p, s);
        if (st) return st;
    }
    char* ws = static_cast<char*>(p->d_ws);
    if (p->count)
        fill_maps_kernel<<<std::min(p->count, 4096), 256, 0, s>>>(p->d_items, p->count, (uint32_t*)(ws + p->map_off),
                                                                  chunks ? (uint32_t*)(ws + p->cmap_off) : nullptr);
    if (cudaGetLastError() != cudaSuccess) return E_CUDA;
    p->variant = variant;
    return OK;
}

// Decides whether every array suits the TMA kernels (data and stream on 16-byte
// boundaries; for 2D/3D a tensor map the driver accepts) and uploads the maps.
static int plan_maps(cuszp_batch_plan* p, cudaStream_t s)
{
    p->tma_ok = tma_allowed();
    std::vector<CUtensorMap> maps(p->dim == 1 ? 0 : (size_t)p->count);
    p->grouped.assign((size_t)p->count, 0);
    for (int a = 0; a < p->count && p->tma_ok; a++) {
        const cuszp_batch_item_t& h = p->host_items[a];
        if (h.nbEle == 0) continue;   // no tiles
        if ((reinterpret_cast<uintptr_t>(h.d_in) | reinterpret_cast<uintptr_t>(h.d_out)) & 15u) p->tma_ok = false;
        if (p->dim == 1 || !p->tma_ok) continue;
        Problem pr;
        if (make_problem(pr, p->type, h.mode, p->dim, h.nbEle, h.dims.x, h.dims.y, h.dims.z)) {
            p->tma_ok = false;
            continue;
        }
        std::memset(&maps[a], 0, sizeof(CUtensorMap));
        bool grouped = false;
        if (!make_block_map(&maps[a], pr, p->compress ? h.d_in : h.d_out, &grouped)) p->tma_ok = false;
        p->grouped[a] = grouped ? 1 : 0;
    }
    if (!p->tma_ok || maps.empty()) return OK;
    const int n = (int)maps.size();
    int st = grow_device(&p->d_maps, &p->cap_maps, n, s);
    if (!st) st = stage_wait(p);
    if (!st) st = grow_pinned(p, &p->h_maps, &p->hcap_maps, n);
    if (st) return st;
    std::memcpy(p->h_maps, maps.data(), sizeof(CUtensorMap) * n);
    if (cudaMemcpyAsync(p->d_maps, p->h_maps, sizeof(CUtensorMap) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaEventRecord(p->staged, s) != cudaSuccess)
        return E_CUDA;
    return OK;
}

static int plan_launch(cuszp_batch_plan* p, unsigned long long* d_sizes, cudaStream_t s)
{
    char* ws = static_cast<char*>(p->d_ws);
    if (p->compress && p->total_chunks) {
        const unsigned grid = (unsigned)std::min<uint64_t>(p->total_chunks, (uint64_t)p->sms * 8);
        double* part = (double*)(ws + p->part_off);
        const uint32_t* cmap = (const uint32_t*)(ws + p->cmap_off);
        if (p->type == 0) {
            range_partial_kernel<float><<<grid, 256, 0, s>>>(p->d_items, cmap, p->total_chunks, part);
            range_finalize_kernel<float><<<(p->count + 127) / 128, 128, 0, s>>>(p->d_items, p->count, part);
        } else {
            range_partial_kernel<double><<<grid, 256, 0, s>>>(p->d_items, cmap, p->total_chunks, part);
            range_finalize_kernel<double><<<(p->count + 127) / 128, 128, 0, s>>>(p->d_items, p->count, part);
        }
    }
    if (p->total_tiles == 0) return cudaGetLastError() == cudaSuccess ? OK : E_CUDA;
    const Variant& v = kVariants[p->variant];
    const void* fn = v.kernel(p->type, p->dim, p->compress);
    const size_t smem = v.smem(p->type, p->dim, p->compress);
    const int threads = v.threads(p->type, p->dim, p->compress);
    const int occ = std::max(1, resident_ctas(fn, threads, smem));
    const int per_sm = p->ctas_per_sm > 0 ? std::min(p->ctas_per_sm, occ) : occ;
    const uint64_t want = (uint64_t)p->sms * per_sm;
    const unsigned grid = (unsigned)std::min<uint64_t>(want, p->total_tiles);
    const BatchItem* items = p->d_items;
    const uint32_t* map = (const uint32_t*)(ws + p->map_off);
    uint64_t total = p->total_tiles;
    WsHeader* hdr = (WsHeader*)ws;
    unsigned long long* status = (unsigned long long*)(ws + p->status_off);
    const CUtensorMap* maps = p->d_maps;
    void* args_cp[] = {(void*)&items, (void*)&map, (void*)&total, (void*)&hdr, (void*)&status, (void*)&d_sizes};
    void* args_tma[] = {(void*)&items, (void*)&map, (void*)&maps, (void*)&total, (void*)&hdr, (void*)&status,
                        (void*)&d_sizes};
    return cudaLaunchKernel(fn, dim3(grid), dim3(threads), v.tma ? args_tma : args_cp, smem, s) == cudaSuccess
               ? OK
               : E_CUDA;
}

extern "C" int cuSZp_batch_plan_create_async(cuszp_batch_plan_t* plan, int count, const cuszp_batch_item_t* items,
                                             cuszp_dim_t dim, cuszp_type_t type, int compress, cudaStream_t stream)
{
    if (!plan || count < 0 || (count && !items)) return E_ARG;
    if (type != CUSZP_TYPE_FLOAT && type != CUSZP_TYPE_DOUBLE) return E_ARG;
    if (dim < CUSZP_DIM_1D || dim > CUSZP_DIM_3D) return E_ARG;
    auto* p = new cuszp_batch_plan;
    p->count = count;
    p->dim = dim;
    p->type = type;
    p->compress = compress != 0;
    p->host_items.assign(items, items + count);
    p->items.resize(count);
    for (int a = 0; a < count; a++) {
        const cuszp_batch_item_t& h = items[a];
        if (h.mode < CUSZP_MODE_FIXED || h.mode > CUSZP_MODE_OUTLIER) { delete p; return E_ARG; }
        if (h.nbEle && (!h.d_in || !h.d_out)) { delete p; return E_ARG; }
        if (h.rel) p->any_rel = true;
    }
    p->sms = std::max(1, sm_count());
    int st = cudaEventCreateWithFlags(&p->staged, cudaEventDisableTiming) == cudaSuccess ? OK : E_CUDA;
    if (!st) st = grow_device(&p->d_items, &p->cap_items, count, stream);
    if (!st) st = plan_maps(p, stream);
    if (!st) st = plan_layout(p, p->tma_ok ? 0 : 1, stream);
    if (st) {
        cuSZp_batch_plan_destroy_async(p, stream);
        return st;
    }
    *plan = p;
    return OK;
}

extern "C" int cuSZp_batch_plan_update(cuszp_batch_plan_t p, int count, const cuszp_batch_item_t* items,
                                       cudaStream_t stream)
{
    if (!p || count < 0 || (count && !items)) return E_ARG;
    for (int a = 0; a < count; a++) {
        const cuszp_batch_item_t& h = items[a];
        if (h.mode < CUSZP_MODE_FIXED || h.mode > CUSZP_MODE_OUTLIER) return E_ARG;
        if (h.nbEle && (!h.d_in || !h.d_out)) return E_ARG;
    }
    p->count = count;
    p->host_items.assign(items, items + count);
    p->items.resize(count);
    p->any_rel = false;
    for (int a = 0; a < count; a++)
        if (items[a].rel) p->any_rel = true;
    int st = grow_device(&p->d_items, &p->cap_items, count, stream);
    if (!st) st = plan_maps(p, stream);
    if (st) return st;
    // a configured kernel pair is kept where the new arrays allow it; otherwise the default
    int variant = p->configured ? p->variant : (p->tma_ok ? 0 : 1);
    if (kVariants[variant].tma && !p->tma_ok) variant = 1;
    return plan_layout(p, variant, stream);
}

extern "C" int cuSZp_batch_plan_create(cuszp_batch_plan_t* plan, int count, const cuszp_batch_item_t* items,
                                       cuszp_dim_t dim, cuszp_type_t type, int compress)
{
    const int st = cuSZp_batch_plan_create_async(plan, count, items, dim, type, compress, 0);
    if (st) return st;
    return cudaStreamSynchronize(0) == cudaSuccess ? OK : E_CUDA;
}

extern "C" int cuSZp_batch_plan_execute(cuszp_batch_plan_t p, unsigned long long* d_sizes, cudaStream_t stream)
{
    if (!p || (p->count && !d_sizes)) return E_ARG;
    return plan_launch(p, d_sizes, stream);
}

extern "C" int cuSZp_batch_plan_check(cuszp_batch_plan_t p, cudaStream_t stream)
{
    if (!p) return E_ARG;
    return cuSZp_workspace_check(p->d_ws, p->ws_bytes, stream);
}

extern "C" int cuSZp_batch_plan_error_async(cuszp_batch_plan_t p, unsigned int* h_err, cudaStream_t stream)
{
    if (!p || !h_err) return E_ARG;
    if (!p->d_ws) {
        *h_err = 0u;
        return OK;
    }
    const char* w = static_cast<const char*>(p->d_ws) + offsetof(WsHeader, err);
    return cudaMemcpyAsync(h_err, w, sizeof(unsigned int), cudaMemcpyDeviceToHost, stream) == cudaSuccess ? OK : E_CUDA;
}

extern "C" int cuSZp_batch_plan_variant(cuszp_batch_plan_t p, int* variant, int* threadsPerBlock, int* tma)
{
    if (!p) return E_ARG;
    if (variant) *variant = p->variant;
    if (threadsPerBlock) *threadsPerBlock = kVariants[p->variant].threads(p->type, p->dim, p->compress);
    if (tma) *tma = kVariants[p->variant].tma ? 1 : 0;
    return OK;
}

extern "C" int cuSZp_batch_plan_config(cuszp_batch_plan_t p, int* warps, int* blocks_per_warp, int* ctas_per_sm)
{
    if (!p) return E_ARG;
    if (warps) *warps = kVariants[p->variant].warps;
    if (blocks_per_warp) *blocks_per_warp = p->dim == 1 ? kVariants[p->variant].bpw1 : kVariants[p->variant].bpwn;
    if (ctas_per_sm) *ctas_per_sm = p->ctas_per_sm;
    return OK;
}

// Autotuner: times every tile shape x CTAs-per-SM candidate on this plan's own
// arrays (CUDA events on `stream`, best of `reps`) and keeps the fastest.
extern "C" int cuSZp_batch_plan_tune(cuszp_batch_plan_t p, unsigned long long* d_sizes, int reps, cudaStream_t stream)
{
    if (!p || (p->count && !d_sizes)) return E_ARG;
    if (reps < 1) reps = 1;
    struct Events {
        cudaEvent_t e0, e1;
        Events() { cudaEventCreate(&e0); cudaEventCreate(&e1); }
        ~Events() { cudaEventDestroy(e0); cudaEventDestroy(e1); }
    } ev;
    cudaEvent_t e0 = ev.e0, e1 = ev.e1;
    float best = 1e30f;
    int best_v = p->tma_ok ? 0 : 1, best_c = 0;
    for (int v = 0; v < kNumVariants; v++) {
        if (kVariants[v].tma && !p->tma_ok) continue;
        int st = plan_layout(p, v, stream);
        if (st) return st;
        const void* fn = kVariants[v].kernel(p->type, p->dim, p->compress);
        const size_t smem = kVariants[v].smem(p->type, p->dim, p->compress);
        const int occ = resident_ctas(fn, kVariants[v].threads(p->type, p->dim, p->compress), smem);
        for (int c = 1; c <= std::max(1, occ); c++) {
            p->ctas_per_sm = c;
            plan_launch(p, d_sizes, stream);   // warm
            float t_best = 1e30f;
            for (int r = 0; r < reps; r++) {
                cudaEventRecord(e0, stream);
                plan_launch(p, d_sizes, stream);
                cudaEventRecord(e1, stream);
                cudaEventSynchronize(e1);
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                t_best = std::min(t_best, ms);
            }
            if (t_best < best) { best = t_best; best_v = v; best_c = c; }
        }
        if (cuSZp_workspace_check(p->d_ws, p->ws_bytes, stream)) return E_TIMEOUT;
    }
    int st = plan_layout(p, best_v, stream);
    p->ctas_per_sm = best_c;
    p->configured = true;
    if (!st && cudaStreamSynchronize(stream) != cudaSuccess) st = E_CUDA;
    return st;
}

extern "C" int cuSZp_batch_plan_set_config(cuszp_batch_plan_t p, int variant, int ctas_per_sm)
{
    if (!p || variant < 0 || variant >= kNumVariants) return E_ARG;
    if (kVariants[variant].tma && !p->tma_ok) return E_UNSUPPORTED;
    const int st = plan_layout(p, variant, 0);
    p->ctas_per_sm = ctas_per_sm;
    p->configured = true;
    if (st) return st;
    return cudaStreamSynchronize(0) == cudaSuccess ? OK : E_CUDA;
}

extern "C" void cuSZp_batch_plan_destroy_async(cuszp_batch_plan_t p, cudaStream_t stream)
{
    if (!p) return;
    if (p->d_items) cudaFreeAsync(p->d_items, stream);
    if (p->d_ws) cudaFreeAsync(p->d_ws, stream);
    if (p->d_maps) cudaFreeAsync(p->d_maps, stream);
    // pinned staging: freed once the uploads that read it are done (freeing pinned
    // memory waits for the device; a plan is destroyed outside any hot loop)
    if (p->h_items || p->h_maps || !p->h_old.empty()) {
        if (p->staged) cudaEventSynchronize(p->staged);
        if (p->h_items) cudaFreeHost(p->h_items);
        if (p->h_maps) cudaFreeHost(p->h_maps);
        for (void* q : p->h_old) cudaFreeHost(q);
    }
    if (p->staged) cudaEventDestroy(p->staged);
    delete p;
}

extern "C" void cuSZp_batch_plan_destroy(cuszp_batch_plan_t p)
{
    if (!p) return;
    cudaDeviceSynchronize();
    cuSZp_batch_plan_destroy_async(p, 0);
    cudaStreamSynchronize(0);
}

extern "C" int cuSZp_batch_plan_eb(cuszp_batch_plan_t p, float* errorBounds, cudaStream_t stream)
{
    if (!p || !errorBounds) return E_ARG;
    std::vector<BatchItem> tmp(p->count);
    if (p->count) {
        if (cudaMemcpyAsync(tmp.data(), p->d_items, sizeof(BatchItem) * p->count, cudaMemcpyDeviceToHost, stream) != cudaSuccess)
            return E_CUDA;
        if (cudaStreamSynchronize(stream) != cudaSuccess) return E_CUDA;
    }
    for (int a = 0; a < p->count; a++) errorBounds[a] = tmp[a].eb;
    return OK;
}

// compress_tma.cuh -- warp-specialised compress kernel for inputs that start on a
// 16-byte boundary (every torch allocation and every cudaMalloc'd buffer).
//
// One CTA = 8 codec warps + 1 loader warp + 1 resolver warp.  Tiles are the
// same as the other compress kernels' (128 blocks in 1D, 64 in 2D/3D), so the
// workspace and stream are identical.  A tile's bytes are produced at once but
// written DEFER tiles later, once its offset is known:
//
//   loader warp: takes tile tickets and loads each tile into an input slot with the
//     Tensor Memory Accelerator -- one `cp.async.bulk` of the tile's contiguous
//     elements in 1D; in 2D/3D one box of 8 whole blocks per codec warp where the
//     array's map allows it (grouped 2D maps: block order; f32 3D row boxes: 32 x 4 x 4,
//     128-byte swizzled), else one `cp.async.bulk.tensor.3d` box per data block in the
//     block's element order; OOB elements zero-filled -- completing on an mbarrier.
//     It refills a slot as soon as the codec warps are done with it.
//   codec warps (tile k): quantize + Lorenzo delta from the input slot, block rates
//     -> rate bytes, and sign maps + bit-planes packed into a span of the warp's
//     staging ring; the last warp to finish posts the tile aggregate.
//   resolver warp: runs the decoupled look-back of the CTA's tiles in order and
//     publishes their offsets.
//   codec warps, DEFER tiles later: the span is written to the stream with 16-byte
//     stores at the published offset.
// Codes never go through shared memory, so the input slots can be deep (three for
// f32, two for f64) at two CTAs per SM.  Every wait is bounded; on timeout the error
// word records it and the kernel ends.
#pragma once

#include <cuda.h>

#include <type_traits>

#include "codec_kernels.cuh"

namespace cuszp {

template <typename T, int DIM>
struct TmaCfg {
    // codec warps x data blocks per codec warp: f64 2D/3D tiles go to four codec warps of
    // 16 blocks (a warp's fixed per-tile costs spread over twice the blocks: 3 % faster on
    // the 8192^2 f64 array; f32 measured slower so), everything else to eight warps
    static constexpr bool WIDE = DIM != 1 && sizeof(T) == 8;
    static constexpr int WARPS = WIDE ? 4 : 8;
    // tiles between packing and writing out: a tile's offset must be resolved by then
    // (the look-back takes about as long as two f32 tiles, or three f64 tiles: f64
    // tiles are load-bound and shorter)
    static constexpr int DEFER = sizeof(T) == 4 ? 2 : 3;
    static constexpr int NC = DEFER + 1;                      // tile states (sizes, offsets, barriers)
    // Resolver r takes the tiles k = r, r + RESOLVERS, ...; RESOLVERS divides NC, so each
    // tile state has one resolver that takes its tiles in order and never waits on a
    // phase of a state barrier whose previous phase is still open (mbarrier parity
    // waits cannot tell a phase two ahead from one behind).
    // (one resolver keeps up with the codec warps and leaves them the issue slots:
    // measured 3-7 % faster than two or three)
    static constexpr int RESOLVERS = 1;
    static_assert(NC % RESOLVERS == 0, "each tile state has one resolver");
    static constexpr int LOADER = WARPS;                      // warp index of the loader
    static constexpr int THREADS = 32 * (WARPS + 1 + RESOLVERS);
    static constexpr int BPW = DIM == 1 || WIDE ? 16 : 8;     // data blocks per codec warp
    static constexpr int TB = WARPS * BPW;                    // data blocks per tile
    static constexpr int BLK = DIM == 1 ? 32 : 64;            // elements per data block
    static constexpr int TILE_ELEMS = TB * BLK;               // 4096
    static constexpr int TILE_BYTES = TILE_ELEMS * (int)sizeof(T);
    static constexpr int NIN = sizeof(T) == 4 ? 3 : 2;        // input slots
    static constexpr int MAXBLK = DIM == 1 ? 4 + 4 + 4 * 32 : 4 + 8 + 8 * 32;   // worst block payload
    // one warp's share of a tile at worst
    static constexpr int REGION = (BPW * MAXBLK + 15) / 16 * 16;
    // staging ring per codec warp (a circular buffer of its packed, not yet written
    // spans): room for three worst-case spans in f32, two in f64 (typical spans are far
    // smaller; one worst-case span is the least the allocator needs)
    static constexpr int RING = (sizeof(T) == 4 ? 3 : 2) * REGION;
    static constexpr int OFF_IN = 0;
    static constexpr int OFF_STG = NIN * TILE_BYTES;
    static constexpr int BYTES = OFF_STG + WARPS * RING + 16;   // + what a copy-out may read past a ring
    // base alignment: 3D input slots take 128-byte swizzled boxes, whose pattern follows
    // the shared address bits and so needs 1024-byte aligned slots
    static constexpr unsigned ALIGN = DIM == 3 ? 1024u : 128u;
    static constexpr size_t smem_bytes() { return (size_t)BYTES + ALIGN; }
    static_assert(TB == Tiling<DIM>::TB, "tiles must match the workspace layout");
    static_assert(DIM == 1 || TB % kGroup == 0, "tiles hold whole groups");
};

// ------------------------------------------------------------------ mbarrier / TMA

constexpr int kWaitLimit = 1 << 18;       // bounded mbarrier waits: attempts of up to kWaitSliceNs each
constexpr uint32_t kWaitSliceNs = 8192;  // (so a wait gives up after about two seconds)

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(uint64_t* b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// try_wait with an explicit suspend-time hint: the warp sleeps in the barrier unit until
// the phase completes (it then wakes at once) or `ns` nanoseconds pass -- waiting costs
// no issue slots.
__device__ __forceinline__ bool mbar_try_wait_ns(uint64_t* b, uint32_t parity, uint32_t ns)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity), "r"(ns)
        : "memory");
    return ok != 0;
}
// Non-blocking poll (try_wait may suspend the thread for a while before it fails).
__device__ __forceinline__ bool mbar_test(uint64_t* b, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase with `parity` to complete; false (and the error bit set) if it
// did not within the limit, or at once false when another wait of the launch gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, uint32_t* err)
{
    if (mbar_try_wait_ns(b, parity, kWaitSliceNs)) return true;
    const int limit = wait_limit(err, kWaitLimit);
    for (int i = 1; i < limit; i++) {
        if (timed_out(err)) return false;   // another wait gave up
        if (mbar_try_wait_ns(b, parity, kWaitSliceNs)) return true;
    }
    atomicOr(err, ERR_WAIT_TIMEOUT);
    return false;
}
// Waits for the completion of a bulk copy already issued into this CTA's shared memory
// (the phase with `parity` of its barrier), whatever else gave up: a CTA must not end
// while a copy still writes its shared memory.  Bounded by the default limit (a copy
// from the GPU's own memory completes in microseconds).
__device__ __forceinline__ void mbar_drain(uint64_t* b, uint32_t parity, uint32_t* err)
{
    for (int i = 0; i < kWaitLimit; i++)
        if (mbar_try_wait_ns(b, parity, kWaitSliceNs)) return;
    atomicOr(err, ERR_WAIT_TIMEOUT);
}

// One tensor box (coordinates x fastest) into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}
// kGroup whole 2D blocks from a grouped map (dims: column in block, row in block, block
// column, block row, slice) into shared memory in block order, completing on `bar`.
__device__ __forceinline__ void tma_load_group(void* dst, const CUtensorMap* map, int bx, int by, int z, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(0), "r"(bx), "r"(by), "r"(z),
          "r"(smem_u32(bar))
        : "memory");
}
// Starts fetching the same box as tma_load_group into L2, with no completion to wait for.
__device__ __forceinline__ void tma_prefetch_group(const CUtensorMap* map, int bx, int by, int z)
{
    asm volatile("cp.async.bulk.prefetch.tensor.5d.L2.global.tile [%0, {%1, %2, %3, %4, %5}];"
                 ::"l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(0), "r"(bx), "r"(by), "r"(z) : "memory");
}
// `bytes` (a multiple of 16) contiguous bytes from global `src` (16-byte aligned).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// ------------------------------------------------------------------ shared state

template <typename T, int DIM>
struct TmaShared {
    using C = TmaCfg<T, DIM>;
    uint64_t full[C::NIN];             // input slot loaded (TMA bytes + loader arrival)
    uint64_t freed[C::NIN];            // input slot consumed (one arrival per codec warp)
    uint64_t aggd[C::NC];              // tile aggregate posted (last codec warp)
    uint64_t based[C::NC];             // tile offset published (resolver)
    int64_t tick[C::NIN];              // tile held by each input slot (>= total: no more tiles)
    int64_t local[C::NIN];             // ... its index inside its array
    int64_t tile_of[C::NC];            // tile held by each tile state
    int64_t local_of[C::NC];           // ... its index inside its array
    int32_t arr[C::NIN];               // array of each input slot's tile (batches)
    int32_t arr_of[C::NC];             // array of each tile state's tile
    unsigned long long agg[C::NC];     // tile payload bytes
    unsigned long long base[C::NC];    // tile payload offset (exclusive prefix)
    uint32_t wt[C::NC][C::WARPS];      // warp payload bytes
    uint32_t woff[C::NC][C::WARPS];    // warp offsets inside the tile
    uint32_t cnt[C::NC];               // codec warps done with the tile
    int kend;                          // index in this CTA's sequence of the first missing tile
};

// ------------------------------------------------------------------ codes and payloads

// Row boxes: 3D arrays whose block rows hold whole boxes move as 128-byte-swizzled TMA
// boxes of 128 / sizeof(T) / 4 x 4 x 4 elements (BPB = 8 f32 or 4 f64 blocks), 2048
// bytes in 16 rows of 128 bytes: row r = 4z + y, and 16-byte chunk c of row r stored at
// chunk c ^ (r & 7).  Lane l handles element x = l & 3, row l >> 2 of each block (the
// block's second half, z + 2, is 8 rows = 1024 bytes on); at(j) is its byte offset in
// block j of a run of boxes.  The 32 lanes of a half-block then read or write distinct
// banks (f32) or two 8-byte words per bank (f64), the least possible.
template <typename T>
struct RowBox {
    static constexpr int BPB = 128 / (4 * (int)sizeof(T));   // blocks per box
    static constexpr int CPB = 4 * (int)sizeof(T) / 16;      // 16-byte chunks per block row
    static constexpr int EPC = 16 / (int)sizeof(T);          // elements per chunk
    uint32_t base;   // row start + offset inside the chunk
    uint32_t k;      // (lane's chunk inside the block row ^ row) << 4
    __device__ __forceinline__ explicit RowBox(int lane)
    {
        const uint32_t r = (uint32_t)lane >> 2, x = (uint32_t)lane & 3u;
        base = r * 128u + (x % EPC) * (uint32_t)sizeof(T);
        k = ((x / EPC) ^ (r & 7u)) << 4;
    }
    __device__ __forceinline__ uint32_t at(int j) const
    {
        return base + (uint32_t)(j / BPB) * 2048u + ((((uint32_t)(j % BPB) * CPB) << 4) ^ k);
    }
};

// A codec warp's codes of one tile, kept in registers from the code phase to the
// pack phase: lane l holds element l (1D: of each block; 2D/3D: elements l and l+32).
template <int DIM, typename C>
struct WarpCodes {
    int32_t c0[C::BPW];
    int32_t c1[DIM == 1 ? 1 : C::BPW];
    uint32_t rb;   // lane j < BPW: rate byte of block j
    uint32_t o;    // 2D/3D outlier mode, lane j < BPW: magnitude of block j's element 0
};

// 1D code phase: the warp's 16 blocks of tile `t` (elements in `tin`) -> codes, rate
// bytes (to the stream and to K.rb).  Returns the warp's payload bytes.
template <typename T, int MODE, typename C>
__device__ __forceinline__ uint32_t codes_1d(saddr_t tin, WarpCodes<1, C>& K, int warp, int64_t t, const Geom& g,
                                             T recip, uint8_t* __restrict__ cmp, int lane)
{
    const uint64_t b0 = (uint64_t)t * C::TB + (uint64_t)warp * C::BPW;
    uint32_t M = 0, O = 0;   // lane j: block j's reduced magnitudes
    const saddr_t wb = tin + (warp * C::BPW * 32 + lane) * (uint32_t)sizeof(T);
    const bool ragged = (b0 + C::BPW) * 32 > g.nbEle;   // also: no element at all
#pragma unroll
    for (int j = 0; j < C::BPW; j += 2) {
        const int32_t qA = quantize(lds_val<T>(wb + j * 32 * sizeof(T)), recip);
        const int32_t qB = quantize(lds_val<T>(wb + (j + 1) * 32 * sizeof(T)), recip);
        int32_t cA = qA, cB = qB;
        if constexpr (MODE != MODE_FIXED) {
            const int32_t uA = __shfl_up_sync(FULL, qA, 1), uB = __shfl_up_sync(FULL, qB, 1);
            cA = wsub(qA, lane ? uA : 0);
            cB = wsub(qB, lane ? uB : 0);
        }
        if (ragged) {   // elements past the array: code 0 (stale slot contents)
            const uint64_t i = (b0 + j) * 32 + lane;
            cA = i < g.nbEle ? cA : 0;
            cB = i + 32 < g.nbEle ? cB : 0;
        }
        K.c0[j] = cA;
        K.c0[j + 1] = cB;
        uint32_t oA, oB;
        const uint32_t mA = block_max<1, MODE>(uabs(cA), 0u, lane, oA);
        const uint32_t mB = block_max<1, MODE>(uabs(cB), 0u, lane, oB);
        if (lane == j) { M = mA; O = oA; }
        if (lane == j + 1) { M = mB; O = oB; }
    }
    K.rb = lane < C::BPW ? rate_byte<1, MODE>(M, O) : 0u;
    K.o = O;
    if (lane < C::BPW && b0 + lane < g.rate_bytes) cmp[b0 + lane] = (uint8_t)K.rb;
    return __reduce_add_sync(FULL, payload_size<1, MODE>(K.rb));
}

// 2D/3D code phase: the warp's blocks.  Lane l codes element l and l + 32 of each block
// (element k = 8r + c in 2D, 16z + 4y + x in 3D).  In the input slot the block's 64
// elements are contiguous, or with SWZ (3D row boxes) the warp's blocks are a run of
// swizzled boxes (RowBox).
template <typename T, int DIM, int MODE, typename C, bool SWZ = false>
__device__ __forceinline__ uint32_t codes_nd(saddr_t tin, WarpCodes<DIM, C>& K, int warp, int64_t t, const Geom& g,
                                             T recip, uint8_t* __restrict__ cmp, int lane)
{
    constexpr uint32_t B = DIM == 2 ? 8 : 4;
    static_assert(C::BPW % 4 == 0, "blocks are coded four at a time");
    static_assert(!SWZ || (DIM == 3 && C::BPW % RowBox<T>::BPB == 0), "row boxes: 3D, whole boxes per warp");
    const uint64_t b0 = (uint64_t)t * C::TB + (uint64_t)warp * C::BPW;
    // this lane's element of block j (and of its second half, H1 bytes on)
    const saddr_t wb = tin + (warp * C::BPW * 64 + (SWZ ? 0 : lane)) * (uint32_t)sizeof(T);
    const RowBox<T> rbx(lane);
    constexpr uint32_t H1 = SWZ ? 1024u : 32u * (uint32_t)sizeof(T);
    auto blk_at = [&](int j) -> saddr_t { return SWZ ? wb + rbx.at(j) : wb + j * 64 * sizeof(T); };
    const uint32_t nblk = b0 < g.nblocks ? (uint32_t)min((uint64_t)C::BPW, g.nblocks - b0) : 0u;
    // partial blocks exist only along axes the block size does not divide
    const bool ragged = (g.dx % B) || (g.dy % B) || (DIM == 3 && (g.dz % 4));
    auto code_pair = [&](saddr_t blk, int32_t& c0, int32_t& c1) {
        const int32_t q0 = quantize(lds_val<T>(blk), recip);
        const int32_t q1 = quantize(lds_val<T>(blk + H1), recip);
        c0 = q0;
        c1 = q1;
        if constexpr (MODE != MODE_FIXED) {
            int32_t p0, p1;
            predecessors<DIM>(q0, q1, lane, p0, p1);
            c0 = wsub(q0, p0);
            c1 = wsub(q1, p1);
        }
    };
    if (!ragged && nblk == C::BPW) {
        // every block whole: no masks, four independent blocks per step
#pragma unroll
        for (int j = 0; j < C::BPW; j++) code_pair(blk_at(j), K.c0[j], K.c1[j]);
    } else {
        // blocks past the warp's last (nblk) or elements past the array: code 0
        const BlockPos bp = block_pos(b0 < g.nblocks ? b0 : 0, g);
        uint32_t bx = bp.x, by = bp.y, bz = bp.z;
        const uint32_t cx = DIM == 2 ? (lane & 7) : (lane & 3);
        const uint32_t ry0 = DIM == 2 ? (lane >> 3) : ((lane >> 2) & 3);
        const uint32_t ry1 = DIM == 2 ? ry0 + 4 : ry0;
        const uint32_t rz0 = DIM == 2 ? 0 : (lane >> 4);
        const uint32_t rz1 = DIM == 2 ? 0 : rz0 + 2;
#pragma unroll
        for (int j = 0; j < C::BPW; j++) {
            int32_t c0, c1;
            code_pair(blk_at(j), c0, c1);
            const uint32_t xb = bx * B, yb = by * B, zb = DIM == 2 ? bz : bz * 4;
            const bool inx = xb + cx < g.dx;
            const bool ok0 = (uint32_t)j < nblk && inx && yb + ry0 < g.dy && (DIM == 2 || zb + rz0 < g.dz);
            const bool ok1 = (uint32_t)j < nblk && inx && yb + ry1 < g.dy && (DIM == 2 || zb + rz1 < g.dz);
            K.c0[j] = ok0 ? c0 : 0;
            K.c1[j] = ok1 ? c1 : 0;
            if (++bx == g.bxn) {
                bx = 0;
                if (++by == g.byn) { by = 0; ++bz; }
            }
        }
    }
    // per block one reduction; lane j then derives block j's rate byte
    uint32_t M = 0, O = 0;
#pragma unroll
    for (int j = 0; j < C::BPW; j++) {
        uint32_t o;
        const uint32_t m = block_max<DIM, MODE>(uabs(K.c0[j]), uabs(K.c1[j]), lane, o);
        if (lane == j) { M = m; O = o; }
    }
    K.rb = lane < C::BPW ? rate_byte<DIM, MODE>(M, O) : 0u;
    if constexpr (MODE == MODE_OUTLIER) {
        // element 0 of a block flagged as outlier goes ahead of its planes in whole bytes
        // (written by the pack phase from K.o); its planes carry magnitude 0, sign kept
        K.o = O;
        const uint32_t head = __ballot_sync(FULL, K.rb & 0x80u);
        if (lane == 0) {
#pragma unroll
            for (int j = 0; j < C::BPW; j++)
                if ((head >> j) & 1u) K.c0[j] = (int32_t)((uint32_t)K.c0[j] & 0x80000000u);
        }
    }
    if (lane < C::BPW && b0 + lane < g.rate_bytes) cmp[b0 + lane] = (uint8_t)K.rb;
    return __reduce_add_sync(FULL, payload_size<DIM, MODE>(K.rb));
}

// Pack phase: sign maps and bit-planes of the warp's blocks, in stream order at `out`.
template <int DIM, int MODE, typename C>
__device__ __forceinline__ void pack_codes(const WarpCodes<DIM, C>& K, saddr_t out, int lane, const XposeLane& xl)
{
    const uint32_t mine = lane < C::BPW ? K.rb : 0u;
    const uint32_t sz = lane < C::BPW ? payload_size<DIM, MODE>(mine) : 0u;
    uint32_t incl = sz;
#pragma unroll
    for (int o = 1; o < C::BPW; o <<= 1) {
        const uint32_t v = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += v;
    }
    uint32_t myoff = incl - sz;
    if constexpr (DIM == 1) {
        const uint32_t n = MODE == MODE_OUTLIER ? (mine & 0x1fu) : mine;
        if (__all_sync(FULL, n <= 15)) {
            // every block narrow: four blocks per step, no branches between them; lane j
            // holds block j's plane mask and sign-word offset
            uint32_t ps = myoff, heads = 0;
            if constexpr (MODE == MODE_OUTLIER) {
                // element 0's bytes of every outlier block: lane 4j + i writes byte i of
                // block j, eight blocks per step; the sign words follow them
                const uint32_t ob = (mine & 0x80u) ? ((mine & 0x60u) >> 5) + 1u : 0u;
                const uint32_t i = lane & 3;
#pragma unroll
                for (int h = 0; h < C::BPW; h += 8) {
                    const int src = h + (lane >> 2);
                    const uint32_t nb = __shfl_sync(FULL, ob, src), v = __shfl_sync(FULL, K.o, src);
                    const uint32_t at = __shfl_sync(FULL, myoff, src);
                    if (i < nb) sts_u8(out + at + i, v >> (8 * i));
                }
                heads = __ballot_sync(FULL, ob != 0);
                ps += ob;
            }
            const uint32_t mask = plane_mask(mine, n);
            const int half = lane >> 4;
            const uint32_t pl = (uint32_t)(lane ^ 7) & 15u;
            const uint32_t o = pl == 15 ? 0u : 4u + 4u * pl;
#pragma unroll
            for (int j = 0; j < C::BPW; j += 4) {
                const uint32_t k1 = __shfl_sync(FULL, mask, j + half), k2 = __shfl_sync(FULL, mask, j + 2 + half);
                const uint32_t p1 = __shfl_sync(FULL, ps, j + half), p2 = __shfl_sync(FULL, ps, j + 2 + half);
                int32_t cA = K.c0[j], cB = K.c0[j + 1], cC = K.c0[j + 2], cD = K.c0[j + 3];
                if constexpr (MODE == MODE_OUTLIER) {
                    // magnitude 0 in the planes where element 0 went ahead of them, sign kept
                    if (lane == 0) {
                        if ((heads >> j) & 1u) cA = (int32_t)((uint32_t)cA & 0x80000000u);
                        if ((heads >> (j + 1)) & 1u) cB = (int32_t)((uint32_t)cB & 0x80000000u);
                        if ((heads >> (j + 2)) & 1u) cC = (int32_t)((uint32_t)cC & 0x80000000u);
                        if ((heads >> (j + 3)) & 1u) cD = (int32_t)((uint32_t)cD & 0x80000000u);
                    }
                }
                pack_quad_1d_narrow<MODE>(cA, cB, cC, cD, k1, out + p1, k2, out + p2, pl, o, xl);
            }
            return;
        }
    }
    if constexpr (DIM != 1) {
        if constexpr (MODE == MODE_OUTLIER) {
            // element 0's bytes of every outlier block: lane 4j + i writes byte i of block j,
            // eight blocks per step; the planes then start past them (myoff: sign words)
            const uint32_t ob = (mine & 0x80u) ? ((mine & 0x60u) >> 5) + 1u : 0u;
            const uint32_t i = lane & 3;
#pragma unroll
            for (int h = 0; h < C::BPW; h += 8) {   // eight blocks per step
                const int src = h + (lane >> 2);
                const uint32_t n = __shfl_sync(FULL, ob, src), v = __shfl_sync(FULL, K.o, src);
                const uint32_t at = __shfl_sync(FULL, myoff, src);
                if (i < n) sts_u8(out + at + i, v >> (8 * i));
            }
            myoff += ob;
        }
        const uint32_t n = MODE == MODE_OUTLIER ? (mine & 0x1fu) : mine;
        if (__all_sync(FULL, n <= 15)) {
            // every block narrow: all pairs unrolled, no branches between them; lane j
            // holds block j's plane mask
            const uint32_t mask = plane_mask(mine, n);
            if constexpr (DIM == 3) {
                // four blocks per step (2D measured faster in pairs)
#pragma unroll
                for (int j = 0; j < C::BPW; j += 4) {
                    uint32_t k4[4];
                    saddr_t p4[4];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        k4[i] = __shfl_sync(FULL, mask, j + i);
                        p4[i] = out + __shfl_sync(FULL, myoff, j + i);
                    }
                    pack_quad_narrow<MODE>(k4, &K.c0[j], &K.c1[j], p4, lane, xl);
                }
            } else {
#pragma unroll
                for (int j = 0; j < C::BPW; j += 2) {
                    const uint32_t ka = __shfl_sync(FULL, mask, j), kb = __shfl_sync(FULL, mask, j + 1);
                    const uint32_t oa = __shfl_sync(FULL, myoff, j), ob = __shfl_sync(FULL, myoff, j + 1);
                    // byte-wise outlier stores in 2D (3D measured 1 % slower with them)
                    pack_pair_narrow<MODE, true>(ka, kb, K.c0[j], K.c1[j], K.c0[j + 1], K.c1[j + 1], out + oa,
                                                 out + ob, lane, xl);
                }
            }
            return;
        }
    }
#pragma unroll
    for (int j = 0; j < C::BPW; j += 2) {
        const uint32_t ra = __shfl_sync(FULL, mine, j), rb = __shfl_sync(FULL, mine, j + 1);
        if ((ra | rb) == 0) continue;
        const uint32_t oa = __shfl_sync(FULL, myoff, j), ob = __shfl_sync(FULL, myoff, j + 1);
        if constexpr (DIM == 1)
            pack_pair_1d<MODE>(ra, rb, K.c0[j], K.c0[j + 1], out + oa, out + ob, lane, xl);
        else
            pack_pair_nd<MODE, true>(ra, rb, K.c0[j], K.c1[j], K.c0[j + 1], K.c1[j + 1], out + oa, out + ob, lane,
                                     xl);
    }
}

// Warp-cooperative write of `n` staged bytes (`src` 16-byte aligned in shared memory)
// to global `dst` (any alignment): 16-byte stores for the aligned units inside the
// range, one byte store per lane for the ragged first and last units.
__device__ __forceinline__ void warp_copy_out(saddr_t src, uint32_t n, uint8_t* __restrict__ dst, int lane)
{
    if (n == 0) return;
    const uint32_t d = (uint32_t)((uintptr_t)dst & 15);
    uint8_t* first = dst - d;
    const uint32_t u0 = d ? 1u : 0u;          // first unit entirely inside [d, d + n)
    const uint32_t u1 = (d + n) >> 4;         // one past the last such unit
    if (d == 0) {
        // destination on a 16-byte boundary (fixed/plain 2D/3D payloads keep it so):
        // unit u is bytes [16u, 16u + 16) of the span, one 16-byte shared load
        for (uint32_t u = lane; u < u1; u += 32)
            __stcs(reinterpret_cast<uint4*>(first + 16 * u), lds_u128(src + 16 * u));
    } else
    for (uint32_t u = u0 + lane; u < u1; u += 32) {
        const uint32_t so = 16 * u - d;
        const saddr_t w = src + (so & ~3u);
        const uint32_t sh = (so & 3u) * 8;
        const uint32_t w0 = lds_u32(w), w1 = lds_u32(w + 4), w2 = lds_u32(w + 8), w3 = lds_u32(w + 12);
        uint4 v;
        if (sh == 0) {
            v = make_uint4(w0, w1, w2, w3);
        } else {
            const uint32_t w4 = lds_u32(w + 16);
            v = make_uint4(__funnelshift_r(w0, w1, sh), __funnelshift_r(w1, w2, sh), __funnelshift_r(w2, w3, sh),
                           __funnelshift_r(w3, w4, sh));
        }
        __stcs(reinterpret_cast<uint4*>(first + 16 * u), v);
    }
    // ragged units: unit 0 when d != 0 (lanes 0-15), unit u1 when the range ends inside
    // it and it is not unit 0 again (lanes 16-31)
    const bool head = d != 0;
    const bool tail = ((d + n) & 15u) != 0 && !(head && u1 == 0);
    const uint32_t unit = lane < 16 ? 0u : u1;
    if ((lane < 16 && head) || (lane >= 16 && tail)) {
        const uint32_t pos = 16 * unit + (uint32_t)(lane & 15);
        if (pos >= d && pos < d + n) first[pos] = (uint8_t)lds_u8(src + (pos - d));
    }
}

// ------------------------------------------------------------------ tile sources

// Where a tile's array lives: what the passes need beyond the tile's own data.
struct TileArray {
    void* data;                       // the array's elements (compress: read; decompress: written)
    uint8_t* cmp;                     // its stream (compress: written; decompress: read)
    const Geom* g;                    // its geometry
    unsigned long long* status;       // its tile status words (indexed by local tile)
    unsigned long long* total_out;    // its stream length
    const CUtensorMap* tmap;          // its block boxes (2D/3D)
    float eb;                         // its absolute bound (batches, where it is set on the device)
    int mode;
};

// One array; everything is a kernel parameter and the encoding mode a constant.
// `scale` is the reciprocal 0.5/eb when compressing and eb when decompressing.
template <typename T, int MODE>
struct SingleTiles {
    const CUtensorMap* tmap;
    void* data;
    uint8_t* cmp;
    const Geom* g;
    T scale;
    unsigned long long* status;
    unsigned long long* total_out;
    int tickets = 1;   // decompress: tiles per ticket (1 or up to kMaxTicketTiles)
    __device__ __forceinline__ uint64_t total() const { return g->ntiles; }
    __device__ __forceinline__ unsigned long long* size_out() const { return g->size_out; }
    __device__ __forceinline__ int ticket_tiles() const { return tickets; }
    __device__ __forceinline__ void locate(int64_t t, int32_t& a, int64_t& local) const { a = 0; local = t; }
    __device__ __forceinline__ TileArray array(int32_t) const
    {
        return TileArray{data, cmp, g, status, total_out, tmap, 0.f, MODE};
    }
    __device__ __forceinline__ T recip_of(const TileArray&) const { return scale; }
    __device__ __forceinline__ T eb_of(const TileArray&) const { return scale; }
    __device__ __forceinline__ void acquire_map(const CUtensorMap*) const {}   // a kernel parameter
    template <typename F>
    __device__ __forceinline__ void with_mode(int, F&& f) const { f(std::integral_constant<int, MODE>{}); }
};

// ------------------------------------------------------------------ the kernel body

template <typename T, int DIM, typename Src>
__device__ __forceinline__ void compress_tma_body(const Src& src, WsHeader* __restrict__ hdr,
                                                  unsigned long long* __restrict__ status_all)
{
    using C = TmaCfg<T, DIM>;
    extern __shared__ unsigned char dsm[];
    unsigned char* base = dsm + ((C::ALIGN - (smem_u32(dsm) & (C::ALIGN - 1u))) & (C::ALIGN - 1u));
    T* inbuf = reinterpret_cast<T*>(base + C::OFF_IN);
    uint8_t* stg = base + C::OFF_STG;
    __shared__ __align__(8) TmaShared<T, DIM> sh;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t* err = &hdr->err;
    const uint64_t ntotal = src.total();

    if (threadIdx.x == 0) {
        for (int i = 0; i < C::NIN; i++) {
            mbar_init(&sh.full[i], 1);
            mbar_init(&sh.freed[i], C::WARPS);
        }
        for (int i = 0; i < C::NC; i++) {
            mbar_init(&sh.aggd[i], 1);
            mbar_init(&sh.based[i], 1);
            sh.cnt[i] = 0;
        }
        sh.kend = 0x7fffffff;
        mbar_fence_init();
    }
    __syncthreads();

    if (warp > C::LOADER) {
        // ---------------------------------------------------------------- resolver warps
        for (int k = warp - C::LOADER - 1;; k += C::RESOLVERS) {
            const int c = k % C::NC;
            const uint32_t parity = (uint32_t)(k / C::NC) & 1u;
            bool ready = false;
            int limit = 1;   // read once a first attempt failed
            for (int i = 0; i < limit; i++) {   // tile k coded and its size posted, or no tile k
                // the loader marks the end of the CTA's tiles well before the last one is
                // coded: look first, rather than sleep in a wait that nothing completes
                // (measured: the CTA's last wait cost up to 4 us on every call)
                if (k >= *reinterpret_cast<volatile int*>(&sh.kend)) break;
                if (mbar_try_wait_ns(&sh.aggd[c], parity, kWaitSliceNs / 4)) { ready = true; break; }
                if (k >= *reinterpret_cast<volatile int*>(&sh.kend)) break;
                if (timed_out(err)) break;
                if (i == 0) limit = 4 * min(wait_limit(err, kWaitLimit), kWaitLimit);
            }
            if (!ready) break;
            const TileArray A = src.array(sh.arr_of[c]);
            const int64_t lt = sh.local_of[c];
            const unsigned long long agg = sh.agg[c];
            const uint64_t excl = lt > 0 ? warp_lookback(A.status, lt, err) : 0;
            if (lane == 0) {
                if (lt > 0) st_post(A.status + lt, ST_INC | ((excl + agg) & ST_VAL));
                if ((uint64_t)lt == A.g->ntiles - 1) *A.total_out = A.g->rate_bytes + excl + agg;
                sh.base[c] = excl;
                mbar_arrive(&sh.based[c]);
            }
        }
    } else if (warp == C::LOADER) {
        // ---------------------------------------------------------------- loader warp
        bool ended = false;
        int issued = 0;   // issue() calls so far; slots are used round-robin
        // Takes a ticket for input slot s and starts its load.  Returns false once the
        // tickets ran past the last tile (the slot then completes with no bytes).
        auto issue = [&](int s) -> bool {
            int64_t t = 0;
            issued++;
            if (lane == 0) t = (int64_t)atomicAdd(&hdr->ticket, 1u);
            t = __shfl_sync(FULL, t, 0);
            T* dst = inbuf + s * C::TILE_ELEMS;
            if ((uint64_t)t >= ntotal) {
                if (lane == 0) {
                    sh.tick[s] = t;
                    *reinterpret_cast<volatile int*>(&sh.kend) = issued - 1;   // issue order = tile order
                    mbar_arrive(&sh.full[s]);
                }
                return false;
            }
            int32_t a;
            int64_t lt;
            src.locate(t, a, lt);
            const TileArray A = src.array(a);
            const Geom g = *A.g;
            const T* in = static_cast<const T*>(A.data);
            if constexpr (DIM == 1) {
                const uint64_t e0 = (uint64_t)lt * C::TILE_ELEMS;
                const uint64_t cnt = e0 < g.nbEle ? min((uint64_t)C::TILE_ELEMS, g.nbEle - e0) : 0;
                const uint32_t bytes = (uint32_t)cnt * (uint32_t)sizeof(T);
                const uint32_t main = bytes & ~15u;
                const uint32_t tail = (bytes - main) / (uint32_t)sizeof(T);   // < 16 bytes of elements
                if ((uint32_t)lane < tail) dst[main / sizeof(T) + lane] = in[e0 + main / sizeof(T) + lane];
                __syncwarp();
                if (lane == 0) {
                    sh.tick[s] = t;
                    sh.arr[s] = a;
                    sh.local[s] = lt;
                    mbar_arrive_tx(&sh.full[s], main);
                    if (main) bulk_load(dst, in + e0, main, &sh.full[s]);
                }
            } else {
                const uint64_t b0 = (uint64_t)lt * C::TB;
                const uint32_t nvalid = (uint32_t)min((uint64_t)C::TB, g.nblocks - b0);
                if (lane == 0) {
                    sh.tick[s] = t;
                    sh.arr[s] = a;
                    sh.local[s] = lt;
                    mbar_arrive_tx(&sh.full[s], nvalid * 64u * (uint32_t)sizeof(T));
                }
                __syncwarp();
                if ((uint32_t)lane < nvalid) src.acquire_map(A.tmap);
                if (DIM == 3 && g.grouped) {
                    // row boxes of BPB blocks (nvalid is a multiple of BPB: block rows hold
                    // whole boxes), landing in the slot in tile order
                    constexpr uint32_t BPB = RowBox<T>::BPB;
                    if ((uint32_t)lane < C::TB / BPB && (uint32_t)lane * BPB < nvalid) {
                        const BlockPos p = block_pos(b0 + lane * BPB, g);
                        tma_load_3d(dst + lane * BPB * 64, A.tmap, (int)(p.x * 4), (int)(p.y * 4), (int)(p.z * 4),
                                    &sh.full[s]);
                    }
                } else if (DIM == 2 && g.grouped) {
                    // kGroup whole blocks per box, landing in block order (nvalid is a
                    // multiple of kGroup: rows hold whole groups)
                    if ((uint32_t)lane * kGroup < nvalid) {
                        const BlockPos p = block_pos(b0 + lane * kGroup, g);
                        tma_load_group(dst + lane * kGroup * 64, A.tmap, (int)p.x, (int)p.y, (int)p.z, &sh.full[s]);
                    }
                } else
                for (uint32_t j = lane; j < nvalid; j += 32) {
                    const BlockPos p = block_pos(b0 + j, g);
                    if constexpr (DIM == 2)
                        tma_load_3d(dst + j * 64, A.tmap, (int)(p.x * 8), (int)(p.y * 8), (int)p.z, &sh.full[s]);
                    else
                        tma_load_3d(dst + j * 64, A.tmap, (int)(p.x * 4), (int)(p.y * 4), (int)(p.z * 4), &sh.full[s]);
                }
            }
            if constexpr (DIM == 2) {
                // Grouped 2D: bring the tile about one ticket round ahead (one tile per CTA
                // later) into L2, so that the load that takes it finds it there.  Measured
                // 3 % faster on 8192^2 f64; per-block prefetches (3D, ungrouped 2D) cost
                // more issue slots than they save, and 1D gained nothing.
                const uint64_t tp = (uint64_t)t + gridDim.x;
                if (tp < ntotal) {
                    int32_t a2;
                    int64_t lt2;
                    src.locate((int64_t)tp, a2, lt2);
                    const TileArray A2 = src.array(a2);
                    const Geom g2 = *A2.g;
                    if (g2.grouped) {
                        const uint64_t b0 = (uint64_t)lt2 * C::TB;
                        const uint32_t nvalid = (uint32_t)min((uint64_t)C::TB, g2.nblocks - b0);
                        if ((uint32_t)lane * kGroup < nvalid) {
                            src.acquire_map(A2.tmap);
                            const BlockPos p = block_pos(b0 + lane * kGroup, g2);
                            tma_prefetch_group(A2.tmap, (int)p.x, (int)p.y, (int)p.z);
                        }
                    }
                }
            }
            return true;
        };
        for (int s = 0; s < C::NIN && !ended; s++) ended = !issue(s);
        for (int k = 0;; k++) {
            const int s = k % C::NIN;
            __syncwarp();
            const int64_t t = *reinterpret_cast<volatile int64_t*>(&sh.tick[s]);
            if ((uint64_t)t >= ntotal) break;
            if (!mbar_wait(&sh.freed[s], (uint32_t)(k / C::NIN) & 1u, err)) break;
            if (!ended) ended = !issue(s);   // tile k's elements are consumed: load tile k + NIN
        }
        // no load may still be writing shared memory when the CTA ends (only reachable
        // with loads outstanding after a timed-out wait)
        if (lane == 0) {
            for (int s = 0; s < C::NIN; s++) {
                const int uses = issued / C::NIN + (s < issued % C::NIN ? 1 : 0);
                if (uses) mbar_drain(&sh.full[s], (uint32_t)(uses - 1) & 1u, err);
            }
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------------- codec warps
        // The warp's staging ring is a circular buffer of the spans it packed but has
        // not yet written out (at most DEFER between tiles, oldest first in q[0..]).  A
        // tile's span (its exact size is known before packing) goes at the 16-byte
        // aligned write position, or at the start of the ring when it does not fit
        // before the end; when neither is free of live spans, the oldest span is
        // written out first (waiting for its offset).  `lap` counts wraps of the write
        // position, so "ahead of the oldest span" needs no full/empty flag.
        struct Span {
            int k;        // CTA tile index (< 0: none)
            uint32_t at;  // ring offset
            int lap;      // ... and its lap
            uint32_t n;   // payload bytes
        };
        const saddr_t ring = saddr(stg + warp * C::RING);
        const XposeLane xl(lane ^ 7);
        Span q[C::DEFER];   // live spans, oldest first; q[i].k < 0: none (then none after it)
#pragma unroll
        for (int i = 0; i < C::DEFER; i++) q[i] = Span{-1, 0, 0, 0};
        Span& q0 = q[0];
        uint32_t head = 0;   // write position
        int lap = 0;
        bool ok = true;
        auto pop = [&]() -> bool {   // write the oldest span out
            const int c = q0.k % C::NC;
            const bool done = mbar_wait(&sh.based[c], (uint32_t)(q0.k / C::NC) & 1u, err);
            if (done) {
                const TileArray A = src.array(sh.arr_of[c]);
                const uint64_t at = A.g->rate_bytes + sh.base[c] + sh.woff[c][warp];
                if (at + q0.n <= A.g->cap) warp_copy_out(ring + q0.at, q0.n, A.cmp + at, lane);
                else if (lane == 0) atomicOr(err, ERR_CAPACITY);   // nothing written past the buffer
                __syncwarp();
            }
#pragma unroll
            for (int i = 0; i + 1 < C::DEFER; i++) q[i] = q[i + 1];
            q[C::DEFER - 1].k = -1;
            return done;
        };
        // ring offset (and lap) for a new span of n bytes
        auto place = [&](uint32_t n, int& span_lap) -> uint32_t {
            for (;;) {
                if (q0.k < 0) {   // empty ring: start over
                    head = n;
                    lap = 0;
                    span_lap = 0;
                    return 0;
                }
                const uint32_t h = (head + 15u) & ~15u;
                if (lap == q0.lap) {   // free: [h, RING) and [0, q0.at)
                    if (h + n <= (uint32_t)C::RING) {
                        head = h + n;
                        span_lap = lap;
                        return h;
                    }
                    if (n <= q0.at) {
                        head = n;
                        span_lap = ++lap;
                        return 0;
                    }
                } else if (h + n <= q0.at) {   // free: [h, q0.at)
                    head = h + n;
                    span_lap = lap;
                    return h;
                }
                if (!pop()) ok = false;   // a timed-out wait still frees the span
            }
        };
        for (int k = 0;; k++) {
            const int s = k % C::NIN, c = k % C::NC;
            if (!mbar_wait(&sh.full[s], (uint32_t)(k / C::NIN) & 1u, err)) { ok = false; break; }
            const int64_t t = *reinterpret_cast<volatile int64_t*>(&sh.tick[s]);
            if ((uint64_t)t >= ntotal) break;
            const int32_t a = sh.arr[s];
            const int64_t lt = sh.local[s];
            const TileArray A = src.array(a);
            const Geom g = *A.g;
            const T recip = src.recip_of(A);
            const saddr_t tin = saddr(inbuf + s * C::TILE_ELEMS);
            src.with_mode(A.mode, [&](auto m) {
                constexpr int MODE = decltype(m)::value;
                WarpCodes<DIM, C> K;
                uint32_t total;
                if constexpr (DIM == 1)
                    total = codes_1d<T, MODE, C>(tin, K, warp, lt, g, recip, A.cmp, lane);
                else if constexpr (DIM == 3)
                    total = g.grouped ? codes_nd<T, DIM, MODE, C, true>(tin, K, warp, lt, g, recip, A.cmp, lane)
                                      : codes_nd<T, DIM, MODE, C, false>(tin, K, warp, lt, g, recip, A.cmp, lane);
                else
                    total = codes_nd<T, DIM, MODE, C>(tin, K, warp, lt, g, recip, A.cmp, lane);
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&sh.freed[s]);   // this warp is done with the input slot
                    sh.wt[c][warp] = total;
                    __threadfence_block();
                    if (atomicAdd(&sh.cnt[c], 1u) == C::WARPS - 1) {   // last warp of the tile
                        __threadfence_block();
                        uint32_t acc = 0;
                        for (int w = 0; w < C::WARPS; w++) {
                            const uint32_t x = *reinterpret_cast<volatile uint32_t*>(&sh.wt[c][w]);
                            sh.woff[c][w] = acc;
                            acc += x;
                        }
                        sh.agg[c] = acc;
                        sh.tile_of[c] = t;
                        sh.arr_of[c] = a;
                        sh.local_of[c] = lt;
                        sh.cnt[c] = 0;
                        st_post(A.status + lt, (lt == 0 ? ST_INC : ST_AGG) | acc);
                        mbar_arrive(&sh.aggd[c]);
                    }
                }
                int span_lap = 0;
                const uint32_t at = place(total, span_lap);
                pack_codes<DIM, MODE, C>(K, ring + at, lane, xl);
                __syncwarp();
                if (q0.k >= 0 && q0.k <= k - C::DEFER && !pop()) ok = false;
                const Span e{k, at, span_lap, total};
                bool put = false;   // into the first free entry (compile-time indices only)
#pragma unroll
                for (int i = 0; i < C::DEFER; i++)
                    if (!put && q[i].k < 0) {
                        q[i] = e;
                        put = true;
                    }
            });
            if (!ok) break;
        }
        while (ok && q0.k >= 0) ok = pop();
    }
    finish_cta(hdr, status_all, ntotal, src.size_out());
}

template <typename T, int DIM, int MODE>
__global__ void __launch_bounds__(TmaCfg<T, DIM>::THREADS, 2)
compress_tma_kernel(const __grid_constant__ CUtensorMap tmap, const T* __restrict__ in, uint8_t* __restrict__ cmp,
                    const __grid_constant__ Geom g, T recip, WsHeader* __restrict__ hdr,
                    unsigned long long* __restrict__ status)
{
    const SingleTiles<T, MODE> src{&tmap, const_cast<T*>(in), cmp, &g, recip, status, &hdr->total, 1};
    compress_tma_body<T, DIM>(src, hdr, status);
}

}  // namespace cuszp

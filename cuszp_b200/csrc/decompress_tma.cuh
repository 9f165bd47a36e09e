// decompress_tma.cuh -- warp-specialised decompress kernel for streams and outputs that
// start on a 16-byte boundary.
//
// One CTA = 8 codec warps + FRONT front warps.  Same tiles as the compress kernels.
//
//   front warp f owns payload slot f.  Per tile it takes a ticket, reads the tile's
//     rate bytes, posts the tile aggregate at once (payload sizes follow from the rate
//     bytes alone, so no tile ever waits on a predecessor that is itself waiting),
//     runs the decoupled look-back, and loads the tile's payload bytes with one
//     `cp.async.bulk` into its slot.  When the codec warps have decoded the slot it
//     takes the next ticket.
//   codec warps: take the slots round-robin; each decodes its blocks from shared
//     memory (sign map and bit-planes -> inverse transpose -> signs -> inverse Lorenzo
//     -> dequantize) into its own output buffer and writes them with TMA stores: one
//     `cp.async.bulk.tensor.3d` box per 2D/3D block (elements outside the array are
//     not written), or one `cp.async.bulk` of the warp's contiguous 1D elements.
// Every wait is bounded; on timeout the error word records it and the kernel ends.
#pragma once

#include "compress_tma.cuh"

namespace cuszp {

// DIRECT: grouped 2D arrays, whose codec warps write straight from registers (each store
// instruction covers four 64-byte row pieces of whole blocks): no output buffers, so a
// third CTA fits on an SM (measured 5.6 % faster on 8192^2 f64).
template <typename T, int DIM, bool DIRECT = false>
struct DecCfg {
    static constexpr int WARPS = 8;                           // codec warps
    // front warps = payload slots.  Fewer of them make a smaller CTA that more CTAs can
    // share an SM with: 1D two (measured 17 % faster than four), f32 3D three (three CTAs
    // per SM, 6 % faster); otherwise four.
    static constexpr bool SMALL3D = DIM == 3 && sizeof(T) == 4;
    static constexpr int FRONT = DIM == 1 ? 2 : SMALL3D ? 3 : 4;
    static constexpr int THREADS = 32 * (WARPS + FRONT);
    static constexpr int BPW = DIM == 1 ? 16 : 8;             // data blocks per codec warp
    static constexpr int TB = WARPS * BPW;                    // data blocks per tile
    static constexpr int BLK = DIM == 1 ? 32 : 64;            // elements per data block
    static constexpr int MAXBLK = DIM == 1 ? 4 + 4 + 4 * 32 : 4 + 8 + 8 * 32;   // worst block payload
    // a tile's payload plus the 16-byte rounding at both ends and word-read slack
    static constexpr int SLOT = (TB * MAXBLK + 48 + 127) / 128 * 128;
    static constexpr int OUTW = BPW * BLK * (int)sizeof(T);   // a codec warp's decoded elements
    static constexpr int OFF_SLOT = 0;
    // 3D output buffers take 128-byte swizzled row boxes (arrays whose block rows hold
    // whole boxes), whose pattern follows the shared address bits: 1024-byte aligned
    static constexpr unsigned ALIGN = DIM == 3 ? 1024u : 128u;
    static constexpr int OFF_OUT = (FRONT * SLOT + (int)ALIGN - 1) / (int)ALIGN * (int)ALIGN;
    static constexpr int BYTES = DIRECT ? OFF_OUT : OFF_OUT + WARPS * OUTW;
    static constexpr int MIN_CTAS = (DIRECT || SMALL3D) ? 3 : 2;   // per SM (register budget)
    static constexpr size_t smem_bytes() { return (size_t)BYTES + ALIGN; }
    static_assert(!DIRECT || DIM == 2, "direct stores are for grouped 2D arrays");
    static_assert(TB == Tiling<DIM>::TB, "tiles must match the workspace layout");
    static_assert(FRONT <= 8, "slot parities are kept in one byte");
    static_assert(DIM == 1 || BPW == (int)kGroup, "a codec warp's 2D blocks are one grouped box");
};

constexpr uint32_t kBadSlot = 0xffffffffu;   // payload offset (toff) of a tile whose rate bytes are invalid
constexpr int kMaxTicketTiles = 16;          // decompress: most tiles per ticket (one look-back each)
// decompress: most tiles per slot fill.  A front warp packs a group's consecutive tiles into
// one fill while their payloads fit a slot (one load, one slot release for several tiles).
// Only 1D arrays in 4-tile tickets use it: measured 5.5 % faster on the 512^3 f32 1D
// decompress, but 1-7 % slower in 2D and 3D and with 2-tile tickets, where a codec warp's
// second tile of a fill waits for the first tile's output store to leave its buffer.
// The direct-store 2D kernel, which has no output buffer, was 3 % slower with it too
// (8192^2 f64 fixed).
constexpr int kFillTiles = 4;

template <typename T, int DIM>
struct DecShared {
    using C = DecCfg<T, DIM>;
    static constexpr int FT = DIM == 1 ? kFillTiles : 1;   // most tiles per fill
    uint64_t full[C::FRONT];           // slot filled (payload bytes + front arrival)
    uint64_t freed[C::FRONT];          // slot decoded (one arrival per codec warp)
    int64_t tile[C::FRONT];            // first tile in each slot's fill (>= total: the front warp has ended)
    int64_t local[C::FRONT];           // ... its index inside its array
    int32_t arr[C::FRONT];             // ... its array (batches)
    int32_t cnt[C::FRONT];             // tiles in the fill (consecutive tiles of one array)
    uint32_t toff[C::FRONT][FT];       // each tile's payload start inside the slot
    // per slot and fill parity (the front warp prepares fill m while fill m - 1 decodes):
    uint32_t woff[C::FRONT][2][FT][C::WARPS];   // codec warp offsets inside each tile's payload
    uint8_t rates[C::FRONT][2][FT][C::TB];      // block rate bytes
};

// ------------------------------------------------------------------ payload words

// Word at byte offset `o` of shared memory `p` (any alignment in outlier mode; the
// payload of fixed/plain streams sits at 4-byte offsets).
template <int MODE>
__device__ __forceinline__ uint32_t lds32(saddr_t p, uint32_t o)
{
    if constexpr (MODE == MODE_OUTLIER) {
        const saddr_t w = p + (o & ~3u);
        const uint32_t sh = (o & 3u) * 8;
        const uint32_t lo = lds_u32(w);
        return sh ? __funnelshift_r(lo, lds_u32(w + 4), sh) : lo;
    } else {
        return lds_u32(p + o);
    }
}
// lds32 where `c` holds, 0 elsewhere, without a branch on `c`.
template <int MODE>
__device__ __forceinline__ uint32_t lds32_if(bool c, saddr_t p, uint32_t o)
{
    if constexpr (MODE == MODE_OUTLIER) {
        const saddr_t w = p + (o & ~3u);
        const uint32_t sh = (o & 3u) * 8;
        const uint32_t lo = lds_u32_if(c, w), hi = lds_u32_if(c && sh, w + 4);
        return sh ? __funnelshift_r(lo, hi, sh) : lo;
    } else {
        return lds_u32_if(c, p + o);
    }
}
// Element 0's magnitude stored in `ob` (1..4) little-endian bytes at offset `o`: one
// unaligned word read, masked (the bytes after it belong to the same payload).
__device__ __forceinline__ uint32_t ld_outlier(saddr_t p, uint32_t o, uint32_t ob)
{
    const uint32_t w = lds32<MODE_OUTLIER>(p, o);
    return ob >= 4 ? w : w & ((1u << (8 * ob)) - 1u);
}

// ------------------------------------------------------------------ block decode

// Decodes the 1D block pair (rates rA, rB at payload offsets oA, oB of `pay`) into the
// codes of this lane's elements (dA, dB).
template <int MODE>
__device__ __forceinline__ void decode_pair_1d(saddr_t pay, uint32_t rA, uint32_t rB, uint32_t oA, uint32_t oB,
                                               int32_t& dA, int32_t& dB, int lane, const XposeLane& xl)
{
    uint32_t nA = rA, nB = rB, obA = 0, obB = 0;
    if constexpr (MODE == MODE_OUTLIER) {
        nA = rA & 0x1f; nB = rB & 0x1f;
        if (rA & 0x80) obA = ((rA & 0x60) >> 5) + 1;
        if (rB & 0x80) obB = ((rB & 0x60) >> 5) + 1;
    }
    const bool hasA = payload_size<1, MODE>(rA) != 0, hasB = payload_size<1, MODE>(rB) != 0;
    const uint32_t pA = oA + obA, pB = oB + obB;   // sign words
    uint32_t magA = 0, magB = 0;
    if (nA <= 15 && nB <= 15) {
        // the compressor's transpose carried each element's sign as plane 15 (the sign
        // word): loading it there gives magnitudes and signs in one transpose
        const uint32_t p = lane & 15;
        const bool b = lane >= 16;
        const uint32_t n = b ? nB : nA, base = b ? pB : pA;
        uint32_t w = 0;
        if (p < n) w = lds32<MODE>(pay, base + 4 + 4 * p);
        else if (p == 15 && (b ? hasB : hasA)) w = lds32<MODE>(pay, base);
        uint32_t x = 0;
        if (hasA | hasB) x = warp_transpose32(from_stream_word(w), xl);
        magA = x & 0x7fffu;
        magB = (x >> 16) & 0x7fffu;
        if constexpr (MODE == MODE_OUTLIER) {
            if (lane == 0) {
                if (obA) magA = ld_outlier(pay, oA, obA);
                if (obB) magB = ld_outlier(pay, oB, obB);
            }
        }
        dA = (x & 0x8000u) ? (int32_t)(0u - magA) : (int32_t)magA;
        dB = (x & 0x80000000u) ? (int32_t)(0u - magB) : (int32_t)magB;
        return;
    }
    if (nA <= 16 && nB <= 16) {
        const uint32_t p = lane & 15;
        uint32_t w = 0;
        if (lane < 16) { if (p < nA) w = lds32<MODE>(pay, pA + 4 + 4 * p); }
        else           { if (p < nB) w = lds32<MODE>(pay, pB + 4 + 4 * p); }
        if (nA | nB) {
            const uint32_t x = warp_transpose32(from_stream_word(w), xl);
            magA = x & 0xffffu;
            magB = x >> 16;
        }
    } else {
        const uint32_t wA = (uint32_t)lane < nA ? lds32<MODE>(pay, pA + 4 + 4 * lane) : 0u;
        const uint32_t wB = (uint32_t)lane < nB ? lds32<MODE>(pay, pB + 4 + 4 * lane) : 0u;
        magA = from_stream_word(wA);
        magB = from_stream_word(wB);
        warp_transpose32x2(magA, magB, xl);
    }
    if constexpr (MODE == MODE_OUTLIER) {
        if (lane == 0) {
            if (obA) magA = ld_outlier(pay, oA, obA);
            if (obB) magB = ld_outlier(pay, oB, obB);
        }
    }
    const uint32_t sA = hasA ? from_stream_word(lds32<MODE>(pay, pA)) : 0u;
    const uint32_t sB = hasB ? from_stream_word(lds32<MODE>(pay, pB)) : 0u;
    dA = hasA ? (((sA >> lane) & 1u) ? (int32_t)(0u - magA) : (int32_t)magA) : 0;
    dB = hasB ? (((sB >> lane) & 1u) ? (int32_t)(0u - magB) : (int32_t)magB) : 0;
}

// Decodes one 2D/3D block (rate r at payload offset o) into the codes of this lane's
// two elements (d0: element lane, d1: element lane + 32).
template <int MODE>
__device__ __forceinline__ void decode_block_nd(saddr_t pay, uint32_t r, uint32_t o, int32_t& d0, int32_t& d1,
                                                int lane, const XposeLane& xl)
{
    if (payload_size<2, MODE>(r) == 0) { d0 = 0; d1 = 0; return; }
    uint32_t n = r, ob = 0;
    if constexpr (MODE == MODE_OUTLIER) {
        n = r & 0x1f;
        if (r & 0x80) ob = ((r & 0x60) >> 5) + 1;
    }
    const uint32_t p = o + ob;   // sign words
    uint32_t mag0, mag1;
    if (n <= 16) {
        const uint32_t pl = lane & 15;
        const uint32_t w = pl < n ? lds32<MODE>(pay, p + 8 + 8 * pl + (lane >> 4) * 4) : 0u;
        const uint32_t x = warp_transpose32(from_stream_word(w), xl);
        mag0 = x & 0xffffu;
        mag1 = x >> 16;
    } else {
        mag0 = (uint32_t)lane < n ? from_stream_word(lds32<MODE>(pay, p + 8 + 8 * lane)) : 0u;
        mag1 = (uint32_t)lane < n ? from_stream_word(lds32<MODE>(pay, p + 12 + 8 * lane)) : 0u;
        warp_transpose32x2(mag0, mag1, xl);
    }
    if constexpr (MODE == MODE_OUTLIER) {
        if (ob && lane == 0) mag0 = ld_outlier(pay, o, ob);
    }
    const uint32_t s0 = from_stream_word(lds32<MODE>(pay, p)), s1 = from_stream_word(lds32<MODE>(pay, p + 4));
    d0 = ((s0 >> lane) & 1u) ? (int32_t)(0u - mag0) : (int32_t)mag0;
    d1 = ((s1 >> lane) & 1u) ? (int32_t)(0u - mag1) : (int32_t)mag1;
}

// Two 2D/3D blocks with payloads of rate <= 15 (na, nb planes; sign words at pa / pb),
// their transposes interleaved.  Lane l loads plane (l & 15) of half l >> 4, and the
// half's sign word in place of plane 15 (the compressor's transpose carried the signs
// there): one transpose per block gives magnitudes (bits 0-14, 16-30) and signs (bits
// 15, 31).  Outlier mode: ha / hb tell whether element 0's magnitude is stored ahead of
// the planes; it is ma / mb then (read by lane 0 only).
template <int MODE>
__device__ __forceinline__ void decode_pair_narrow(saddr_t pay, uint32_t pa, uint32_t pb, uint32_t na, uint32_t nb,
                                                   bool ha, bool hb, uint32_t ma, uint32_t mb, int32_t& d0a,
                                                   int32_t& d1a, int32_t& d0b, int32_t& d1b, int lane,
                                                   const XposeLane& xl)
{
    // one load per lane and block: lane l takes plane (l ^ 7) & 15 of half l >> 4, or in
    // slot 15 the half's sign word, as stored; the stream-order transpose (xl: this
    // lane's XposeLane(lane)) then leaves element p's planes in bits 0-14 / 16-30 of lane p
    const uint32_t pl = (uint32_t)(lane ^ 7) & 15, h4 = (uint32_t)(lane >> 4) * 4;
    const uint32_t op = 8 + 8 * pl + h4;
    const uint32_t oa = pl < na ? op : h4, ob = pl < nb ? op : h4;
    uint32_t xa = lds32_if<MODE>(pl < na || pl == 15, pay, pa + oa);
    uint32_t xb = lds32_if<MODE>(pl < nb || pl == 15, pay, pb + ob);
    warp_transpose32x2_stream(xa, xb, xl);
    uint32_t m0a = xa & 0x7fffu, m1a = (xa >> 16) & 0x7fffu, m0b = xb & 0x7fffu, m1b = (xb >> 16) & 0x7fffu;
    if constexpr (MODE == MODE_OUTLIER) {
        if (lane == 0) {
            if (ha) m0a = ma;
            if (hb) m0b = mb;
        }
    }
    d0a = (xa & 0x8000u) ? (int32_t)(0u - m0a) : (int32_t)m0a;
    d1a = (xa & 0x80000000u) ? (int32_t)(0u - m1a) : (int32_t)m1a;
    d0b = (xb & 0x8000u) ? (int32_t)(0u - m0b) : (int32_t)m0b;
    d1b = (xb & 0x80000000u) ? (int32_t)(0u - m1b) : (int32_t)m1b;
}

// Four 1D blocks with at most 15 planes each: the pairs (A, B) and (C, D) take one
// stream-order transpose each, interleaved.  Lane l loads plane pl = (l ^ 7) & 15 of block
// A / C (l < 16) or B / D (l >= 16), or in slot 15 that block's sign word, when that bit
// of the block's plane mask k1 / k2 is set (sign-word offsets p1 / p2, `o` as in the
// compressor: 0 for the sign word, 4 + 4 pl for a plane); afterwards lane e holds element
// e of both blocks of a pair: magnitudes in bits 0-14 / 16-30, signs in bits 15 / 31.
// Outlier mode: lane 0 replaces element 0's magnitude of a block whose head bit (hA..hD)
// is set by the stored value (mA..mD).
template <int MODE>
__device__ __forceinline__ void decode_quad_1d_narrow(saddr_t pay, uint32_t k1, uint32_t p1, uint32_t k2, uint32_t p2,
                                                      uint32_t pl, uint32_t o, uint32_t heads, uint32_t mA,
                                                      uint32_t mB, uint32_t mC, uint32_t mD, int32_t& dA,
                                                      int32_t& dB, int32_t& dC, int32_t& dD, int lane,
                                                      const XposeLane& xl)
{
    uint32_t x1 = lds32_if<MODE>((k1 >> pl) & 1u, pay, p1 + o);
    uint32_t x2 = lds32_if<MODE>((k2 >> pl) & 1u, pay, p2 + o);
    warp_transpose32x2_stream(x1, x2, xl);
    uint32_t a = x1 & 0x7fffu, b = (x1 >> 16) & 0x7fffu, c = x2 & 0x7fffu, d = (x2 >> 16) & 0x7fffu;
    if constexpr (MODE == MODE_OUTLIER) {
        if (lane == 0) {
            if (heads & 1u) a = mA;
            if (heads & 2u) b = mB;
            if (heads & 4u) c = mC;
            if (heads & 8u) d = mD;
        }
    }
    dA = (x1 & 0x8000u) ? (int32_t)(0u - a) : (int32_t)a;
    dB = (x1 & 0x80000000u) ? (int32_t)(0u - b) : (int32_t)b;
    dC = (x2 & 0x8000u) ? (int32_t)(0u - c) : (int32_t)c;
    dD = (x2 & 0x80000000u) ? (int32_t)(0u - d) : (int32_t)d;
}

// Two 2D/3D blocks at once: when both have payloads of rate <= 15 their transposes run
// interleaved (signs included); otherwise one after the other.
template <int MODE>
__device__ __forceinline__ void decode_pair_nd(saddr_t pay, uint32_t ra, uint32_t rb, uint32_t oa, uint32_t ob_,
                                               int32_t& d0a, int32_t& d1a, int32_t& d0b, int32_t& d1b, int lane,
                                               const XposeLane& xl)
{
    uint32_t na = ra, nb = rb, oba = 0, obb = 0;
    if constexpr (MODE == MODE_OUTLIER) {
        na = ra & 0x1f; nb = rb & 0x1f;
        if (ra & 0x80) oba = ((ra & 0x60) >> 5) + 1;
        if (rb & 0x80) obb = ((rb & 0x60) >> 5) + 1;
    }
    if (na > 15 || nb > 15 || payload_size<2, MODE>(ra) == 0 || payload_size<2, MODE>(rb) == 0) {
        decode_block_nd<MODE>(pay, ra, oa, d0a, d1a, lane, xl);
        decode_block_nd<MODE>(pay, rb, ob_, d0b, d1b, lane, xl);
        return;
    }
    uint32_t ma = 0, mb = 0;
    if constexpr (MODE == MODE_OUTLIER) {
        if (lane == 0) {
            if (oba) ma = ld_outlier(pay, oa, oba);
            if (obb) mb = ld_outlier(pay, ob_, obb);
        }
    }
    decode_pair_narrow<MODE>(pay, oa + oba, ob_ + obb, na, nb, oba != 0, obb != 0, ma, mb, d0a, d1a, d0b, d1b, lane,
                             xl);
}

// ------------------------------------------------------------------ TMA stores

__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, int x, int y, int z, const void* src)
{
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];"
                 ::"l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(src))
                 : "memory");
}
// kGroup whole 2D blocks (block order in shared `src`) to a grouped map's box.
__device__ __forceinline__ void tma_store_group(const CUtensorMap* map, int bx, int by, int z, const void* src)
{
    asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];"
                 ::"l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(0), "r"(bx), "r"(by), "r"(z), "r"(smem_u32(src))
                 : "memory");
}
// `bytes` (a multiple of 16) from shared `src` to global `dst` (16-byte aligned).
__device__ __forceinline__ void bulk_store(void* dst, const void* src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
                 "r"(bytes)
                 : "memory");
}
// Starts fetching `bytes` (a multiple of 16) from global `src` (16-byte aligned) into L2,
// with no completion to wait for: a later bulk load of the same bytes then reads L2.
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Decodes a codec warp's blocks of the tile in payload slot f into its output buffer
// `ob` and starts their stores (the caller waits for the previous stores first).
// SWZ (3D arrays with row boxes): the buffer holds the warp's blocks as a run of
// swizzled row boxes (RowBox, as the compressor's input slots), `obs` is its start, and
// one lane per box stores it with one TMA store.
template <typename T, int DIM, int MODE, bool DIRECT, bool SWZ, typename Src>
__device__ __forceinline__ void decode_and_store(const Src& src, const TileArray& A, DecShared<T, DIM>& sh, int f,
                                                 int rb, int kt, bool last, int64_t lt, saddr_t pay, T* ob,
                                                 saddr_t obs, const XposeLane& xl, bool& stored, int warp, int lane)
{
    using C = DecCfg<T, DIM>;
    static_assert(!SWZ || (DIM == 3 && C::BPW % RowBox<T>::BPB == 0), "row boxes: 3D, whole boxes per warp");
    const Geom g = *A.g;
    const T eb = src.eb_of(A);
    const LorenzoLane<DIM> ll(lane);
    T* out = static_cast<T*>(A.data);
    const uint32_t poff = sh.toff[f][kt];
    const bool bad = poff == kBadSlot;
    // this warp's blocks: rate bytes, payload offsets (lane j: block j)
    const uint32_t myr = lane < C::BPW && !bad ? sh.rates[f][rb][kt][warp * C::BPW + lane] : 0u;
    const uint32_t mysz = lane < C::BPW ? payload_size<DIM, MODE>(myr) : 0u;
    uint32_t incl = mysz;
#pragma unroll
    for (int o = 1; o < C::BPW; o <<= 1) {
        const uint32_t v = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += v;
    }
    const uint32_t myo = bad ? 0u : poff + sh.woff[f][rb][kt][warp] + incl - mysz;
    const uint64_t b0 = (uint64_t)lt * C::TB + (uint64_t)warp * C::BPW;
    // 2D/3D: lane j derives block j's plane count, sign-word offset and (outlier mode)
    // element 0's magnitude once; a warp whose blocks all have payloads of rate <= 15
    // then decodes every pair on the narrow path without per-pair rate arithmetic
    uint32_t myn = myr, myps = myo, mym = 0, heads = 0;
    bool narrow = false;
    if constexpr (DIM != 1) {
        if constexpr (MODE == MODE_OUTLIER) {
            myn = myr & 0x1fu;
            const uint32_t myob = (myr & 0x80u) ? ((myr & 0x60u) >> 5) + 1u : 0u;
            if (myob) mym = ld_outlier(pay, myo, myob);
            myps = myo + myob;
            heads = __ballot_sync(FULL, myob != 0);
        }
        narrow = __all_sync(FULL, lane >= C::BPW || (mysz != 0 && myn <= 15));
    }
    // blocks j, j + 1; `nar` is `narrow`, passed as a constant by for_pairs
    auto decode = [&](int j, bool nar, int32_t& d0a, int32_t& d1a, int32_t& d0b, int32_t& d1b, bool& za,
                      bool& zb) {
        if (nar) {
            const uint32_t pa = __shfl_sync(FULL, myps, j), pb = __shfl_sync(FULL, myps, j + 1);
            const uint32_t na = __shfl_sync(FULL, myn, j), nb = __shfl_sync(FULL, myn, j + 1);
            uint32_t ma = 0, mb = 0;
            if constexpr (MODE == MODE_OUTLIER) {
                ma = __shfl_sync(FULL, mym, j);
                mb = __shfl_sync(FULL, mym, j + 1);
            }
            decode_pair_narrow<MODE>(pay, pa, pb, na, nb, (heads >> j) & 1u, (heads >> (j + 1)) & 1u, ma, mb, d0a,
                                     d1a, d0b, d1b, lane, xl);
            za = zb = false;
        } else {
            const uint32_t ra = __shfl_sync(FULL, myr, j), oa = __shfl_sync(FULL, myo, j);
            const uint32_t rb2 = __shfl_sync(FULL, myr, j + 1), ob2 = __shfl_sync(FULL, myo, j + 1);
            decode_pair_nd<MODE>(pay, ra, rb2, oa, ob2, d0a, d1a, d0b, d1b, lane, xl);
            // blocks without payload decode to 0.0
            za = payload_size<DIM, MODE>(ra) == 0;
            zb = payload_size<DIM, MODE>(rb2) == 0;
        }
    };
    // pair(j, nar) for j = 0, 2, ..: a narrow warp runs its pairs fully unrolled, with no
    // branch between them (measured 7-8 % faster decompress of 512^3 f32 in 2D and 3D);
    // otherwise one pair per iteration
    auto for_pairs = [&](auto&& pair) {
        if (narrow) {
#pragma unroll
            for (int j = 0; j < C::BPW; j += 2) pair(j, true);
        } else {
#pragma unroll 1
            for (int j = 0; j < C::BPW; j += 2) pair(j, false);
        }
    };
    if constexpr (DIRECT) {
        // the warp's kGroup whole blocks lie in one block row (or past the array)
        T* q = nullptr;
        if (b0 < g.nblocks) {
            const BlockPos p = block_pos(b0, g);
            const uint64_t row = (uint64_t)p.z * g.dy + (uint64_t)p.y * 8 + (uint32_t)(lane >> 3);
            q = out + row * g.dx + (uint64_t)p.x * 8 + (uint32_t)(lane & 7);
        }
        const uint64_t half = 4ull * g.dx;   // element l + 32 is four rows down
        for_pairs([&](int j, bool nar) {
            int32_t d0a, d1a, d0b, d1b;
            bool za, zb;
            decode(j, nar, d0a, d1a, d0b, d1b, za, zb);
            if constexpr (MODE != MODE_FIXED) {
                lorenzo_inverse<DIM>(d0a, d1a, lane, ll);
                lorenzo_inverse<DIM>(d0b, d1b, lane, ll);
            }
            if (q) {
                T* qa = q + (uint32_t)j * 8;
                qa[0] = za ? T(0) : dequant(d0a, eb);
                qa[half] = za ? T(0) : dequant(d1a, eb);
                qa[8] = zb ? T(0) : dequant(d0b, eb);
                qa[8 + half] = zb ? T(0) : dequant(d1b, eb);
            }
        });
        __syncwarp();
        if (lane == 0 && last) mbar_arrive(&sh.freed[f]);   // done with the payload slot
        return;
    }
    // the output buffer is free once the previous stores have read it
    if (stored) bulk_wait_read();
    __syncwarp();
    if constexpr (DIM == 1) {
        // every block with at most 15 planes (rate-0 blocks included): four blocks per
        // step, each lane's block facts read by shuffles, no per-block rate arithmetic
        uint32_t n1 = myr, ps1 = myo, m1 = 0, heads1 = 0;
        if constexpr (MODE == MODE_OUTLIER) {
            n1 = myr & 0x1fu;
            const uint32_t ob1 = (myr & 0x80u) ? ((myr & 0x60u) >> 5) + 1u : 0u;
            if (ob1) m1 = ld_outlier(pay, myo, ob1);
            ps1 = myo + ob1;
            heads1 = __ballot_sync(FULL, ob1 != 0);
        }
        if (__all_sync(FULL, lane >= C::BPW || n1 <= 15)) {
            const uint32_t mask = plane_mask(myr, n1);
            const uint32_t has = __ballot_sync(FULL, mysz != 0);   // bit j: block j has a payload
            const int half = lane >> 4;
            const uint32_t pl = (uint32_t)(lane ^ 7) & 15u;
            const uint32_t o = pl == 15 ? 0u : 4u + 4u * pl;
#pragma unroll 1
            for (int j = 0; j < C::BPW; j += 4) {
                const uint32_t k1 = __shfl_sync(FULL, mask, j + half), k2 = __shfl_sync(FULL, mask, j + 2 + half);
                const uint32_t p1 = __shfl_sync(FULL, ps1, j + half), p2 = __shfl_sync(FULL, ps1, j + 2 + half);
                uint32_t mA = 0, mB = 0, mC = 0, mD = 0;
                if constexpr (MODE == MODE_OUTLIER) {
                    mA = __shfl_sync(FULL, m1, j);
                    mB = __shfl_sync(FULL, m1, j + 1);
                    mC = __shfl_sync(FULL, m1, j + 2);
                    mD = __shfl_sync(FULL, m1, j + 3);
                }
                int32_t dA, dB, dC, dD;
                decode_quad_1d_narrow<MODE>(pay, k1, p1, k2, p2, pl, o, heads1 >> j, mA, mB, mC, mD, dA, dB, dC, dD,
                                            lane, xl);
                if constexpr (MODE != MODE_FIXED) {
                    int32_t z = 0;
                    lorenzo_inverse<1>(dA, z, lane, ll);
                    lorenzo_inverse<1>(dB, z, lane, ll);
                    lorenzo_inverse<1>(dC, z, lane, ll);
                    lorenzo_inverse<1>(dD, z, lane, ll);
                }
                // blocks without payload decode to 0.0
                const uint32_t hj = has >> j;
                sts_val(obs + j * 32 * sizeof(T), (hj & 1u) ? dequant(dA, eb) : T(0));
                sts_val(obs + (j + 1) * 32 * sizeof(T), (hj & 2u) ? dequant(dB, eb) : T(0));
                sts_val(obs + (j + 2) * 32 * sizeof(T), (hj & 4u) ? dequant(dC, eb) : T(0));
                sts_val(obs + (j + 3) * 32 * sizeof(T), (hj & 8u) ? dequant(dD, eb) : T(0));
            }
        } else
#pragma unroll 1
        for (int j = 0; j < C::BPW; j += 2) {
            const uint32_t rA = __shfl_sync(FULL, myr, j), rB = __shfl_sync(FULL, myr, j + 1);
            const uint32_t oA = __shfl_sync(FULL, myo, j), oB = __shfl_sync(FULL, myo, j + 1);
            int32_t dA, dB;
            decode_pair_1d<MODE>(pay, rA, rB, oA, oB, dA, dB, lane, xl);
            if constexpr (MODE != MODE_FIXED) {
                int32_t z = 0;
                lorenzo_inverse<1>(dA, z, lane, ll);
                lorenzo_inverse<1>(dB, z, lane, ll);
            }
            // blocks without payload decode to 0.0
            sts_val(obs + j * 32 * sizeof(T), payload_size<1, MODE>(rA) ? dequant(dA, eb) : T(0));
            sts_val(obs + (j + 1) * 32 * sizeof(T), payload_size<1, MODE>(rB) ? dequant(dB, eb) : T(0));
        }
    } else {
        for_pairs([&](int j, bool nar) {
            int32_t d0a, d1a, d0b, d1b;
            bool za, zb;
            decode(j, nar, d0a, d1a, d0b, d1b, za, zb);
            if constexpr (MODE != MODE_FIXED) {
                lorenzo_inverse<DIM>(d0a, d1a, lane, ll);
                lorenzo_inverse<DIM>(d0b, d1b, lane, ll);
            }
            if constexpr (SWZ) {
                // this lane's elements of blocks j and j + 1; second halves 8 rows on
                const RowBox<T> rbx(lane);
                const saddr_t oa = obs + rbx.at(j), obb = obs + rbx.at(j + 1);
                sts_val(oa, za ? T(0) : dequant(d0a, eb));
                sts_val(oa + 1024u, za ? T(0) : dequant(d1a, eb));
                sts_val(obb, zb ? T(0) : dequant(d0b, eb));
                sts_val(obb + 1024u, zb ? T(0) : dequant(d1b, eb));
            } else {
                const saddr_t oj = obs + j * 64 * sizeof(T);
                sts_val(oj, za ? T(0) : dequant(d0a, eb));
                sts_val(oj + 32 * sizeof(T), za ? T(0) : dequant(d1a, eb));
                sts_val(oj + 64 * sizeof(T), zb ? T(0) : dequant(d0b, eb));
                sts_val(oj + 96 * sizeof(T), zb ? T(0) : dequant(d1b, eb));
            }
        });
    }
    __syncwarp();
    if (lane == 0 && last) mbar_arrive(&sh.freed[f]);   // done with the payload slot
    fence_proxy_async_smem();                  // decoded values -> async proxy
    __syncwarp();
    if constexpr (DIM == 1) {
        // the warp's 512 contiguous elements, clipped to the array
        const uint64_t e0 = b0 * 32;
        const uint64_t cnt = e0 < g.nbEle ? min((uint64_t)(C::BPW * 32), g.nbEle - e0) : 0;
        const uint32_t bytes = (uint32_t)cnt * (uint32_t)sizeof(T);
        const uint32_t main = bytes & ~15u;
        const uint32_t tail = (bytes - main) / (uint32_t)sizeof(T);
        if ((uint32_t)lane < tail) out[e0 + main / sizeof(T) + lane] = ob[main / sizeof(T) + lane];
        if (lane == 0 && main) {
            bulk_store(out + e0, ob, main);
            bulk_commit();
            stored = true;
        }
    } else {
        // lane j stores block j (bulk groups are per thread: each storing lane
        // commits and later waits for its own)
        if (SWZ) {
            // lane i stores row box i of the warp (block rows hold whole boxes: each box
            // is inside the array or past its last block)
            constexpr uint32_t BPB = RowBox<T>::BPB;
            if ((uint32_t)lane < C::BPW / BPB && b0 + lane * BPB < g.nblocks) {
                const BlockPos p = block_pos(b0 + lane * BPB, g);
                src.acquire_map(A.tmap);
                tma_store_3d(A.tmap, (int)(p.x * 4), (int)(p.y * 4), (int)(p.z * 4), ob + lane * BPB * 64);
                bulk_commit();
                stored = true;
            }
        } else if (DIM == 2 && g.grouped) {
            // the warp's kGroup blocks are one box (a whole group, or none past the array)
            if (lane == 0 && b0 < g.nblocks) {
                const BlockPos p = block_pos(b0, g);
                src.acquire_map(A.tmap);
                tma_store_group(A.tmap, (int)p.x, (int)p.y, (int)p.z, ob);
                bulk_commit();
                stored = true;
            }
        } else if ((uint64_t)lane < C::BPW && b0 + lane < g.nblocks) {
            const BlockPos p = block_pos(b0 + lane, g);
            src.acquire_map(A.tmap);
            if constexpr (DIM == 2)
                tma_store_3d(A.tmap, (int)(p.x * 8), (int)(p.y * 8), (int)p.z, ob + lane * 64);
            else
                tma_store_3d(A.tmap, (int)(p.x * 4), (int)(p.y * 4), (int)(p.z * 4), ob + lane * 64);
            bulk_commit();
            stored = true;
        }
    }
}

// ------------------------------------------------------------------ the kernel body

template <typename T, int DIM, bool DIRECT, typename Src>
__device__ __forceinline__ void decompress_tma_body(const Src& src, WsHeader* __restrict__ hdr,
                                                    unsigned long long* __restrict__ status_all)
{
    using C = DecCfg<T, DIM, DIRECT>;
    extern __shared__ unsigned char dsm[];
    unsigned char* base = dsm + ((C::ALIGN - (smem_u32(dsm) & (C::ALIGN - 1u))) & (C::ALIGN - 1u));
    uint8_t* slots = base + C::OFF_SLOT;
    T* obuf = reinterpret_cast<T*>(base + C::OFF_OUT);
    __shared__ __align__(8) DecShared<T, DIM> sh;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t* err = &hdr->err;
    const uint64_t ntotal = src.total();
    if (threadIdx.x == 0) {
        for (int i = 0; i < C::FRONT; i++) {
            mbar_init(&sh.full[i], 1);
            mbar_init(&sh.freed[i], C::WARPS);
        }
        mbar_fence_init();
    }
    __syncthreads();

    if (warp >= C::WARPS) {
        // ---------------------------------------------------------------- front warps
        const int f = warp - C::WARPS;
        uint8_t* slot = slots + f * C::SLOT;
        // A ticket is a group of G consecutive tiles of one array (G = Src::ticket_tiles(),
        // up to kMaxTicketTiles): their rate bytes give the group's payload size at once,
        // and one status word per group carries the look-back, so the chain of inclusive
        // prefixes advances G tiles per step.  The group's tiles then fill the slot one
        // after another (their rate bytes read again, from the cache).  Fill m is prepared
        // while the codec warps still decode fill m - 1; only its payload load waits for
        // the slot.
        constexpr int PER = C::TB / 32;   // rate bytes per lane and tile (4 in 1D, 2 in 2D/3D)
        constexpr int LPW = C::BPW / PER; // lanes per codec warp
        const int G = max(1, min(src.ticket_tiles(), kMaxTicketTiles));
        int m = 0;                        // fills of the slot so far
        bool failed = false;              // left after a wait gave up
        // A tile's rate bytes (this lane's PER consecutive blocks): block sizes, their sum,
        // and the warp-exclusive prefix of the sums (where this lane's blocks start).
        auto tile_sizes = [&](const TileArray& A, const Geom& g, int64_t lt, uint32_t* rb, uint32_t& lane_off,
                              uint32_t& total) {
            const uint64_t b0 = (uint64_t)lt * C::TB;
            uint32_t rsum = 0;
#pragma unroll
            for (int e = 0; e < PER; e++) {
                const uint64_t b = b0 + (uint64_t)lane * PER + e;   // lane holds consecutive blocks
                const uint32_t r = b < g.nblocks ? __ldg(A.cmp + b) : 0u;
                rb[e] = r;
                uint32_t sz = 0;
                src.with_mode(A.mode, [&](auto md) { sz = payload_size<DIM, decltype(md)::value>(r); });
                rsum += sz;
            }
            uint32_t incl = rsum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t v = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += v;
            }
            lane_off = incl - rsum;
            total = __shfl_sync(FULL, incl, 31);
        };
        for (;;) {
            int64_t gi = 0;
            if (lane == 0) gi = (int64_t)atomicAdd(&hdr->ticket, 1u);
            gi = __shfl_sync(FULL, gi, 0);
            const int64_t t0 = gi * G;
            if ((uint64_t)t0 >= ntotal) {   // no more tiles: an empty fill ends the slot
                if (m > 0 && !mbar_wait(&sh.freed[f], (uint32_t)(m - 1) & 1u, err)) { failed = true; break; }
                if (lane == 0) {
                    sh.tile[f] = t0;
                    mbar_arrive(&sh.full[f]);
                }
                break;
            }
            const int n = (int)min((uint64_t)G, ntotal - (uint64_t)t0);   // tiles in the group
            int32_t a;
            int64_t lt0;
            src.locate(t0, a, lt0);   // a group's tiles are consecutive tiles of one array
            const TileArray A = src.array(a);
            const Geom g = *A.g;
            const uint8_t* cmp = A.cmp;
            unsigned long long* status = A.status;
            const int64_t grp = lt0 / G;   // status word of the group
            // the group's payload bytes: every tile's rate bytes -> sizes -> sum (the group's
            // tiles are read again as they fill the slot, from the cache)
            unsigned long long gagg = 0;
            for (int i = 0; i < n; i++) {
                uint32_t rb[PER], lo, tot;
                tile_sizes(A, g, lt0 + i, rb, lo, tot);
                gagg += tot;
            }
            if (lane == 0) st_post(status + grp, (grp == 0 ? ST_INC : ST_AGG) | gagg);
            const uint64_t excl = grp > 0 ? warp_lookback(status, grp, err) : 0;
            if (lane == 0) {
                if (grp > 0) st_post(status + grp, ST_INC | ((excl + gagg) & ST_VAL));
                if ((uint64_t)(lt0 + n) == g.ntiles) *A.total_out = g.rate_bytes + excl + gagg;
            }
            uint64_t p0 = g.rate_bytes + excl;   // payload start of the group's next tile
            bool stop = false;
            const int fill_max = DIM == 1 && G >= 4 ? DecShared<T, DIM>::FT : 1;
            for (int i = 0; i < n;) {
                // one fill: the group's next tiles while their payloads fit one slot
                const int rb = m & 1;
                const int first = i;
                const uint64_t a0 = p0 & ~15ull;
                uint64_t pend = p0;                 // end of the fill's payload
                uint32_t mytoff = kBadSlot;         // lane k: tile k's payload start in the slot
                int cnt = 0;
                bool bad = false;
                while (i < n && cnt < fill_max) {
                    uint32_t rbyte[PER], wo, agg;
                    tile_sizes(A, g, lt0 + i, rbyte, wo, agg);
                    // rate bytes no valid stream holds (rate > 32 outside outlier mode) could
                    // claim more than a slot: such a tile goes alone, is not loaded and decodes
                    // to zeros
                    const bool fits = agg <= (uint32_t)(C::TB * C::MAXBLK);
                    if (!fits && cnt > 0) break;
                    if (fits && cnt > 0 && ((pend + agg + 15) & ~15ull) - a0 > (uint64_t)C::TB * C::MAXBLK + 30) break;
#pragma unroll
                    for (int e = 0; e < PER; e++) sh.rates[f][rb][cnt][lane * PER + e] = (uint8_t)rbyte[e];
                    if (lane % LPW == 0) sh.woff[f][rb][cnt][lane / LPW] = wo;
                    if (lane == cnt) mytoff = fits ? (uint32_t)(pend - a0) : kBadSlot;
                    pend += agg;
                    cnt++;
                    i++;
                    if (!fits) {
                        if (lane == 0) atomicOr(err, ERR_CAPACITY);
                        bad = true;
                        break;
                    }
                }
                const uint64_t a1 = (pend + 15) & ~15ull;
                const uint32_t bytes = !bad && pend > p0 ? (uint32_t)(a1 - a0) : 0u;
                // the payload's address is known before the slot is free: bring it into L2
                // now, so that the slot's load, once the codec warps release it, reads L2
                if (lane == 0 && bytes) bulk_prefetch_l2(cmp + a0, bytes);
                // the slot: fill m - 1 decoded
                if (m > 0 && !mbar_wait(&sh.freed[f], (uint32_t)(m - 1) & 1u, err)) { stop = true; break; }
                if (lane < cnt) sh.toff[f][lane] = mytoff;
                __syncwarp();   // rates and offsets are written before lane 0 publishes the fill
                if (lane == 0) {
                    sh.tile[f] = t0 + first;
                    sh.local[f] = lt0 + first;
                    sh.arr[f] = a;
                    sh.cnt[f] = cnt;
                    mbar_arrive_tx(&sh.full[f], bytes);
                    if (bytes) bulk_load(slot, cmp + a0, bytes, &sh.full[f]);
                }
                __syncwarp();
                p0 = pend;
                m++;
            }
            if (stop) { failed = true; break; }
        }
        // fill m - 1 may still be loading when a wait gave up: the CTA must not end
        // before that copy into its shared memory has landed
        if (failed && m > 0 && lane == 0) mbar_drain(&sh.full[f], (uint32_t)(m - 1) & 1u, err);
        __syncwarp();
    } else {
        // ---------------------------------------------------------------- codec warps
        T* ob = obuf + warp * (C::BPW * C::BLK);
        const saddr_t obs = saddr(ob) + lane * (uint32_t)sizeof(T);   // this lane's element of block 0
        const XposeLane xl(lane);
        uint32_t parity = 0;      // bit f: phase parity of slot f's next fill
        uint32_t ended = 0;       // bit f: front warp f has no more tiles
        bool stored = false;      // this warp has bulk stores in flight
        for (int k = 0; ended != (1u << C::FRONT) - 1u; k++) {
            const int f = k % C::FRONT;
            if ((ended >> f) & 1u) continue;
            const uint32_t ph = (parity >> f) & 1u;
            parity ^= 1u << f;
            if (!mbar_wait(&sh.full[f], ph, err)) break;
            const int64_t t = *reinterpret_cast<volatile int64_t*>(&sh.tile[f]);
            if ((uint64_t)t >= ntotal) { ended |= 1u << f; continue; }
            const TileArray A = src.array(sh.arr[f]);
            const int64_t lt0 = sh.local[f];
            const int nt = DIM == 1 ? sh.cnt[f] : 1;   // multi-tile fills: 1D only
            const saddr_t pay = saddr(slots + f * C::SLOT);
            for (int kt = 0; kt < nt; kt++) {   // the fill's tiles; the last one frees the slot
                const int64_t lt = lt0 + kt;
                const bool last = kt == nt - 1;
                src.with_mode(A.mode, [&](auto m) {
                    constexpr int MODE = decltype(m)::value;
                    if constexpr (DIM == 3) {
                        if (A.g->grouped)   // row boxes: the buffer's start
                            decode_and_store<T, DIM, MODE, DIRECT, true>(src, A, sh, f, (int)ph, kt, last, lt, pay, ob,
                                                                         saddr(ob), xl, stored, warp, lane);
                        else
                            decode_and_store<T, DIM, MODE, DIRECT, false>(src, A, sh, f, (int)ph, kt, last, lt, pay,
                                                                          ob, obs, xl, stored, warp, lane);
                    } else {
                        decode_and_store<T, DIM, MODE, DIRECT, false>(src, A, sh, f, (int)ph, kt, last, lt, pay, ob,
                                                                      obs, xl, stored, warp, lane);
                    }
                });
                __syncwarp();
            }
        }
        if (stored) bulk_wait_all();
        __syncwarp();
    }
    finish_cta(hdr, status_all, ntotal);
}

template <typename T, int DIM, int MODE, bool DIRECT = false>
__global__ void __launch_bounds__(DecCfg<T, DIM, DIRECT>::THREADS, DecCfg<T, DIM, DIRECT>::MIN_CTAS)
decompress_tma_kernel(const __grid_constant__ CUtensorMap tmap, T* __restrict__ out, const uint8_t* __restrict__ cmp,
                      const __grid_constant__ Geom g, T eb, WsHeader* __restrict__ hdr,
                      unsigned long long* __restrict__ status, int ticket_tiles)
{
    const SingleTiles<T, MODE> src{&tmap, out, const_cast<uint8_t*>(cmp), &g, eb, status, &hdr->total, ticket_tiles};
    decompress_tma_body<T, DIM, DIRECT>(src, hdr, status);
}

}  // namespace cuszp

// codec.cuh -- device building blocks of the fused cuSZp block codec for sm_100a.
//
// Format (identical bytes to the reference, independent of how work is tiled):
//   [rate region: one byte per data block]  [payload of block 0][payload of block 1]...
//   data block = 32 consecutive elements (1D), 8x8 elements of one z-slice (2D,
//   element k = 8*row + col), or 4x4x4 elements (3D, k = 16*z + 4*y + x).
//   payload = sign map (W bytes) + `rate` bit-planes of W bytes (W = 4 in 1D, 8 in 2D/3D);
//   in outlier mode optionally preceded by element 0's magnitude in 1..4 LE bytes.
//   Reference: src/cuSZp_kernels_1D_f32.cu:31-296 (layout), :1165-1183 (outlier choice).
//
// Work decomposition (B200-first, not the reference's): persistent CTAs of 8 warps
// pull tiles of consecutive data blocks from an atomic ticket; a warp owns one data
// block at a time with one element per lane (two in 2D/3D), so sign maps are warp
// ballots and bit-planes come out of one 32x32 register transpose across the warp.
// Payload offsets come from a single-pass decoupled look-back over tiles.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace cuszp {

constexpr unsigned FULL = 0xffffffffu;
constexpr int kWarps = 8;                 // default warps per CTA of the single-array kernels
constexpr int kThreads = kWarps * 32;

enum Mode : int { MODE_FIXED = 0, MODE_PLAIN = 1, MODE_OUTLIER = 2 };

// Error bits reported through the workspace error word.  The two timeout bits make
// every other bounded wait of the launch give up as well; ERR_CAPACITY (a stream that
// does not fit the caller's buffer, or rate bytes no valid stream holds) does not stop
// the launch: its other tiles complete normally.
enum : uint32_t { ERR_LOOKBACK_TIMEOUT = 1u, ERR_CAPACITY = 2u, ERR_WAIT_TIMEOUT = 4u };
constexpr uint32_t kTimeoutErrs = ERR_LOOKBACK_TIMEOUT | ERR_WAIT_TIMEOUT;

// Tile status word: [63:62] = 0 none / 1 aggregate / 2 inclusive prefix, [61:0] value.
constexpr uint64_t ST_AGG = 1ull << 62;
constexpr uint64_t ST_INC = 2ull << 62;
constexpr uint64_t ST_VAL = (1ull << 62) - 1;

// Upper bound on look-back polls before a tile gives up (a few hundred ms).
constexpr int kSpinLimit = 1 << 21;

// Workspace header; followed by one uint64 status word per tile.
struct WsHeader {
    uint32_t ticket;     // next tile to hand out
    uint32_t done;       // CTAs that finished (last one resets the workspace)
    uint32_t err;        // sticky error bits, read and cleared by the host
    uint32_t wait_cap;   // 0: default wait limits; else every bounded wait gives up after
                         // this many polls (look-back) or sleep slices (mbarrier waits)
    unsigned long long total;   // true stream length S of the last call (~0 after a timeout)
    unsigned long long pad2[3];
};
static_assert(sizeof(WsHeader) == 48, "header layout");
static_assert(offsetof(WsHeader, wait_cap) == offsetof(WsHeader, err) + 4, "wait_cap follows err");

// A wait's limit: the workspace's wait_cap when set (read through the error word's
// address: the cap is the header word after it), else the default.  Waits read it only
// once a first attempt has failed, so a wait that is already satisfied costs no load.
__device__ __forceinline__ int wait_limit(const uint32_t* err, int dflt)
{
    const uint32_t cap = *reinterpret_cast<const volatile uint32_t*>(err + 1);
    return cap ? (int)min(cap, 0x7fffffffu) : dflt;
}
// Whether a bounded wait elsewhere in the launch has given up.
__device__ __forceinline__ bool timed_out(const uint32_t* err)
{
    return (*reinterpret_cast<const volatile uint32_t*>(err) & kTimeoutErrs) != 0;
}

// Unsigned 32-bit division by an invariant divisor d >= 1 as a multiply-high and shifts
// (Granlund & Montgomery, "Division by invariant integers using multiplication",
// PLDI 1994): with l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1,
// n / d = (t + ((n - t) >> 1)) >> (l - 1), t = umulhi(m, n); d == 1 is n itself.
struct FastDiv {
    uint32_t m, s1, s2;   // multiplier and the two shifts (s1 = 1, s2 = l - 1; both 0 for d == 1)
    __host__ __device__ static FastDiv make(uint32_t d)
    {
        FastDiv f{0u, 0u, 0u};
        if (d <= 1) return f;
        uint32_t l = 0;
        while (l < 32 && (1ull << l) < d) l++;
        f.m = (uint32_t)((((1ull << l) - d) << 32) / d + 1);
        f.s1 = 1;
        f.s2 = l - 1;
        return f;
    }
    __device__ __forceinline__ uint32_t div(uint32_t n) const
    {
        const uint32_t t = __umulhi(m, n);
        return (t + ((n - t) >> s1)) >> s2;
    }
};

struct Geom {
    uint64_t nbEle;        // 1D element count
    uint32_t dx, dy, dz;   // dims.x fastest
    uint32_t bxn, byn;     // blocks along x and y (2D/3D)
    uint64_t nblocks;      // data blocks that exist
    uint64_t rate_bytes;   // size of the rate region
    uint64_t ntiles;       // tiles handed out (1D: covers the whole rate region)
    FastDiv div_bx;        // division by bxn
    FastDiv div_plane;     // division by bxn * byn
    uint32_t grouped;      // TMA kernels, 2D: the tensor map's box is kGroup whole blocks
    uint64_t cap;          // compress: bytes the stream buffer holds (~0: not checked); a
                           // payload span that would end past it is not written and
                           // ERR_CAPACITY is raised (the stream length is still computed)
    unsigned long long* size_out;   // single-array compress: the CTA that finishes last
                                    // writes the stream length here (null: not asked)
};

// Blocks per tensor-map box of the TMA kernels' grouped 2D maps (one codec warp's share
// of a tile in 2D/3D).
constexpr uint32_t kGroup = 8;

// ------------------------------------------------------------------ scalar helpers

__device__ __forceinline__ int32_t wsub(int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); }
__device__ __forceinline__ int32_t wadd(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
__device__ __forceinline__ uint32_t uabs(int32_t a) { return a < 0 ? 0u - (uint32_t)a : (uint32_t)a; }
__device__ __forceinline__ int bitlen(uint32_t x) { return 32 - __clz(x); }

// Quantizer of src/cuSZp_kernels_1D_f32.cu:3-20 (f32) and 1D_f64.cu:3-8 (f64):
//   p = x*r; s = (p >= -0.5) ? 0 : 1; q = rzi(p + 0.5) - s.
// kFusedQuant selects how p + 0.5 is rounded: as a separately rounded add, or as
// one fma(x, r, 0.5).  The reference build for sm_100 rounds them separately; the
// golden vectors' rounding-trap inputs (where the two truncate differently) pin it.
// The conversion is the same cvt.rzi instruction the reference uses, so NaN and
// out-of-range products convert identically (f32: NaN -> 0, f64: NaN -> INT_MIN).
#ifndef CUSZP_FUSED_QUANT
#define CUSZP_FUSED_QUANT 0
#endif
constexpr bool kFusedQuant = CUSZP_FUSED_QUANT != 0;

__device__ __forceinline__ int32_t quantize(float x, float r)
{
    float p = __fmul_rn(x, r);
    int32_t s = (p >= -0.5f) ? 0 : 1;
    float t = kFusedQuant ? __fmaf_rn(x, r, 0.5f) : __fadd_rn(p, 0.5f);
    return wsub(__float2int_rz(t), s);
}
__device__ __forceinline__ int32_t quantize(double x, double r)
{
    double p = __dmul_rn(x, r);
    int32_t s = (p >= -0.5) ? 0 : 1;
    double t = kFusedQuant ? __fma_rn(x, r, 0.5) : __dadd_rn(p, 0.5);
    return wsub(__double2int_rz(t), s);
}

// Reconstruction ((T)q * eb) * 2 of src/cuSZp_kernels_1D_f32.cu:490.
__device__ __forceinline__ float dequant(int32_t q, float eb) { return __fmul_rn(__fmul_rn(__int2float_rn(q), eb), 2.0f); }
__device__ __forceinline__ double dequant(int32_t q, double eb) { return __dmul_rn(__dmul_rn((double)q, eb), 2.0); }

// Streaming loads/stores (touched once).
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }
__device__ __forceinline__ double ld_stream(const double* p) { return __ldcs(p); }
__device__ __forceinline__ void st_stream(float* p, float v) { __stcs(p, v); }
__device__ __forceinline__ void st_stream(double* p, double v) { __stcs(p, v); }

// ------------------------------------------------------------------ shared-memory access

// Shared memory addressed through 32-bit shared-window addresses: address arithmetic
// stays 32-bit and the accesses compile to LDS/STS whatever the compiler can prove
// about a pointer's origin.  Volatile with a memory clobber: they are never moved
// across mbarrier waits or warp barriers.
using saddr_t = uint32_t;
__device__ __forceinline__ saddr_t saddr(const void* p) { return (saddr_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void sts_u8(saddr_t a, uint32_t v)
{
    asm volatile("st.shared.u8 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ void sts_u16(saddr_t a, uint32_t v)
{
    asm volatile("st.shared.u16 [%0], %1;" ::"r"(a), "h"((unsigned short)v) : "memory");
}
__device__ __forceinline__ void sts_u32(saddr_t a, uint32_t v)
{
    asm volatile("st.shared.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t lds_u8(saddr_t a)
{
    uint32_t v;
    asm volatile("ld.shared.u8 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
    return v;
}
__device__ __forceinline__ uint32_t lds_u32(saddr_t a)
{
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
    return v;
}
// Stores and loads that take effect only where `c` holds, as predicated instructions:
// lanes that skip them do not branch, so a warp whose lanes disagree does not diverge.
__device__ __forceinline__ void sts_u32_if(bool c, saddr_t a, uint32_t v)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %2, 0;\n\t@p st.shared.u32 [%0], %1;\n\t}"
                 ::"r"(a), "r"(v), "r"((uint32_t)c) : "memory");
}
__device__ __forceinline__ void sts_u16_if(bool c, saddr_t a, uint32_t v)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %2, 0;\n\t@p st.shared.u16 [%0], %1;\n\t}"
                 ::"r"(a), "h"((unsigned short)v), "r"((uint32_t)c) : "memory");
}
__device__ __forceinline__ void sts_u8_if(bool c, saddr_t a, uint32_t v)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %2, 0;\n\t@p st.shared.u8 [%0], %1;\n\t}"
                 ::"r"(a), "r"(v), "r"((uint32_t)c) : "memory");
}
// 0 where `c` does not hold.
__device__ __forceinline__ uint32_t lds_u32_if(bool c, saddr_t a)
{
    uint32_t v;
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %2, 0;\n\tmov.u32 %0, 0;\n\t@p ld.shared.u32 %0, [%1];\n\t}"
                 : "=r"(v) : "r"(a), "r"((uint32_t)c) : "memory");
    return v;
}
// 16 bytes from a 16-byte aligned shared address.
__device__ __forceinline__ uint4 lds_u128(saddr_t a)
{
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a) : "memory");
    return v;
}
__device__ __forceinline__ void sts_val(saddr_t a, float v) { asm volatile("st.shared.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory"); }
__device__ __forceinline__ void sts_val(saddr_t a, double v) { asm volatile("st.shared.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory"); }
template <typename T> __device__ __forceinline__ T lds_val(saddr_t a);
template <> __device__ __forceinline__ float lds_val<float>(saddr_t a)
{
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a) : "memory");
    return v;
}
template <> __device__ __forceinline__ double lds_val<double>(saddr_t a)
{
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a) : "memory");
    return v;
}

// ------------------------------------------------------------------ warp bit transpose

// 32x32 bit-matrix transpose across a warp: on entry the lane whose row index is
// `row` holds row `row` (bit b = M[row][b]); on exit lane p holds column p (bit r =
// M[r][p]).  5 butterfly stages of one shuffle, one rotate and one LOP3: in the stage
// of distance j a lane keeps its own half of each 2j-bit group and takes the other
// half from its partner, whose bits sit j places away -- (y >> j) for the upper
// partner, (y << j) for the lower one, which under the stage's mask equal rotations
// of y right by j and by 32 - j.
// With row = lane the transpose is the plain one.  With row = lane ^ 7 the element
// held by lane l lands on bit l ^ 7 of every column word -- the reference's byte
// layout (8 elements per byte, first element in the most significant bit) -- so a
// plane word can be stored as it comes out.
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x, int row)
{
#pragma unroll
    for (int j = 16; j >= 1; j >>= 1) {
        const uint32_t m = j == 16 ? 0xFFFF0000u : j == 8 ? 0xFF00FF00u : j == 4 ? 0xF0F0F0F0u
                         : j == 2 ? 0xCCCCCCCCu : 0xAAAAAAAAu;
        const uint32_t y = __shfl_xor_sync(FULL, x, j);
        const bool up = row & j;
        const uint32_t keep = up ? m : ~m;
        const uint32_t sh = __funnelshift_r(y, y, up ? j : 32 - j);
        x = (x & keep) | (sh & ~keep);
    }
    return x;
}

// The per-lane constants of the five butterfly stages for a fixed row index, for loops
// that transpose many words with the same row: keep mask and rotate amount per stage.
// The two whole-byte stages (distances 16 and 8) keep / take whole bytes, so each is one
// byte permute of the lane's and its partner's word (selectors byte16 / byte8) instead
// of a rotate and a masked merge.
struct XposeLane {
    uint32_t keep[5];
    uint32_t rot[5];
    uint32_t byte16, byte8;
    __device__ __forceinline__ explicit XposeLane(int row)
    {
#pragma unroll
        for (int i = 0; i < 5; i++) {
            const int j = 16 >> i;
            const uint32_t m = j == 16 ? 0xFFFF0000u : j == 8 ? 0xFF00FF00u : j == 4 ? 0xF0F0F0F0u
                             : j == 2 ? 0xCCCCCCCCu : 0xAAAAAAAAu;
            const bool up = row & j;
            keep[i] = up ? m : ~m;
            rot[i] = up ? (uint32_t)j : (uint32_t)(32 - j);
        }
        // __byte_perm(x, y, s): selector nibble n picks result byte n from x (0-3) or y (4-7).
        // distance 16: upper lanes keep x's high half and take y's high half as their low
        // half; lower lanes keep x's low half and take y's low half as their high half.
        byte16 = (row & 16) ? 0x3276u : 0x5410u;
        // distance 8: upper lanes keep x's odd bytes and take y's odd bytes into the even
        // positions; lower lanes keep x's even bytes and take y's even bytes into the odd ones.
        byte8 = (row & 8) ? 0x3715u : 0x6240u;
    }
    // One butterfly stage i (distance 16 >> i) of word x with its partner's word y.
    __device__ __forceinline__ uint32_t stage(int i, uint32_t x, uint32_t y) const
    {
        if (i == 0) return __byte_perm(x, y, byte16);
        if (i == 1) return __byte_perm(x, y, byte8);
        return (x & keep[i]) | (__funnelshift_r(y, y, rot[i]) & ~keep[i]);
    }
};
// Two independent transposes, interleaved stage by stage (twice the work per dependent
// step of the butterfly).
__device__ __forceinline__ void warp_transpose32x2(uint32_t& a, uint32_t& b, const XposeLane& xl)
{
#pragma unroll
    for (int i = 0; i < 5; i++) {
        const int j = 16 >> i;
        const uint32_t ya = __shfl_xor_sync(FULL, a, j);
        const uint32_t yb = __shfl_xor_sync(FULL, b, j);
        a = xl.stage(i, a, ya);
        b = xl.stage(i, b, yb);
    }
}
// Two transposes of stream-order words, for the decoder: lane l holds the word of row
// (l ^ 7), whose bit (e ^ 7) is column e (the reference's byte order, 8 columns per byte,
// first one in the most significant bit); on exit lane p holds column p with bit r =
// row r, so no per-word byte-order conversion is needed.  It is the butterfly of
// XposeLane(lane ^ 7), which swaps the keep / rotate roles of the three sub-byte stages:
// those stages keep ~keep and rotate the other way, from the same XposeLane(lane).
__device__ __forceinline__ void warp_transpose32x2_stream(uint32_t& a, uint32_t& b, const XposeLane& xl)
{
#pragma unroll
    for (int i = 0; i < 5; i++) {
        const int j = 16 >> i;
        const uint32_t ya = __shfl_xor_sync(FULL, a, j);
        const uint32_t yb = __shfl_xor_sync(FULL, b, j);
        if (i < 2) {
            a = xl.stage(i, a, ya);
            b = xl.stage(i, b, yb);
        } else {
            a = (a & ~xl.keep[i]) | (__funnelshift_l(ya, ya, xl.rot[i]) & xl.keep[i]);
            b = (b & ~xl.keep[i]) | (__funnelshift_l(yb, yb, xl.rot[i]) & xl.keep[i]);
        }
    }
}
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x, const XposeLane& xl)
{
#pragma unroll
    for (int i = 0; i < 5; i++) {
        const int j = 16 >> i;
        const uint32_t y = __shfl_xor_sync(FULL, x, j);
        x = xl.stage(i, x, y);
    }
    return x;
}

// Word with bit l = element l  <->  stored little-endian word whose byte b holds
// elements 8b..8b+7 most-significant-bit first (the reference's plane/sign bytes).
__device__ __forceinline__ uint32_t to_stream_word(uint32_t bits) { return __byte_perm(__brev(bits), 0, 0x0123); }
__device__ __forceinline__ uint32_t from_stream_word(uint32_t w) { return __brev(__byte_perm(w, 0, 0x0123)); }

// ------------------------------------------------------------------ payload sizes

template <int DIM, int MODE>
__device__ __forceinline__ uint32_t payload_size(uint32_t rb)
{
    constexpr uint32_t W = DIM == 1 ? 4u : 8u;
    if constexpr (MODE != MODE_OUTLIER) {
        return rb ? W + W * rb : 0u;
    } else {
        const uint32_t r = rb & 0x1fu;
        if (rb & 0x80u) return W + (((rb & 0x60u) >> 5) + 1u) + W * r;
        return r ? W + W * r : 0u;
    }
}

// ------------------------------------------------------------------ tile look-back

// Posts a tile's status word (aggregate or inclusive prefix).  The word carries its
// state and value together and publishes no other data, so the store needs no
// release ordering: a relaxed store does not first wait for this thread's earlier
// global writes (rate and payload bytes) to reach L2, which under load costs
// microseconds on the look-back chain.  Should a tile's aggregate ever land after its
// inclusive prefix, readers would only look further back; sums stay exact.
__device__ __forceinline__ void st_post(unsigned long long* p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}
// Status words carry their value (state and prefix in one 64-bit word), so polling
// needs no acquire ordering; relaxed loads let a lane's polls overlap instead of
// waiting out one L2 round trip each.
__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint64_t warp_sum64(uint64_t v)
{
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// Exclusive prefix of tile `tile`, looked back by ONE warp over a window of
// 32 x kLookbackPerLane predecessors per step (poll k reads the 32 consecutive
// status words hi-32k-31 .. hi-32k, one per lane: coalesced).
// The newest inclusive prefix in the window ends the walk; every tile newer than it
// must have posted its aggregate; older prefixes are reached by further steps.  One
// word per lane per poll measured fastest: 3-9 % shorter compress kernels than 8 words
// per lane, and no decompress kernel gained from 4, 8 or 16 (each poll then costs more
// loads and instructions than the steps it saves).  Only the polling warp spins (with
// exponential back-off).  Every wait is bounded: on timeout the error bit is set and
// the partial sum is returned, so no CTA can hang the GPU.
constexpr int kLookbackPerLane = 1;

struct LookbackShared {
    unsigned long long excl;
};

template <int K = kLookbackPerLane>
__device__ __forceinline__ uint64_t warp_lookback(unsigned long long* status, int64_t tile, uint32_t* err)
{
    const int lane = threadIdx.x & 31;
    constexpr long long NONE = -(1ll << 62);
    int limit = 0;   // read at the first poll that finds a predecessor pending
    uint64_t excl = 0;
    int64_t hi = tile - 1;
    while (hi >= 0) {
        int spins = 0;
        unsigned backoff = 32;
        unsigned long long w[K];
        long long jmax;
        while (true) {
            long long j = NONE;
            bool pend_any = false;
#pragma unroll
            for (int k = 0; k < K; k++) {
                const int64_t idx = hi - (int64_t)(k * 32 + lane);
                w[k] = idx >= 0 ? ld_relaxed(status + idx) : (unsigned long long)ST_INC;   // before tile 0: prefix 0
            }
#pragma unroll
            for (int k = K - 1; k >= 0; k--) {
                const int64_t idx = hi - (int64_t)(k * 32 + lane);
                if ((w[k] >> 62) == 2) j = (long long)idx;     // newest inclusive this lane saw
            }
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) j = max(j, (long long)__shfl_xor_sync(FULL, j, o));
            jmax = j;
#pragma unroll
            for (int k = 0; k < K; k++) {
                const int64_t idx = hi - (int64_t)(k * 32 + lane);
                pend_any |= (w[k] >> 62) == 0 && (long long)idx > jmax;
            }
            if (!__any_sync(FULL, pend_any)) break;
            if (limit == 0) limit = wait_limit(err, kSpinLimit);
            if (++spins > limit) {
                if (lane == 0) atomicOr(err, ERR_LOOKBACK_TIMEOUT);
                return excl;
            }
            __nanosleep(backoff);
            backoff = backoff < 256 ? 2 * backoff : 256;
        }
        uint64_t v = 0;
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int64_t idx = hi - (int64_t)(k * 32 + lane);
            if (idx >= 0 && (long long)idx >= jmax) v += w[k] & ST_VAL;
        }
        excl += warp_sum64(v);
        if (jmax != NONE) return excl;
        hi -= 32 * K;
    }
    return excl;
}

// Last CTA out resets the workspace so the next call finds it zeroed.
// The CTA that finishes last resets the workspace for the next call and, when asked
// (size_out), writes the stream length there: it is the last writer, so the length is
// final, and no copy after the kernel is needed.
__device__ __forceinline__ void finish_cta(WsHeader* hdr, unsigned long long* status, uint64_t ntiles,
                                           unsigned long long* size_out = nullptr)
{
    __shared__ int s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t prev = atomicAdd(&hdr->done, 1u);
        s_last = prev == gridDim.x - 1;
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        for (uint64_t i = threadIdx.x; i < ntiles; i += blockDim.x) status[i] = 0ull;
        if (threadIdx.x == 0) {
            hdr->ticket = 0u;
            hdr->done = 0u;
            // a stream length after a timed-out wait may be partial: mark it invalid
            if (timed_out(&hdr->err)) hdr->total = ~0ull;
            if (size_out) *size_out = *reinterpret_cast<volatile unsigned long long*>(&hdr->total);
        }
        __threadfence();
    }
}

// CTA-wide tile prefix in two halves, so a CTA can issue other work between them:
//   scan_begin: each warp posts its payload total (then a barrier);
//   scan_finish: warp 0 scans the totals, publishes the tile aggregate, looks back,
//                publishes the inclusive prefix (then a barrier).
// Afterwards s_warp[w] is warp w's offset inside the tile and *s_base the tile's
// offset inside the payload; the last tile of an array stores S in *total_out.
template <int WARPS>
__device__ __forceinline__ void scan_begin(uint32_t warp_total, uint32_t* s_warp)
{
    if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = warp_total;
    __syncthreads();
}

template <int WARPS>
__device__ __forceinline__ void scan_finish(int64_t tile, uint64_t ntiles, unsigned long long* status, uint32_t* err,
                                            unsigned long long* total_out, uint64_t rate_bytes, uint32_t* s_warp,
                                            uint64_t* s_base, LookbackShared& lb)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp == 0) {
        uint32_t v = lane < WARPS ? s_warp[lane] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < WARPS; o <<= 1) {
            uint32_t t = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += t;
        }
        const uint64_t agg = __shfl_sync(FULL, incl, WARPS - 1);
        __syncwarp();
        if (lane < WARPS) s_warp[lane] = incl - v;
        if (lane == 0) st_post(status + tile, (tile == 0 ? ST_INC : ST_AGG) | agg);
        const uint64_t excl = tile > 0 ? warp_lookback(status, tile, err) : 0;
        if (lane == 0) {
            if (tile > 0) st_post(status + tile, ST_INC | ((excl + agg) & ST_VAL));
            *s_base = excl;
            if ((uint64_t)tile == ntiles - 1) *total_out = rate_bytes + excl + agg;
        }
    }
    __syncthreads();
}

}  // namespace cuszp

// codec_kernels.cuh -- the fused compress and decompress kernels (one of each per
// dtype x dimensionality x encoding mode), built from the pieces in codec.cuh.
//
// Compress, per tile of TB consecutive data blocks (TB = 128 in 1D, 64 in 2D/3D):
//   1. each warp loads its BPW blocks (coalesced, one element per lane; two in 2D/3D),
//      quantizes, applies the Lorenzo delta with warp shuffles, reduces the block
//      maximum with redux.sync and writes the rate bytes;
//   2. warp totals -> tile aggregate -> decoupled look-back -> tile byte offset;
//   3. each warp transposes its magnitudes (one 32x32 warp transpose per block, or
//      per pair of 1D blocks when both rates are <= 16) and stores sign map and
//      planes at their final offsets.
// Decompress mirrors it: rate bytes -> sizes -> look-back -> payload loads ->
// inverse transpose -> prefix-sum Lorenzo inverse -> dequantize -> store.
#pragma once

#include "codec.cuh"

#include <type_traits>

namespace cuszp {

// Tile shape: WARPS warps per CTA, BPW data blocks per warp (TB = WARPS*BPW per tile).
// In 1D a tile count must divide the 1024-block rate-region granule, so TB is a
// power of two <= 1024.
template <int DIM, int WARPS_ = kWarps, int BPW_ = (DIM == 1 ? 16 : 8)> struct Tiling {
    static constexpr int DIMS = DIM;
    static constexpr int WARPS = WARPS_;
    static constexpr int THREADS = 32 * WARPS_;
    static constexpr int BPW = BPW_;                // data blocks per warp per tile
    static constexpr int TB = WARPS_ * BPW_;        // data blocks per tile
    static constexpr int W = DIM == 1 ? 4 : 8;      // bytes per bit-plane
    static_assert(BPW_ % 2 == 0 && BPW_ <= 32, "blocks per warp");
};

// --------------------------------------------------------------- byte stores / loads

// put32 into shared memory.  Outlier-mode words sit at any byte offset; the offset's
// residue mod 4 is the same for every word of a block, so the branch is warp-uniform.
template <int MODE>
__device__ __forceinline__ void put32s(saddr_t a, uint32_t v)
{
    if constexpr (MODE == MODE_OUTLIER) {
        if ((a & 3u) == 0) {
            sts_u32(a, v);
        } else if ((a & 1u) == 0) {
            sts_u16(a, v);
            sts_u16(a + 2, v >> 16);
        } else {
            // odd offset: the middle two bytes are a 2-byte aligned pair
            sts_u8(a, v); sts_u16(a + 1, v >> 8); sts_u8(a + 3, v >> 24);
        }
    } else {
        sts_u32(a, v);
    }
}
// put32s where `c` holds, without a branch on `c`.  Outlier mode: BYTEWISE writes the
// word as four byte stores under one predicate, with no branch at all; otherwise the
// offset's residue mod 4 (uniform over a block's words, so the branch does not
// diverge) picks one word, two halves, or byte + half + byte.  Bytewise measured 8 %
// faster on the 512^3 f32 outlier 1D compress and 3.6 % in 2D, but 1 % slower in 3D.
template <int MODE, bool BYTEWISE = false>
__device__ __forceinline__ void put32s_if(bool c, saddr_t a, uint32_t v)
{
    if constexpr (MODE == MODE_OUTLIER && BYTEWISE) {
        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %5, 0;\n\t"
                     "@p st.shared.u8 [%0], %1;\n\t@p st.shared.u8 [%0+1], %2;\n\t"
                     "@p st.shared.u8 [%0+2], %3;\n\t@p st.shared.u8 [%0+3], %4;\n\t}"
                     ::"r"(a), "r"(v), "r"(v >> 8), "r"(v >> 16), "r"(v >> 24), "r"((uint32_t)c) : "memory");
    } else if constexpr (MODE == MODE_OUTLIER) {
        const uint32_t r = a & 3u;
        if (r == 0) {
            sts_u32_if(c, a, v);
        } else if (r == 2) {
            sts_u16_if(c, a, v);
            sts_u16_if(c, a + 2, v >> 16);
        } else {
            sts_u8_if(c, a, v);
            sts_u16_if(c, a + 1, v >> 8);
            sts_u8_if(c, a + 3, v >> 24);
        }
    } else {
        sts_u32_if(c, a, v);
    }
}
// Outlier-mode payload words sit at any byte offset: read the (at most two) aligned
// words that hold the four bytes and funnel-shift.  Both aligned words contain bytes
// of the payload itself, so the reads never leave the pages the stream occupies.
template <int MODE>
__device__ __forceinline__ uint32_t get32(const uint8_t* p)
{
    if constexpr (MODE == MODE_OUTLIER) {
        const uintptr_t a = reinterpret_cast<uintptr_t>(p);
        const uint32_t* w = reinterpret_cast<const uint32_t*>(a & ~(uintptr_t)3);
        const uint32_t sh = (uint32_t)(a & 3) * 8;
        const uint32_t lo = __ldg(w);
        return sh ? __funnelshift_r(lo, __ldg(w + 1), sh) : lo;
    } else {
        return __ldg(reinterpret_cast<const uint32_t*>(p));
    }
}

// --------------------------------------------------------------- block addressing

struct BlockPos { uint32_t z, y, x; };   // block coordinates (2D: z = slice)

__device__ __forceinline__ BlockPos block_pos(uint64_t b, const Geom& g)
{
    const uint32_t per = g.bxn * g.byn;
    const uint32_t bb = (uint32_t)b;
    BlockPos p;
    p.z = g.div_plane.div(bb);
    const uint32_t r = bb - p.z * per;
    p.y = g.div_bx.div(r);
    p.x = r - p.y * g.bxn;
    return p;
}

// Walks a warp's consecutive 2D/3D blocks without per-block divisions: one
// block_pos() for the first block, then x/y/z carries.  Per-lane element offsets
// inside a block are fixed for an array.
template <int DIM>
struct BlockWalk {
    uint32_t x, y, z;            // block coordinates of the current block
    uint32_t cx, ry0, ry1, rz0, rz1;
    uint64_t o0, o1;             // element offsets of this lane's two elements

    __device__ __forceinline__ BlockWalk(uint64_t b0, const Geom& g, int lane)
    {
        const BlockPos p = block_pos(b0 < g.nblocks ? b0 : 0, g);
        x = p.x; y = p.y; z = p.z;
        if constexpr (DIM == 2) {
            cx = lane & 7; ry0 = lane >> 3; ry1 = ry0 + 4; rz0 = rz1 = 0;
            o0 = (uint64_t)ry0 * g.dx + cx;
            o1 = (uint64_t)ry1 * g.dx + cx;
        } else {
            cx = lane & 3; ry0 = ry1 = (lane >> 2) & 3; rz0 = lane >> 4; rz1 = rz0 + 2;
            o0 = ((uint64_t)rz0 * g.dy + ry0) * g.dx + cx;
            o1 = ((uint64_t)rz1 * g.dy + ry0) * g.dx + cx;
        }
    }
    // Flat index of this lane's half-0 element and validity of both halves.
    __device__ __forceinline__ uint64_t elems(const Geom& g, bool bok, bool& ok0, bool& ok1) const
    {
        constexpr uint32_t B = DIM == 2 ? 8 : 4;
        const uint32_t xb = x * B, yb = y * B, zb = DIM == 2 ? z : z * 4;
        const bool inx = bok && xb + cx < g.dx;
        if constexpr (DIM == 2) {
            ok0 = inx && yb + ry0 < g.dy;
            ok1 = inx && yb + ry1 < g.dy;
        } else {
            const bool iny = inx && yb + ry0 < g.dy;
            ok0 = iny && zb + rz0 < g.dz;
            ok1 = iny && zb + rz1 < g.dz;
        }
        return ((uint64_t)zb * g.dy + yb) * g.dx + xb;
    }
    __device__ __forceinline__ void advance(const Geom& g)
    {
        if (++x == g.bxn) {
            x = 0;
            if (++y == g.byn) { y = 0; ++z; }
        }
    }
};

// Predecessor of each element for the Lorenzo delta (src/cuSZp_kernels_2D_f32.cu:711-760,
// 3D_f32.cu:697-704): returns q(pred) for half 0 (p0) and half 1 (p1).
template <int DIM>
__device__ __forceinline__ void predecessors(int32_t q0, int32_t q1, int lane, int32_t& p0, int32_t& p1)
{
    if constexpr (DIM == 1) {
        int32_t u = __shfl_up_sync(FULL, q0, 1);
        p0 = lane ? u : 0;
        p1 = 0;
    } else {
        // Every element but the block's first has one predecessor inside its own half,
        // at a per-lane source lane: 2D: x-delta inside a row, column 0 against the
        // previous row's column 0; 3D: x-delta, row start against the previous row start,
        // plane start against the previous plane start.  Lane 0 has no predecessor in
        // half 0, and its half-1 predecessor is half 0's element at lane 24 (2D: row 3,
        // column 0) or lane 16 (3D: plane 1 start) -- so lane 0 reads that lane in the
        // half-0 shuffle and one shuffle per half covers the block.
        int src;
        if constexpr (DIM == 2) {
            src = (lane & 7) ? lane - 1 : (lane >= 8 ? lane - 8 : 24);
        } else {
            src = (lane & 3) ? lane - 1 : ((lane >> 2) & 3) ? lane - 4 : (lane ^ 16);
        }
        const int32_t r0 = __shfl_sync(FULL, q0, src);
        const int32_t r1 = __shfl_sync(FULL, q1, src);
        p0 = lane ? r0 : 0;
        p1 = lane ? r1 : r0;
    }
}

// Inverse of the Lorenzo delta: q from codes d (wrapping adds).
template <int DIM>
__device__ __forceinline__ void lorenzo_inverse(int32_t& d0, int32_t& d1, int lane)
{
    if constexpr (DIM == 1) {
#pragma unroll
        for (int s = 1; s < 32; s <<= 1) {
            int32_t t = __shfl_up_sync(FULL, d0, s);
            if (lane >= s) d0 = wadd(d0, t);
        }
    } else if constexpr (DIM == 2) {
        // q[r][c] = sum_{c'<=c} d[r][c'] + sum_{r'<r} d[r'][0]
        int32_t r0 = d0, r1 = d1;
#pragma unroll
        for (int s = 1; s < 8; s <<= 1) {
            int32_t t0 = __shfl_up_sync(FULL, r0, s), t1 = __shfl_up_sync(FULL, r1, s);
            if ((lane & 7) >= s) { r0 = wadd(r0, t0); r1 = wadd(r1, t1); }
        }
        const bool c0 = (lane & 7) == 0;
        int32_t v0 = c0 ? d0 : 0, v1 = c0 ? d1 : 0;
        int32_t i0 = v0, i1 = v1;
#pragma unroll
        for (int s = 8; s < 32; s <<= 1) {
            int32_t t0 = __shfl_up_sync(FULL, i0, s), t1 = __shfl_up_sync(FULL, i1, s);
            if (lane >= s) { i0 = wadd(i0, t0); i1 = wadd(i1, t1); }
        }
        const int32_t tot0 = __shfl_sync(FULL, i0, 24);
        const int32_t e0 = __shfl_sync(FULL, wsub(i0, v0), lane & 24);
        const int32_t e1 = __shfl_sync(FULL, wsub(i1, v1), lane & 24);
        d0 = wadd(r0, e0);
        d1 = wadd(wadd(r1, e1), tot0);
    } else {
        // q(z,y,x) = [E(z) + sum_{y'<=y} d(z,y',0) - d(z,y,0)] + sum_{x'<=x} d(z,y,x'),
        // E(z) = sum_{z'<z} d(z',0,0).
        int32_t x0 = d0, x1 = d1;
#pragma unroll
        for (int s = 1; s < 4; s <<= 1) {
            int32_t t0 = __shfl_up_sync(FULL, x0, s), t1 = __shfl_up_sync(FULL, x1, s);
            if ((lane & 3) >= s) { x0 = wadd(x0, t0); x1 = wadd(x1, t1); }
        }
        const bool rs = (lane & 3) == 0;
        int32_t v0 = rs ? d0 : 0, v1 = rs ? d1 : 0;
        int32_t y0 = v0, y1 = v1;
#pragma unroll
        for (int s = 4; s < 16; s <<= 1) {
            int32_t t0 = __shfl_up_sync(FULL, y0, s), t1 = __shfl_up_sync(FULL, y1, s);
            if ((lane & 15) >= s) { y0 = wadd(y0, t0); y1 = wadd(y1, t1); }
        }
        const int32_t zs0 = __shfl_sync(FULL, d0, 0);
        const int32_t zs1 = wadd(zs0, __shfl_sync(FULL, d0, 16));
        const int32_t zs2 = wadd(zs1, __shfl_sync(FULL, d1, 0));
        const int32_t E0 = lane >= 16 ? zs0 : 0;
        const int32_t E1 = lane >= 16 ? zs2 : zs1;
        const int32_t b0 = __shfl_sync(FULL, wsub(wadd(E0, y0), v0), lane & ~3);
        const int32_t b1 = __shfl_sync(FULL, wsub(wadd(E1, y1), v1), lane & ~3);
        d0 = wadd(x0, b0);
        d1 = wadd(x1, b1);
    }
}

// The same inverse with the lane-dependent parts precomputed per lane as 0/1
// multipliers: every conditional add of the prefix sums is one multiply-add (the FMA
// pipe) instead of a compare and a predicated add (the ALU pipe, which the decoders
// saturate).  Integer arithmetic wraps as in lorenzo_inverse.
template <int DIM>
struct LorenzoLane {
    uint32_t mx[DIM == 1 ? 5 : DIM == 2 ? 3 : 2];   // x-direction prefix steps (1D: all five)
    uint32_t my[2];                                 // 2D: rows, 3D: row starts
    uint32_t first;                                 // 2D: column 0, 3D: row start (x == 0)
    uint32_t hi;                                    // 3D: second half of the block (z >= 2)
    __device__ __forceinline__ explicit LorenzoLane(int lane)
    {
        if constexpr (DIM == 1) {
#pragma unroll
            for (int i = 0; i < 5; i++) mx[i] = lane >= (1 << i) ? 1u : 0u;
            my[0] = my[1] = first = hi = 0;
        } else if constexpr (DIM == 2) {
#pragma unroll
            for (int i = 0; i < 3; i++) mx[i] = (lane & 7) >= (1 << i) ? 1u : 0u;
            my[0] = lane >= 8 ? 1u : 0u;
            my[1] = lane >= 16 ? 1u : 0u;
            first = (lane & 7) == 0 ? 1u : 0u;
            hi = 0;
        } else {
            mx[0] = (lane & 3) >= 1 ? 1u : 0u;
            mx[1] = (lane & 3) >= 2 ? 1u : 0u;
            my[0] = (lane & 15) >= 4 ? 1u : 0u;
            my[1] = (lane & 15) >= 8 ? 1u : 0u;
            first = (lane & 3) == 0 ? 1u : 0u;
            hi = lane >= 16 ? 1u : 0u;
        }
    }
};

// d + t * m with wrapping 32-bit arithmetic (m is 0 or 1).
__device__ __forceinline__ int32_t madd(int32_t d, int32_t t, uint32_t m)
{
    return (int32_t)((uint32_t)d + (uint32_t)t * m);
}

template <int DIM>
__device__ __forceinline__ void lorenzo_inverse(int32_t& d0, int32_t& d1, int lane, const LorenzoLane<DIM>& L)
{
    if constexpr (DIM == 1) {
#pragma unroll
        for (int i = 0; i < 5; i++) d0 = madd(d0, __shfl_up_sync(FULL, d0, 1 << i), L.mx[i]);
    } else if constexpr (DIM == 2) {
        int32_t r0 = d0, r1 = d1;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const int32_t t0 = __shfl_up_sync(FULL, r0, 1 << i), t1 = __shfl_up_sync(FULL, r1, 1 << i);
            r0 = madd(r0, t0, L.mx[i]);
            r1 = madd(r1, t1, L.mx[i]);
        }
        const int32_t v0 = (int32_t)((uint32_t)d0 * L.first), v1 = (int32_t)((uint32_t)d1 * L.first);
        int32_t i0 = v0, i1 = v1;
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const int32_t t0 = __shfl_up_sync(FULL, i0, 8 << i), t1 = __shfl_up_sync(FULL, i1, 8 << i);
            i0 = madd(i0, t0, L.my[i]);
            i1 = madd(i1, t1, L.my[i]);
        }
        const int32_t tot0 = __shfl_sync(FULL, i0, 24);
        const int32_t e0 = __shfl_sync(FULL, wsub(i0, v0), lane & 24);
        const int32_t e1 = __shfl_sync(FULL, wsub(i1, v1), lane & 24);
        d0 = wadd(r0, e0);
        d1 = wadd(wadd(r1, e1), tot0);
    } else {
        int32_t x0 = d0, x1 = d1;
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const int32_t t0 = __shfl_up_sync(FULL, x0, 1 << i), t1 = __shfl_up_sync(FULL, x1, 1 << i);
            x0 = madd(x0, t0, L.mx[i]);
            x1 = madd(x1, t1, L.mx[i]);
        }
        const int32_t v0 = (int32_t)((uint32_t)d0 * L.first), v1 = (int32_t)((uint32_t)d1 * L.first);
        int32_t y0 = v0, y1 = v1;
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const int32_t t0 = __shfl_up_sync(FULL, y0, 4 << i), t1 = __shfl_up_sync(FULL, y1, 4 << i);
            y0 = madd(y0, t0, L.my[i]);
            y1 = madd(y1, t1, L.my[i]);
        }
        const int32_t zs0 = __shfl_sync(FULL, d0, 0);
        const int32_t zs1 = wadd(zs0, __shfl_sync(FULL, d0, 16));
        const int32_t zs2 = wadd(zs1, __shfl_sync(FULL, d1, 0));
        const int32_t E0 = (int32_t)((uint32_t)zs0 * L.hi);
        const int32_t E1 = madd(zs1, wsub(zs2, zs1), L.hi);
        const int32_t b0 = __shfl_sync(FULL, wsub(wadd(E0, y0), v0), lane & ~3);
        const int32_t b1 = __shfl_sync(FULL, wsub(wadd(E1, y1), v1), lane & ~3);
        d0 = wadd(x0, b0);
        d1 = wadd(x1, b1);
    }
}

// --------------------------------------------------------------- value range

// Running NaN-skipping extrema (fmax / fmin) of in[lo, hi) over the threads t = first,
// first + stride, ...: scalar elements up to the first 16-byte boundary, then 16-byte
// vector loads, four in flight per thread, then the scalar tail.  Every element is read
// once, by streaming loads.
template <typename T>
__device__ __forceinline__ void range_accumulate(const T* __restrict__ in, uint64_t lo, uint64_t hi, uint64_t first,
                                                 uint64_t stride, T& mx, T& mn)
{
    using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
    constexpr uint64_t PER = 16 / sizeof(T);
    if (lo >= hi) return;
    const uint64_t skew = ((16u - ((uintptr_t)(in + lo) & 15u)) & 15u) / sizeof(T);
    const uint64_t head = min(hi - lo, skew);
    for (uint64_t i = lo + first; i < lo + head; i += stride) {
        const T v = __ldcs(in + i);
        mx = fmax(mx, v);
        mn = fmin(mn, v);
    }
    const V* body = reinterpret_cast<const V*>(in + lo + head);
    const uint64_t nv = (hi - lo - head) / PER;
    auto take = [&](const V& v) {
        if constexpr (sizeof(T) == 4) {
            mx = fmax(fmax(mx, v.x), fmax(v.y, fmax(v.z, v.w)));
            mn = fmin(fmin(mn, v.x), fmin(v.y, fmin(v.z, v.w)));
        } else {
            mx = fmax(mx, fmax(v.x, v.y));
            mn = fmin(mn, fmin(v.x, v.y));
        }
    };
    uint64_t i = first;
    for (; i + 3 * stride < nv; i += 4 * stride) {
        const V a = __ldcs(body + i), b = __ldcs(body + i + stride), c = __ldcs(body + i + 2 * stride),
                d = __ldcs(body + i + 3 * stride);
        take(a);
        take(b);
        take(c);
        take(d);
    }
    for (; i < nv; i += stride) take(__ldcs(body + i));
    for (uint64_t k = lo + head + nv * PER + first; k < hi; k += stride) {
        const T v = __ldcs(in + k);
        mx = fmax(mx, v);
        mn = fmin(mn, v);
    }
}

// --------------------------------------------------------------- compress phases

template <typename T, int DIM, typename Tl>
struct CompressWork {
    int32_t c0[Tl::BPW];
    int32_t c1[DIM == 1 ? 1 : Tl::BPW];
    uint32_t myrb;    // lane j < BPW: rate byte of the warp's block j
    uint32_t myoff;   // lane j < BPW: its payload offset inside the warp's range
    uint32_t wtot;
};

// A block's rate byte in two steps: the warp-wide reduction of its lanes' code
// magnitudes (a1: 2D/3D second half), then the rate arithmetic on the reduced values.
// Split so that a warp coding several blocks can leave the second step to lane j for
// block j, once for all its blocks.  1D reduces the magnitudes as signed ints
// (|INT_MIN| drops out, as in the reference).
// block_max returns the maximum magnitude -- outlier mode: without element 0, whose
// magnitude goes to `o`.
template <int DIM, int MODE>
__device__ __forceinline__ uint32_t block_max(uint32_t a0, uint32_t a1, int lane, uint32_t& o)
{
    if constexpr (MODE == MODE_OUTLIER) {
        o = __shfl_sync(FULL, a0, 0);
        if constexpr (DIM == 1) return (uint32_t)max(__reduce_max_sync(FULL, lane ? (int)a0 : 0), 0);
        else return __reduce_max_sync(FULL, lane ? max(a0, a1) : a1);
    } else {
        o = 0;
        if constexpr (DIM == 1) return (uint32_t)max(__reduce_max_sync(FULL, (int)a0), 0);
        else return __reduce_max_sync(FULL, max(a0, a1));
    }
}
template <int DIM, int MODE>
__device__ __forceinline__ uint32_t rate_byte(uint32_t m2, uint32_t o)
{
    constexpr int W = DIM == 1 ? 4 : 8;
    if constexpr (MODE == MODE_OUTLIER) {
        // m2: maximum without element 0; m: with it
        const uint32_t m = DIM == 1 ? (uint32_t)max((int)m2, (int)o) : max(m2, o);
        const int fr1 = bitlen(m);
        const int fr2 = bitlen(m2);
        const int ob = (bitlen(o) + 7) / 8;
        const int cost1 = fr1 ? W + fr1 * W : 0;
        const int cost2 = fr2 ? W + fr2 * W + ob : W + ob;
        return cost1 <= cost2 ? (uint32_t)fr1 : (uint32_t)((fr2 | 0x80 | ((ob - 1) << 5)) & 0xff);
    } else {
        return (uint32_t)bitlen(m2);
    }
}
template <int DIM, int MODE>
__device__ __forceinline__ uint32_t block_rate(uint32_t a0, uint32_t a1, int lane)
{
    uint32_t o;
    const uint32_t m = block_max<DIM, MODE>(a0, a1, lane, o);
    return rate_byte<DIM, MODE>(m, o);
}

// Plane-word stores.  Blocks of rate <= 15 (the common case) carry each element's
// sign in bit 15 of its 16-bit magnitude slot, so one 32x32 transpose yields the
// planes and, as plane 15, the sign map already in stream byte order; the lane
// holding plane 15 stores it as the sign word.  Wider blocks transpose the
// magnitudes and take the sign maps from ballots.

// Payload of two 1D blocks A and B (rates rA, rB; codes cA, cB of this lane) at pA / pB.
template <int MODE>
__device__ __forceinline__ void pack_pair_1d(uint32_t rA, uint32_t rB, int32_t cA, int32_t cB, saddr_t pA,
                                             saddr_t pB, int lane, const XposeLane& xl)
{
    uint32_t nA = rA, nB = rB, obA = 0, obB = 0;
    if constexpr (MODE == MODE_OUTLIER) {
        nA = rA & 0x1f; nB = rB & 0x1f;
        if (rA & 0x80) obA = ((rA & 0x60) >> 5) + 1;
        if (rB & 0x80) obB = ((rB & 0x60) >> 5) + 1;
    }
    uint32_t aA = uabs(cA), aB = uabs(cB);
    if constexpr (MODE == MODE_OUTLIER) {
        // element 0's magnitude, little-endian, one byte per lane (lanes 0-3: A, 4-7: B)
        const uint32_t oA = __shfl_sync(FULL, aA, 0), oB = __shfl_sync(FULL, aB, 0);
        const uint32_t i = lane & 3;
        if (lane < 4 && i < obA) sts_u8(pA + i, oA >> (8 * i));
        if (lane >= 4 && lane < 8 && i < obB) sts_u8(pB + i, oB >> (8 * i));
        if (lane == 0) {
            if (obA) aA = 0;
            if (obB) aB = 0;
        }
        pA += obA; pB += obB;
    }
    const bool hasA = payload_size<1, MODE>(rA) != 0, hasB = payload_size<1, MODE>(rB) != 0;
    if (nA <= 15 && nB <= 15) {
        // lane l holds plane (l ^ 7) & 15 of block A (l < 16) or B (l >= 16); plane 15 = signs
        // (masks: a |INT_MIN| code, which the 1D rate ignores, must not reach the sign bits)
        const uint32_t x = (aA & 0x7fffu) | ((aB << 16) & 0x7fff0000u) | (((uint32_t)cA >> 16) & 0x8000u) |
                           ((uint32_t)cB & 0x80000000u);
        const uint32_t y = warp_transpose32(x, xl);
        const uint32_t p = (lane ^ 7) & 15;
        const bool b = lane >= 16;
        const uint32_t n = b ? nB : nA;
        const saddr_t q = b ? pB : pA;
        if (p == 15) {
            if (b ? hasB : hasA) put32s<MODE>(q, y);
        } else if (p < n) {
            put32s<MODE>(q + 4 + 4 * p, y);
        }
    } else {
        const uint32_t sA = to_stream_word(__ballot_sync(FULL, cA < 0));
        const uint32_t sB = to_stream_word(__ballot_sync(FULL, cB < 0));
        if (lane == 0 && hasA) put32s<MODE>(pA, sA);
        if (lane == 16 && hasB) put32s<MODE>(pB, sB);
        uint32_t yA = aA, yB = aB;
        warp_transpose32x2(yA, yB, xl);
        const int p = lane ^ 7;
        if ((uint32_t)p < nA) put32s<MODE>(pA + 4 + 4 * p, yA);
        if ((uint32_t)p < nB) put32s<MODE>(pB + 4 + 4 * p, yB);
    }
}

// Payload of one 2D/3D block (rate r != 0; codes c0, c1 of this lane's two elements) at p.
// HEAD: outlier mode, the caller has written element 0's bytes, zeroed its magnitude
// (sign kept) and passes p past them.
template <int MODE, bool HEAD = false>
__device__ __forceinline__ void pack_block_nd(uint32_t r, int32_t c0, int32_t c1, saddr_t p, int lane,
                                              const XposeLane& xl)
{
    uint32_t n = r, ob = 0;
    if constexpr (MODE == MODE_OUTLIER) {
        n = r & 0x1f;
        if (r & 0x80) ob = ((r & 0x60) >> 5) + 1;
    }
    uint32_t a0 = uabs(c0);
    const uint32_t a1 = uabs(c1);
    if constexpr (MODE == MODE_OUTLIER && !HEAD) {
        // element 0's magnitude, little-endian, one byte per lane
        const uint32_t o = __shfl_sync(FULL, a0, 0);
        if ((uint32_t)lane < ob) sts_u8(p + lane, o >> (8 * lane));
        if (lane == 0 && ob) a0 = 0;
        p += ob;
    }
    if (n <= 15) {
        // lane l holds plane (l ^ 7) & 15 of half l >> 4; plane 15 = the half's signs
        const uint32_t x = (a0 & 0x7fffu) | ((a1 << 16) & 0x7fff0000u) | (((uint32_t)c0 >> 16) & 0x8000u) |
                           ((uint32_t)c1 & 0x80000000u);
        const uint32_t y = warp_transpose32(x, xl);
        const uint32_t pl = (lane ^ 7) & 15;
        const uint32_t h4 = (uint32_t)(lane >> 4) * 4;
        if (pl == 15) put32s<MODE>(p + h4, y);
        else if (pl < n) put32s<MODE>(p + 8 + 8 * pl + h4, y);
    } else {
        const uint32_t s0 = to_stream_word(__ballot_sync(FULL, c0 < 0));
        const uint32_t s1 = to_stream_word(__ballot_sync(FULL, c1 < 0));
        if (lane < 2) put32s<MODE>(p + 4 * lane, lane ? s1 : s0);
        uint32_t ylo = a0, yhi = a1;
        warp_transpose32x2(ylo, yhi, xl);
        const int pl = lane ^ 7;
        if ((uint32_t)pl < n) {
            put32s<MODE>(p + 8 + 8 * pl, ylo);
            put32s<MODE>(p + 12 + 8 * pl, yhi);
        }
    }
}

// The transpose input word of two 16-bit element slots: magnitudes in bits 0-14 (a) and
// 16-30 (b), signs in bits 15 and 31.  A magnitude with bits above 14 (a 1D |INT_MIN|
// code, which the 1D rate ignores) must not reach the sign bits, hence the masks.
__device__ __forceinline__ uint32_t slot_pair(int32_t a, int32_t b)
{
    return (uabs(a) & 0x7fffu) | ((uabs(b) << 16) & 0x7fff0000u) | (((uint32_t)a >> 16) & 0x8000u) |
           ((uint32_t)b & 0x80000000u);
}

// Payloads of four 1D blocks of rate <= 15: the pairs (A, B) and (C, D) take one
// transpose each, interleaved.  After the transposes lane l holds plane pl = (l ^ 7) & 15
// of block A / C (l < 16) or B / D (l >= 16), plane 15 being the block's sign word; the
// lane stores it at its block's sign-word offset p1 / p2 plus `o` (0 for the sign word,
// 4 + 4 pl for a plane) when that bit of the block's plane mask k1 / k2 is set.  In
// outlier mode element 0's magnitude must already be cleared (sign kept) in blocks that
// store element 0 ahead of their planes.
template <int MODE>
__device__ __forceinline__ void pack_quad_1d_narrow(int32_t cA, int32_t cB, int32_t cC, int32_t cD, uint32_t k1,
                                                    saddr_t p1, uint32_t k2, saddr_t p2, uint32_t pl, uint32_t o,
                                                    const XposeLane& xl)
{
    uint32_t x1 = slot_pair(cA, cB), x2 = slot_pair(cC, cD);
    warp_transpose32x2(x1, x2, xl);
    put32s_if<MODE, true>((k1 >> pl) & 1u, p1 + o, x1);
    put32s_if<MODE, true>((k2 >> pl) & 1u, p2 + o, x2);
}

// Payloads of two 2D/3D blocks of rate <= 15, sign words at pa / pb, transposes
// interleaved.  Lane l holds plane (l ^ 7) & 15 of half l >> 4 after the transpose
// (plane 15 = the half's signs) and stores it when that bit of the block's plane mask
// is set (ka / kb: bits 0 .. n-1 and 15 for a block with a payload, 0 without).  In
// outlier mode element 0's magnitude must already be cleared (sign kept) where the
// block stores element 0 ahead of its planes.  BYTEWISE: as for put32s_if.
template <int MODE, bool BYTEWISE = false>
__device__ __forceinline__ void pack_pair_narrow(uint32_t ka, uint32_t kb, int32_t c0a, int32_t c1a, int32_t c0b,
                                                 int32_t c1b, saddr_t pa, saddr_t pb, int lane, const XposeLane& xl)
{
    uint32_t xa = slot_pair(c0a, c1a), xb = slot_pair(c0b, c1b);
    warp_transpose32x2(xa, xb, xl);
    const uint32_t pl = (lane ^ 7) & 15;
    const uint32_t h4 = (uint32_t)(lane >> 4) * 4;
    const uint32_t o = pl == 15 ? h4 : 8 + 8 * pl + h4;
    put32s_if<MODE, BYTEWISE>((ka >> pl) & 1u, pa + o, xa);
    put32s_if<MODE, BYTEWISE>((kb >> pl) & 1u, pb + o, xb);
}

// pack_pair_narrow for four blocks (masks k, codes c0 / c1, sign-word offsets p): four
// transposes interleaved stage by stage, twice the independent work per dependent step
// of the butterfly (measured 1.3 % faster on the 512^3 f32 3D compress, 1 % slower in 2D).
template <int MODE, bool BYTEWISE = false>
__device__ __forceinline__ void pack_quad_narrow(const uint32_t* k, const int32_t* c0, const int32_t* c1,
                                                 const saddr_t* p, int lane, const XposeLane& xl)
{
    uint32_t x[4];
#pragma unroll
    for (int i = 0; i < 4; i++) x[i] = slot_pair(c0[i], c1[i]);
#pragma unroll
    for (int st = 0; st < 5; st++) {
        uint32_t y[4];
#pragma unroll
        for (int i = 0; i < 4; i++) y[i] = __shfl_xor_sync(FULL, x[i], 16 >> st);
#pragma unroll
        for (int i = 0; i < 4; i++) x[i] = xl.stage(st, x[i], y[i]);
    }
    const uint32_t pl = (lane ^ 7) & 15;
    const uint32_t h4 = (uint32_t)(lane >> 4) * 4;
    const uint32_t o = pl == 15 ? h4 : 8 + 8 * pl + h4;
#pragma unroll
    for (int i = 0; i < 4; i++) put32s_if<MODE, BYTEWISE>((k[i] >> pl) & 1u, p[i] + o, x[i]);
}

// Plane mask of a block for pack_pair_narrow (rate byte r, n <= 15 planes).
__device__ __forceinline__ uint32_t plane_mask(uint32_t r, uint32_t n) { return r ? ((1u << n) - 1u) | 0x8000u : 0u; }

// Payloads of two 2D/3D blocks a and b (rates ra, rb) at pa / pb; both blocks'
// transposes run interleaved when both rates are <= 15.  HEAD: as for pack_block_nd.
template <int MODE, bool HEAD = false>
__device__ __forceinline__ void pack_pair_nd(uint32_t ra, uint32_t rb, int32_t c0a, int32_t c1a, int32_t c0b,
                                             int32_t c1b, saddr_t pa, saddr_t pb, int lane, const XposeLane& xl)
{
    uint32_t na = ra, nb = rb, oba = 0, obb = 0;
    if constexpr (MODE == MODE_OUTLIER) {
        na = ra & 0x1f; nb = rb & 0x1f;
        if (ra & 0x80) oba = ((ra & 0x60) >> 5) + 1;
        if (rb & 0x80) obb = ((rb & 0x60) >> 5) + 1;
    }
    if (na > 15 || nb > 15) {
        if (ra) pack_block_nd<MODE, HEAD>(ra, c0a, c1a, pa, lane, xl);
        if (rb) pack_block_nd<MODE, HEAD>(rb, c0b, c1b, pb, lane, xl);
        return;
    }
    if constexpr (MODE == MODE_OUTLIER && !HEAD) {
        // element 0's magnitude, little-endian, one byte per lane (lanes 0-3: a, 4-7: b)
        const uint32_t oa = __shfl_sync(FULL, uabs(c0a), 0), ob = __shfl_sync(FULL, uabs(c0b), 0);
        const uint32_t i = lane & 3;
        if (lane < 4 && i < oba) sts_u8(pa + i, oa >> (8 * i));
        if (lane >= 4 && lane < 8 && i < obb) sts_u8(pb + i, ob >> (8 * i));
        if (lane == 0) {   // magnitude 0 in the planes, sign kept
            if (oba) c0a = (int32_t)((uint32_t)c0a & 0x80000000u);
            if (obb) c0b = (int32_t)((uint32_t)c0b & 0x80000000u);
        }
        pa += oba; pb += obb;
    }
    pack_pair_narrow<MODE>(plane_mask(ra, na), plane_mask(rb, nb), c0a, c1a, c0b, c1b, pa, pb, lane, xl);
}

// Sign maps and bit-planes of the warp's blocks at their final offsets.
template <typename T, int DIM, int MODE, typename Tl>
__device__ __forceinline__ void compress_pack(const CompressWork<T, DIM, Tl>& K, uint8_t* __restrict__ pbase)
{
    constexpr int BPW = Tl::BPW;
    const int lane = threadIdx.x & 31;
    const XposeLane xl(lane ^ 7);
    if constexpr (DIM == 1) {
#pragma unroll
        for (int j = 0; j < BPW; j += 2) {
            const uint32_t rA = __shfl_sync(FULL, K.myrb, j), rB = __shfl_sync(FULL, K.myrb, j + 1);
            if ((rA | rB) == 0) continue;
            pack_pair_1d<MODE>(rA, rB, K.c0[j], K.c0[j + 1], saddr(pbase) + __shfl_sync(FULL, K.myoff, j),
                               saddr(pbase) + __shfl_sync(FULL, K.myoff, j + 1), lane, xl);
        }
    } else {
#pragma unroll
        for (int j = 0; j < BPW; j++) {
            const uint32_t r = __shfl_sync(FULL, K.myrb, j);
            if (r == 0) continue;
            pack_block_nd<MODE>(r, K.c0[j], K.c1[DIM == 1 ? 0 : j], saddr(pbase) + __shfl_sync(FULL, K.myoff, j), lane,
                                xl);
        }
    }
}

// Shared state of one CTA's tile loop.
template <int WARPS>
struct TileShared {
    uint32_t warp[WARPS];
    uint64_t base;
    int64_t ticket[2];
    uint32_t dwarp[2][WARPS];         // decompress: warp offsets of the two tiles in flight
    unsigned long long dagg[2];       // decompress: their aggregates
    LookbackShared lb;
};

// --------------------------------------------------------------- compress pipeline
//
// Per CTA, tiles flow through three overlapped stages:
//   prefetch(t+1): cp.async copies of the next tile's elements into shared memory
//                  (no registers held while they are in flight);
//   encode(t):     quantize, predict, rate bytes, bit-plane pack into a shared staging
//                  buffer at tile-local offsets; post the tile aggregate;
//   flush(t-1):    resolve the previous tile's offset (its aggregate was posted one
//                  tile earlier, so its predecessors are normally done) and write its
//                  staged payload with coalesced 16-byte stores.
// No stage waits on a predecessor while DRAM traffic for the CTA could be flowing.

template <typename T, int DIM, typename Tl>
struct CompressSmem {
    static constexpr int HALVES = DIM == 1 ? 1 : 2;
    static constexpr int IN_ELEMS = Tl::WARPS * Tl::BPW * HALVES * 32;          // one tile of input
    static constexpr int MAXBLK = DIM == 1 ? 4 + 4 + 4 * 31 + 4 : 8 + 4 + 8 * 32;  // worst block payload
    static constexpr int SB_BYTES = (Tl::TB * MAXBLK + 16 + 15) / 16 * 16;     // staged payload + slack
    static constexpr size_t bytes() { return 2 * (size_t)IN_ELEMS * sizeof(T) + 2 * (size_t)SB_BYTES; }
    T* in[2];
    uint8_t* sb[2];
    __device__ __forceinline__ explicit CompressSmem(unsigned char* base)
    {
        in[0] = reinterpret_cast<T*>(base);
        in[1] = in[0] + IN_ELEMS;
        sb[0] = reinterpret_cast<uint8_t*>(in[1] + IN_ELEMS);
        sb[1] = sb[0] + SB_BYTES;
    }
    // this lane's element (block j, half h) inside a tile buffer
    __device__ __forceinline__ static int slot(int warp, int j, int h, int lane)
    {
        return ((warp * Tl::BPW + j) * HALVES + h) * 32 + lane;
    }
};

template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem_dst, const T* gsrc, bool ok)
{
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem_dst);
    const int n = ok ? (int)sizeof(T) : 0;   // 0: zero-fill, nothing read
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(s), "l"(gsrc), "n"(sizeof(T)), "r"(n)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Issue the asynchronous copies of this lane's elements of `tile`.  Returns the 2D/3D
// validity bitmasks (bit j: element of block j inside the array) through ok0/ok1.
template <typename T, int DIM, typename Tl>
__device__ __forceinline__ void compress_prefetch(T* __restrict__ buf, const T* __restrict__ in, const Geom& g,
                                                  int64_t tile, uint32_t& ok0m, uint32_t& ok1m)
{
    using SM = CompressSmem<T, DIM, Tl>;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t b0 = (uint64_t)tile * Tl::TB + (uint64_t)warp * Tl::BPW;
    if constexpr (DIM == 1) {
#pragma unroll
        for (int j = 0; j < Tl::BPW; j++) {
            const uint64_t i = (b0 + j) * 32 + lane;
            const bool ok = i < g.nbEle;
            cp_async_elem(buf + SM::slot(warp, j, 0, lane), ok ? in + i : in, ok);
        }
        ok0m = ok1m = 0;
    } else {
        BlockWalk<DIM> bw(b0, g, lane);
        uint32_t m0 = 0, m1 = 0;
#pragma unroll
        for (int j = 0; j < Tl::BPW; j++) {
            bool ok0, ok1;
            const uint64_t base = bw.elems(g, b0 + j < g.nblocks, ok0, ok1);
            cp_async_elem(buf + SM::slot(warp, j, 0, lane), ok0 ? in + base + bw.o0 : in, ok0);
            cp_async_elem(buf + SM::slot(warp, j, 1, lane), ok1 ? in + base + bw.o1 : in, ok1);
            m0 |= (uint32_t)ok0 << j;
            m1 |= (uint32_t)ok1 << j;
            bw.advance(g);
        }
        ok0m = m0;
        ok1m = m1;
    }
}

// Quantize + predict from the prefetched tile; rate bytes to the stream; per-block
// payload offsets inside the warp's range in lane j (myrb / myoff).
template <typename T, int DIM, int MODE, typename Tl>
__device__ __forceinline__ void compress_codes(const T* __restrict__ buf, uint32_t ok0m, uint32_t ok1m,
                                               CompressWork<T, DIM, Tl>& K, T recip, const Geom& g, int64_t tile,
                                               uint8_t* __restrict__ cmp)
{
    using SM = CompressSmem<T, DIM, Tl>;
    constexpr int BPW = Tl::BPW;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t b0 = (uint64_t)tile * Tl::TB + (uint64_t)warp * BPW;
    if constexpr (DIM == 1) {
#pragma unroll
        for (int j = 0; j < BPW; j++) {
            const uint64_t i = (b0 + j) * 32 + lane;
            const int32_t q = quantize(buf[SM::slot(warp, j, 0, lane)], recip);
            int32_t p0 = 0, p1;
            if constexpr (MODE != MODE_FIXED) predecessors<1>(q, 0, lane, p0, p1);
            K.c0[j] = i < g.nbEle ? wsub(q, p0) : 0;
        }
        K.c1[0] = 0;
    } else {
#pragma unroll
        for (int j = 0; j < BPW; j++) {
            const bool ok0 = (ok0m >> j) & 1u, ok1 = (ok1m >> j) & 1u;
            const int32_t q0 = quantize(buf[SM::slot(warp, j, 0, lane)], recip);
            const int32_t q1 = quantize(buf[SM::slot(warp, j, 1, lane)], recip);
            int32_t p0 = 0, p1 = 0;
            if constexpr (MODE != MODE_FIXED) predecessors<DIM>(q0, q1, lane, p0, p1);
            K.c0[j] = ok0 ? wsub(q0, p0) : 0;
            K.c1[j] = ok1 ? wsub(q1, p1) : 0;
        }
    }
    uint32_t wtot = 0, myrb = 0, myoff = 0;
#pragma unroll
    for (int j = 0; j < BPW; j++) {
        const uint32_t a0 = uabs(K.c0[j]);
        const uint32_t a1 = DIM == 1 ? 0u : uabs(K.c1[DIM == 1 ? 0 : j]);
        const uint32_t r = block_rate<DIM, MODE>(a0, a1, lane);
        if (lane == j) { myrb = r; myoff = wtot; }
        wtot += payload_size<DIM, MODE>(r);
    }
    K.wtot = wtot;
    K.myrb = myrb;
    K.myoff = myoff;
    if (lane < BPW && b0 + lane < g.rate_bytes) cmp[b0 + lane] = (uint8_t)myrb;
}

// Writes `size` staged bytes to global `dst` (any alignment) with 16-byte stores for
// every full aligned unit and byte stores for the two ragged ends.  All threads call.
__device__ __forceinline__ void copy_out(const uint8_t* __restrict__ sb, uint32_t size, uint8_t* __restrict__ dst)
{
    if (size == 0) return;
    const uint32_t d = (uint32_t)((uintptr_t)dst & 15);
    uint8_t* first = dst - d;
    const uint32_t nunits = (d + size + 15) / 16;
    for (uint32_t u = threadIdx.x; u < nunits; u += blockDim.x) {
        const int32_t so = (int32_t)(16 * u) - (int32_t)d;   // staged offset of this unit
        uint8_t* gp = first + 16 * u;
        if (so >= 0 && so + 16 <= (int32_t)size) {
            const uint32_t* w = reinterpret_cast<const uint32_t*>(sb + (so & ~3));
            const uint32_t sh = (uint32_t)(so & 3) * 8;
            uint4 v;
            if (sh == 0) {
                v = make_uint4(w[0], w[1], w[2], w[3]);
            } else {
                const uint32_t w4 = w[4];
                v = make_uint4(__funnelshift_r(w[0], w[1], sh), __funnelshift_r(w[1], w[2], sh),
                               __funnelshift_r(w[2], w[3], sh), __funnelshift_r(w[3], w4, sh));
            }
            __stcs(reinterpret_cast<uint4*>(gp), v);
        } else {
#pragma unroll 1
            for (int b = 0; b < 16; b++) {
                const int32_t o = so + b;
                if (o >= 0 && o < (int32_t)size) gp[b] = sb[o];
            }
        }
    }
}

// Tile context: where a tile's data and stream live (constant for a single array).
struct TileCtx {
    const void* in;
    uint8_t* cmp;
    Geom g;
    unsigned long long* status;     // this array's tile status words
    unsigned long long* total_out;  // this array's stream length
    int64_t local;                  // tile index inside the array
    int mode;
    float eb;                       // batch: bound the recip is derived from
};

template <int WARPS>
struct PipeShared {
    uint32_t wt[WARPS];             // warp payload totals of the tile being encoded
    unsigned long long base;        // resolved offset of the tile being flushed
    int64_t ticket[2];
    uint32_t item[2];
};

// Resolve the offset of a tile whose aggregate `agg` was posted earlier (warp 0;
// the caller's barrier publishes sp.base).
template <int WARPS>
__device__ __forceinline__ void resolve_prev(const TileCtx& c, unsigned long long agg, uint32_t* err,
                                             PipeShared<WARPS>& sp)
{
    if ((threadIdx.x >> 5) == 0) {
        const uint64_t excl = c.local > 0 ? warp_lookback(c.status, c.local, err) : 0;
        if (threadIdx.x == 0) {
            if (c.local > 0) st_post(c.status + c.local, ST_INC | ((excl + agg) & ST_VAL));
            if ((uint64_t)c.local == c.g.ntiles - 1) *c.total_out = c.g.rate_bytes + excl + agg;
            sp.base = excl;
        }
    }
}

// Encode one tile (data already prefetched into `buf`): codes, aggregate, staged pack.
// Returns the tile aggregate (same in every thread).  Contains one barrier.
template <typename T, int DIM, int MODE, typename Tl>
__device__ __forceinline__ unsigned long long encode_tile(const T* __restrict__ buf, uint32_t ok0m, uint32_t ok1m,
                                                          const TileCtx& c, T recip, uint8_t* __restrict__ sb,
                                                          PipeShared<Tl::WARPS>& sp)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    CompressWork<T, DIM, Tl> K;
    compress_codes<T, DIM, MODE, Tl>(buf, ok0m, ok1m, K, recip, c.g, c.local, c.cmp);
    if (lane == 0) sp.wt[warp] = K.wtot;
    __syncthreads();
    uint32_t woff = 0;
    unsigned long long agg = 0;
#pragma unroll
    for (int w = 0; w < Tl::WARPS; w++) {
        const uint32_t t = sp.wt[w];
        woff += w < warp ? t : 0u;
        agg += t;
    }
    if (threadIdx.x == 0) st_post(c.status + c.local, (c.local == 0 ? ST_INC : ST_AGG) | agg);
    compress_pack<T, DIM, MODE, Tl>(K, sb + woff);
    return agg;
}

// Writes a resolved tile's staged payload at its offset, unless it would end past the
// stream buffer's capacity (then nothing is written and ERR_CAPACITY is raised).
__device__ __forceinline__ void flush_tile(const uint8_t* __restrict__ sb, const TileCtx& c, unsigned long long agg,
                                           unsigned long long base, uint32_t* err)
{
    const uint64_t at = c.g.rate_bytes + base;
    if (at + agg <= c.g.cap) copy_out(sb, (uint32_t)agg, c.cmp + at);
    else if (threadIdx.x == 0) atomicOr(err, ERR_CAPACITY);
}

// The tile loop shared by the single-array, batched and allocation-free kernels.
// `Src` supplies tiles: take(sp, k) (thread 0: next ticket into slot k), ctx(sp, k, c)
// (tile context of slot k; false once tiles run out), encode(...) (encode_tile with
// the tile's mode and bound).
template <typename T, int DIM, typename Tl, typename Src>
__device__ __forceinline__ void compress_pipeline(Src& src, unsigned char* smem_raw, uint32_t* err)
{
    CompressSmem<T, DIM, Tl> sm(smem_raw);
    __shared__ PipeShared<Tl::WARPS> sp;
    if (threadIdx.x == 0) {
        src.take(sp, 0);
        src.take(sp, 1);
    }
    __syncthreads();
    TileCtx cur, nxt, prev;
    bool has_cur = src.ctx(sp, 0, cur);
    bool has_nxt = src.ctx(sp, 1, nxt);
    uint32_t ok0c = 0, ok1c = 0, ok0n = 0, ok1n = 0;
    if (has_cur) compress_prefetch<T, DIM, Tl>(sm.in[0], static_cast<const T*>(cur.in), cur.g, cur.local, ok0c, ok1c);
    cp_async_commit();
    __syncthreads();   // every thread has read slot 0 before the loop refills it
    bool has_prev = false;
    unsigned long long prev_agg = 0;
    int prev_buf = 0;
    for (int it = 0; has_cur; it++) {
        const int b = it & 1;
        if (has_nxt)
            compress_prefetch<T, DIM, Tl>(sm.in[b ^ 1], static_cast<const T*>(nxt.in), nxt.g, nxt.local, ok0n, ok1n);
        cp_async_commit();
        if (threadIdx.x == 0) src.take(sp, b);
        cp_async_wait_prev();    // this thread's copies of the current tile have landed
        const unsigned long long agg = src.encode(sm.in[b], ok0c, ok1c, cur, sm.sb[b], sp);
        if (has_prev) resolve_prev<Tl::WARPS>(prev, prev_agg, err, sp);
        __syncthreads();
        if (has_prev) flush_tile(sm.sb[prev_buf], prev, prev_agg, sp.base, err);
        prev = cur;
        prev_agg = agg;
        prev_buf = b;
        has_prev = true;
        cur = nxt;
        has_cur = has_nxt;
        ok0c = ok0n;
        ok1c = ok1n;
        has_nxt = src.ctx(sp, b, nxt);
    }
    cp_async_wait_all();
    if (has_prev) {
        resolve_prev<Tl::WARPS>(prev, prev_agg, err, sp);
        __syncthreads();
        flush_tile(sm.sb[prev_buf], prev, prev_agg, sp.base, err);
    }
}

// Tile source of one array.
template <typename T, int DIM, int MODE, typename Tl>
struct SingleSource {
    const T* in;
    uint8_t* cmp;
    Geom g;
    T recip;
    WsHeader* hdr;
    unsigned long long* status;
    unsigned long long* total_out;
    __device__ __forceinline__ void take(PipeShared<Tl::WARPS>& sp, int k)
    {
        sp.ticket[k] = (int64_t)atomicAdd(&hdr->ticket, 1u);
    }
    __device__ __forceinline__ bool ctx(const PipeShared<Tl::WARPS>& sp, int k, TileCtx& c) const
    {
        c.in = in;
        c.cmp = cmp;
        c.g = g;
        c.status = status;
        c.total_out = total_out;
        c.local = sp.ticket[k];
        c.mode = MODE;
        c.eb = 0.f;
        return (uint64_t)c.local < g.ntiles;
    }
    __device__ __forceinline__ unsigned long long encode(const T* buf, uint32_t ok0, uint32_t ok1, const TileCtx& c,
                                                         uint8_t* sb, PipeShared<Tl::WARPS>& sp) const
    {
        return encode_tile<T, DIM, MODE, Tl>(buf, ok0, ok1, c, recip, sb, sp);
    }
};

template <typename T, int DIM, typename Tl>
constexpr size_t compress_smem_bytes() { return CompressSmem<T, DIM, Tl>::bytes(); }

template <typename T, int DIM, int MODE, typename Tl = Tiling<DIM>>
__global__ void __launch_bounds__(Tl::THREADS, 2)
compress_kernel(const T* __restrict__ in, uint8_t* __restrict__ cmp, Geom g, T recip,
                WsHeader* __restrict__ hdr, unsigned long long* __restrict__ status)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SingleSource<T, DIM, MODE, Tl> src{in, cmp, g, recip, hdr, status, &hdr->total};
    compress_pipeline<T, DIM, Tl>(src, smem_raw, &hdr->err);
    finish_cta(hdr, status, g.ntiles, g.size_out);
}

// --------------------------------------------------------------- decompress phases
//
// Mirror pipeline: tile t's payload loads are issued, then tile t+1's rate bytes are
// scanned and looked back (overlapping those loads), then tile t is decoded and stored.

template <typename Tl>
struct DecompRates {
    uint32_t myrb;    // lane j < BPW: rate byte of block j of this warp
    uint32_t myoff;   // lane j < BPW: payload offset of block j inside the warp's range
    uint32_t wtot;
};

template <int DIM, int MODE, typename Tl>
__device__ __forceinline__ void decompress_rates(DecompRates<Tl>& R, const uint8_t* __restrict__ cmp, const Geom& g,
                                                 int64_t tile)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t b0 = (uint64_t)tile * Tl::TB + (uint64_t)warp * Tl::BPW;
    uint32_t myrb = 0;
    if (lane < Tl::BPW && b0 + lane < g.nblocks) myrb = __ldg(cmp + b0 + lane);
    const uint32_t sz = lane < Tl::BPW ? payload_size<DIM, MODE>(myrb) : 0u;
    uint32_t incl = sz;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += t;
    }
    R.myrb = myrb;
    R.myoff = incl - sz;
    R.wtot = __shfl_sync(FULL, incl, 31);
}

template <int DIM, typename Tl>
struct DecompPayload {
    uint32_t w0[Tl::BPW];
    uint32_t w1[Tl::BPW];
    uint32_t s0[Tl::BPW];
    uint32_t s1[DIM == 1 ? 1 : Tl::BPW];
    uint32_t m0[Tl::BPW];
};

// Issue the payload loads of the warp's blocks (plane words, sign words, outlier bytes).
template <int DIM, int MODE, typename Tl>
__device__ __forceinline__ void decompress_load(DecompPayload<DIM, Tl>& P, const DecompRates<Tl>& R,
                                                const uint8_t* __restrict__ pbase)
{
    constexpr int BPW = Tl::BPW;
    const int lane = threadIdx.x & 31;
    if constexpr (DIM == 1) {
#pragma unroll
        for (int k = 0; k < BPW / 2; k++) {
            const int j = 2 * k;
            const uint32_t rA = __shfl_sync(FULL, R.myrb, j), rB = __shfl_sync(FULL, R.myrb, j + 1);
            const uint32_t oA = __shfl_sync(FULL, R.myoff, j), oB = __shfl_sync(FULL, R.myoff, j + 1);
            uint32_t nA = rA, nB = rB, obA = 0, obB = 0;
            if constexpr (MODE == MODE_OUTLIER) {
                nA = rA & 0x1f; nB = rB & 0x1f;
                if (rA & 0x80) obA = ((rA & 0x60) >> 5) + 1;
                if (rB & 0x80) obB = ((rB & 0x60) >> 5) + 1;
            }
            const uint8_t* pA = pbase + oA;
            const uint8_t* pB = pbase + oB;
            P.m0[j] = 0; P.m0[j + 1] = 0;
            if constexpr (MODE == MODE_OUTLIER) {
                for (uint32_t i = 0; i < obA; i++) P.m0[j] |= (uint32_t)pA[i] << (8 * i);
                for (uint32_t i = 0; i < obB; i++) P.m0[j + 1] |= (uint32_t)pB[i] << (8 * i);
                pA += obA; pB += obB;
            }
            const bool hasA = payload_size<DIM, MODE>(rA) != 0, hasB = payload_size<DIM, MODE>(rB) != 0;
            P.s0[j] = hasA ? get32<MODE>(pA) : 0u;
            P.s0[j + 1] = hasB ? get32<MODE>(pB) : 0u;
            P.w0[k] = 0; P.w1[k] = 0;
            if (nA <= 16 && nB <= 16) {
                const int p = lane & 15;
                if (lane < 16) { if ((uint32_t)p < nA) P.w0[k] = get32<MODE>(pA + 4 + 4 * p); }
                else           { if ((uint32_t)p < nB) P.w0[k] = get32<MODE>(pB + 4 + 4 * p); }
            } else {
                if ((uint32_t)lane < nA) P.w0[k] = get32<MODE>(pA + 4 + 4 * lane);
                if ((uint32_t)lane < nB) P.w1[k] = get32<MODE>(pB + 4 + 4 * lane);
            }
        }
    } else {
#pragma unroll
        for (int j = 0; j < BPW; j++) {
            const uint32_t r = __shfl_sync(FULL, R.myrb, j);
            const uint32_t o = __shfl_sync(FULL, R.myoff, j);
            uint32_t n = r, ob = 0;
            if constexpr (MODE == MODE_OUTLIER) {
                n = r & 0x1f;
                if (r & 0x80) ob = ((r & 0x60) >> 5) + 1;
            }
            const uint8_t* p = pbase + o;
            P.m0[j] = 0;
            if constexpr (MODE == MODE_OUTLIER) {
                for (uint32_t i = 0; i < ob; i++) P.m0[j] |= (uint32_t)p[i] << (8 * i);
                p += ob;
            }
            const bool has = payload_size<DIM, MODE>(r) != 0;
            P.s0[j] = has ? get32<MODE>(p) : 0u;
            P.s1[j] = has ? get32<MODE>(p + 4) : 0u;
            P.w0[j] = 0; P.w1[j] = 0;
            if (n <= 16) {
                const int pl = lane & 15;
                if ((uint32_t)pl < n) P.w0[j] = get32<MODE>(p + 8 + 8 * pl + (lane >> 4) * 4);
            } else if ((uint32_t)lane < n) {
                P.w0[j] = get32<MODE>(p + 8 + 8 * lane);
                P.w1[j] = get32<MODE>(p + 12 + 8 * lane);
            }
        }
    }
}

// Inverse transpose, signs, inverse Lorenzo, dequantize, store.
template <typename T, int DIM, int MODE, typename Tl>
__device__ __forceinline__ void decompress_store(const DecompPayload<DIM, Tl>& P, const DecompRates<Tl>& R,
                                                 T* __restrict__ out, const Geom& g, T eb, int64_t tile)
{
    constexpr int BPW = Tl::BPW;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t b0 = (uint64_t)tile * Tl::TB + (uint64_t)warp * BPW;
    if constexpr (DIM == 1) {
#pragma unroll
        for (int k = 0; k < BPW / 2; k++) {
            const uint32_t rA = __shfl_sync(FULL, R.myrb, 2 * k), rB = __shfl_sync(FULL, R.myrb, 2 * k + 1);
            uint32_t nA = rA, nB = rB;
            if constexpr (MODE == MODE_OUTLIER) { nA = rA & 0x1f; nB = rB & 0x1f; }
            uint32_t magA = 0, magB = 0;
            if (nA <= 16 && nB <= 16) {
                if ((nA | nB) != 0) {
                    const uint32_t x = warp_transpose32(from_stream_word(P.w0[k]), lane);
                    magA = x & 0xffffu;
                    magB = x >> 16;
                }
            } else {
                magA = warp_transpose32(from_stream_word(P.w0[k]), lane);
                magB = warp_transpose32(from_stream_word(P.w1[k]), lane);
            }
            if constexpr (MODE == MODE_OUTLIER) {
                if (lane == 0) {
                    if (rA & 0x80) magA = P.m0[2 * k];
                    if (rB & 0x80) magB = P.m0[2 * k + 1];
                }
            }
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const uint32_t r = s ? rB : rA;
                const uint64_t i = (b0 + 2 * k + s) * 32 + lane;
                if (payload_size<DIM, MODE>(r) == 0) {
                    if (i < g.nbEle) st_stream(out + i, T(0));
                    continue;
                }
                const uint32_t mag = s ? magB : magA;
                const uint32_t sg = from_stream_word(P.s0[2 * k + s]);
                int32_t d = ((sg >> lane) & 1u) ? (int32_t)(0u - mag) : (int32_t)mag;
                int32_t dummy = 0;
                if constexpr (MODE != MODE_FIXED) lorenzo_inverse<1>(d, dummy, lane);
                if (i < g.nbEle) st_stream(out + i, dequant(d, eb));
            }
        }
    } else {
        BlockWalk<DIM> bw(b0, g, lane);
#pragma unroll
        for (int j = 0; j < BPW; j++) {
            bool ok0, ok1;
            const uint64_t base = bw.elems(g, b0 + j < g.nblocks, ok0, ok1);
            bw.advance(g);
            const uint64_t i0 = base + bw.o0, i1 = base + bw.o1;
            const uint32_t r = __shfl_sync(FULL, R.myrb, j);
            if (payload_size<DIM, MODE>(r) == 0) {
                if (ok0) st_stream(out + i0, T(0));
                if (ok1) st_stream(out + i1, T(0));
                continue;
            }
            uint32_t n = r;
            if constexpr (MODE == MODE_OUTLIER) n = r & 0x1f;
            uint32_t mag0, mag1;
            if (n <= 16) {
                const uint32_t x = warp_transpose32(from_stream_word(P.w0[j]), lane);
                mag0 = x & 0xffffu;
                mag1 = x >> 16;
            } else {
                mag0 = warp_transpose32(from_stream_word(P.w0[j]), lane);
                mag1 = warp_transpose32(from_stream_word(P.w1[j]), lane);
            }
            if constexpr (MODE == MODE_OUTLIER) {
                if ((r & 0x80) && lane == 0) mag0 = P.m0[j];
            }
            const uint32_t s0 = from_stream_word(P.s0[j]), s1 = from_stream_word(P.s1[DIM == 1 ? 0 : j]);
            int32_t d0 = ((s0 >> lane) & 1u) ? (int32_t)(0u - mag0) : (int32_t)mag0;
            int32_t d1 = ((s1 >> lane) & 1u) ? (int32_t)(0u - mag1) : (int32_t)mag1;
            if constexpr (MODE != MODE_FIXED) lorenzo_inverse<DIM>(d0, d1, lane);
            if (ok0) st_stream(out + i0, dequant(d0, eb));
            if (ok1) st_stream(out + i1, dequant(d1, eb));
        }
    }
}

// Posts a tile's aggregate as soon as its rate bytes are scanned -- before any
// waiting -- so that no tile ever waits on a predecessor that is itself waiting.
template <int WARPS>
__device__ __forceinline__ void post_aggregate(uint32_t warp_total, int64_t tile, unsigned long long* status,
                                               uint32_t* s_w, unsigned long long* s_agg)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_w[warp] = warp_total;
    __syncthreads();
    if (warp == 0) {
        uint32_t v = lane < WARPS ? s_w[lane] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < WARPS; o <<= 1) {
            uint32_t t = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += t;
        }
        const uint64_t agg = __shfl_sync(FULL, incl, WARPS - 1);
        __syncwarp();
        if (lane < WARPS) s_w[lane] = incl - v;
        if (lane == 0) {
            st_post(status + tile, (tile == 0 ? ST_INC : ST_AGG) | agg);
            *s_agg = agg;
        }
    }
    __syncthreads();
}

// Look-back for a tile whose aggregate was posted earlier (warp 0 polls, the CTA
// waits at one barrier); returns its exclusive payload offset in every thread and
// publishes its inclusive prefix.
template <int WARPS>
__device__ __forceinline__ uint64_t resolve_tile(int64_t tile, uint64_t ntiles, unsigned long long* status,
                                                 uint32_t* err, unsigned long long* total_out, uint64_t rate_bytes,
                                                 unsigned long long agg, LookbackShared& lb)
{
    if ((threadIdx.x >> 5) == 0) {
        const uint64_t excl = tile > 0 ? warp_lookback(status, tile, err) : 0;
        if (threadIdx.x == 0) {
            if (tile > 0) st_post(status + tile, ST_INC | ((excl + agg) & ST_VAL));
            if ((uint64_t)tile == ntiles - 1) *total_out = rate_bytes + excl + agg;
            lb.excl = excl;
        }
    }
    __syncthreads();
    return lb.excl;
}

template <typename T, int DIM, int MODE, typename Tl = Tiling<DIM>>
__global__ void __launch_bounds__(Tl::THREADS, 2)
decompress_kernel(T* __restrict__ out, const uint8_t* __restrict__ cmp, Geom g, T eb,
                  WsHeader* __restrict__ hdr, unsigned long long* __restrict__ status)
{
    __shared__ TileShared<Tl::WARPS> sh;
    if (threadIdx.x == 0) sh.ticket[0] = (int64_t)atomicAdd(&hdr->ticket, 1u);
    __syncthreads();
    int64_t tile = sh.ticket[0];
    int slot = 0;
    DecompRates<Tl> R;
    if ((uint64_t)tile < g.ntiles) {
        decompress_rates<DIM, MODE, Tl>(R, cmp, g, tile);
        post_aggregate<Tl::WARPS>(R.wtot, tile, status, sh.dwarp[0], &sh.dagg[0]);
    }
    for (int it = 1; (uint64_t)tile < g.ntiles; it++) {
        if (threadIdx.x == 0) sh.ticket[it & 1] = (int64_t)atomicAdd(&hdr->ticket, 1u);
        __syncthreads();
        const int64_t next = sh.ticket[it & 1];
        DecompRates<Tl> Rn = R;
        if ((uint64_t)next < g.ntiles) {
            decompress_rates<DIM, MODE, Tl>(Rn, cmp, g, next);
            post_aggregate<Tl::WARPS>(Rn.wtot, next, status, sh.dwarp[slot ^ 1], &sh.dagg[slot ^ 1]);
        }
        const uint64_t excl = resolve_tile<Tl::WARPS>(tile, g.ntiles, status, &hdr->err, &hdr->total, g.rate_bytes,
                                                      sh.dagg[slot], sh.lb);
        const uint8_t* pbase = cmp + g.rate_bytes + excl + sh.dwarp[slot][threadIdx.x >> 5];
        DecompPayload<DIM, Tl> P;
        decompress_load<DIM, MODE, Tl>(P, R, pbase);
        decompress_store<T, DIM, MODE, Tl>(P, R, out, g, eb, tile);
        tile = next;
        R = Rn;
        slot ^= 1;
    }
    finish_cta(hdr, status, g.ntiles);
}

}  // namespace cuszp

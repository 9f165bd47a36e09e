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

template <int MODE>
__device__ __forceinline__ void put32(uint8_t* p, uint32_t v)
{
    if constexpr (MODE == MODE_OUTLIER) {   // outlier payloads sit at any byte offset
        p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); p[2] = (uint8_t)(v >> 16); p[3] = (uint8_t)(v >> 24);
    } else {
        *reinterpret_cast<uint32_t*>(p) = v;
    }
}
template <int MODE>
__device__ __forceinline__ uint32_t get32(const uint8_t* p)
{
    if constexpr (MODE == MODE_OUTLIER) {
        return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
    } else {
        return *reinterpret_cast<const uint32_t*>(p);
    }
}

// --------------------------------------------------------------- block addressing

struct BlockPos { uint32_t z, y, x; };   // block coordinates (2D: z = slice)

__device__ __forceinline__ BlockPos block_pos(uint64_t b, const Geom& g)
{
    const uint32_t per = g.bxn * g.byn;
    const uint32_t bb = (uint32_t)b;
    BlockPos p;
    p.z = bb / per;
    const uint32_t r = bb - p.z * per;
    p.y = r / g.bxn;
    p.x = r - p.y * g.bxn;
    return p;
}

// Element (half h, lane l) of a 2D/3D block: returns the flat index and validity.
template <int DIM>
__device__ __forceinline__ bool elem_index(const BlockPos& bp, bool block_ok, int h, int lane, const Geom& g,
                                           uint64_t& idx)
{
    uint32_t x, y, z;
    if constexpr (DIM == 2) {
        x = bp.x * 8 + (lane & 7);
        y = bp.y * 8 + (lane >> 3) + 4 * h;
        z = bp.z;
    } else {
        x = bp.x * 4 + (lane & 3);
        y = bp.y * 4 + ((lane >> 2) & 3);
        z = bp.z * 4 + (lane >> 4) + 2 * h;
    }
    const bool ok = block_ok && x < g.dx && y < g.dy && z < g.dz;
    idx = ((uint64_t)z * g.dy + y) * g.dx + x;
    return ok;
}

// Predecessor of each element for the Lorenzo delta (src/cuSZp_kernels_2D_f32.cu:711-760,
// 3D_f32.cu:697-704): returns q(pred) for half 0 (p0) and half 1 (p1).
template <int DIM>
__device__ __forceinline__ void predecessors(int32_t q0, int32_t q1, int lane, int32_t& p0, int32_t& p1)
{
    if constexpr (DIM == 1) {
        int32_t u = __shfl_up_sync(FULL, q0, 1);
        p0 = lane ? u : 0;
        p1 = 0;
    } else if constexpr (DIM == 2) {
        // x-delta inside a row, column 0 against the previous row's column 0.
        const int32_t u1a = __shfl_up_sync(FULL, q0, 1), u8a = __shfl_up_sync(FULL, q0, 8);
        const int32_t u1b = __shfl_up_sync(FULL, q1, 1), u8b = __shfl_up_sync(FULL, q1, 8);
        const int32_t r3 = __shfl_sync(FULL, q0, 24);
        const bool c0 = (lane & 7) == 0;
        p0 = !c0 ? u1a : (lane >= 8 ? u8a : 0);
        p1 = !c0 ? u1b : (lane >= 8 ? u8b : r3);
    } else {
        // x-delta; row start against previous row start; plane start against previous plane start.
        const int32_t u1a = __shfl_up_sync(FULL, q0, 1), u4a = __shfl_up_sync(FULL, q0, 4), u16a = __shfl_up_sync(FULL, q0, 16);
        const int32_t u1b = __shfl_up_sync(FULL, q1, 1), u4b = __shfl_up_sync(FULL, q1, 4), u16b = __shfl_up_sync(FULL, q1, 16);
        const int32_t z1 = __shfl_sync(FULL, q0, 16);
        const int xx = lane & 3, yy = (lane >> 2) & 3;
        p0 = xx ? u1a : yy ? u4a : (lane >= 16 ? u16a : 0);
        p1 = xx ? u1b : yy ? u4b : (lane >= 16 ? u16b : z1);
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

// --------------------------------------------------------------- compress

template <typename T, int DIM, int MODE, typename Tl = Tiling<DIM>>
__device__ __forceinline__ void compress_tile(const T* __restrict__ in, uint8_t* __restrict__ cmp, const Geom& g,
                                              T recip, int64_t tile, unsigned long long* __restrict__ status,
                                              uint32_t* err, unsigned long long* total_out, uint32_t* s_warp,
                                              uint64_t* s_base)
{
    constexpr int BPW = Tl::BPW;
    constexpr int W = Tl::W;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    {
        const uint64_t b0 = (uint64_t)tile * Tl::TB + (uint64_t)warp * BPW;

        // ---- 1. load, quantize, predict
        int32_t c0[BPW], c1[BPW];
        if constexpr (DIM == 1) {
            T v[BPW];
#pragma unroll
            for (int j = 0; j < BPW; j++) {
                const uint64_t i = (b0 + j) * 32 + lane;
                v[j] = i < g.nbEle ? ld_stream(in + i) : T(0);
            }
#pragma unroll
            for (int j = 0; j < BPW; j++) {
                const uint64_t i = (b0 + j) * 32 + lane;
                const int32_t q = quantize(v[j], recip);
                int32_t p0 = 0, p1;
                if constexpr (MODE != MODE_FIXED) predecessors<1>(q, 0, lane, p0, p1);
                c0[j] = i < g.nbEle ? wsub(q, p0) : 0;
                c1[j] = 0;
            }
        } else {
            T v0[BPW], v1[BPW];
            bool ok0[BPW], ok1[BPW];
#pragma unroll
            for (int j = 0; j < BPW; j++) {
                const uint64_t b = b0 + j;
                const bool bok = b < g.nblocks;
                const BlockPos bp = block_pos(bok ? b : 0, g);
                uint64_t i0, i1;
                ok0[j] = elem_index<DIM>(bp, bok, 0, lane, g, i0);
                ok1[j] = elem_index<DIM>(bp, bok, 1, lane, g, i1);
                v0[j] = ok0[j] ? ld_stream(in + i0) : T(0);
                v1[j] = ok1[j] ? ld_stream(in + i1) : T(0);
            }
#pragma unroll
            for (int j = 0; j < BPW; j++) {
                const int32_t q0 = quantize(v0[j], recip), q1 = quantize(v1[j], recip);
                int32_t p0 = 0, p1 = 0;
                if constexpr (MODE != MODE_FIXED) predecessors<DIM>(q0, q1, lane, p0, p1);
                c0[j] = ok0[j] ? wsub(q0, p0) : 0;
                c1[j] = ok1[j] ? wsub(q1, p1) : 0;
            }
        }

        // ---- rate byte per block (block maxima: signed in 1D, unsigned in 2D/3D)
        uint32_t rb[BPW], off[BPW];
        uint32_t wtot = 0, myrb = 0;
#pragma unroll
        for (int j = 0; j < BPW; j++) {
            const uint32_t a0 = uabs(c0[j]), a1 = uabs(c1[j]);
            uint32_t m, m2 = 0;
            if constexpr (DIM == 1) {
                m = (uint32_t)max(__reduce_max_sync(FULL, (int)a0), 0);
                if constexpr (MODE == MODE_OUTLIER) m2 = (uint32_t)max(__reduce_max_sync(FULL, lane ? (int)a0 : 0), 0);
            } else {
                m = __reduce_max_sync(FULL, max(a0, a1));
                if constexpr (MODE == MODE_OUTLIER) m2 = __reduce_max_sync(FULL, lane ? max(a0, a1) : a1);
            }
            const int fr1 = bitlen(m);
            uint32_t r;
            if constexpr (MODE == MODE_OUTLIER) {
                const int fr2 = bitlen(m2);
                const int ob = (bitlen(__shfl_sync(FULL, a0, 0)) + 7) / 8;
                const int cost1 = fr1 ? W + fr1 * W : 0;
                const int cost2 = fr2 ? W + fr2 * W + ob : W + ob;
                r = cost1 <= cost2 ? (uint32_t)fr1 : (uint32_t)((fr2 | 0x80 | ((ob - 1) << 5)) & 0xff);
            } else {
                r = (uint32_t)fr1;
            }
            rb[j] = r;
            off[j] = wtot;
            wtot += payload_size<DIM, MODE>(r);
            if (lane == j) myrb = r;
        }
        if (lane < BPW && b0 + lane < g.rate_bytes) cmp[b0 + lane] = (uint8_t)myrb;

        // ---- 2. tile offset
        tile_scan<Tl::WARPS>(wtot, tile, g.ntiles, status, err, total_out, g.rate_bytes, s_warp, s_base);
        uint8_t* const pbase = cmp + g.rate_bytes + *s_base + s_warp[warp];

        // ---- 3. sign maps and bit-planes
        if constexpr (DIM == 1) {
#pragma unroll
            for (int j = 0; j < BPW; j += 2) {
                const uint32_t rA = rb[j], rB = rb[j + 1];
                if ((rA | rB) == 0) continue;
                uint32_t nA = rA, nB = rB, obA = 0, obB = 0;
                if constexpr (MODE == MODE_OUTLIER) {
                    nA = rA & 0x1f; nB = rB & 0x1f;
                    if (rA & 0x80) obA = ((rA & 0x60) >> 5) + 1;
                    if (rB & 0x80) obB = ((rB & 0x60) >> 5) + 1;
                }
                uint32_t aA = uabs(c0[j]), aB = uabs(c0[j + 1]);
                uint8_t* pA = pbase + off[j];
                uint8_t* pB = pbase + off[j + 1];
                if constexpr (MODE == MODE_OUTLIER) {
                    if (lane == 0) {
                        for (uint32_t i = 0; i < obA; i++) pA[i] = (uint8_t)(aA >> (8 * i));
                        for (uint32_t i = 0; i < obB; i++) pB[i] = (uint8_t)(aB >> (8 * i));
                        if (obA) aA = 0;
                        if (obB) aB = 0;
                    }
                    pA += obA; pB += obB;
                }
                const uint32_t sA = to_stream_word(__ballot_sync(FULL, c0[j] < 0));
                const uint32_t sB = to_stream_word(__ballot_sync(FULL, c0[j + 1] < 0));
                const bool hasA = payload_size<DIM, MODE>(rA) != 0, hasB = payload_size<DIM, MODE>(rB) != 0;
                if (lane == 0 && hasA) put32<MODE>(pA, sA);
                if (lane == 16 && hasB) put32<MODE>(pB, sB);
                if (nA <= 16 && nB <= 16) {
                    const uint32_t y = to_stream_word(warp_transpose32((aA & 0xffffu) | (aB << 16), lane));
                    const int p = lane & 15;
                    if (lane < 16) { if ((uint32_t)p < nA) put32<MODE>(pA + 4 + 4 * p, y); }
                    else           { if ((uint32_t)p < nB) put32<MODE>(pB + 4 + 4 * p, y); }
                } else {
                    const uint32_t yA = to_stream_word(warp_transpose32(aA, lane));
                    const uint32_t yB = to_stream_word(warp_transpose32(aB, lane));
                    if ((uint32_t)lane < nA) put32<MODE>(pA + 4 + 4 * lane, yA);
                    if ((uint32_t)lane < nB) put32<MODE>(pB + 4 + 4 * lane, yB);
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < BPW; j++) {
                const uint32_t r = rb[j];
                if (r == 0) continue;
                uint32_t n = r, ob = 0;
                if constexpr (MODE == MODE_OUTLIER) {
                    n = r & 0x1f;
                    if (r & 0x80) ob = ((r & 0x60) >> 5) + 1;
                }
                uint32_t a0 = uabs(c0[j]);
                const uint32_t a1 = uabs(c1[j]);
                uint8_t* p = pbase + off[j];
                if constexpr (MODE == MODE_OUTLIER) {
                    if (lane == 0) {
                        for (uint32_t i = 0; i < ob; i++) p[i] = (uint8_t)(a0 >> (8 * i));
                        if (ob) a0 = 0;
                    }
                    p += ob;
                }
                const uint32_t s0 = to_stream_word(__ballot_sync(FULL, c0[j] < 0));
                const uint32_t s1 = to_stream_word(__ballot_sync(FULL, c1[j] < 0));
                if (lane == 0) put32<MODE>(p, s0);
                if (lane == 1) put32<MODE>(p + 4, s1);
                if (n <= 16) {
                    const uint32_t y = to_stream_word(warp_transpose32((a0 & 0xffffu) | (a1 << 16), lane));
                    const int pl = lane & 15;
                    if ((uint32_t)pl < n) put32<MODE>(p + 8 + 8 * pl + (lane >> 4) * 4, y);
                } else {
                    const uint32_t ylo = to_stream_word(warp_transpose32(a0, lane));
                    const uint32_t yhi = to_stream_word(warp_transpose32(a1, lane));
                    if ((uint32_t)lane < n) {
                        put32<MODE>(p + 8 + 8 * lane, ylo);
                        put32<MODE>(p + 12 + 8 * lane, yhi);
                    }
                }
            }
        }
    }
}

template <typename T, int DIM, int MODE>
__global__ void __launch_bounds__(kThreads)
compress_kernel(const T* __restrict__ in, uint8_t* __restrict__ cmp, Geom g, T recip,
                WsHeader* __restrict__ hdr, unsigned long long* __restrict__ status)
{
    __shared__ uint32_t s_warp[kWarps];
    __shared__ uint64_t s_base;
    __shared__ int64_t s_tile;
    for (;;) {
        if (threadIdx.x == 0) s_tile = (int64_t)atomicAdd(&hdr->ticket, 1u);
        __syncthreads();
        const int64_t tile = s_tile;
        if ((uint64_t)tile >= g.ntiles) break;
        compress_tile<T, DIM, MODE>(in, cmp, g, recip, tile, status, &hdr->err, &hdr->total, s_warp, &s_base);
    }
    finish_cta(hdr, status, g.ntiles);
}

// --------------------------------------------------------------- decompress

template <typename T, int DIM, int MODE, typename Tl = Tiling<DIM>>
__device__ __forceinline__ void decompress_tile(T* __restrict__ out, const uint8_t* __restrict__ cmp, const Geom& g,
                                                T eb, int64_t tile, unsigned long long* __restrict__ status,
                                                uint32_t* err, unsigned long long* total_out, uint32_t* s_warp,
                                                uint64_t* s_base)
{
    constexpr int BPW = Tl::BPW;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    {
        const uint64_t b0 = (uint64_t)tile * Tl::TB + (uint64_t)warp * BPW;

        // ---- rate bytes -> payload sizes -> warp-local offsets
        uint32_t myrb = 0;
        if (lane < BPW && b0 + lane < g.nblocks) myrb = cmp[b0 + lane];
        const uint32_t sz = lane < BPW ? payload_size<DIM, MODE>(myrb) : 0u;
        uint32_t incl = sz;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += t;
        }
        const uint32_t myoff = incl - sz;
        const uint32_t wtot = __shfl_sync(FULL, incl, 31);

        tile_scan<Tl::WARPS>(wtot, tile, g.ntiles, status, err, total_out, g.rate_bytes, s_warp, s_base);
        const uint8_t* const pbase = cmp + g.rate_bytes + *s_base + s_warp[warp];

        if constexpr (DIM == 1) {
            // ---- load phase: plane words and sign words of all blocks
            constexpr int NP = BPW / 2;
            uint32_t wA[NP], wB[NP], sgA[NP], sgB[NP], m0A[NP], m0B[NP];
#pragma unroll
            for (int k = 0; k < NP; k++) {
                const int j = 2 * k;
                const uint32_t rA = __shfl_sync(FULL, myrb, j), rB = __shfl_sync(FULL, myrb, j + 1);
                const uint32_t oA = __shfl_sync(FULL, myoff, j), oB = __shfl_sync(FULL, myoff, j + 1);
                uint32_t nA = rA, nB = rB, obA = 0, obB = 0;
                if constexpr (MODE == MODE_OUTLIER) {
                    nA = rA & 0x1f; nB = rB & 0x1f;
                    if (rA & 0x80) obA = ((rA & 0x60) >> 5) + 1;
                    if (rB & 0x80) obB = ((rB & 0x60) >> 5) + 1;
                }
                const uint8_t* pA = pbase + oA;
                const uint8_t* pB = pbase + oB;
                m0A[k] = 0; m0B[k] = 0;
                if constexpr (MODE == MODE_OUTLIER) {
                    for (uint32_t i = 0; i < obA; i++) m0A[k] |= (uint32_t)pA[i] << (8 * i);
                    for (uint32_t i = 0; i < obB; i++) m0B[k] |= (uint32_t)pB[i] << (8 * i);
                    pA += obA; pB += obB;
                }
                const bool hasA = payload_size<DIM, MODE>(rA) != 0, hasB = payload_size<DIM, MODE>(rB) != 0;
                sgA[k] = hasA ? get32<MODE>(pA) : 0u;
                sgB[k] = hasB ? get32<MODE>(pB) : 0u;
                wA[k] = 0; wB[k] = 0;
                if (nA <= 16 && nB <= 16) {
                    const int p = lane & 15;
                    if (lane < 16) { if ((uint32_t)p < nA) wA[k] = get32<MODE>(pA + 4 + 4 * p); }
                    else           { if ((uint32_t)p < nB) wA[k] = get32<MODE>(pB + 4 + 4 * p); }
                } else {
                    if ((uint32_t)lane < nA) wA[k] = get32<MODE>(pA + 4 + 4 * lane);
                    if ((uint32_t)lane < nB) wB[k] = get32<MODE>(pB + 4 + 4 * lane);
                }
            }
            // ---- decode phase: one warp transpose per pair (two if a rate exceeds 16)
#pragma unroll
            for (int k = 0; k < NP; k++) {
                const uint32_t rA = __shfl_sync(FULL, myrb, 2 * k), rB = __shfl_sync(FULL, myrb, 2 * k + 1);
                uint32_t nA = rA, nB = rB;
                if constexpr (MODE == MODE_OUTLIER) { nA = rA & 0x1f; nB = rB & 0x1f; }
                uint32_t magA = 0, magB = 0;
                if (nA <= 16 && nB <= 16) {
                    if ((nA | nB) != 0) {
                        const uint32_t x = warp_transpose32(from_stream_word(wA[k]), lane);
                        magA = x & 0xffffu;
                        magB = x >> 16;
                    }
                } else {
                    magA = warp_transpose32(from_stream_word(wA[k]), lane);
                    magB = warp_transpose32(from_stream_word(wB[k]), lane);
                }
                if constexpr (MODE == MODE_OUTLIER) {
                    if (lane == 0) {
                        if (rA & 0x80) magA = m0A[k];
                        if (rB & 0x80) magB = m0B[k];
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
                    const uint32_t sg = from_stream_word(s ? sgB[k] : sgA[k]);
                    int32_t d = ((sg >> lane) & 1u) ? (int32_t)(0u - mag) : (int32_t)mag;
                    int32_t dummy = 0;
                    if constexpr (MODE != MODE_FIXED) lorenzo_inverse<1>(d, dummy, lane);
                    if (i < g.nbEle) st_stream(out + i, dequant(d, eb));
                }
            }
        } else {
            // ---- load phase
            uint32_t w0[BPW], w1[BPW], sg0[BPW], sg1[BPW], m0[BPW];
#pragma unroll
            for (int j = 0; j < BPW; j++) {
                const uint32_t r = __shfl_sync(FULL, myrb, j);
                const uint32_t o = __shfl_sync(FULL, myoff, j);
                uint32_t n = r, ob = 0;
                if constexpr (MODE == MODE_OUTLIER) {
                    n = r & 0x1f;
                    if (r & 0x80) ob = ((r & 0x60) >> 5) + 1;
                }
                const uint8_t* p = pbase + o;
                m0[j] = 0;
                if constexpr (MODE == MODE_OUTLIER) {
                    for (uint32_t i = 0; i < ob; i++) m0[j] |= (uint32_t)p[i] << (8 * i);
                    p += ob;
                }
                const bool has = payload_size<DIM, MODE>(r) != 0;
                sg0[j] = has ? get32<MODE>(p) : 0u;
                sg1[j] = has ? get32<MODE>(p + 4) : 0u;
                w0[j] = 0; w1[j] = 0;
                if (n <= 16) {
                    const int pl = lane & 15;
                    if ((uint32_t)pl < n) w0[j] = get32<MODE>(p + 8 + 8 * pl + (lane >> 4) * 4);
                } else if ((uint32_t)lane < n) {
                    w0[j] = get32<MODE>(p + 8 + 8 * lane);
                    w1[j] = get32<MODE>(p + 12 + 8 * lane);
                }
            }
            // ---- decode phase
#pragma unroll
            for (int j = 0; j < BPW; j++) {
                const uint64_t b = b0 + j;
                const bool bok = b < g.nblocks;
                const BlockPos bp = block_pos(bok ? b : 0, g);
                uint64_t i0, i1;
                const bool ok0 = elem_index<DIM>(bp, bok, 0, lane, g, i0);
                const bool ok1 = elem_index<DIM>(bp, bok, 1, lane, g, i1);
                const uint32_t r = __shfl_sync(FULL, myrb, j);
                if (payload_size<DIM, MODE>(r) == 0) {
                    if (ok0) st_stream(out + i0, T(0));
                    if (ok1) st_stream(out + i1, T(0));
                    continue;
                }
                uint32_t n = r;
                if constexpr (MODE == MODE_OUTLIER) n = r & 0x1f;
                uint32_t mag0, mag1;
                if (n <= 16) {
                    const uint32_t x = warp_transpose32(from_stream_word(w0[j]), lane);
                    mag0 = x & 0xffffu;
                    mag1 = x >> 16;
                } else {
                    mag0 = warp_transpose32(from_stream_word(w0[j]), lane);
                    mag1 = warp_transpose32(from_stream_word(w1[j]), lane);
                }
                if constexpr (MODE == MODE_OUTLIER) {
                    if ((r & 0x80) && lane == 0) mag0 = m0[j];
                }
                const uint32_t s0 = from_stream_word(sg0[j]), s1 = from_stream_word(sg1[j]);
                int32_t d0 = ((s0 >> lane) & 1u) ? (int32_t)(0u - mag0) : (int32_t)mag0;
                int32_t d1 = ((s1 >> lane) & 1u) ? (int32_t)(0u - mag1) : (int32_t)mag1;
                if constexpr (MODE != MODE_FIXED) lorenzo_inverse<DIM>(d0, d1, lane);
                if (ok0) st_stream(out + i0, dequant(d0, eb));
                if (ok1) st_stream(out + i1, dequant(d1, eb));
            }
        }
    }
}

template <typename T, int DIM, int MODE>
__global__ void __launch_bounds__(kThreads)
decompress_kernel(T* __restrict__ out, const uint8_t* __restrict__ cmp, Geom g, T eb,
                  WsHeader* __restrict__ hdr, unsigned long long* __restrict__ status)
{
    __shared__ uint32_t s_warp[kWarps];
    __shared__ uint64_t s_base;
    __shared__ int64_t s_tile;
    for (;;) {
        if (threadIdx.x == 0) s_tile = (int64_t)atomicAdd(&hdr->ticket, 1u);
        __syncthreads();
        const int64_t tile = s_tile;
        if ((uint64_t)tile >= g.ntiles) break;
        decompress_tile<T, DIM, MODE>(out, cmp, g, eb, tile, status, &hdr->err, &hdr->total, s_warp, &s_base);
    }
    finish_cta(hdr, status, g.ntiles);
}

}  // namespace cuszp

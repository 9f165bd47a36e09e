/*
 * cuszp_oracle.c -- CPU restatement of cuSZp's fixed-length block codec.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: tests, the smoke
 * check and the CPU-baseline leg of bench.py call it to check or time against;
 * the product path (cuszp_b200/csrc) never links it and never falls back to it.
 *
 * It restates, block by block, what the reference GPU kernels compute, so that
 * the compressed stream and the reconstruction can be compared byte for byte:
 *
 *   quantizer f32     src/cuSZp_kernels_1D_f32.cu:3-20   (inline PTX mul/setp/add/cvt.rzi)
 *   quantizer f64     src/cuSZp_kernels_1D_f64.cu:3-8
 *   bit length        src/cuSZp_kernels_1D_f32.cu:23-28  (32 - clz)
 *   1D fixed / plain  src/cuSZp_kernels_1D_f32.cu:31-296, :523-799 (compress)
 *                     src/cuSZp_kernels_1D_f32.cu:299-520, :802-1034 (decompress)
 *   1D outlier        src/cuSZp_kernels_1D_f32.cu:1037-1662 / :1665-2260
 *   2D (8x8 blocks)   src/cuSZp_kernels_2D_f32.cu:31-3229 (f64 twin 2D_f64.cu)
 *   3D (4x4x4 blocks) src/cuSZp_kernels_3D_f32.cu:32-3094 (f64 twin 3D_f64.cu)
 *   reported cmpSize  src/cuSZp_entry_1D_f32.cu:42-43, src/cuSZp_entry_2D_f64.cu:46-47
 *
 * Stream layout (independent of the reference's CTA tiling):
 *   [rate region: one byte per data block; 1D: round_up(n,32768)/32 bytes,
 *    2D/3D: round_up(blockNum,4) bytes]  [block payloads in block order]
 *
 * Integer semantics follow the device code exactly: 32-bit two's complement
 * wrap for deltas, abs(INT_MIN) == INT_MIN, signed maxima in 1D and unsigned
 * maxima in 2D/3D, and cvt.rzi saturation (NaN: see cvt_rzi_*).  Built with
 * -ffp-contract=off so that the only fused multiply-add is the explicit one
 * selected by `fused`.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { ORC_F32 = 0, ORC_F64 = 1 };
enum { ORC_FIXED = 0, ORC_PLAIN = 1, ORC_OUTLIER = 2 };

typedef struct {
    int type, mode, dim;
    size_t nbEle;
    uint32_t dx, dy, dz;       /* dims.x fastest */
    uint64_t nblocks;          /* data blocks that exist */
    uint64_t rate_bytes;       /* size of the rate region */
    uint32_t bx, by;           /* blocks along x and y (2D/3D) */
    int n;                     /* elements per block: 32 (1D) or 64 */
    int W;                     /* bytes per bit-plane: 4 or 8 */
} geom_t;

/* ---------------------------------------------------------------- scalar ops */

static inline int32_t wrap_sub(int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); }
static inline int32_t wrap_add(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
static inline int32_t wrap_neg(int32_t a) { return (int32_t)(0u - (uint32_t)a); }
static inline uint32_t abs_u(int32_t a) { return a < 0 ? (uint32_t)wrap_neg(a) : (uint32_t)a; }

static inline int bitlen(uint32_t x) { return x ? 32 - __builtin_clz(x) : 0; }

/* cvt.rzi.s32.f32 / .f64: truncate and saturate.  NaN converts to 0 through the
 * f32 path and to INT_MIN through the f64 path on the reference build (pinned by
 * the eb == 0 golden vectors, where 0 * inf = NaN). */
static inline int32_t cvt_rzi_f32(float t)
{
    if (t != t) return 0;
    if (t >= 2147483648.0f) return INT32_MAX;
    if (t < -2147483648.0f) return INT32_MIN;
    return (int32_t)t;
}
static inline int32_t cvt_rzi_f64(double t)
{
    if (t != t) return INT32_MIN;
    if (t >= 2147483648.0) return INT32_MAX;
    if (t <= -2147483649.0) return INT32_MIN;
    return (int32_t)t;
}

/* src/cuSZp_kernels_1D_f32.cu:3-20: p = x*r; s = !(p >= -0.5); q = rzi(p + 0.5) - s.
 * `fused` evaluates p + 0.5 as one fma(x, r, 0.5), as a code generator may; the
 * reference build rounds the two operations separately (fused = 0), which the
 * golden vectors' rounding-trap inputs pin. */
static inline int32_t quant_f32(float x, float r, int fused)
{
    float p = x * r;
    int32_t s = (p >= -0.5f) ? 0 : 1;
    float t = fused ? fmaf(x, r, 0.5f) : (p + 0.5f);
    return wrap_sub(cvt_rzi_f32(t), s);
}
/* src/cuSZp_kernels_1D_f64.cu:3-8 */
static inline int32_t quant_f64(double x, double r, int fused)
{
    double p = x * r;
    int32_t s = (p >= -0.5) ? 0 : 1;
    double t = fused ? fma(x, r, 0.5) : (p + 0.5);
    return wrap_sub(cvt_rzi_f64(t), s);
}

/* ---------------------------------------------------------------- geometry */

static int make_geom(geom_t* g, int type, int mode, int dim, size_t nbEle,
                     uint32_t dx, uint32_t dy, uint32_t dz)
{
    memset(g, 0, sizeof(*g));
    g->type = type; g->mode = mode; g->dim = dim; g->nbEle = nbEle;
    g->dx = dx; g->dy = dy; g->dz = dz;
    if (type != ORC_F32 && type != ORC_F64) return -1;
    if (mode < 0 || mode > 2) return -1;
    if (dim == 1) {
        g->n = 32; g->W = 4;
        g->nblocks = (nbEle + 31) / 32;
        /* src/cuSZp_kernels_1D_f32.cu:47 rate_ofs = round_up(n, 32*1024)/32 */
        g->rate_bytes = ((uint64_t)nbEle + 32767) / 32768 * 32768 / 32;
    } else if (dim == 2) {
        g->n = 64; g->W = 8;
        g->bx = (dx + 7) / 8; g->by = (dy + 7) / 8;
        g->nblocks = (uint64_t)dz * g->by * g->bx;
        g->rate_bytes = (g->nblocks + 3) / 4 * 4;      /* 2D_f32.cu:46 */
    } else if (dim == 3) {
        g->n = 64; g->W = 8;
        g->bx = (dx + 3) / 4; g->by = (dy + 3) / 4;
        g->nblocks = (uint64_t)((dz + 3) / 4) * g->by * g->bx;
        g->rate_bytes = (g->nblocks + 3) / 4 * 4;      /* 3D_f32.cu:41 */
    } else {
        return -1;
    }
    return 0;
}

/* Quantized value at flat element index i. */
static inline int32_t qat(const geom_t* g, const void* data, size_t i, double recip, int fused)
{
    if (g->type == ORC_F32) return quant_f32(((const float*)data)[i], (float)recip, fused);
    return quant_f64(((const double*)data)[i], recip, fused);
}

/*
 * Per-block prediction codes (src/cuSZp_kernels_*: the quantize/delta loops).
 * code[k] for element k of the block, in the block's element order:
 *   1D k = lane offset; 2D k = 8*row + col; 3D k = 16*z + 4*y + x.
 * Elements outside the array get code 0 and never update a predictor.
 */
static void block_codes(const geom_t* g, const void* data, uint64_t b, double recip,
                        int fused, int32_t* code)
{
    const int lorenzo = g->mode != ORC_FIXED;
    if (g->dim == 1) {
        int32_t prev = 0;
        for (int k = 0; k < 32; k++) {
            uint64_t i = b * 32 + (uint64_t)k;
            if (i < g->nbEle) {
                int32_t q = qat(g, data, i, recip, fused);
                code[k] = lorenzo ? wrap_sub(q, prev) : q;
                prev = q;
            } else {
                code[k] = 0;
            }
        }
    } else if (g->dim == 2) {
        uint64_t per_slice = (uint64_t)g->by * g->bx;
        uint64_t z = b / per_slice, rem = b % per_slice;
        uint64_t byi = rem / g->bx, bxi = rem % g->bx;
        uint64_t x0 = bxi * 8;
        int32_t prev_y = 0;
        for (int r = 0; r < 8; r++) {
            uint64_t y = byi * 8 + (uint64_t)r;
            int32_t prev = 0;
            for (int c = 0; c < 8; c++) {
                int k = r * 8 + c;
                /* 2D_f32.cu:92,120: rows past dims.y and the x half-block past
                 * dims.x are zero codes (dims.x % 4 == 0 is required). */
                int valid = (y < g->dy) && (x0 + (uint64_t)c < g->dx);
                if (!valid) { code[k] = 0; continue; }
                uint64_t i = (z * g->dy + y) * g->dx + x0 + (uint64_t)c;
                int32_t q = qat(g, data, i, recip, fused);
                if (!lorenzo) { code[k] = q; continue; }
                if (c == 0) { code[k] = wrap_sub(q, prev_y); prev_y = q; }
                else        { code[k] = wrap_sub(q, prev); }
                prev = q;
            }
        }
    } else {
        uint64_t per_slice = (uint64_t)g->by * g->bx;
        uint64_t bz = b / per_slice, rem = b % per_slice;
        uint64_t byi = rem / g->bx, bxi = rem % g->bx;
        int32_t prev_z = 0;
        for (int zz = 0; zz < 4; zz++) {
            uint64_t z = bz * 4 + (uint64_t)zz;
            int32_t prev_y = 0;
            for (int yy = 0; yy < 4; yy++) {
                uint64_t y = byi * 4 + (uint64_t)yy;
                int32_t prev_x = 0;
                for (int xx = 0; xx < 4; xx++) {
                    int k = zz * 16 + yy * 4 + xx;
                    uint64_t x = bxi * 4 + (uint64_t)xx;
                    int valid = (z < g->dz) && (y < g->dy) && (x < g->dx);
                    if (!valid) { code[k] = 0; continue; }
                    uint64_t i = (z * g->dy + y) * g->dx + x;
                    int32_t q = qat(g, data, i, recip, fused);
                    if (!lorenzo) { code[k] = q; continue; }
                    /* 3D_f32.cu:697-704: x-delta; row start from previous row
                     * start; plane start from previous plane start. */
                    if (xx == 0) {
                        if (yy) code[k] = wrap_sub(q, prev_y);
                        else { code[k] = wrap_sub(q, prev_z); prev_z = q; }
                        prev_y = q;
                    } else {
                        code[k] = wrap_sub(q, prev_x);
                    }
                    prev_x = q;
                }
            }
        }
    }
}

/* Block summary: rate byte and payload size (as decoded from the rate byte). */
typedef struct { uint8_t rate; uint32_t size; } bsum_t;

static inline uint32_t size_from_rate(const geom_t* g, uint8_t rb)
{
    const uint32_t W = (uint32_t)g->W;
    if (g->mode != ORC_OUTLIER) return rb ? W + W * rb : 0;
    /* 1D_f32.cu:1701-1707 (decompress) and :1268-1269 (compress write phase) */
    uint32_t sel = rb >> 7, ob = ((rb & 0x60u) >> 5) + 1, r = rb & 0x1fu;
    if (!sel) return r ? W + W * r : 0;
    return W + ob + W * r;
}

static uint8_t block_rate(const geom_t* g, const int32_t* code)
{
    const int n = g->n;
    const int W = g->W;
    /* maxima: signed in 1D (int), unsigned in 2D/3D (unsigned int) */
    uint32_t mx = 0, mx2 = 0;
    int32_t smx = 0, smx2 = 0;
    for (int k = 0; k < n; k++) {
        uint32_t a = abs_u(code[k]);
        if (g->dim == 1) {
            if ((int32_t)a > smx) smx = (int32_t)a;
            if (k && (int32_t)a > smx2) smx2 = (int32_t)a;
        } else {
            if (a > mx) mx = a;
            if (k && a > mx2) mx2 = a;
        }
    }
    if (g->dim == 1) { mx = (uint32_t)smx; mx2 = (uint32_t)smx2; }
    int fr1 = bitlen(mx);
    if (g->mode != ORC_OUTLIER) return (uint8_t)fr1;
    /* 1D_f32.cu:1165-1183 */
    int fr2 = bitlen(mx2);
    int ob = (bitlen(abs_u(code[0])) + 7) / 8;
    int c1 = fr1 ? W + fr1 * W : 0;
    int c2 = fr2 ? W + fr2 * W + ob : W + ob;
    if (c1 <= c2) return (uint8_t)fr1;
    return (uint8_t)(fr2 | 0x80 | ((ob - 1) << 5));
}

static void put_word_be(uint8_t* p, uint32_t w)
{
    p[0] = (uint8_t)(w >> 24); p[1] = (uint8_t)(w >> 16); p[2] = (uint8_t)(w >> 8); p[3] = (uint8_t)w;
}

/* Writes one block's payload at `out` (src/cuSZp_kernels_1D_f32.cu:1282-1660). */
static void block_write(const geom_t* g, const int32_t* code, uint8_t rb, uint8_t* out)
{
    const int n = g->n;
    uint32_t sel = 0, ob = 0, r = rb;
    if (g->mode == ORC_OUTLIER) { sel = rb >> 7; ob = ((rb & 0x60u) >> 5) + 1; r = rb & 0x1fu; }
    if (!sel && r == 0) return;
    uint32_t mag[64];
    uint32_t sign[2] = {0, 0};
    for (int k = 0; k < n; k++) {
        mag[k] = abs_u(code[k]);
        if (code[k] < 0) sign[k >> 5] |= 1u << (31 - (k & 31));
    }
    size_t o = 0;
    if (sel) {
        uint32_t m0 = mag[0];
        for (uint32_t i = 0; i < ob; i++) { out[o++] = (uint8_t)(m0 & 0xff); m0 >>= 8; }
        mag[0] = 0;   /* element 0 carries no plane bits once stored as outlier */
    }
    put_word_be(out + o, sign[0]); o += 4;
    if (n == 64) { put_word_be(out + o, sign[1]); o += 4; }
    for (uint32_t p = 0; p < r; p++) {
        for (int b = 0; b < n / 8; b++) {
            uint8_t v = 0;
            for (int j = 0; j < 8; j++) v |= (uint8_t)(((mag[8 * b + j] >> p) & 1u) << (7 - j));
            out[o++] = v;
        }
    }
}

/* ---------------------------------------------------------------- public API */

/*
 * Compress.  Returns the true stream length S (rate region + all payloads),
 * or 0 on a bad argument / insufficient capacity.  *ref_cmpSize receives the
 * value the reference's launcher reports (src/cuSZp_entry_1D_f32.cu:42-43,
 * src/cuSZp_entry_2D_f64.cu:46-47), which is short of S for single-CTA grids
 * and, in 2D/3D, by the rate-region padding.
 */
size_t orc_compress(const void* data, int type, int mode, int dim, size_t nbEle,
                    uint32_t dx, uint32_t dy, uint32_t dz, double eb, int fused,
                    uint8_t* out, size_t out_cap, size_t* ref_cmpSize)
{
    geom_t g;
    if (make_geom(&g, type, mode, dim, nbEle, dx, dy, dz)) return 0;
    if (dim != 1 && (dx % 4) != 0) return 0;
    /* f32: recip = 0.5f/eb in float; f64: 0.5f promoted, so 0.5/eb in double */
    double recip = (type == ORC_F32) ? (double)(0.5f / (float)eb) : 0.5 / eb;
    const uint64_t nb = g.nblocks;
    uint8_t* rates = (uint8_t*)calloc(nb ? nb : 1, 1);
    uint64_t* offs = (uint64_t*)malloc(sizeof(uint64_t) * (nb + 1));
    if (!rates || !offs) { free(rates); free(offs); return 0; }

    #pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < (int64_t)nb; b++) {
        int32_t code[64];
        block_codes(&g, data, (uint64_t)b, recip, fused, code);
        rates[b] = block_rate(&g, code);
    }
    offs[0] = 0;
    for (uint64_t b = 0; b < nb; b++) offs[b + 1] = offs[b] + size_from_rate(&g, rates[b]);
    const uint64_t total = offs[nb];
    const uint64_t S = g.rate_bytes + total;
    if (S > out_cap) { free(rates); free(offs); return 0; }

    memset(out, 0, g.rate_bytes);
    memcpy(out, rates, nb);
    #pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < (int64_t)nb; b++) {
        if (!size_from_rate(&g, rates[b])) continue;
        int32_t code[64];
        block_codes(&g, data, (uint64_t)b, recip, fused, code);
        block_write(&g, code, rates[b], out + g.rate_bytes + offs[b]);
    }
    if (ref_cmpSize) {
        uint64_t grid, glob;
        if (dim == 1) grid = ((uint64_t)nbEle + 32767) / 32768;
        else grid = (nb + (uint64_t)(32 * (type == ORC_F32 ? 16 : 32)) - 1) / (uint64_t)(32 * (type == ORC_F32 ? 16 : 32));
        glob = grid > 1 ? (uint32_t)total : 0;   /* 1D_f32.cu:702-708: only warp>0 writes */
        *ref_cmpSize = (size_t)(glob + (dim == 1 ? g.rate_bytes : nb));
    }
    free(rates); free(offs);
    return (size_t)S;
}

/* Decompress one block from its payload (src/cuSZp_kernels_1D_f32.cu:1820-2258). */
static void block_decode(const geom_t* g, const uint8_t* in, uint8_t rb, int32_t* q)
{
    const int n = g->n;
    uint32_t sel = 0, ob = 0, r = rb;
    if (g->mode == ORC_OUTLIER) { sel = rb >> 7; ob = ((rb & 0x60u) >> 5) + 1; r = rb & 0x1fu; }
    uint32_t mag[64] = {0};
    uint32_t sign[2] = {0, 0};
    size_t o = 0;
    uint32_t m0 = 0;
    if (sel) { for (uint32_t i = 0; i < ob; i++) m0 |= (uint32_t)in[o++] << (8 * i); }
    sign[0] = ((uint32_t)in[o] << 24) | ((uint32_t)in[o + 1] << 16) | ((uint32_t)in[o + 2] << 8) | in[o + 3];
    o += 4;
    if (n == 64) {
        sign[1] = ((uint32_t)in[o] << 24) | ((uint32_t)in[o + 1] << 16) | ((uint32_t)in[o + 2] << 8) | in[o + 3];
        o += 4;
    }
    for (uint32_t p = 0; p < r; p++) {
        for (int b = 0; b < n / 8; b++) {
            uint8_t v = in[o++];
            for (int j = 0; j < 8; j++) mag[8 * b + j] |= (uint32_t)((v >> (7 - j)) & 1) << p;
        }
    }
    if (sel) mag[0] = m0;
    for (int k = 0; k < n; k++) {
        int neg = (sign[k >> 5] >> (31 - (k & 31))) & 1;
        q[k] = neg ? wrap_neg((int32_t)mag[k]) : (int32_t)mag[k];
    }
}

static inline void store_val(const geom_t* g, void* out, size_t i, int32_t q, double eb)
{
    if (g->type == ORC_F32) ((float*)out)[i] = ((float)q * (float)eb) * 2.0f;
    else ((double*)out)[i] = ((double)q * eb) * 2.0;
}

/*
 * Decompress.  Blocks whose rate byte is 0 are left untouched, as in the
 * reference (src/cuSZp_kernels_1D_f32.cu:431); callers pre-zero `out`.
 * Returns the stream length consumed, or 0 on a bad argument.
 */
size_t orc_decompress(void* out, int type, int mode, int dim, size_t nbEle,
                      uint32_t dx, uint32_t dy, uint32_t dz, double eb,
                      const uint8_t* cmp, size_t cmp_len)
{
    geom_t g;
    if (make_geom(&g, type, mode, dim, nbEle, dx, dy, dz)) return 0;
    if (dim != 1 && (dx % 4) != 0) return 0;
    const uint64_t nb = g.nblocks;
    if (cmp_len < g.rate_bytes) return 0;
    uint64_t* offs = (uint64_t*)malloc(sizeof(uint64_t) * (nb + 1));
    if (!offs) return 0;
    offs[0] = 0;
    for (uint64_t b = 0; b < nb; b++) offs[b + 1] = offs[b] + size_from_rate(&g, cmp[b]);
    const uint64_t S = g.rate_bytes + offs[nb];
    if (S > cmp_len) { free(offs); return 0; }
    const double ebv = (type == ORC_F32) ? (double)(float)eb : eb;

    #pragma omp parallel for schedule(static)
    for (int64_t bb = 0; bb < (int64_t)nb; bb++) {
        uint64_t b = (uint64_t)bb;
        uint8_t rb = cmp[b];
        if (!size_from_rate(&g, rb)) continue;
        int32_t d[64], q;
        block_decode(&g, cmp + g.rate_bytes + offs[b], rb, d);
        const int lorenzo = g.mode != ORC_FIXED;
        if (g.dim == 1) {
            int32_t prev = 0;
            for (int k = 0; k < 32; k++) {
                q = lorenzo ? wrap_add(d[k], prev) : d[k];
                prev = q;
                uint64_t i = b * 32 + (uint64_t)k;
                if (i < g.nbEle) store_val(&g, out, i, q, ebv);
            }
        } else if (g.dim == 2) {
            uint64_t per_slice = (uint64_t)g.by * g.bx;
            uint64_t z = b / per_slice, rem = b % per_slice;
            uint64_t byi = rem / g.bx, bxi = rem % g.bx;
            int32_t prev_y = 0;
            for (int r = 0; r < 8; r++) {
                uint64_t y = byi * 8 + (uint64_t)r;
                if (y >= g.dy) continue;
                int32_t prev = 0;
                for (int c = 0; c < 8; c++) {
                    uint64_t x = bxi * 8 + (uint64_t)c;
                    if (x >= g.dx) continue;
                    int k = r * 8 + c;
                    if (!lorenzo) q = d[k];
                    else if (c == 0) { q = wrap_add(d[k], prev_y); prev_y = q; }
                    else q = wrap_add(d[k], prev);
                    prev = q;
                    store_val(&g, out, (size_t)((z * g.dy + y) * g.dx + x), q, ebv);
                }
            }
        } else {
            uint64_t per_slice = (uint64_t)g.by * g.bx;
            uint64_t bz = b / per_slice, rem = b % per_slice;
            uint64_t byi = rem / g.bx, bxi = rem % g.bx;
            int32_t prev_z = 0;
            for (int zz = 0; zz < 4; zz++) {
                uint64_t z = bz * 4 + (uint64_t)zz;
                if (z >= g.dz) continue;
                int32_t prev_y = 0;
                for (int yy = 0; yy < 4; yy++) {
                    uint64_t y = byi * 4 + (uint64_t)yy;
                    if (y >= g.dy) continue;
                    int32_t prev_x = 0;
                    for (int xx = 0; xx < 4; xx++) {
                        uint64_t x = bxi * 4 + (uint64_t)xx;
                        int k = zz * 16 + yy * 4 + xx;
                        if (!lorenzo) q = d[k];
                        else if (xx == 0) {
                            if (yy) q = wrap_add(d[k], prev_y);
                            else { q = wrap_add(d[k], prev_z); prev_z = q; }
                            prev_y = q;
                        } else q = wrap_add(d[k], prev_x);
                        prev_x = q;
                        if (x < g.dx) store_val(&g, out, (size_t)((z * g.dy + y) * g.dx + x), q, ebv);
                    }
                }
            }
        }
    }
    free(offs);
    return (size_t)S;
}

/* Geometry queries used by the tests. */
uint64_t orc_rate_bytes(int type, int mode, int dim, size_t nbEle, uint32_t dx, uint32_t dy, uint32_t dz)
{
    geom_t g;
    if (make_geom(&g, type, mode, dim, nbEle, dx, dy, dz)) return 0;
    return g.rate_bytes;
}
uint64_t orc_num_blocks(int type, int mode, int dim, size_t nbEle, uint32_t dx, uint32_t dy, uint32_t dz)
{
    geom_t g;
    if (make_geom(&g, type, mode, dim, nbEle, dx, dy, dz)) return 0;
    return g.nblocks;
}

/* Exact value range (src/examples/cuSZp.cpp:176-187 f32, :199-210 f64) and the
 * error bound the CLI derives from it: f32 eb*(max-min) in float, f64
 * eb*(float)(max-min). */
float orc_rel_eb(const void* data, int type, size_t n, float rel)
{
    if (!n) return 0.0f;
    if (type == ORC_F32) {
        const float* d = (const float*)data;
        float mx = d[0], mn = d[0];
        for (size_t i = 0; i < n; i++) { if (d[i] > mx) mx = d[i]; else if (d[i] < mn) mn = d[i]; }
        return rel * (mx - mn);
    }
    const double* d = (const double*)data;
    double mx = d[0], mn = d[0];
    for (size_t i = 0; i < n; i++) { if (d[i] > mx) mx = d[i]; else if (d[i] < mn) mn = d[i]; }
    return rel * (float)(mx - mn);
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

#ifndef CUSZP_H
#define CUSZP_H

/*
 * cuSZp -- error-bounded lossy compressor for f32/f64 arrays, B200 (sm_100a) build.
 *
 * Drop-in for the reference cuSZp interface:
 *   - enums and the two C-linkage entry points below keep the reference's names,
 *     values and signatures (reference include/cuSZp.h:20-45, src/cuSZp.cu:4,86),
 *     so `ctypes.CDLL("libcuSZp.so").cuSZp_compress` binds unchanged;
 *   - the 36 per-mode C++ entry points (cuSZp/cuSZp_entry_*.h), TimingGPU and the
 *     *_Yafan file helpers keep the reference's C++ signatures.
 * The compressed stream is byte-identical to the reference's for the same input,
 * error bound, mode and dimensionality.
 *
 * The extensions at the end (no counterpart in the reference) return a status,
 * take caller-provided workspace, never synchronize, and report the exact stream
 * length.
 */

#include <cuda_runtime.h>
#include <stddef.h>
#ifdef __cplusplus
#include <cstddef>
#include "cuSZp/cuSZp_utility.h"
#include "cuSZp/cuSZp_timer.h"
#include "cuSZp/cuSZp_entry_1D_f32.h"
#include "cuSZp/cuSZp_entry_1D_f64.h"
#include "cuSZp/cuSZp_entry_2D_f32.h"
#include "cuSZp/cuSZp_entry_2D_f64.h"
#include "cuSZp/cuSZp_entry_3D_f32.h"
#include "cuSZp/cuSZp_entry_3D_f64.h"
#endif
#include <stdio.h>

#ifdef __cplusplus
#define CUSZP_DEFAULT_STREAM = 0
extern "C" {
#else
#define CUSZP_DEFAULT_STREAM
#endif

typedef enum {
    CUSZP_DIM_1D = 1, // 1D processing (any array)
    CUSZP_DIM_2D = 2, // 2D processing: 8x8 blocks of each [dim_y x dim_x] slice
    CUSZP_DIM_3D = 3  // 3D processing: 4x4x4 blocks
} cuszp_dim_t;

typedef enum {
    CUSZP_MODE_FIXED   = 0, // no-delta fixed-length encoding
    CUSZP_MODE_PLAIN   = 1, // Lorenzo delta + fixed-length encoding
    CUSZP_MODE_OUTLIER = 2  // Lorenzo delta + outlier-preserving fixed-length encoding
} cuszp_mode_t;

typedef enum {
    CUSZP_TYPE_FLOAT  = 0,  // f32
    CUSZP_TYPE_DOUBLE = 1   // f64
} cuszp_type_t;

/*
 * Reference entry points (include/cuSZp.h:38-45 of the reference).
 * All pointers are device pointers.  dims = {x (fastest), y, z}; 1D ignores dims,
 * 2D/3D ignore nbEle and need dims.x % 4 == 0.  f64 data uses (double)errorBound.
 * compress: returns once the stream is complete and *cmpSize holds its length.
 *   The length reported is the true stream length S (rate region + every block
 *   payload).  The reference reports less than S for single-CTA launches and,
 *   in 2D/3D, omits the rate-region padding; cuSZp_reference_cmpsize() gives
 *   that value when it is wanted.
 * decompress: returns once d_decData holds the reconstruction.  Blocks encoded
 *   at rate 0 are written as 0.0 (the reference leaves them untouched and its
 *   CLI pre-zeroes the output, so results agree).
 * Errors are printed to stderr; compress then sets *cmpSize = 0.
 */
void cuSZp_compress(void* d_oriData, unsigned char* d_cmpBytes,
                    size_t nbEle, size_t* cmpSize, float errorBound,
                    cuszp_dim_t dim, uint3 dims, cuszp_type_t type, cuszp_mode_t mode,
                    cudaStream_t stream CUSZP_DEFAULT_STREAM);
void cuSZp_decompress(void* d_decData, unsigned char* d_cmpBytes,
                      size_t nbEle, size_t cmpSize, float errorBound,
                      cuszp_dim_t dim, uint3 dims, cuszp_type_t type, cuszp_mode_t mode,
                      cudaStream_t stream CUSZP_DEFAULT_STREAM);

/* ------------------------------------------------------------------ extensions
 * No counterpart in the reference: it has no error reporting, allocates and frees
 * scratch on every call (src/cuSZp_entry_1D_f32.cu:29-48) and blocks on a 4-byte
 * device-to-host copy.  These calls let a pipeline keep buffers resident and stay
 * asynchronous. */

typedef enum {
    CUSZP_SUCCESS                = 0,
    CUSZP_ERROR_INVALID_ARGUMENT = 1,
    CUSZP_ERROR_UNSUPPORTED      = 2, /* 2D/3D with dims.x % 4 != 0 */
    CUSZP_ERROR_CUDA             = 3,
    CUSZP_ERROR_TIMEOUT          = 4, /* a bounded device-side wait gave up */
    CUSZP_ERROR_WORKSPACE        = 5,
    CUSZP_ERROR_CAPACITY         = 6
} cuszp_status_t;

/* Capacity that holds the stream of any input of this geometry. */
size_t cuSZp_max_compressed_size(size_t nbEle, cuszp_dim_t dim, uint3 dims,
                                 cuszp_type_t type, cuszp_mode_t mode);

/* Device workspace one compress/decompress call of this geometry needs.  A new
 * workspace must be zero-filled once; every completed call leaves it zeroed. */
size_t cuSZp_workspace_size(size_t nbEle, cuszp_dim_t dim, uint3 dims,
                            cuszp_type_t type, cuszp_mode_t mode);

/* Enqueue compression on `stream` without synchronizing.  `cmpCapacity` is the size of
 * d_cmpBytes in bytes: nothing is written past it (cuSZp_max_compressed_size() always
 * suffices).  A stream that does not fit is reported by cuSZp_workspace_check() as
 * CUSZP_ERROR_CAPACITY; *d_cmpSize then still receives the length S it needs.  A
 * capacity below the rate region fails at once with CUSZP_ERROR_CAPACITY.  S is
 * written to *d_cmpSize (a device uint64) when d_cmpSize is non-null (~0 if a device
 * wait timed out).  Calls that share a workspace must be ordered (same stream or
 * explicit dependencies). */
int cuSZp_compress_async(const void* d_oriData, unsigned char* d_cmpBytes, size_t cmpCapacity,
                         size_t nbEle, float errorBound, cuszp_dim_t dim, uint3 dims,
                         cuszp_type_t type, cuszp_mode_t mode, void* d_workspace,
                         size_t workspaceBytes, unsigned long long* d_cmpSize, cudaStream_t stream);

/* Enqueue decompression on `stream` without synchronizing. */
int cuSZp_decompress_async(void* d_decData, const unsigned char* d_cmpBytes, size_t nbEle,
                           float errorBound, cuszp_dim_t dim, uint3 dims, cuszp_type_t type,
                           cuszp_mode_t mode, void* d_workspace, size_t workspaceBytes,
                           cudaStream_t stream);

/* Synchronize `stream`, then read and clear the workspace's error word:
 * CUSZP_SUCCESS; CUSZP_ERROR_TIMEOUT if a device-side wait gave up (the workspace is
 * re-zeroed so it can be reused); CUSZP_ERROR_CAPACITY if a compressed stream did not
 * fit its buffer, or a decompressed stream held rate bytes no valid stream holds.
 * Word 3 of a workspace (uint32 at byte offset 12, normally 0) caps every bounded
 * device-side wait of the calls using it at that many polls / sleep slices instead
 * of the default of about two seconds; tests use it to make a wait run out fast. */
int cuSZp_workspace_check(void* d_workspace, size_t workspaceBytes, cudaStream_t stream);
/* No reference counterpart.  Enqueue on `stream` a copy of the workspace's sticky error
 * word (0: no error) into *h_err (pinned host memory), without synchronizing; a caller
 * that polls for completion calls cuSZp_workspace_check() only when it is non-zero. */
int cuSZp_workspace_error_async(void* d_workspace, unsigned int* h_err, cudaStream_t stream);
/* No reference counterpart: one request of a serving lane in one host call.  `stream`
 * first waits for the work queued so far on `producer` (through `order`, recorded here;
 * skipped when `order` is NULL or producer == stream).  Then it runs
 * cuSZp_compress_async (compress != 0; d_in values, d_out stream of outCapacity bytes)
 * or cuSZp_decompress_async (d_in stream, d_out values) with the workspace.  Next it
 * copies the workspace's error word and stream length into the 16 pinned host bytes
 * at h_words: bytes 0-3 hold the error word, bytes 8-15 the compressed length.  Last,
 * it records `done` on `stream` (skipped when NULL).  h_words must not be the target
 * of a copy still in flight: the call zeroes it from the host first, which leaves an
 * empty array's length 0. */
int cuSZp_serve_submit_async(int compress, const void* d_in, void* d_out, size_t outCapacity, size_t nbEle,
                             float errorBound, cuszp_dim_t dim, uint3 dims, cuszp_type_t type, cuszp_mode_t mode,
                             void* d_workspace, size_t workspaceBytes, void* h_words, cudaStream_t producer,
                             cudaEvent_t order, cudaEvent_t done, cudaStream_t stream);

/* Synchronous forms with a status and the true stream length; workspace is taken
 * from the device's stream-ordered memory pool.  Compress writes nothing past
 * `cmpCapacity` bytes of d_cmpBytes; when the stream does not fit it returns
 * CUSZP_ERROR_CAPACITY and *cmpSize receives the capacity needed. */
int cuSZp_compress_ex(const void* d_oriData, unsigned char* d_cmpBytes, size_t cmpCapacity,
                      size_t nbEle, size_t* cmpSize, float errorBound, cuszp_dim_t dim, uint3 dims,
                      cuszp_type_t type, cuszp_mode_t mode, cudaStream_t stream);
int cuSZp_decompress_ex(void* d_decData, const unsigned char* d_cmpBytes, size_t nbEle,
                        size_t cmpSize, float errorBound, cuszp_dim_t dim, uint3 dims,
                        cuszp_type_t type, cuszp_mode_t mode, cudaStream_t stream);

/* The compressed size the reference launcher reports for a stream of length
 * `streamBytes` (src/cuSZp_entry_1D_f32.cu:42-43, src/cuSZp_entry_2D_f64.cu:46-47). */
size_t cuSZp_reference_cmpsize(size_t streamBytes, size_t nbEle, cuszp_dim_t dim, uint3 dims,
                               cuszp_type_t type, cuszp_mode_t mode);

/* Relative error bound as the reference CLI derives it for `-eb rel`
 * (examples/cuSZp.cpp:176-187 f32, :199-210 f64): rel * (max - min), evaluated in
 * float (f64: rel * (float)(max - min)); min/max are reduced on the device. */
int cuSZp_rel_error_bound(const void* d_data, size_t nbEle, cuszp_type_t type, float rel,
                          float* errorBound, cudaStream_t stream);

/* Device min/max with the CLI's NaN semantics, returned as doubles. */
int cuSZp_value_range(const void* d_data, size_t nbEle, cuszp_type_t type,
                      double* minValue, double* maxValue, cudaStream_t stream);

/* ------------------------------------------------------------------ batches
 * Many arrays compressed (or decompressed) by ONE persistent kernel launch that
 * pulls tiles of all arrays from a device work queue; every array keeps its own
 * look-back chain, so each array's stream is byte-identical to cuSZp_compress's.
 * A plan owns the device item table and workspace; executing it only enqueues
 * kernels, so it can be captured in a CUDA graph and replayed.  All arrays of a
 * plan share dim and type; modes may differ per array. */

typedef struct {
    const void* d_in;      /* compress: data;   decompress: stream */
    void* d_out;           /* compress: stream buffer (>= cuSZp_max_compressed_size); decompress: data */
    size_t nbEle;
    uint3 dims;
    float errorBound;      /* absolute, or relative to the array's value range when rel != 0 */
    int rel;               /* compress only: derive eb = errorBound*(max-min) on the device */
    cuszp_mode_t mode;
} cuszp_batch_item_t;

typedef struct cuszp_batch_plan* cuszp_batch_plan_t;

int cuSZp_batch_plan_create(cuszp_batch_plan_t* plan, int count, const cuszp_batch_item_t* items,
                            cuszp_dim_t dim, cuszp_type_t type, int compress);
/* Same, with every device step (stream-ordered allocation, table upload, map build)
 * enqueued on `stream` and no synchronization: for request loops that keep other
 * work in flight. */
int cuSZp_batch_plan_create_async(cuszp_batch_plan_t* plan, int count, const cuszp_batch_item_t* items,
                                  cuszp_dim_t dim, cuszp_type_t type, int compress, cudaStream_t stream);
/* Re-targets a plan at a new list of arrays (same dim, type and direction), reusing its
 * device buffers (grown when the new list needs more) and its pinned staging memory, so
 * a request loop keeps one plan per lane instead of creating and destroying one per
 * batch.  Stream-ordered on `stream`, no device synchronization; work that still uses
 * the plan must be ordered before `stream`.  The kernel pair chosen for the plan is kept
 * where the new arrays allow it. */
int cuSZp_batch_plan_update(cuszp_batch_plan_t plan, int count, const cuszp_batch_item_t* items,
                            cudaStream_t stream);
/* Enqueue the batch on `stream`; stream lengths go to d_sizes[count] (device u64). */
int cuSZp_batch_plan_execute(cuszp_batch_plan_t plan, unsigned long long* d_sizes, cudaStream_t stream);
/* Autotuner: time each tile shape (warps per CTA x blocks per warp) and CTAs per SM on
 * this plan's arrays and keep the fastest (runs the batch several times). */
int cuSZp_batch_plan_tune(cuszp_batch_plan_t plan, unsigned long long* d_sizes, int reps, cudaStream_t stream);
int cuSZp_batch_plan_set_config(cuszp_batch_plan_t plan, int variant, int ctasPerSM);
int cuSZp_batch_plan_config(cuszp_batch_plan_t plan, int* warps, int* blocksPerWarp, int* ctasPerSM);
/* The kernel pair in use: variant index, threads per CTA, and whether it is the TMA
 * pair (variant 0, chosen by default when every array and stream starts on a 16-byte
 * boundary; set_config returns CUSZP_ERROR_UNSUPPORTED for it otherwise). */
int cuSZp_batch_plan_variant(cuszp_batch_plan_t plan, int* variant, int* threadsPerBlock, int* tma);
/* Absolute bounds the last execution used (derived on the device for rel items). */
int cuSZp_batch_plan_eb(cuszp_batch_plan_t plan, float* errorBounds, cudaStream_t stream);
/* Synchronize and report a timed-out device wait (CUSZP_ERROR_TIMEOUT). */
int cuSZp_batch_plan_check(cuszp_batch_plan_t plan, cudaStream_t stream);
/* No reference counterpart.  Enqueue on `stream` a copy of the plan's sticky error word
 * (0: no error) into *h_err (pinned host memory), without synchronizing: a caller that
 * polls for completion reads it once the stream's work is done, and calls
 * cuSZp_batch_plan_check() only when it is non-zero. */
int cuSZp_batch_plan_error_async(cuszp_batch_plan_t plan, unsigned int* h_err, cudaStream_t stream);
void cuSZp_batch_plan_destroy(cuszp_batch_plan_t plan);
/* Release a plan once the work already enqueued on `stream` is done (stream-ordered free). */
void cuSZp_batch_plan_destroy_async(cuszp_batch_plan_t plan, cudaStream_t stream);

/* Compression without any allocation -- no counterpart in the reference.  For callers
 * that cannot allocate device memory when they compress (allocation forbidden or too
 * slow where they run, or all memory owned by a host framework): the look-back scratch
 * is a fixed 1 MiB array inside this library on each device, so the call allocates
 * nothing and needs no workspace.  Limit: 131,066 tiles of look-back state, i.e. 1D
 * arrays of at most 536,838,144 elements (tiles of 4,096 elements, counted in whole
 * 32,768-element rate granules) and 2D/3D arrays of at most 8,388,224 data blocks
 * (tiles of 64 blocks; 536,846,336 elements when every block is whole); larger arrays
 * are rejected with CUSZP_ERROR_WORKSPACE and a message on stderr.  Asynchronous on `stream`; the stream
 * length goes to *d_cmpSize (device uint64, required), or ~0 if a bounded device-side
 * wait gave up.  The first call on a device looks up the array's device address; make
 * that first call before any stream capture.  All calls on a device share the array:
 * calls that can overlap on the GPU race and must be ordered (same stream or explicit
 * dependencies).  Output bytes are identical to cuSZp_compress_async's. */
int cuSZp_compress_noalloc(const void* d_oriData, unsigned char* d_cmpBytes, size_t nbEle,
                           float errorBound, cuszp_dim_t dim, uint3 dims, cuszp_type_t type,
                           cuszp_mode_t mode, unsigned long long* d_cmpSize, cudaStream_t stream);

/* Version string of the library. */
const char* cuSZp_version(void);

#ifdef __cplusplus
}
#endif

#endif // CUSZP_H

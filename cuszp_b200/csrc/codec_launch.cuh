// codec_launch.cuh -- host-side geometry, workspace sizing and kernel launches for
// the fused codec.  Internal to libcuSZp; the exported C ABI lives in api.cu.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "codec.cuh"

namespace cuszp {

// Status codes of the extended C ABI (mirrored in include/cuSZp.h).
enum Status : int {
    OK = 0,
    E_ARG = 1,          // invalid argument (enum, shape, pointer, size)
    E_UNSUPPORTED = 2,  // shape the format does not define (2D/3D with dims.x % 4 != 0)
    E_CUDA = 3,         // a CUDA runtime call failed
    E_TIMEOUT = 4,      // a bounded device-side wait gave up
    E_WORKSPACE = 5,    // workspace missing or too small
    E_CAPACITY = 6,     // output buffer smaller than the stream
};

struct Problem {
    int type;   // 0 f32, 1 f64
    int mode;   // 0 fixed, 1 plain, 2 outlier
    int dim;    // 1, 2, 3
    Geom g;
};

// Builds the block geometry; returns a Status.  Reference geometry:
// 1D src/cuSZp_entry_1D_f32.cu:20-22 + kernels_1D_f32.cu:47 (rate region),
// 2D src/cuSZp_entry_2D_f64.cu:21-25, 3D src/cuSZp_entry_3D_f64.cu:21-25.
int make_problem(Problem& p, int type, int mode, int dim, size_t nbEle, unsigned dx, unsigned dy, unsigned dz);

// Bytes of workspace (header + one status word per tile) a call needs.
size_t workspace_bytes(const Problem& p);

// Worst-case stream length for this geometry (all blocks at rate 32, plus the
// largest outlier prefix), i.e. a capacity that can never overflow.
size_t max_stream_bytes(const Problem& p);

// Enqueue the fused kernels.  `ws` must point at a zeroed workspace of at least
// workspace_bytes(p) (the kernels leave it zeroed again, except for the error
// word and the stream length in the header).  eb is the absolute error bound
// (float for f32, double for f64 -- the generic API widens a float).
// d_size: when non-null, the kernel writes the stream length there (~0 after a
// timed-out wait), as the workspace header's `total`.
int launch_compress(const Problem& p, const void* d_in, uint8_t* d_cmp, double eb, void* ws, cudaStream_t s,
                    unsigned long long* d_size = nullptr);
int launch_decompress(const Problem& p, void* d_out, const uint8_t* d_cmp, double eb, void* ws, cudaStream_t s);

// The TMA kernels: whether the environment allows them (CUSZP_NO_TMA=1 turns them
// off), and the 2D/3D tensor map of an array (false when the driver rejects the
// geometry, e.g. a row pitch that is not a multiple of 16 bytes).  *grouped: the map
// is a grouped 2D map (kGroup whole blocks per box), to be recorded in Geom::grouped.
bool tma_allowed();
bool make_block_map(CUtensorMap* m, const Problem& p, const void* data, bool* grouped);

// Per-device kernel set-up shared by every launch path, thread-safe and cached per
// (device, kernel): enable_dynamic_smem sets a kernel's dynamic shared-memory limit the
// first time it is needed on the current device (false if the runtime refused; the next
// call tries again); resident_ctas is the kernel's occupancy in CTAs per SM (0 if the
// query failed); sm_count is the current device's SM count (0 on failure).
bool enable_dynamic_smem(const void* fn, size_t bytes);
int resident_ctas(const void* fn, int threads, size_t smem);
int sm_count();

// Value range (min, max) of a device array with the reference CLI's semantics
// (examples/cuSZp.cpp:176-187): NaNs are skipped unless the first element is NaN.
// Writes two values of the array's type to d_minmax; needs range_ws_bytes() of workspace.
size_t range_ws_bytes(size_t n);
int launch_range(const void* d_in, size_t n, int type, void* d_minmax, void* ws, cudaStream_t s);

}  // namespace cuszp

// batch.cuh -- many arrays in one persistent launch.
//
// Every array keeps its own stream layout and its own chain of look-back tiles;
// the arrays' tiles are numbered into one global sequence that CTAs pull from a
// single atomic ticket, so short arrays fill the tail of long ones and the whole
// batch is one launch (capturable in a CUDA graph: no host synchronization, the
// workspace resets itself).  A per-tile table maps a global tile to its array.
#pragma once

#include <cstdint>
#include "codec.cuh"

namespace cuszp {

// One array of a batch.  Host-built; `eb` may be overwritten on the device by the
// batched value-range pass (relative bounds).
struct BatchItem {
    const void* in;        // compress: data;   decompress: stream
    void* out;             // compress: stream; decompress: data
    Geom g;
    uint64_t tile_start;   // first global tile of this array
    uint64_t chunk_start;  // first value-range chunk of this array
    uint64_t nchunks;
    float eb;              // absolute error bound used by the codec
    float rel;             // relative bound (when the batch derives eb on the device)
    int32_t mode;          // 0 fixed, 1 plain, 2 outlier
    int32_t pad;
};

// Batch workspace: WsHeader, then status[total_tiles] (u64), tile_map[total_tiles]
// (u32, padded to 16 B), range partials[total_chunks] (2 x f64).
struct BatchLayout {
    uint64_t total_tiles;
    uint64_t total_chunks;
    size_t status_off, map_off, part_off, bytes;
};

constexpr uint64_t kRangeChunk = 1 << 16;   // elements per value-range partial

inline BatchLayout batch_layout(uint64_t total_tiles, uint64_t total_chunks)
{
    BatchLayout L;
    L.total_tiles = total_tiles;
    L.total_chunks = total_chunks;
    L.status_off = sizeof(WsHeader);
    L.map_off = L.status_off + 8 * (total_tiles ? total_tiles : 1);
    L.part_off = (L.map_off + 4 * (total_tiles ? total_tiles : 1) + 15) / 16 * 16;
    L.bytes = L.part_off + 16 * (total_chunks ? total_chunks : 1);
    return L;
}

}  // namespace cuszp

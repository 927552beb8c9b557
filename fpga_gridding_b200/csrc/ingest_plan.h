// How the drop-in splits its visibilities into upload chunks (host code, no
// CUDA).
#pragma once

#include <algorithm>
#include <cstddef>

namespace b200 {

// Points per chunk ahead of the last one: chunk k is gridded while chunk
// k + 1 crosses PCIe.  The first chunks are small (kFirstChunk, doubling up
// to kHeadChunkMax) so that the gridding starts soon after the call; later
// ones large, as each chunk pays the pipeline's fixed costs again (a 10 M
// cap measured 31.1 ms end to end at plain_large against 31.4 ms with 5 M).
constexpr size_t kIngestChunk = size_t(5) << 20;
constexpr size_t kFirstChunk = size_t(5) << 18;
constexpr size_t kHeadChunkMax = size_t(10) << 20;
// The last chunk holds about this fraction of the points (all of them when
// there are at most kIngestChunk).  It is gridded band by band (rows of
// coarse tiles), and each band of the result goes back to the host as soon
// as no later band can touch it, so the download of the grid overlaps the
// gridding.  The earlier chunks should be gridded by the time it has landed
// (uploads run a little faster than the gridding), and the less of the
// gridding is left after the upload, the sooner the rows become final: at
// plain_large 0.30 measured 29.8 ms end to end, 0.25 29.8 ms, 0.35
// 30.2 ms, 0.45 30.9 ms (a CUDA timeline of 0.45 showed the gridding idle
// for 3 ms while the large last chunk uploaded, then the heavy central
// bands holding back half the grid's download).
constexpr double kTailFraction = 0.30;

// Chunk boundaries for n points: chunk k covers [bound[k], bound[k + 1]),
// the last chunk is the tail.  At most max_chunks chunks (max_chunks >= 2);
// bound must hold max_chunks + 1 entries.  Returns the number of chunks
// (at least 1; the only chunk is empty when n == 0).
inline int ingest_chunks(size_t n, int max_chunks, size_t* bound)
{
    const size_t tail = n <= kIngestChunk ? n
                                          : (size_t)((double)n * kTailFraction);
    const size_t head = n - tail;
    int chunks = 0;
    bound[0] = 0;
    for (size_t at = 0, size = kFirstChunk; at < head;)
    {
        size_t e = std::min(head, at + size);
        // no short remainder, and room left for the tail
        if (head - e < kFirstChunk || chunks == max_chunks - 2) e = head;
        bound[++chunks] = e;
        at = e;
        size = std::min(kHeadChunkMax, 2 * size);
    }
    bound[++chunks] = n;
    return chunks;
}

}  // namespace b200

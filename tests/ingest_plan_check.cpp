// Checks b200::ingest_chunks (fpga_gridding_b200/csrc/ingest_plan.h): the
// chunks cover the points in order without gaps or overlaps, there are at
// most max_chunks of them, only the last may be empty (when there are no
// points at all), the ones ahead of the last grow from kFirstChunk up to at
// most kHeadChunkMax (the last of them may also take a short remainder), and
// the last holds about kTailFraction of the points.  Prints "ok" and exits
// 0, or prints the first violation and exits 1.
#include <cmath>
#include <cstdio>
#include <vector>

#include "ingest_plan.h"

using namespace b200;

static int check(size_t n, int max_chunks)
{
    std::vector<size_t> bound(max_chunks + 1, ~size_t(0));
    const int c = ingest_chunks(n, max_chunks, bound.data());
    auto fail = [&](const char* what) {
        std::printf("n=%zu max=%d chunks=%d: %s\n", n, max_chunks, c, what);
        return 1;
    };
    if (c < 1 || c > max_chunks) return fail("chunk count");
    if (bound[0] != 0 || bound[c] != n) return fail("coverage");
    for (int k = 0; k < c; ++k)
        if (bound[k + 1] < bound[k] || (bound[k + 1] == bound[k] && n > 0))
            return fail("order or empty chunk");
    const size_t tail = n - bound[c - 1];
    if (n <= kIngestChunk && c != 1) return fail("small job not one chunk");
    if (n > kIngestChunk &&
        std::fabs((double)tail - kTailFraction * (double)n) > 1.0)
        return fail("tail fraction");
    for (int k = 0; k + 1 < c; ++k)
    {
        const size_t size = bound[k + 1] - bound[k];
        const bool last_head = k + 2 == c;
        if (!last_head && size > kHeadChunkMax) return fail("head chunk too big");
        if (k == 0 && !last_head && size != kFirstChunk)
            return fail("first chunk size");
        if (last_head && c < max_chunks && size > kHeadChunkMax + kFirstChunk)
            return fail("last head chunk too big");
    }
    return 0;
}

int main()
{
    const size_t ns[] = {0, 1, 1000, kIngestChunk, kIngestChunk + 1,
                         11u << 20, 39244800, 164370927, 392000000,
                         4000000000ull};
    for (size_t n : ns)
        for (int max_chunks : {2, 3, 5, 15})
            if (check(n, max_chunks)) return 1;
    std::printf("ok\n");
    return 0;
}

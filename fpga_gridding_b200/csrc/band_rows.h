// Which rows of the grid a band-ordered gridding pass has finished, step by
// step (host code, no CUDA).  Used by the drop-in to copy finished rows back
// while later bands still grid.
#pragma once

#include <algorithm>
#include <vector>

namespace b200 {

// A run of grid rows [r0, r1) that becomes final at `step`.
struct FinalRows
{
    int step;
    long long r0, r1;
};

// Band b holds the points of grid rows [b << row_shift, (b + 1) << row_shift)
// (clipped to the grid); their footprints reach at most `halo` rows beyond
// the band.  Bands are gridded in `order` (a permutation of
// 0 .. num_bands - 1).  A row is final once every band that can reach it has
// been gridded.  Returns, in step order, the maximal runs of rows that
// become final at each step; each row of the grid appears in exactly one.
inline std::vector<FinalRows> final_rows(int num_bands, const int* order,
                                         int row_shift, long long halo,
                                         long long grid_size)
{
    std::vector<FinalRows> out;
    std::vector<unsigned char> sent((size_t)grid_size, 0);
    std::vector<unsigned char> done((size_t)num_bands, 0);
    const long long H = 1ll << row_shift;
    auto final_row = [&](long long q) {
        if (sent[(size_t)q]) return false;
        // bands whose reach [b*H - halo, (b+1)*H - 1 + halo] holds q
        const long long b0 = std::max(0ll, (q - halo) >> row_shift);
        const long long b1 = std::min((long long)num_bands - 1,
                                      (q + halo) >> row_shift);
        for (long long x = b0; x <= b1; ++x)
            if (!done[(size_t)x]) return false;
        return true;
    };
    for (int i = 0; i < num_bands; ++i)
    {
        const int b = order[i];
        done[(size_t)b] = 1;
        // only rows within this band's reach can have changed state
        const long long lo = std::max(0ll, (long long)b * H - halo);
        const long long hi = std::min(grid_size, (long long)(b + 1) * H +
                                                     halo);
        for (long long r = lo; r < hi;)
        {
            if (!final_row(r))
            {
                ++r;
                continue;
            }
            long long e = r + 1;
            while (e < hi && final_row(e)) ++e;
            for (long long q = r; q < e; ++q) sent[(size_t)q] = 1;
            out.push_back(FinalRows{i, r, e});
            r = e;
        }
    }
    return out;
}

}  // namespace b200

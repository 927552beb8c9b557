// Checks b200::final_rows (fpga_gridding_b200/csrc/band_rows.h) on many
// band layouts: every grid row is returned exactly once, never before every
// band that can reach it has been gridded, and runs come in step order.
// Prints "ok" and exits 0, or prints the first violation and exits 1.
#include <cstdio>
#include <vector>

#include "band_rows.h"

static int check(int grid_size, int row_shift, int halo, bool outside_in)
{
    const long long H = 1ll << row_shift;
    const int nb = (int)((grid_size + H - 1) / H);
    // the drop-in's outside-in order (0, last, 1, last - 1, ...), or the
    // bands from the last to the first
    std::vector<int> order(nb);
    if (outside_in)
        for (int i = 0, lo = 0, hi = nb - 1; lo <= hi; ++i)
            order[i] = (i & 1) ? hi-- : lo++;
    else
        for (int i = 0; i < nb; ++i) order[i] = nb - 1 - i;
    std::vector<int> step_of_band(nb);
    for (int i = 0; i < nb; ++i) step_of_band[order[i]] = i;
    std::vector<int> seen(grid_size, 0);
    int last_step = -1;
    for (const b200::FinalRows& f :
         b200::final_rows(nb, order.data(), row_shift, halo, grid_size))
    {
        if (f.step < last_step || f.r0 >= f.r1 || f.r0 < 0 ||
            f.r1 > grid_size)
        {
            std::printf("bad run G=%d rs=%d halo=%d step %d [%lld, %lld)\n",
                        grid_size, row_shift, halo, f.step, f.r0, f.r1);
            return 1;
        }
        last_step = f.step;
        for (long long r = f.r0; r < f.r1; ++r)
        {
            ++seen[r];
            // every band whose points lie within `halo` rows of r
            for (int b = 0; b < nb; ++b)
            {
                const long long b_lo = b * H - halo;
                const long long b_hi = (b + 1) * H - 1 + halo;
                if (r >= b_lo && r <= b_hi && step_of_band[b] > f.step)
                {
                    std::printf("row %lld of G=%d rs=%d halo=%d returned at "
                                "step %d before band %d (step %d)\n", r,
                                grid_size, row_shift, halo, f.step, b,
                                step_of_band[b]);
                    return 1;
                }
            }
        }
    }
    for (int r = 0; r < grid_size; ++r)
        if (seen[r] != 1)
        {
            std::printf("row %d of G=%d rs=%d halo=%d returned %d times\n", r,
                        grid_size, row_shift, halo, seen[r]);
            return 1;
        }
    return 0;
}

int main()
{
    const int grids[] = {1, 63, 64, 65, 200, 256, 1000, 1024, 4097};
    const int shifts[] = {4, 6, 8};
    const int halos[] = {0, 1, 3, 36, 70, 127};
    for (int g : grids)
        for (int rs : shifts)
            for (int h : halos)
                for (int oi = 0; oi < 2; ++oi)
                {
                    if (((long long)g >> rs) > 16) continue;   // <= 16 bands
                    if (check(g, rs, h, oi == 0)) return 1;
                }
    std::printf("ok\n");
    return 0;
}

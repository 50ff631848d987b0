// merge.h -- host-side MERGE_VOID on cube records and the small host helpers
// of the post-processing.
#pragma once

#include <stdint.h>
#include <vector>

namespace avism {

struct MergeIn {
    int32_t nvoid;
    int low1, low2, periodic;
    float dx, rx1, lado0plus;
    const int32_t *x0, *x1, *y0, *y1, *z0, *z1, *icx, *icy, *icz, *father;
    const float *rix, *rfx, *riy, *rfy, *riz, *rfz;
    const int32_t *indice;          // cube ids by volume, largest first
    // neighbour lists (CSR over cubes, 0-based ids): cubes of the same father
    // whose 1-cell halo boxes overlap, with the squared distance of the initial
    // centres and whether it lies inside the cube's ball-search radius
    const int32_t *nbr_start, *nbr;
    const float *nbr_d2;
    const uint8_t *nbr_inball;
};

// ball-search radius**2 of MERGE_VOID for a cube of volume v (src/voidfinding.f90:913-916)
float merge_ball_r2(float vol, float dx);

struct MergeOut {
    std::vector<int32_t> uvoid;     // -1 main void, >0 owner id
    std::vector<float> gxc, gyc, gzc, volnew;
    std::vector<int32_t> paint_time;   // order in which each cube painted its box
    std::vector<int32_t> paint_owner;  // void id painted by that cube
    int32_t nvoid2 = 0;
};

void merge_cubes_host(const MergeIn &in, MergeOut &out);

}  // namespace avism

// nbr_iter.cuh -- walks a particle's neighbour list in the reference order.
//
// The list of the particle at cell-order position t (see StepArgs) holds the
// real neighbours' positions in the order of MCM/mcm_ll_neighbours.f90
// (same-material neighbours, then contacts, :239-252); the particle itself
// follows for disctype 1 (:288-299), then the ghost neighbours (:181-229,
// :254-266).  The visitors receive cell-order positions (real) or ghost
// indices.
#pragma once
#include "kernels.h"

namespace mcm {

__device__ __forceinline__ void cell_coords(int key, const int *gl, int &bx, int &by, int &bz) {
    bx = key % gl[0] + 1;
    int r = key / gl[0];
    by = r % gl[1] + 1;
    bz = r / gl[1] + 1;
}

constexpr unsigned kPosMask = 0x3ffffffu;   // position bits of a neighbour entry

// Real neighbours stored for position t (the self entry of disctype 1 is not stored).
__device__ __forceinline__ int stored_neighbours(const StepArgs &a, int t) {
    return a.nnbr[t] - (a.prm.disctype == 1 ? 1 : 0);
}

// FR: void(int position, bool is_self); FG: void(int ghost)
template <typename FR, typename FG>
__device__ __forceinline__ void for_each_neighbour(const StepArgs &a, const DevGrid &g, int t, FR &&real, FG &&ghost) {
    (void)g;
    const unsigned *list = a.nidx + (size_t)t * a.nstride;
    const int nreal = stored_neighbours(a, t);
    for (int k = 0; k < nreal; ++k) real((int)(list[k] & kPosMask), false);
    if (a.prm.disctype == 1) real(t, true);
    const int gn = a.gnnbr[t];
    for (int k = 0; k < gn; ++k) ghost(a.gnbr[(size_t)k * a.npad + t]);
}

}  // namespace mcm

// nbr_iter.cuh -- walks a particle's neighbour list in the reference order.
//
// The list of the particle at cell-order position t (see StepArgs) is
// decoded row by row: for the rows (nz, my) of its 27-cell neighbourhood in
// the z, y order of MCM/mcm_ll_neighbours.f90:122-124, `cnt` one-byte
// offsets into the contiguous range of positions that the row's three
// x-adjacent cells occupy.  Same-material neighbours first, then contacts
// (:239-252), then the particle itself for disctype 1 (:288-299), then ghost
// neighbours (:181-229, :254-266).  The visitors receive cell-order positions
// (real) or ghost indices.
#pragma once
#include "kernels.h"

namespace mcm {

__device__ __forceinline__ void cell_coords(int key, const int *gl, int &bx, int &by, int &bz) {
    bx = key % gl[0] + 1;
    int r = key / gl[0];
    by = r % gl[1] + 1;
    bz = r / gl[1] + 1;
}

// FR: void(int position, bool is_self); FG: void(int ghost)
template <typename FR, typename FG>
__device__ __forceinline__ void for_each_neighbour(const StepArgs &a, const DevGrid &g, int t, FR &&real, FG &&ghost) {
    const int key = a.ckey[t];
    const int np = a.npad;
    if (key >= 0) {
        int bx, by, bz;
        cell_coords(key, g.gridlim, bx, by, bz);
        const int lo0 = bx > 1 ? bx - 1 : 1, hi0 = bx < g.gridlim[0] ? bx + 1 : g.gridlim[0];
        const int lo1 = by > 1 ? by - 1 : 1, hi1 = by < g.gridlim[1] ? by + 1 : g.gridlim[1];
        const int lo2 = bz > 1 ? bz - 1 : 1, hi2 = bz < g.gridlim[2] ? bz + 1 : g.gridlim[2];
        unsigned int word = 0;
        int nb = 0, w = 0;
        const int passes = a.nmat > 1 ? 2 : 1;
        for (int pass = 0; pass < passes; ++pass) {
            unsigned long long hdr = a.nhdr[(size_t)pass * np + t];
            int r = 0;
            for (int nz = lo2; nz <= hi2; ++nz) {
                for (int my = lo1; my <= hi1; ++my, ++r) {
                    int cnt = (int)((hdr >> (7 * r)) & 127ull);
                    if (cnt == 0) continue;
                    const int rs = a.cell_start[(int)cell_key(lo0, my, nz, g.gridlim)];
                    for (int c = 0; c < cnt; ++c) {
                        if (nb == 0) {
                            word = a.nlist[(size_t)w * np + t];
                            ++w;
                            nb = 4;
                        }
                        const int off = (int)(word & 255u);
                        word >>= 8;
                        --nb;
                        real(rs + off, false);
                    }
                }
            }
        }
    }
    if (a.prm.disctype == 1) real(t, true);
    const int gn = a.gnnbr[t];
    for (int k = 0; k < gn; ++k) ghost(a.gnbr[(size_t)k * np + t]);
}

}  // namespace mcm

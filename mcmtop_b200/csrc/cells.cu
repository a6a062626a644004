// cells.cu -- device cell list, boundary ghosts and the warp-cooperative
// neighbour search of the MCM explicit step.
//
// Replaces MCM/mcm_setuplist.f90 (linked-list grid), MCM/mcm_ghost_setup.f90
// (ghost particles) and MCM/mcm_ll_neighbours.f90 (27-cell search).  The cell
// list is a counting sort by cell key (one radix digit of width = number of
// cells) followed by a per-cell sort into descending reference index, which is
// the order in which the reference walks a head-inserted linked list.  Rows of
// three x-adjacent cells are contiguous in that order, so the search visits
// candidates exactly in the reference's z/y/x cell order and the neighbour
// lists come out as the same sequences, not only the same sets.
//
// Compiled without fused multiply-add: the cell index int(gridsize*(x-gridmin))
// and the predicate d^2 < (h_i+h_j)^2 are evaluated exactly as the reference
// does in FP64, so borderline pairs resolve identically.
#include "kernels.h"

namespace mcm {

// ------------------------------------------------------------- grid set-up
// MCM/mcm_setuplist.f90:240-291 (one thread).
__global__ void k_grid_setup(StepArgs a) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (a.status->code) return;
    const DevParams &P = a.prm;
    const double factor = 2.0;
    DevGrid g;
    for (int i = 0; i < 3; ++i) {
        g.gridmin[i] = 0.0;
        g.gridlim[i] = 1;
        g.gridsize[i] = 1.0 / (factor * P.hmax);
    }
    bool bad = false;
    for (int i = 0; i < P.ndim; ++i) {
        double span = 0.0;
        switch (P.planes.type[i]) {
            case 1:
                g.gridmin[i] = a.bbox[i] - 0.01 * P.hmax;
                span = g.gridsize[i] * (a.bbox[3 + i] - g.gridmin[i]);
                if (!(span < 1.0e9)) { bad = true; span = 0; }
                g.gridlim[i] = (int)span + 1;
                break;
            case 2:
                g.gridmin[i] = P.planes.bx[0][i];
                span = g.gridsize[i] * (a.bbox[3 + i] - g.gridmin[i]);
                if (!(span < 1.0e9)) { bad = true; span = 0; }
                g.gridlim[i] = (int)span + 1;
                break;
            case 3:
                span = g.gridsize[i] * (P.planes.bx[1][i] - a.bbox[i]);
                if (!(span < 1.0e9)) { bad = true; span = 0; }
                g.gridlim[i] = (int)span + 1;
                g.gridmin[i] = P.planes.bx[1][i] - g.gridlim[i] * factor * P.hmax;
                break;
            case 4:
                g.gridmin[i] = P.planes.bx[0][i];
                span = g.gridsize[i] * (P.planes.bx[1][i] - P.planes.bx[0][i]);
                if (!(span < 1.0e9)) { bad = true; span = 0; }
                g.gridlim[i] = (int)span;
                g.gridlim[i] = g.gridlim[i] > 1 ? g.gridlim[i] : 1;
                g.gridsize[i] = (double)(float)g.gridlim[i] / (P.planes.bx[1][i] - P.planes.bx[0][i]);
                break;
        }
    }
    for (int i = 0; i < P.ndim; ++i) {
        int c0 = P.planes.code[0][i];
        if (c0 == 1 || c0 == 2) {
            g.gridlim[i] = g.gridlim[i] + 1;
            g.gridmin[i] = g.gridmin[i] - (1.0 / g.gridsize[i]);
        }
        int c1 = P.planes.code[1][i];
        if (c1 == 1 || c1 == 2) g.gridlim[i] = g.gridlim[i] + 1;
    }
    g.pad = 0;
    g.ncells = (long long)g.gridlim[0] * g.gridlim[1] * g.gridlim[2];
    if (bad || g.ncells >= (1LL << 31)) {
        raise_status(a.status, MCM_EGRID_TOO_LARGE);
    } else if (g.ncells > a.cell_cap) {
        a.status->req_cells = g.ncells;
        raise_status(a.status, MCM_EGRID_OVERFLOW);
    }
    *a.grid = g;
    *a.ngp = 0;
}

// --------------------------------------------------------------- cell keys
// MCM/mcm_setuplist.f90:316-345: particles outside the grid get no cell.
__global__ void k_cell_keys(StepArgs a) {
    if (a.status->code) return;
    const DevGrid g = *a.grid;
    const int ndim = a.prm.ndim;
    const double *X[3] = {a.F.f[FX], a.F.f[FY], a.F.f[FZ]};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        int box[3] = {1, 1, 1};
        bool in = true;
        for (int j = 0; j < ndim; ++j) {
            double t = g.gridsize[j] * (X[j][i] - g.gridmin[j]);
            // int() of the reference truncates toward zero; out-of-range values are outside anyway
            if (!(t > -2.0e9 && t < 2.0e9)) { in = false; continue; }
            box[j] = (int)t + 1;
            if (box[j] < 1 || box[j] > g.gridlim[j]) in = false;
        }
        int key = in ? (int)cell_key(box[0], box[1], box[2], g.gridlim) : kNoCell;
        a.key[i] = key;
        if (key >= 0) atomicAdd(&a.cell_count[key], 1);
    }
}

// ------------------------------------------------------------------- scan
// Exclusive scan of cell_count[0, ncells) into cell_start[0, ncells].
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanChunk = kScanThreads * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int *smem, int &total) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = (lane < (int)(blockDim.x >> 5)) ? smem[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        smem[lane] = s;
    }
    __syncthreads();
    int prefix = (w > 0 ? smem[w - 1] : 0) + x - v;
    total = smem[(blockDim.x >> 5) - 1];
    __syncthreads();
    return prefix;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_blocks(const int *in, int *out, int *sums, const long long *np_dev,
                                                              long long n_static) {
    __shared__ int smem[32];
    long long n = np_dev ? *np_dev : n_static;
    long long base = (long long)blockIdx.x * kScanChunk;
    int v[kScanItems];
    int local = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        long long idx = base + (long long)threadIdx.x * kScanItems + k;
        v[k] = (idx < n) ? in[idx] : 0;
        local += v[k];
    }
    int total;
    int pre = block_exclusive_scan(local, smem, total);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        long long idx = base + (long long)threadIdx.x * kScanItems + k;
        if (idx < n) out[idx] = pre;
        pre += v[k];
    }
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_sums(int *sums, int nblocks) {
    __shared__ int smem[32];
    int carry = 0;
    for (int base = 0; base < nblocks; base += kScanThreads) {
        int idx = base + threadIdx.x;
        int v = idx < nblocks ? sums[idx] : 0;
        int total;
        int pre = block_exclusive_scan(v, smem, total);
        if (idx < nblocks) sums[idx] = pre + carry;
        carry += total;
    }
    if (threadIdx.x == 0) sums[nblocks] = carry;
}

__global__ void k_scan_add(int *out, const int *sums, const long long *np_dev, long long n_static, int nblocks) {
    long long n = np_dev ? *np_dev : n_static;
    long long base = (long long)blockIdx.x * kScanChunk;
    int add = sums[blockIdx.x];
    for (int k = threadIdx.x; k < kScanChunk; k += blockDim.x) {
        long long idx = base + k;
        if (idx < n) out[idx] += add;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = sums[nblocks];
}

static void device_exclusive_scan(const int *in, int *out, int *sums, const long long *n_dev, long long cap,
                                  cudaStream_t s) {
    int nblocks = (int)((cap + kScanChunk - 1) / kScanChunk);
    if (nblocks < 1) nblocks = 1;
    k_scan_blocks<<<nblocks, kScanThreads, 0, s>>>(in, out, sums, n_dev, cap);
    k_scan_sums<<<1, kScanThreads, 0, s>>>(sums, nblocks);
    k_scan_add<<<nblocks, 256, 0, s>>>(out, sums, n_dev, cap, nblocks);
}

// --------------------------------------------------------------- scatter
__global__ void k_cell_scatter(StepArgs a) {
    if (a.status->code) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        int key = a.key[i];
        if (key < 0) continue;
        int slot = atomicSub(&a.cell_count[key], 1) - 1;
        a.cell_list[a.cell_start[key] + slot] = i;
    }
}

// Per-cell order: descending reference index (head insertion in
// MCM/mcm_setuplist.f90:336-340 over i = 1..np ascending).
__global__ void k_cell_sort(StepArgs a) {
    if (a.status->code) return;
    const long long ncells = a.grid->ncells;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncells;
         c += (long long)gridDim.x * blockDim.x) {
        int s = a.cell_start[c], e = a.cell_start[c + 1];
        if (e - s < 2) continue;
        for (int k = s + 1; k < e; ++k) {
            int v = a.cell_list[k];
            int ov = a.F.orig[v];
            int m = k - 1;
            while (m >= s && a.F.orig[a.cell_list[m]] < ov) {
                a.cell_list[m + 1] = a.cell_list[m];
                --m;
            }
            a.cell_list[m + 1] = v;
        }
    }
}

static int grid_blocks(long long work, int threads) {
    long long b = (work + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148LL * 32) b = 148LL * 32;
    return (int)b;
}

void launch_grid_setup(const StepArgs &a, cudaStream_t s) { k_grid_setup<<<1, 32, 0, s>>>(a); }

void launch_cell_build(const StepArgs &a, cudaStream_t s) {
    cudaMemsetAsync(a.cell_count, 0, sizeof(int) * (size_t)a.cell_cap, s);
    k_cell_keys<<<grid_blocks(a.n, 256), 256, 0, s>>>(a);
    device_exclusive_scan(a.cell_count, a.cell_start, a.scan_sums, &a.grid->ncells, a.cell_cap, s);
    k_cell_scatter<<<grid_blocks(a.n, 256), 256, 0, s>>>(a);
    k_cell_sort<<<grid_blocks(a.cell_cap, 128), 128, 0, s>>>(a);
}

// ------------------------------------------------------------------ ghosts
// MCM/mcm_ghost_setup.f90:29-284.  Planes in the order xmin xmax ymin ymax
// zmin zmax; each plane walks the 2-D layer of source cells in the
// reference's loop order and emits, per source cell, its members in chain
// order.  A destination cell receives the ghosts of exactly one source cell;
// its chain order (newest first) is the reverse of the emission order.

struct PlaneGeom {
    int d, side, src, dst, a_dim, b_dim;
    long long L;
};

__device__ __forceinline__ PlaneGeom plane_geom(const StepArgs &a, int plane) {
    PlaneGeom p;
    p.d = plane >> 1;
    p.side = plane & 1;
    const int *gl = a.grid->gridlim;
    int code = a.prm.planes.code[p.side][p.d];
    if (p.side == 0) p.src = (code == 1) ? 2 : gl[p.d] - 1;
    else p.src = (code == 1) ? gl[p.d] - 1 : 2;
    p.dst = (p.side == 0) ? 1 : gl[p.d];
    if (p.d == 0) { p.a_dim = 2; p.b_dim = 1; }
    else if (p.d == 1) { p.a_dim = 2; p.b_dim = 0; }
    else { p.a_dim = 1; p.b_dim = 0; }
    p.L = (long long)gl[p.a_dim] * gl[p.b_dim];
    return p;
}

__device__ __forceinline__ void layer_cells(const StepArgs &a, const PlaneGeom &p, long long t, int &cs, int &cd) {
    const int *gl = a.grid->gridlim;
    int bcount = gl[p.b_dim];
    int aa = (int)(t / bcount) + 1, bb = (int)(t % bcount) + 1;
    int c[3];
    c[p.a_dim] = aa; c[p.b_dim] = bb;
    c[p.d] = p.src;
    cs = (int)cell_key(c[0], c[1], c[2], gl);
    c[p.d] = p.dst;
    cd = (int)cell_key(c[0], c[1], c[2], gl);
}

__global__ void k_ghost_count(StepArgs a, int plane) {
    if (a.status->code) return;
    PlaneGeom p = plane_geom(a, plane);
    if (p.L > a.layer_cap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) raise_status(a.status, MCM_EGRID_OVERFLOW);
        return;
    }
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < p.L; t += (long long)gridDim.x * blockDim.x) {
        int cs, cd;
        layer_cells(a, p, t, cs, cd);
        int nreal = a.cell_start[cs + 1] - a.cell_start[cs];
        int ng = a.gcell[cs].y;
        if (nreal > 0 && ng > 0) raise_status(a.status, MCM_EGHOST_LAYER, cs);
        int cnt = nreal > 0 ? nreal : ng;
        if (cnt > 0) {
            int dreal = a.cell_start[cd + 1] - a.cell_start[cd];
            if (dreal > 0 || a.gcell[cd].y > 0) raise_status(a.status, MCM_EGHOST_LAYER, cd);
        }
        a.layer_count[t] = cnt;
    }
}

__global__ void __launch_bounds__(kScanThreads) k_ghost_layer_scan(StepArgs a, int plane) {
    __shared__ int smem[32];
    if (a.status->code) return;
    PlaneGeom p = plane_geom(a, plane);
    int carry = 0;
    for (long long base = 0; base < p.L; base += kScanThreads) {
        long long idx = base + threadIdx.x;
        int v = idx < p.L ? a.layer_count[idx] : 0;
        int total;
        int pre = block_exclusive_scan(v, smem, total);
        if (idx < p.L) a.layer_off[idx] = pre + carry;
        carry += total;
    }
    if (threadIdx.x == 0) {
        int base = *a.ngp;
        *a.plane_base = base;
        long long need = (long long)base + carry;
        if (need > a.ghost_cap) {
            if (need > a.status->req_ngp) a.status->req_ngp = (int)need;
            raise_status(a.status, MCM_EGHOST_OVERFLOW);
        }
        *a.ngp = (int)need;
    }
}

__global__ void k_ghost_emit(StepArgs a, int plane) {
    if (a.status->code) return;
    PlaneGeom p = plane_geom(a, plane);
    const double *mult = a.prm.planes.mult[plane];
    const double *add = a.prm.planes.add[plane];
    const int base = *a.plane_base;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < p.L; t += (long long)gridDim.x * blockDim.x) {
        int cnt = a.layer_count[t];
        if (cnt == 0) continue;
        int cs, cd;
        layer_cells(a, p, t, cs, cd);
        int g0 = base + a.layer_off[t];
        a.gcell[cd] = make_int2(g0, cnt);
        int rs = a.cell_start[cs];
        int nreal = a.cell_start[cs + 1] - rs;
        int2 src = a.gcell[cs];
        for (int r = 0; r < cnt; ++r) {
            int g = g0 + r;
            if (nreal > 0) {
                // MCM/mcm_ghost_setup.f90:324-355 (create_ghost_from_real)
                int j = a.cell_list[rs + r];
                a.gpar[g] = j;
                a.gmat[g] = a.F.mat[j];
                a.gmass[g] = a.F.f[FMASS][j];
                a.gh[g] = a.F.f[FH][j];
                a.ghold[g] = a.F.f[FHOLD][j];
                a.grho[g] = a.F.f[FRHO][j];
                a.gx[g] = a.F.f[FX][j] * mult[0] + add[0];
                a.gy[g] = a.F.f[FY][j] * mult[1] + add[1];
                a.gz[g] = a.F.f[FZ][j] * mult[2] + add[2];
                a.gvx[g] = a.F.f[FVX][j] * mult[0];
                a.gvy[g] = a.F.f[FVY][j] * mult[1];
                a.gvz[g] = a.F.f[FVZ][j] * mult[2];
            } else {
                // MCM/mcm_ghost_setup.f90:392-423 (create_ghost_from_ghost); chain order = newest first
                int q = src.x + src.y - 1 - r;
                a.gpar[g] = a.gpar[q];
                a.gmat[g] = a.gmat[q];
                a.gmass[g] = a.gmass[q];
                a.gh[g] = a.gh[q];
                a.ghold[g] = a.ghold[q];
                a.grho[g] = a.grho[q];
                a.gx[g] = a.gx[q] * mult[0] + add[0];
                a.gy[g] = a.gy[q] * mult[1] + add[1];
                a.gz[g] = a.gz[q] * mult[2] + add[2];
                a.gvx[g] = a.gvx[q] * mult[0];
                a.gvy[g] = a.gvy[q] * mult[1];
                a.gvz[g] = a.gvz[q] * mult[2];
            }
        }
    }
}

void launch_ghosts(const StepArgs &a, cudaStream_t s) {
    cudaMemsetAsync(a.gcell, 0, sizeof(int2) * (size_t)a.cell_cap, s);
    for (int plane = 0; plane < 6; ++plane) {
        int code = a.prm.planes.code[plane & 1][plane >> 1];
        if (code != 1 && code != 2) continue;
        if ((plane >> 1) >= a.prm.ndim) continue;
        int blocks = grid_blocks(a.layer_cap, 256);
        if (blocks > 592) blocks = 592;
        k_ghost_count<<<blocks, 256, 0, s>>>(a, plane);
        k_ghost_layer_scan<<<1, kScanThreads, 0, s>>>(a, plane);
        k_ghost_emit<<<blocks, 256, 0, s>>>(a, plane);
    }
}

// ------------------------------------------------------------------ search
// MCM/mcm_ll_neighbours.f90:96-299.  One warp per particle; the candidates of
// a row of three x-adjacent cells are spread over the lanes and accepted
// pairs are compacted in lane order with ballots, which keeps the
// reference's order.  A block handles a tile of 32 consecutive particles and
// writes its lists column-major with coalesced stores.

constexpr int kSearchWarps = 8;
constexpr int kSearchTile = 32;

size_t search_smem_bytes(const StepArgs &a) {
    return sizeof(int) * ((size_t)kSearchTile * (a.stride + a.gstride) + (size_t)kSearchWarps * (a.stride + a.gstride) +
                          2 * kSearchTile);
}

__device__ __forceinline__ double exact_d2(double xi, double yi, double zi, double xj, double yj, double zj, int ndim) {
    double d = __dsub_rn(xj, xi);
    double s = __dmul_rn(d, d);
    if (ndim > 1) { d = __dsub_rn(yj, yi); s = __dadd_rn(s, __dmul_rn(d, d)); }
    if (ndim > 2) { d = __dsub_rn(zj, zi); s = __dadd_rn(s, __dmul_rn(d, d)); }
    return s;
}

__global__ void __launch_bounds__(kSearchWarps * 32) k_search(StepArgs a) {
    extern __shared__ int smem[];
    if (a.status->code) return;
    const int stride = a.stride, gstride = a.gstride;
    int *s_nbr = smem;                                    // [tile][stride]
    int *s_gnbr = s_nbr + kSearchTile * stride;           // [tile][gstride]
    int *s_cont = s_gnbr + kSearchTile * gstride;         // [warps][stride]
    int *s_gcont = s_cont + kSearchWarps * stride;        // [warps][gstride]
    int *s_nn = s_gcont + kSearchWarps * gstride;         // [tile]
    int *s_gn = s_nn + kSearchTile;                       // [tile]

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    const DevGrid g = *a.grid;
    const int ndim = a.prm.ndim;
    const double *X = a.F.f[FX], *Y = a.F.f[FY], *Z = a.F.f[FZ], *H = a.F.f[FH];
    const int *MAT = a.F.mat;
    const int tile0 = blockIdx.x * kSearchTile;
    const bool with_self = (a.prm.disctype == 1);

    for (int p = warp; p < kSearchTile; p += kSearchWarps) {
        const int i = tile0 + p;
        int nn = 0, gn = 0;
        double mind = 1.0e20;
        bool inside = false;
        if (i < a.n && a.key[i] >= 0) {
            inside = true;
            const double xi = X[i], yi = Y[i], zi = Z[i], hi = H[i];
            const int mati = MAT[i];
            int box[3] = {1, 1, 1}, lo[3] = {1, 1, 1}, hi_[3] = {1, 1, 1};
            const double xv[3] = {xi, yi, zi};
            for (int j = 0; j < ndim; ++j) {
                box[j] = (int)(g.gridsize[j] * (xv[j] - g.gridmin[j])) + 1;
                lo[j] = box[j] - 1 > 1 ? box[j] - 1 : 1;
                hi_[j] = box[j] + 1 < g.gridlim[j] ? box[j] + 1 : g.gridlim[j];
            }
            int n_same = 0, n_cont = 0, g_same = 0, g_cont = 0;
            double lmin = 1.0e20, lminc = 1.0e20;
            int *my_nbr = s_nbr + p * stride;
            int *my_gnbr = s_gnbr + p * gstride;
            int *my_cont = s_cont + warp * stride;
            int *my_gcont = s_gcont + warp * gstride;
            for (int nz = lo[2]; nz <= hi_[2]; ++nz) {
                for (int my = lo[1]; my <= hi_[1]; ++my) {
                    const int k0 = (int)cell_key(lo[0], my, nz, g.gridlim);
                    const int k1 = k0 + (hi_[0] - lo[0]);
                    // real particles of the row, in reference chain order
                    const int rs = a.cell_start[k0], re = a.cell_start[k1 + 1];
                    for (int b = rs; b < re; b += 32) {
                        const int idx = b + lane;
                        bool acc = false, same = false;
                        int j = -1;
                        if (idx < re) {
                            j = a.cell_list[idx];
                            if (j != i) {
                                double d2 = exact_d2(xi, yi, zi, X[j], Y[j], Z[j], ndim);
                                double hs = __dadd_rn(H[j], hi);
                                double hsq = __dmul_rn(hs, hs);
                                if (d2 < hsq) {
                                    acc = true;
                                    same = (MAT[j] == mati);
                                    if (same) lmin = fmin(lmin, d2);
                                    else lminc = fmin(lminc, d2);
                                }
                            }
                        }
                        unsigned bs = __ballot_sync(0xffffffffu, acc && same);
                        unsigned bc = __ballot_sync(0xffffffffu, acc && !same);
                        if (acc && same) {
                            int pos = n_same + __popc(bs & lt_mask);
                            if (pos < stride) my_nbr[pos] = j;
                        } else if (acc) {
                            int pos = n_cont + __popc(bc & lt_mask);
                            if (pos < stride) my_cont[pos] = j;
                        }
                        n_same += __popc(bs);
                        n_cont += __popc(bc);
                    }
                    // ghost cells of the row, one cell at a time (newest ghost first)
                    if (a.prm.boundary) {
                        for (int c = k0; c <= k1; ++c) {
                            const int2 gc = a.gcell[c];
                            for (int b = 0; b < gc.y; b += 32) {
                                const int r = b + lane;
                                bool acc = false, same = false;
                                int q = -1;
                                if (r < gc.y) {
                                    q = gc.x + gc.y - 1 - r;
                                    double d2 = exact_d2(xi, yi, zi, a.gx[q], a.gy[q], a.gz[q], ndim);
                                    double hs = __dadd_rn(a.gh[q], hi);
                                    double hsq = __dmul_rn(hs, hs);
                                    if (d2 < hsq) {
                                        acc = true;
                                        same = (a.gmat[q] == mati);
                                        if (same) lmin = fmin(lmin, d2);
                                        else lminc = fmin(lminc, d2);
                                    }
                                }
                                unsigned bs = __ballot_sync(0xffffffffu, acc && same);
                                unsigned bc = __ballot_sync(0xffffffffu, acc && !same);
                                if (acc && same) {
                                    int pos = g_same + __popc(bs & lt_mask);
                                    if (pos < gstride) my_gnbr[pos] = q;
                                } else if (acc) {
                                    int pos = g_cont + __popc(bc & lt_mask);
                                    if (pos < gstride) my_gcont[pos] = q;
                                }
                                g_same += __popc(bs);
                                g_cont += __popc(bc);
                            }
                        }
                    }
                }
            }
            __syncwarp();
            // kernel contact (contacttype 0): contacts follow the same-material list
            for (int k = lane; k < n_cont; k += 32) {
                int pos = n_same + k;
                if (pos < stride && k < stride) my_nbr[pos] = my_cont[k];
            }
            nn = n_same + n_cont;
            if (a.prm.boundary) {
                for (int k = lane; k < g_cont; k += 32) {
                    int pos = g_same + k;
                    if (pos < gstride && k < gstride) my_gnbr[pos] = my_gcont[k];
                }
                gn = g_same + g_cont;
            } else {
                gn = g_same;
            }
            // mindist (MCM/mcm_ll_neighbours.f90:152,167,252,268)
            double m = fmin(lmin, lminc);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
            mind = sqrt(m);
            if (with_self) {
                // MCM/mcm_ll_neighbours.f90:288-299
                if (lane == 0 && nn < stride) my_nbr[nn] = i;
                nn += 1;
            }
            __syncwarp();
        }
        if (lane == 0) {
            s_nn[p] = nn;
            s_gn[p] = gn;
            if (i < a.n) {
                a.nnbr[i] = nn;
                a.gnnbr[i] = gn;
                if (a.prm.tcrit_opt == 2 || a.prm.diag) a.F.f[FMINDIST][i] = inside ? mind : 1.0e20;
                if (nn > stride) { atomicMax(&a.status->req_stride, nn); raise_status(a.status, MCM_ENBR_OVERFLOW, i); }
                if (gn > gstride) { atomicMax(&a.status->req_gstride, gn); raise_status(a.status, MCM_ENBR_OVERFLOW, i); }
                atomicMax(&a.status->max_nbr, nn);
                atomicMax(&a.status->max_gnbr, gn);
            }
        }
    }
    __syncthreads();
    // coalesced column-major write-out of the tile
    int maxn = 0, maxg = 0;
    for (int p = 0; p < kSearchTile; ++p) {
        maxn = max(maxn, min(s_nn[p], stride));
        maxg = max(maxg, min(s_gn[p], gstride));
    }
    for (int t = threadIdx.x; t < maxn * kSearchTile; t += blockDim.x) {
        int k = t / kSearchTile, p = t % kSearchTile;
        int i = tile0 + p;
        if (i < a.npad) a.nbr[(size_t)k * a.npad + i] = (k < s_nn[p]) ? s_nbr[p * stride + k] : -1;
    }
    for (int t = threadIdx.x; t < maxg * kSearchTile; t += blockDim.x) {
        int k = t / kSearchTile, p = t % kSearchTile;
        int i = tile0 + p;
        if (i < a.npad) a.gnbr[(size_t)k * a.npad + i] = (k < s_gn[p]) ? s_gnbr[p * gstride + k] : -1;
    }
}

void launch_search(const StepArgs &a, cudaStream_t s) {
    size_t smem = search_smem_bytes(a);
    static size_t configured = 0;
    if (smem > 48 * 1024 && smem > configured) {
        cudaFuncSetAttribute(k_search, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        configured = smem;
    }
    int blocks = (a.n + kSearchTile - 1) / kSearchTile;
    k_search<<<blocks, kSearchWarps * 32, smem, s>>>(a);
}

}  // namespace mcm

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
#include "nbr_iter.cuh"

namespace mcm {

// ------------------------------------------------------------- grid set-up
// MCM/mcm_setuplist.f90:30-81 (one thread).
__global__ void k_grid_setup(StepArgs a) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (a.status->code) return;
    const DevParams &P = a.prm;
    const double factor = 2.0;
    const double hmax = a.hmax[0];   // fixed, or the last mcm_update_h's maximum
    DevGrid g;
    for (int i = 0; i < 3; ++i) {
        g.gridmin[i] = 0.0;
        g.gridlim[i] = 1;
        g.gridsize[i] = 1.0 / (factor * hmax);
    }
    bool bad = false;
    for (int i = 0; i < P.ndim; ++i) {
        double span = 0.0;
        switch (P.planes.type[i]) {
            case 1:
                g.gridmin[i] = a.bbox[i] - 0.01 * hmax;
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
                g.gridmin[i] = P.planes.bx[1][i] - g.gridlim[i] * factor * hmax;
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
    g.hcut = 0.0;   // raised by k_cell_records
    *a.grid = g;
    *a.ngp = 0;
    *a.n_inside = 0;
}

// --------------------------------------------------------------- cell keys
// MCM/mcm_setuplist.f90:110-135: particles outside the grid get no cell.
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
        // lanes of one cell add their count once (the particles are mostly in
        // cell order, so a warp holds few distinct cells)
        const unsigned act = __activemask();
        const unsigned grp = __match_any_sync(act, key);
        if (key >= 0 && (threadIdx.x & 31) == __ffs(grp) - 1) atomicAdd(&a.cell_count[key], __popc(grp));
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
// Particles outside the grid (llpointer = -1 in the reference) take the
// positions after the last cell; they have no neighbours and are never one.
__global__ void k_cell_scatter(StepArgs a) {
    if (a.status->code) return;
    const int base_out = a.cell_start[a.grid->ncells];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        int key = a.key[i];
        const unsigned act = __activemask();
        const unsigned grp = __match_any_sync(act, key);
        if (key < 0) {
            a.cell_list[base_out + atomicAdd(a.n_inside, 1)] = i;
            continue;
        }
        // one atomic per cell and warp: the group's slots are the n below the
        // returned count, one per lane in lane order
        const int lane = threadIdx.x & 31, lead = __ffs(grp) - 1;
        int top = 0;
        if (lane == lead) top = atomicSub(&a.cell_count[key], __popc(grp));
        top = __shfl_sync(grp, top, lead);
        int slot = top - 1 - __popc(grp & ((1u << lane) - 1u));
        a.cell_list[a.cell_start[key] + slot] = i;
    }
}

// Candidate records in cell order (positions at neighbour time).
// Candidate records in cell order: FP64 position and h, and an FP32 copy of
// the position relative to the origin of the particle's own cell, which the
// search uses to decide all but the near-tie candidates.
__global__ void __launch_bounds__(256) k_cell_records(StepArgs a) {
    __shared__ unsigned long long smax[8];
    if (a.status->code) return;
    const double *X = a.F.f[FX], *Y = a.F.f[FY], *Z = a.F.f[FZ], *H = a.F.f[FH];
    const DevGrid g = *a.grid;
    unsigned long long hbits = 0ull;   // h > 0: the bit pattern orders like the value
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += gridDim.x * blockDim.x) {
        int i = a.cell_list[p];
        const double x = X[i], y = Y[i], z = Z[i], h = H[i];
        a.cpos[p] = make_double4(x, y, z, h);
        if (a.pos_of) a.pos_of[i] = p;
        a.cmat[p] = a.F.mat[i];
        const int key = a.key[i];
        a.ckey[p] = key;
        float4 r = make_float4(0.f, 0.f, 0.f, (float)h);
        if (key >= 0) {
            int bx, by, bz;
            cell_coords(key, g.gridlim, bx, by, bz);
            r.x = (float)(x - cell_origin(g, 0, bx));
            r.y = (float)(y - cell_origin(g, 1, by));
            r.z = (float)(z - cell_origin(g, 2, bz));
            const unsigned long long hb = (unsigned long long)__double_as_longlong(h);
            hbits = hb > hbits ? hb : hbits;
        }
        a.cposf[p] = r;
        // the windowed search's copy: x relative to the grid origin, so that the
        // candidates of a row's two or three cells share one frame in x
        if (a.cposg) a.cposg[p] = make_float4((float)(x - g.gridmin[0]), r.y, r.z, r.w);
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long v = __shfl_xor_sync(0xffffffffu, hbits, o);
        hbits = v > hbits ? v : hbits;
    }
    if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = hbits;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) hbits = smax[w] > hbits ? smax[w] : hbits;
        atomicMax(reinterpret_cast<unsigned long long *>(&a.grid->hcut), hbits);
    }
}

// Per-cell order: descending reference index (head insertion in
// MCM/mcm_setuplist.f90:126-130 over i = 1..np ascending), the order of the
// reference's lists.  With xsort (steps whose sums do not follow that order)
// ascending x, ties by descending reference index: a row of x-adjacent cells
// is then one x-sorted range, which the search windows in x.
// One warp per cell: each lane takes one of the cell's particles (cells of up
// to 32, the common case) or up to kSortPer of them, and counts how many of
// the cell's particles come before each (a rank sort: the order is total, so
// the ranks are a permutation); all ranks are known before any entry is
// written back.  Cells of more than 32 * kSortPer particles are sorted by
// insertion in one lane.
constexpr int kSortPer = 4;
__device__ __forceinline__ bool cell_before(bool xs, double xa, int oa, double xb, int ob) {
    return xs ? (xa < xb || (xa == xb && oa > ob)) : oa > ob;
}
__global__ void __launch_bounds__(256) k_cell_sort(StepArgs a) {
    if (a.status->code) return;
    const long long ncells = a.grid->ncells;
    const bool xs = a.prm.xsort != 0;
    const double *X = a.F.f[FX];
    const int lane = threadIdx.x & 31;
    const long long nw = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long c = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < ncells; c += nw) {
        const int s = a.cell_start[c], e = a.cell_start[c + 1];
        const int n = e - s;
        if (n < 2) continue;   // warp-uniform
        if (n <= 32) {
            // one particle per lane (the common case)
            const bool on = lane < n;
            const int v = on ? a.cell_list[s + lane] : 0;
            const int o = on ? a.F.orig[v] : 0;
            const double x = (on && xs) ? X[v] : 0.0;
            int rank = 0;
            for (int k = 0; k < n; ++k) {
                const double xb = __shfl_sync(0xffffffffu, x, k);
                const int ob = __shfl_sync(0xffffffffu, o, k);
                rank += cell_before(xs, xb, ob, x, o) ? 1 : 0;
            }
            __syncwarp();
            if (on) a.cell_list[s + rank] = v;
            __syncwarp();
        } else if (n <= 32 * kSortPer) {
            int v[kSortPer], o[kSortPer], rank[kSortPer];
            double x[kSortPer];
#pragma unroll
            for (int u = 0; u < kSortPer; ++u) {
                const int j = lane + 32 * u;
                v[u] = j < n ? a.cell_list[s + j] : 0;
                o[u] = j < n ? a.F.orig[v[u]] : 0;
                x[u] = (j < n && xs) ? X[v[u]] : 0.0;
                rank[u] = 0;
            }
            for (int k0 = 0; k0 < n; k0 += 32) {
                // the chunk's keys, one per lane, broadcast by shuffles
                const int uk = k0 >> 5;
                double xk = 0.0;
                int ok = 0;
#pragma unroll
                for (int u = 0; u < kSortPer; ++u)
                    if (u == uk) { xk = x[u]; ok = o[u]; }
                const int m = n - k0 < 32 ? n - k0 : 32;
                for (int k = 0; k < m; ++k) {
                    const double xb = __shfl_sync(0xffffffffu, xk, k);
                    const int ob = __shfl_sync(0xffffffffu, ok, k);
#pragma unroll
                    for (int u = 0; u < kSortPer; ++u)
                        if (lane + 32 * u < n && cell_before(xs, xb, ob, x[u], o[u])) ++rank[u];
                }
            }
            __syncwarp();
#pragma unroll
            for (int u = 0; u < kSortPer; ++u)
                if (lane + 32 * u < n) a.cell_list[s + rank[u]] = v[u];
            __syncwarp();
        } else if (lane == 0) {
            for (int k = s + 1; k < e; ++k) {
                const int v = a.cell_list[k];
                const int ov = a.F.orig[v];
                const double xv = xs ? X[v] : 0.0;
                int m = k - 1;
                while (m >= s) {
                    const int u = a.cell_list[m];
                    if (!cell_before(xs, xv, ov, xs ? X[u] : 0.0, a.F.orig[u])) break;
                    a.cell_list[m + 1] = u;
                    --m;
                }
                a.cell_list[m + 1] = v;
            }
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
    {
        long long b = (a.cell_cap + 7) / 8;   // 8 warps (cells) per block
        if (b > 148LL * 8) b = 148LL * 8;
        k_cell_sort<<<(unsigned)(b < 1 ? 1 : b), 256, 0, s>>>(a);
    }
    k_cell_records<<<grid_blocks(a.n, 256) < 148 * 8 ? grid_blocks(a.n, 256) : 148 * 8, 256, 0, s>>>(a);
}

// ------------------------------------------------------------- re-sorting
// Permutes the particle state into the cell order of the last step's list,
// so that the gathers of later steps walk memory nearly in order.  Results do
// not depend on it: every order used by the step is defined by cell keys and
// reference indices, not by storage positions.
__global__ void k_permute_int(const int *src, int *dst, const int *perm, int n) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) dst[p] = src[perm[p]];
}
__global__ void k_copy_back_int(const int *src, int *dst, int n) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) dst[p] = src[p];
}

// A group of nf consecutive fields (field k of the group at base + k np),
// permuted into tmp (padding copied as it is) in one pass over the positions.
__global__ void k_permute_group(const double *base, size_t np, int nf, double *tmp, const int *perm, int n) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < np; p += (size_t)gridDim.x * blockDim.x) {
        const size_t j = p < (size_t)n ? (size_t)perm[p] : p;
        for (int k = 0; k < nf; ++k) tmp[k * np + p] = base[k * np + j];
    }
}

void launch_reorder(const StepArgs &a, cudaStream_t s) {
    const int b = grid_blocks(a.n, 256);
    // the fields lie at F.f[0] + f npad: each group is one contiguous range
    const size_t np = (size_t)a.npad;
    for (int f0 = 0; f0 < NFIELD; f0 += kReorderGroup) {
        const int nf = NFIELD - f0 < kReorderGroup ? NFIELD - f0 : kReorderGroup;
        k_permute_group<<<b, 256, 0, s>>>(a.F.f[f0], np, nf, a.reorder_grp, a.cell_list, a.n);
        cudaMemcpyAsync(a.F.f[f0], a.reorder_grp, sizeof(double) * nf * np, cudaMemcpyDeviceToDevice, s);
    }
    int *ints[4] = {a.F.mat, a.F.dispbc, a.F.orig, a.F.ptype};
    for (int *p : ints) {
        k_permute_int<<<b, 256, 0, s>>>(p, (int *)a.reorder_tmp, a.cell_list, a.n);
        k_copy_back_int<<<b, 256, 0, s>>>((const int *)a.reorder_tmp, p, a.n);
    }
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
    // axes this plane mirrors (bit d: x_d -> -x_d + add_d); composed along ghost chains
    const int flips = (mult[0] < 0.0 ? 1 : 0) | (mult[1] < 0.0 ? 2 : 0) | (mult[2] < 0.0 ? 4 : 0);
    // one warp per layer cell, its lanes over the cell's ghosts (the sources
    // are real particles or ghosts of earlier planes, so no ghost of this
    // launch reads another)
    const int lane = threadIdx.x & 31;
    const long long nw = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long t = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); t < p.L; t += nw) {
        int cnt = a.layer_count[t];
        if (cnt == 0) continue;
        int cs, cd;
        layer_cells(a, p, t, cs, cd);
        int g0 = base + a.layer_off[t];
        if (lane == 0) a.gcell[cd] = make_int2(g0, cnt);
        int rs = a.cell_start[cs];
        int nreal = a.cell_start[cs + 1] - rs;
        int2 src = a.gcell[cs];
        for (int r = lane; r < cnt; r += 32) {
            int g = g0 + r;
            if (nreal > 0) {
                // MCM/mcm_ghost_setup.f90:324-355 (create_ghost_from_real)
                int j = a.cell_list[rs + r];
                a.gpar[g] = j;
                a.gflip[g] = flips;
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
                a.gflip[g] = a.gflip[q] ^ flips;
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
        long long eb = ((long long)a.layer_cap + 7) / 8;   // 8 warps (layer cells) per block
        if (eb > 148LL * 8) eb = 148LL * 8;
        k_ghost_emit<<<(unsigned)(eb < 1 ? 1 : eb), 256, 0, s>>>(a, plane);
    }
}

// ------------------------------------------------------------------ search
// MCM/mcm_ll_neighbours.f90:96-299.  One thread per cell-order position t;
// the threads of a warp (neighbouring positions, mostly one cell) walk the
// same rows, so their candidate loads hit the same cache lines.  Candidates
// are visited in the reference order (rows of the 27-cell neighbourhood in
// z, y order, cells in x order, each cell's contiguous range of positions),
// and accepted ones are appended to t's list in that order.  The distance
// test runs first in FP32 on positions relative to cell origins; only
// candidates within a narrow band around the cutoff (or all accepted ones
// when the FP64 minimum distance is wanted) are decided by the reference's
// FP64 expression, so the sets are the reference's.  Cells whose box lies
// beyond h_i + max h cannot hold a neighbour and are skipped.

__device__ __forceinline__ double exact_d2(double4 a, double4 b) {
    double d = __dsub_rn(b.x, a.x);
    double s = __dmul_rn(d, d);
    d = __dsub_rn(b.y, a.y);
    s = __dadd_rn(s, __dmul_rn(d, d));
    d = __dsub_rn(b.z, a.z);
    s = __dadd_rn(s, __dmul_rn(d, d));
    return s;
}

// Variants of the search, fixed at compile time so that the candidate loop of
// the common case (one material, no repulsive contact, no minimum distance)
// tests none of these flags per candidate.
enum { kSrchContact = 1, kSrchTwoPass = 2, kSrchMind = 4, kSrchXWin = 8 };

template <int V>
__global__ void __launch_bounds__(256, 4) k_search(StepArgs a) {
    constexpr bool contact = (V & kSrchContact) != 0;   // contacttype > 0: other materials -> contact list
    constexpr bool two_pass = (V & kSrchTwoPass) != 0;  // kernel contact between materials: own material first
    constexpr bool want_mind = (V & kSrchMind) != 0;    // FP64 minimum distance (tcrit option 2, diagnostics)
    constexpr bool xwin = (V & kSrchXWin) != 0;         // cells in x order: each row windowed in x
    if (a.status->code) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    const int np = a.npad;
    const int cap = a.nstride;
    const int key = a.ckey[t];
    const int i = a.cell_list[t];
    const bool with_self = (a.prm.disctype == 1);
    int nn = 0, gn = 0, nc = 0, gcn = 0;
    double mind = 1.0e20;
    if (key >= 0) {
        const DevGrid g = *a.grid;
        int bx, by, bz;
        cell_coords(key, g.gridlim, bx, by, bz);
        const int lo1 = by > 1 ? by - 1 : 1, hi1 = by < g.gridlim[1] ? by + 1 : g.gridlim[1];
        const int lo2 = bz > 1 ? bz - 1 : 1, hi2 = bz < g.gridlim[2] ? bz + 1 : g.gridlim[2];
        const bool has_l = bx > 1, has_r = bx < g.gridlim[0];
        const double4 xi = a.cpos[t];
        const float4 ui = a.cposf[t];
        const float cs[3] = {(float)(1.0 / g.gridsize[0]), (float)(1.0 / g.gridsize[1]), (float)(1.0 / g.gridsize[2])};
        const float csm = fmaxf(cs[0], fmaxf(cs[1], cs[2]));
        // FP32 decision band around the cutoff: the FP32 rounding of d2 and
        // (h_i + h_j)^2 (a few hundred ulps of csm^2 at most) stays far inside it
        const float kb = 2.44140625e-4f * csm * csm;
        const float khi = 1.0f + 2.44140625e-4f, klo = 1.0f - 2.44140625e-4f;
        const float reach = ui.w + (float)g.hcut;
        const float reach2 = reach * reach * 1.0009765625f + 9.765625e-4f * csm * csm;
        // this particle relative to the origins of the left, own and right cell of a row
        const float qxl = ui.x + cs[0], qxr = ui.x - cs[0];
        const float gxl = fmaxf(ui.x, 0.0f), gxr = fmaxf(cs[0] - ui.x, 0.0f);
        // windowed rows: x relative to the grid origin (one frame for the whole
        // row); its rounding (up to gridlim(1) cells of magnitude) widens the
        // decision band by gridlim(1) 2^-16 cell^2, 32 times that error's bound
        const float ugx = xwin ? a.cposg[t].x : 0.0f;
        const float kbx = kb + (xwin ? (float)g.gridlim[0] * 1.52587890625e-5f * csm * csm : 0.0f);
        const int mati = a.cmat[t];
        unsigned *out = a.nidx + (size_t)t * cap;
        // MCM/mcm_ll_neighbours.f90:150-174, 238-267: other materials'
        // particles are appended after the own material's with kernel contact
        // (a second walk), and form the contact list otherwise (the same walk,
        // each list in walk order)
        unsigned *cout = contact ? a.cidx + (size_t)t * a.cstride : nullptr;
        // Windowed common case: accepted entries collect in four registers and
        // leave as one 16-byte store per four (t's row starts at t * cap
        // entries, cap a multiple of 4), so a warp's lanes, whose rows lie cap
        // entries apart, send a quarter of the scattered store requests.
        const bool vec = (cap & 3) == 0;
        unsigned b0 = 0u, b1 = 0u, b2 = 0u, b3 = 0u;
#pragma unroll 1
        for (int pass = 0; pass < (two_pass ? 2 : 1); ++pass) {
            for (int nz = lo2; nz <= hi2; ++nz) {
                const float qz = ui.z + (float)(bz - nz) * cs[2];
                const float gz = fmaxf(nz < bz ? ui.z : (nz > bz ? cs[2] - ui.z : 0.0f), 0.0f);
                for (int my = lo1; my <= hi1; ++my) {
                    const float qy = ui.y + (float)(by - my) * cs[1];
                    const float gy = fmaxf(my < by ? ui.y : (my > by ? cs[1] - ui.y : 0.0f), 0.0f);
                    const float gyz = gy * gy + gz * gz;
                    if (gyz > reach2) continue;
                    // the row's x-adjacent cells are contiguous in position
                    // order: one range from the first to the last cell whose
                    // box is within reach (the own cell always is)
                    const int kc = (int)cell_key(bx, my, nz, g.gridlim);
                    const int s1 = a.cell_start[kc], s2 = a.cell_start[kc + 1];
                    const int rb = (has_l && !(gyz + gxl * gxl > reach2)) ? a.cell_start[kc - 1] : s1;
                    const int re = (has_r && !(gyz + gxr * gxr > reach2)) ? a.cell_start[kc + 2] : s2;
                    const unsigned code_yz = (unsigned)(3 * (my - by + 1) + 9 * (nz - bz + 1));
                    int pb = rb, pe = re;
                    if (xwin) {
                        // the row is x-sorted: candidates farther than rxw in x
                        // are beyond reach (with a margin for FP32 rounding);
                        // the window's ends by bisection
                        const float rxw = sqrtf(fmaxf(reach2 - gyz, 0.0f)) * 1.0009765625f + 9.765625e-4f * csm;
                        int hi = re;
                        while (pb < hi) {
                            const int mid = (pb + hi) >> 1;
                            if (ugx - a.cposg[mid].x > rxw) pb = mid + 1;
                            else hi = mid;
                        }
                        int lo = pb;
                        while (lo < pe) {
                            const int mid = (lo + pe) >> 1;
                            if (ugx - a.cposg[mid].x < -rxw) pe = mid;
                            else lo = mid + 1;
                        }
                    }
                    if constexpr (xwin && !contact && !two_pass && !want_mind) {
                        // windowed rows, one material, no minimum distance: the
                        // accept path is a predicated store, so the lanes stay
                        // converged (measured: 1.41 against 1.46 ms on the 2M
                        // bar; on the unwindowed rows of the reference order it
                        // is slower than the branching loop)
                        for (int p = pb; p < pe; ++p) {
                            const float4 c = a.cposg[p];
                            const float dx = ugx - c.x, dy = qy - c.y, dz = qz - c.z;
                            const float d2f = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                            const float hsf = ui.w + c.w;
                            const float r2f = hsf * hsf;
                            bool in = d2f < fmaf(r2f, khi, kbx) && p != t;
                            if (in && d2f > fmaf(r2f, klo, -kbx)) {
                                // near tie: the reference's FP64 test
                                const double4 cd = a.cpos[p];
                                const double hs = __dadd_rn(cd.w, xi.w);
                                in = exact_d2(xi, cd) < __dmul_rn(hs, hs);
                            }
                            const unsigned entry = (unsigned)p | ((code_yz + (p < s1 ? 0u : (p >= s2 ? 2u : 1u))) << 26);
                            if (vec) {
                                if (in) { b0 = b1; b1 = b2; b2 = b3; b3 = entry; }
                                nn += in ? 1 : 0;
                                if (in && (nn & 3) == 0 && nn <= cap)
                                    *reinterpret_cast<uint4 *>(out + (nn - 4)) = make_uint4(b0, b1, b2, b3);
                            } else {
                                if (in && nn < cap) out[nn] = entry;
                                nn += in ? 1 : 0;
                            }
                        }
                    } else {
                    for (int p = pb; p < pe; ++p) {
                        const float4 c = a.cposf[p];
                        const bool left = p < s1, right = p >= s2;
                        const float qx = left ? qxl : (right ? qxr : ui.x);
                        const float dx = qx - c.x, dy = qy - c.y, dz = qz - c.z;
                        const float d2f = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                        const float hsf = ui.w + c.w;
                        const float r2f = hsf * hsf;
                        if (d2f >= fmaf(r2f, khi, kb)) continue;
                        if (p == t) continue;
                        double d2 = 0.0;
                        if (want_mind || d2f > fmaf(r2f, klo, -kb)) {
                            // near tie (or mindist wanted): the reference's FP64 test
                            const double4 cd = a.cpos[p];
                            d2 = exact_d2(xi, cd);
                            const double hs = __dadd_rn(cd.w, xi.w);
                            if (!(d2 < __dmul_rn(hs, hs))) continue;
                        }
                        const unsigned code = (code_yz + (left ? 0u : (right ? 2u : 1u))) << 26;
                        if (contact) {
                            if (a.cmat[p] != mati) {
                                if (nc < a.cstride) cout[nc] = (unsigned)p | code;
                                ++nc;
                                continue;
                            }
                        } else if (two_pass) {
                            if ((a.cmat[p] == mati) != (pass == 0)) continue;
                        }
                        if (want_mind) mind = fmin(mind, d2);
                        if (nn < cap) out[nn] = (unsigned)p | code;
                        ++nn;
                    }
                    }
                }
            }
        }
        if constexpr (xwin && !contact && !two_pass && !want_mind) {
            if (vec) {
                // the last nn % 4 accepted entries are still in b(4 - nn % 4) .. b3
                const int r = nn & 3;
                if (r >= 3 && nn - 3 < cap) out[nn - 3] = b1;
                if (r >= 2 && nn - 2 < cap) out[nn - 2] = b2;
                if (r >= 1 && nn - 1 < cap) out[nn - 1] = b3;
            }
        }
        if (nn > cap) {
            atomicMax(&a.status->req_stride, nn);
            raise_status(a.status, MCM_ENBR_OVERFLOW, i);
        }
        if (contact && nc > a.cstride) {
            atomicMax(&a.status->req_cstride, nc);
            raise_status(a.status, MCM_ENBR_OVERFLOW, i);
        }
        // ghosts: only neighbourhoods that reach a ghost layer
        if (a.prm.boundary) {
            const int lo0 = has_l ? bx - 1 : bx, hi0 = has_r ? bx + 1 : bx;
            const DevPlanes &pl = a.prm.planes;
            const bool near = (lo0 == 1 && pl.code[0][0]) || (hi0 == g.gridlim[0] && pl.code[1][0]) ||
                              (lo1 == 1 && pl.code[0][1]) || (hi1 == g.gridlim[1] && pl.code[1][1]) ||
                              (lo2 == 1 && pl.code[0][2]) || (hi2 == g.gridlim[2] && pl.code[1][2]);
            if (near) {
#pragma unroll 1
                for (int pass = 0; pass < (two_pass ? 2 : 1); ++pass) {
                    for (int nz = lo2; nz <= hi2; ++nz)
                        for (int my = lo1; my <= hi1; ++my)
                            for (int lx = lo0; lx <= hi0; ++lx) {
                                const int2 gc = a.gcell[(int)cell_key(lx, my, nz, g.gridlim)];
                                for (int r = 0; r < gc.y; ++r) {
                                    const int q = gc.x + gc.y - 1 - r;   // chain order: newest first
                                    const double4 c = make_double4(a.gx[q], a.gy[q], a.gz[q], a.gh[q]);
                                    const double d2 = exact_d2(xi, c);
                                    const double hs = __dadd_rn(c.w, xi.w);
                                    if (d2 < __dmul_rn(hs, hs)) {
                                        if (contact) {
                                            if (a.gmat[q] != mati) {
                                                if (gcn < a.gcstride) a.gcont[(size_t)gcn * np + t] = q;
                                                ++gcn;
                                                continue;
                                            }
                                        } else if (two_pass) {
                                            if ((a.gmat[q] == mati) != (pass == 0)) continue;
                                        }
                                        mind = fmin(mind, d2);
                                        if (gn < a.gstride) a.gnbr[(size_t)gn * np + t] = q;
                                        ++gn;
                                    }
                                }
                            }
                }
                if (gn > a.gstride) {
                    atomicMax(&a.status->req_gstride, gn);
                    raise_status(a.status, MCM_ENBR_OVERFLOW, i);
                }
                if (contact && gcn > a.gcstride) {
                    atomicMax(&a.status->req_gcstride, gcn);
                    raise_status(a.status, MCM_ENBR_OVERFLOW, i);
                }
            }
        }
        mind = sqrt(mind);
    }
    if (with_self) nn += 1;   // MCM/mcm_ll_neighbours.f90:288-299 (for every particle)
    a.nnbr[t] = nn;
    a.gnnbr[t] = gn;
    if (contact) { a.ncont[t] = nc; a.gncont[t] = gcn; }
    if (want_mind) a.F.f[FMINDIST][i] = mind;
    atomicMax(&a.status->max_nbr, nn);
    atomicMax(&a.status->max_gnbr, gn);
}

// The same search with one warp per position t (search_kind 2; on the
// 2 034 720-particle bar it takes 2.1x the time of k_search, whose threads
// share candidate rows through L1, so it is only a tuning alternative for
// small bodies).  The lanes take consecutive
// candidates of a row (the up to three cells of a row are contiguous in
// position order), so every lane runs the same loop and the candidate loads
// are coalesced.  Accepted candidates are compacted with a ballot in lane
// order, which is position order, so t's list is the one k_search builds:
// rows in z, y order, cells in x order, positions ascending.  The FP32
// decision and the FP64 tie test are k_search's expressions.
__global__ void __launch_bounds__(256) k_search_warp(StepArgs a) {
    if (a.status->code) return;
    const int lane = threadIdx.x & 31;
    const int t = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    if (t >= a.n) return;                       // warp-uniform
    const unsigned below = (1u << lane) - 1u;
    const int np = a.npad;
    const int cap = a.nstride;
    const int key = a.ckey[t];
    const int i = a.cell_list[t];
    const bool with_self = (a.prm.disctype == 1);
    const bool want_mind = (a.prm.tcrit_opt == 2 || a.prm.diag);
    int nn = 0, gn = 0, nc = 0, gcn = 0;
    double mind = 1.0e20;
    const bool contact = a.prm.contact != 0;
    if (key >= 0) {
        const DevGrid g = *a.grid;
        int bx, by, bz;
        cell_coords(key, g.gridlim, bx, by, bz);
        const int lo0 = bx > 1 ? bx - 1 : 1, hi0 = bx < g.gridlim[0] ? bx + 1 : g.gridlim[0];
        const int lo1 = by > 1 ? by - 1 : 1, hi1 = by < g.gridlim[1] ? by + 1 : g.gridlim[1];
        const int lo2 = bz > 1 ? bz - 1 : 1, hi2 = bz < g.gridlim[2] ? bz + 1 : g.gridlim[2];
        const double4 xi = a.cpos[t];
        const float4 ui = a.cposf[t];
        const float cs[3] = {(float)(1.0 / g.gridsize[0]), (float)(1.0 / g.gridsize[1]), (float)(1.0 / g.gridsize[2])};
        const float csm = fmaxf(cs[0], fmaxf(cs[1], cs[2]));
        const float kb = 2.44140625e-4f * csm * csm;
        const float khi = 1.0f + 2.44140625e-4f, klo = 1.0f - 2.44140625e-4f;
        const float reach = ui.w + (float)g.hcut;
        const float reach2 = reach * reach * 1.0009765625f + 9.765625e-4f * csm * csm;
        const int mati = a.cmat[t];
        unsigned *out = a.nidx + (size_t)t * cap;
        // x extent of the rows: the own column always, a side column when its
        // box can hold a neighbour (the test of k_search's cell loop)
        const float gxl = ui.x, gxr = fmaxf(cs[0] - ui.x, 0.0f);
        unsigned *cout = contact ? a.cidx + (size_t)t * a.cstride : nullptr;
        const int passes = (a.nmat > 1 && a.prm.contacttype == 0) ? 2 : 1;
        for (int pass = 0; pass < passes; ++pass) {
            for (int nz = lo2; nz <= hi2; ++nz) {
                const float qz = ui.z + (float)(bz - nz) * cs[2];
                const float gz = fmaxf(nz < bz ? ui.z : (nz > bz ? cs[2] - ui.z : 0.0f), 0.0f);
                for (int my = lo1; my <= hi1; ++my) {
                    const float qy = ui.y + (float)(by - my) * cs[1];
                    const float gy = fmaxf(my < by ? ui.y : (my > by ? cs[1] - ui.y : 0.0f), 0.0f);
                    const float gyz = gy * gy + gz * gz;
                    if (gyz > reach2) continue;
                    const int lf = (lo0 < bx && !(gyz + fmaxf(gxl, 0.0f) * fmaxf(gxl, 0.0f) > reach2)) ? lo0 : bx;
                    const int ll = (hi0 > bx && !(gyz + gxr * gxr > reach2)) ? hi0 : bx;
                    const int kf = (int)cell_key(lf, my, nz, g.gridlim);
                    const int cb = a.cell_start[kf];
                    const int ce = a.cell_start[kf + (ll - lf) + 1];
                    // first positions of the second and third cell of the range
                    const int s1 = a.cell_start[kf + 1];
                    const int s2 = (ll - lf >= 2) ? a.cell_start[kf + 2] : ce;
                    const unsigned code_yz = (unsigned)(3 * (my - by + 1) + 9 * (nz - bz + 1));
                    for (int base = cb; base < ce; base += 32) {
                        const int p = base + lane;
                        bool acc = false, accc = false;
                        double d2 = 0.0;
                        int lx = lf;
                        if (p < ce) {
                            lx = lf + (p >= s1 ? 1 : 0) + (p >= s2 ? 1 : 0);
                            const float4 c = a.cposf[p];
                            const float qx = ui.x + (float)(bx - lx) * cs[0];
                            const float dx = qx - c.x, dy = qy - c.y, dz = qz - c.z;
                            const float d2f = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                            const float hsf = ui.w + c.w;
                            const float r2f = hsf * hsf;
                            acc = (d2f < fmaf(r2f, khi, kb)) && (p != t);
                            if (acc && (d2f > fmaf(r2f, klo, -kb) || want_mind)) {
                                const double4 cd = a.cpos[p];
                                d2 = exact_d2(xi, cd);
                                const double hs = __dadd_rn(cd.w, xi.w);
                                acc = d2 < __dmul_rn(hs, hs);
                            }
                            if (acc && contact) {
                                accc = (a.cmat[p] != mati);
                                acc = !accc;
                            } else if (acc && a.nmat > 1) {
                                acc = ((a.cmat[p] == mati) == (pass == 0));
                            }
                        }
                        const unsigned bal = __ballot_sync(0xffffffffu, acc);
                        if (acc) {
                            if (want_mind) mind = fmin(mind, d2);
                            const int pos = nn + __popc(bal & below);
                            if (pos < cap) out[pos] = (unsigned)p | ((code_yz + (unsigned)(lx - bx + 1)) << 26);
                        }
                        nn += __popc(bal);
                        if (contact) {
                            const unsigned cbal = __ballot_sync(0xffffffffu, accc);
                            if (accc) {
                                const int pos = nc + __popc(cbal & below);
                                if (pos < a.cstride) cout[pos] = (unsigned)p | ((code_yz + (unsigned)(lx - bx + 1)) << 26);
                            }
                            nc += __popc(cbal);
                        }
                    }
                }
            }
        }
        // ghosts: only neighbourhoods that reach a ghost layer; a cell's ghosts
        // are visited newest first (the chain order of the reference)
        if (a.prm.boundary) {
            const DevPlanes &pl = a.prm.planes;
            const bool near = (lo0 == 1 && pl.code[0][0]) || (hi0 == g.gridlim[0] && pl.code[1][0]) ||
                              (lo1 == 1 && pl.code[0][1]) || (hi1 == g.gridlim[1] && pl.code[1][1]) ||
                              (lo2 == 1 && pl.code[0][2]) || (hi2 == g.gridlim[2] && pl.code[1][2]);
            if (near) {
                const int gpasses = (a.nmat > 1 && a.prm.contacttype == 0) ? 2 : 1;
                for (int pass = 0; pass < gpasses; ++pass) {
                    for (int nz = lo2; nz <= hi2; ++nz)
                        for (int my = lo1; my <= hi1; ++my)
                            for (int lx = lo0; lx <= hi0; ++lx) {
                                const int2 gc = a.gcell[(int)cell_key(lx, my, nz, g.gridlim)];
                                for (int base = 0; base < gc.y; base += 32) {
                                    const int r = base + lane;
                                    bool acc = false, accc = false;
                                    double d2 = 0.0;
                                    int q = 0;
                                    if (r < gc.y) {
                                        q = gc.x + gc.y - 1 - r;
                                        const double4 c = make_double4(a.gx[q], a.gy[q], a.gz[q], a.gh[q]);
                                        d2 = exact_d2(xi, c);
                                        const double hs = __dadd_rn(c.w, xi.w);
                                        acc = d2 < __dmul_rn(hs, hs);
                                        if (acc && contact) {
                                            accc = (a.gmat[q] != mati);
                                            acc = !accc;
                                        } else if (acc && a.nmat > 1) {
                                            acc = ((a.gmat[q] == mati) == (pass == 0));
                                        }
                                    }
                                    const unsigned bal = __ballot_sync(0xffffffffu, acc);
                                    if (acc) {
                                        mind = fmin(mind, d2);
                                        const int pos = gn + __popc(bal & below);
                                        if (pos < a.gstride) a.gnbr[(size_t)pos * np + t] = q;
                                    }
                                    gn += __popc(bal);
                                    if (contact) {
                                        const unsigned cbal = __ballot_sync(0xffffffffu, accc);
                                        if (accc) {
                                            const int pos = gcn + __popc(cbal & below);
                                            if (pos < a.gcstride) a.gcont[(size_t)pos * np + t] = q;
                                        }
                                        gcn += __popc(cbal);
                                    }
                                }
                            }
                }
            }
        }
        for (int o = 16; o > 0; o >>= 1) mind = fmin(mind, __shfl_xor_sync(0xffffffffu, mind, o));
        mind = sqrt(mind);
    }
    if (lane != 0) return;
    if (nn > cap) {
        atomicMax(&a.status->req_stride, nn);
        raise_status(a.status, MCM_ENBR_OVERFLOW, i);
    }
    if (gn > a.gstride) {
        atomicMax(&a.status->req_gstride, gn);
        raise_status(a.status, MCM_ENBR_OVERFLOW, i);
    }
    if (contact && nc > a.cstride) {
        atomicMax(&a.status->req_cstride, nc);
        raise_status(a.status, MCM_ENBR_OVERFLOW, i);
    }
    if (contact && gcn > a.gcstride) {
        atomicMax(&a.status->req_gcstride, gcn);
        raise_status(a.status, MCM_ENBR_OVERFLOW, i);
    }
    if (with_self) nn += 1;   // MCM/mcm_ll_neighbours.f90:288-299 (for every particle)
    a.nnbr[t] = nn;
    a.gnnbr[t] = gn;
    if (contact) { a.ncont[t] = nc; a.gncont[t] = gcn; }
    if (want_mind) a.F.f[FMINDIST][i] = mind;
    atomicMax(&a.status->max_nbr, nn);
    atomicMax(&a.status->max_gnbr, gn);
}

// The same search with one warp per cell (search_kind 3): the lanes are the
// particles of one cell (32 at a time), so every lane walks the same rows of
// the same 27-cell neighbourhood and the loop control is warp-uniform.  Each
// row's contiguous candidate range is staged 32 records at a time in shared
// memory by one coalesced load per lane and then read by every lane as a
// broadcast, so the inner loop has no global load.  Candidates are visited in
// k_search's order and tested with its FP32 decision and FP64 tie test, so
// the lists are k_search's, entry for entry.
constexpr int kCellWarps = 8;
__global__ void __launch_bounds__(kCellWarps * 32, 3) k_search_cell(StepArgs a) {
    __shared__ float4 stage[kCellWarps][32];
    __shared__ int stage_mat[kCellWarps][32];
    if (a.status->code) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long ncells = a.grid->ncells;
    const int gl0 = a.grid->gridlim[0], gl1 = a.grid->gridlim[1], gl2 = a.grid->gridlim[2];
    // cell keys from scalars (an array passed by pointer would live in local memory)
    auto key_of = [gl0, gl1](int x, int y, int z) { return (x - 1) + gl0 * ((y - 1) + gl1 * (z - 1)); };
    const float hcut = (float)a.grid->hcut;
    const int np = a.npad;
    const int cap = a.nstride;
    const bool with_self = (a.prm.disctype == 1);
    const bool want_mind = (a.prm.tcrit_opt == 2 || a.prm.diag);
    const bool contact = a.prm.contact != 0;
    const bool multi = a.nmat > 1;
    const float cs[3] = {(float)(1.0 / a.grid->gridsize[0]), (float)(1.0 / a.grid->gridsize[1]),
                         (float)(1.0 / a.grid->gridsize[2])};
    const float csm = fmaxf(cs[0], fmaxf(cs[1], cs[2]));
    const float kb = 2.44140625e-4f * csm * csm;
    const float khi = 1.0f + 2.44140625e-4f, klo = 1.0f - 2.44140625e-4f;
    float4 *st = stage[w];
    int *stm = stage_mat[w];
    const long long nwarps = (long long)gridDim.x * kCellWarps;
    for (long long c = (long long)blockIdx.x * kCellWarps + w; c < ncells; c += nwarps) {
        const int c0 = a.cell_start[c], c1 = a.cell_start[c + 1];
        if (c0 == c1) continue;   // warp-uniform
        const int bx = (int)(c % gl0) + 1;
        const int by = (int)((c / gl0) % gl1) + 1;
        const int bz = (int)(c / ((long long)gl0 * gl1)) + 1;
        const int lo0 = bx > 1 ? bx - 1 : 1, hi0 = bx < gl0 ? bx + 1 : gl0;
        const int lo1 = by > 1 ? by - 1 : 1, hi1 = by < gl1 ? by + 1 : gl1;
        const int lo2 = bz > 1 ? bz - 1 : 1, hi2 = bz < gl2 ? bz + 1 : gl2;
        for (int base = c0; base < c1; base += 32) {
            const int t = base + lane;
            const bool live = t < c1;
            double4 xi = make_double4(0.0, 0.0, 0.0, 0.0);
            float4 ui = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            int mati = 0, i = 0;
            if (live) {
                xi = a.cpos[t];
                ui = a.cposf[t];
                mati = a.cmat[t];
                i = a.cell_list[t];
            }
            const float reach = ui.w + hcut;
            const float reach2 = reach * reach * 1.0009765625f + 9.765625e-4f * csm * csm;
            unsigned *out = a.nidx + (size_t)(live ? t : 0) * cap;
            unsigned *cout = contact ? a.cidx + (size_t)(live ? t : 0) * a.cstride : nullptr;
            int nn = 0, gn = 0, nc = 0, gcn = 0;
            double mind = 1.0e20;
            // x extent of the own cell's neighbours: distance to the side columns
            const float gxl = fmaxf(ui.x, 0.0f), gxr = fmaxf(cs[0] - ui.x, 0.0f);
            const int passes = (multi && a.prm.contacttype == 0) ? 2 : 1;
            for (int pass = 0; pass < passes; ++pass) {
                for (int nz = lo2; nz <= hi2; ++nz) {
                    const float qz = ui.z + (float)(bz - nz) * cs[2];
                    const float gz = fmaxf(nz < bz ? ui.z : (nz > bz ? cs[2] - ui.z : 0.0f), 0.0f);
                    for (int my = lo1; my <= hi1; ++my) {
                        const float qy = ui.y + (float)(by - my) * cs[1];
                        const float gy = fmaxf(my < by ? ui.y : (my > by ? cs[1] - ui.y : 0.0f), 0.0f);
                        const float gyz = gy * gy + gz * gz;
                        const bool rowok = live && !(gyz > reach2);
                        if (!__any_sync(0xffffffffu, rowok)) continue;
                        // per lane: which of the row's cells can hold a neighbour
                        const bool okl = rowok && !(gyz + gxl * gxl > reach2);
                        const bool okr = rowok && !(gyz + gxr * gxr > reach2);
                        const int k0 = key_of(lo0, my, nz);
                        const int rb = a.cell_start[k0];
                        const int re = a.cell_start[k0 + (hi0 - lo0) + 1];
                        const int s1 = a.cell_start[k0 + 1];
                        const int s2 = (hi0 - lo0 >= 2) ? a.cell_start[k0 + 2] : re;
                        const unsigned code_yz = (unsigned)(3 * (my - by + 1) + 9 * (nz - bz + 1));
                        for (int chunk = rb; chunk < re; chunk += 32) {
                            const int pc = chunk + lane;
                            if (pc < re) {
                                st[lane] = a.cposf[pc];
                                if (multi) stm[lane] = a.cmat[pc];
                            }
                            __syncwarp();
                            const int m = (re - chunk) < 32 ? (re - chunk) : 32;
                            if (rowok) {
                                for (int k = 0; k < m; ++k) {
                                    const int p = chunk + k;
                                    const int lx = lo0 + (p >= s1 ? 1 : 0) + (p >= s2 ? 1 : 0);
                                    if (lx < bx ? !okl : (lx > bx ? !okr : false)) continue;
                                    const float4 cd4 = st[k];
                                    const float qx = ui.x + (float)(bx - lx) * cs[0];
                                    const float dx = qx - cd4.x, dy = qy - cd4.y, dz = qz - cd4.z;
                                    const float d2f = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                                    const float hsf = ui.w + cd4.w;
                                    const float r2f = hsf * hsf;
                                    if (d2f >= fmaf(r2f, khi, kb)) continue;
                                    if (p == t) continue;
                                    double d2 = 0.0;
                                    if (d2f > fmaf(r2f, klo, -kb) || want_mind) {
                                        const double4 cd = a.cpos[p];
                                        d2 = exact_d2(xi, cd);
                                        const double hs = __dadd_rn(cd.w, xi.w);
                                        if (!(d2 < __dmul_rn(hs, hs))) continue;
                                    }
                                    const unsigned code = (code_yz + (unsigned)(lx - bx + 1)) << 26;
                                    if (contact) {
                                        if (stm[k] != mati) {
                                            if (nc < a.cstride) cout[nc] = (unsigned)p | code;
                                            ++nc;
                                            continue;
                                        }
                                    } else if (multi && (stm[k] == mati) != (pass == 0)) {
                                        continue;
                                    }
                                    if (want_mind) mind = fmin(mind, d2);
                                    if (nn < cap) out[nn] = (unsigned)p | code;
                                    ++nn;
                                }
                            }
                            __syncwarp();
                        }
                    }
                }
            }
            // ghosts: only neighbourhoods that reach a ghost layer (warp-uniform test)
            if (a.prm.boundary && live) {
                const DevPlanes &pl = a.prm.planes;
                const bool near = (lo0 == 1 && pl.code[0][0]) || (hi0 == gl0 && pl.code[1][0]) ||
                                  (lo1 == 1 && pl.code[0][1]) || (hi1 == gl1 && pl.code[1][1]) ||
                                  (lo2 == 1 && pl.code[0][2]) || (hi2 == gl2 && pl.code[1][2]);
                if (near) {
                    const int gpasses = (multi && a.prm.contacttype == 0) ? 2 : 1;
                    for (int pass = 0; pass < gpasses; ++pass) {
                        for (int nz = lo2; nz <= hi2; ++nz)
                            for (int my = lo1; my <= hi1; ++my)
                                for (int lx = lo0; lx <= hi0; ++lx) {
                                    const int2 gcl = a.gcell[key_of(lx, my, nz)];
                                    for (int r = 0; r < gcl.y; ++r) {
                                        const int q = gcl.x + gcl.y - 1 - r;   // chain order: newest first
                                        const double4 gq = make_double4(a.gx[q], a.gy[q], a.gz[q], a.gh[q]);
                                        const double d2 = exact_d2(xi, gq);
                                        const double hs = __dadd_rn(gq.w, xi.w);
                                        if (d2 < __dmul_rn(hs, hs)) {
                                            if (contact) {
                                                if (a.gmat[q] != mati) {
                                                    if (gcn < a.gcstride) a.gcont[(size_t)gcn * np + t] = q;
                                                    ++gcn;
                                                    continue;
                                                }
                                            } else if (multi && (a.gmat[q] == mati) != (pass == 0)) {
                                                continue;
                                            }
                                            mind = fmin(mind, d2);
                                            if (gn < a.gstride) a.gnbr[(size_t)gn * np + t] = q;
                                            ++gn;
                                        }
                                    }
                                }
                    }
                }
            }
            if (!live) continue;
            if (nn > cap) {
                atomicMax(&a.status->req_stride, nn);
                raise_status(a.status, MCM_ENBR_OVERFLOW, i);
            }
            if (gn > a.gstride) {
                atomicMax(&a.status->req_gstride, gn);
                raise_status(a.status, MCM_ENBR_OVERFLOW, i);
            }
            if (contact && nc > a.cstride) {
                atomicMax(&a.status->req_cstride, nc);
                raise_status(a.status, MCM_ENBR_OVERFLOW, i);
            }
            if (contact && gcn > a.gcstride) {
                atomicMax(&a.status->req_gcstride, gcn);
                raise_status(a.status, MCM_ENBR_OVERFLOW, i);
            }
            mind = sqrt(mind);
            if (with_self) nn += 1;   // MCM/mcm_ll_neighbours.f90:288-299 (for every particle)
            a.nnbr[t] = nn;
            a.gnnbr[t] = gn;
            if (contact) { a.ncont[t] = nc; a.gncont[t] = gcn; }
            if (want_mind) a.F.f[FMINDIST][i] = mind;
            atomicMax(&a.status->max_nbr, nn);
            atomicMax(&a.status->max_gnbr, gn);
        }
    }
    // particles outside the grid (the last positions) have no neighbours
    const int first_out = a.cell_start[ncells];
    for (int t = first_out + blockIdx.x * blockDim.x + threadIdx.x; t < a.n; t += gridDim.x * blockDim.x) {
        const int nn = with_self ? 1 : 0;
        a.nnbr[t] = nn;
        a.gnnbr[t] = 0;
        if (contact) { a.ncont[t] = 0; a.gncont[t] = 0; }
        if (want_mind) a.F.f[FMINDIST][a.cell_list[t]] = 1.0e20;
        atomicMax(&a.status->max_nbr, nn);
    }
}

// ------------------------------------------------------------- skin lists
// For the FP64-fast and mixed steps, whose sums do not follow the reference's
// neighbour order: the neighbour lists of a step are filtered from a skin
// list, a superset of each particle's neighbours kept from the last build.
// A pair (i, j) missing from the skin list was at least h_i + h_j + skin apart
// at the build; while every particle has moved less than skin/2 since then,
// it is still at least h_i + h_j apart, so it cannot be a neighbour.  The
// step rebuilds the skin lists when the largest displacement reaches skin/2
// (or on request), and filters them every step with k_search's FP32 decision
// and FP64 tie test, among the candidates in the 27 cells around the
// particle's cell of the current grid (the only ones the reference examines),
// so the neighbour sets are the reference's; their order is the skin list's.

// Largest squared displacement since the last build (state order).
__global__ void __launch_bounds__(256) k_skin_disp(StepArgs a) {
    __shared__ unsigned long long sm[8];
    if (a.status->code) return;
    unsigned long long best = 0ull;
    const double *X = a.F.f[FX], *Y = a.F.f[FY], *Z = a.F.f[FZ];
    const size_t np = a.npad;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const double dx = X[i] - a.xref[i], dy = Y[i] - a.xref[np + i], dz = Z[i] - a.xref[2 * np + i];
        const double d2 = dx * dx + dy * dy + dz * dz;   // >= 0: the bit pattern orders like the value
        const unsigned long long b = (unsigned long long)__double_as_longlong(d2);
        best = b > best ? b : best;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long v = __shfl_xor_sync(0xffffffffu, best, o);
        best = v > best ? v : best;
    }
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) best = sm[w] > best ? sm[w] : best;
        atomicMax(a.skin_d2, best);
    }
}

// One thread: build when asked to, or when 2 * max displacement >= skin.
__global__ void k_skin_decide(StepArgs a) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (a.status->code) return;
    const double dmax = sqrt(__longlong_as_double((long long)*a.skin_d2));
    const double skin = a.prm.skin * a.hmax[0];
    const int need = (a.skin_flags[0] != 0 || !(2.0 * dmax < skin)) ? 1 : 0;
    a.skin_flags[1] = need;
    a.skin_flags[0] = 0;
    if (need) a.skin_flags[2] += 1;
    *a.skin_d2 = 0ull;
}

// The skin lists: one thread per cell-order position, candidates in the
// cells within reach (up to two cells away), accepted when their FP32
// distance lies below h_i + h_j + skin with a margin (a superset needs no
// exact test).  Positions outside the grid keep an empty list.
__global__ void __launch_bounds__(256) k_skin_build(StepArgs a) {
    if (a.status->code || !a.skin_flags[1]) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    const int i = a.cell_list[t];
    const size_t np = a.npad;
    const double4 xi = a.cpos[t];
    a.xref[i] = xi.x;
    a.xref[np + i] = xi.y;
    a.xref[2 * np + i] = xi.z;
    const int key = a.ckey[t];
    int nn = 0;
    if (key >= 0) {
        const int gl0 = a.grid->gridlim[0], gl1 = a.grid->gridlim[1], gl2 = a.grid->gridlim[2];
        const int bx = key % gl0 + 1, by = (key / gl0) % gl1 + 1, bz = key / (gl0 * gl1) + 1;
        const float cs[3] = {(float)(1.0 / a.grid->gridsize[0]), (float)(1.0 / a.grid->gridsize[1]),
                             (float)(1.0 / a.grid->gridsize[2])};
        const float skin = (float)(a.prm.skin * a.hmax[0]);
        const float4 ui = a.cposf[t];
        const float reach = ui.w + (float)a.grid->hcut + skin;
        const float reach2 = reach * reach * 1.001f + 1.0e-3f * cs[0] * cs[0];
        int *out = a.sup + (size_t)i * a.sstride;
        for (int nz = max(bz - 2, 1); nz <= min(bz + 2, gl2); ++nz) {
            const float qz = ui.z + (float)(bz - nz) * cs[2];
            const float gz = nz < bz ? ui.z + (float)(bz - nz - 1) * cs[2] : (nz > bz ? (float)(nz - bz) * cs[2] - ui.z : 0.0f);
            for (int my = max(by - 2, 1); my <= min(by + 2, gl1); ++my) {
                const float qy = ui.y + (float)(by - my) * cs[1];
                const float gy = my < by ? ui.y + (float)(by - my - 1) * cs[1] : (my > by ? (float)(my - by) * cs[1] - ui.y : 0.0f);
                const float gyz = fmaxf(gy, 0.0f) * fmaxf(gy, 0.0f) + fmaxf(gz, 0.0f) * fmaxf(gz, 0.0f);
                if (gyz > reach2) continue;
                for (int lx = max(bx - 2, 1); lx <= min(bx + 2, gl0); ++lx) {
                    const float gx = lx < bx ? ui.x + (float)(bx - lx - 1) * cs[0] : (lx > bx ? (float)(lx - bx) * cs[0] - ui.x : 0.0f);
                    if (gyz + fmaxf(gx, 0.0f) * fmaxf(gx, 0.0f) > reach2) continue;
                    const int k = (lx - 1) + gl0 * ((my - 1) + gl1 * (nz - 1));
                    const int cb = a.cell_start[k], ce = a.cell_start[k + 1];
                    const float qx = ui.x + (float)(bx - lx) * cs[0];
                    for (int p = cb; p < ce; ++p) {
                        if (p == t) continue;
                        const float4 c = a.cposf[p];
                        const float dx = qx - c.x, dy = qy - c.y, dz = qz - c.z;
                        const float d2f = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                        const float r = ui.w + c.w + skin;
                        if (d2f >= r * r * 1.001f + 1.0e-3f * cs[0] * cs[0]) continue;
                        if (nn < a.sstride) out[nn] = a.cell_list[p];
                        ++nn;
                    }
                }
            }
        }
    }
    a.supn[i] = nn;
    if (nn > a.sstride) {
        atomicMax(&a.status->req_sstride, nn);
        raise_status(a.status, MCM_ENBR_OVERFLOW, i);
    }
}

// The step's neighbour lists from the skin lists: k_search's decisions on
// the candidates that lie in the 27 cells around the particle's cell, in
// skin-list order; ghosts, contacts, minimum distances and counts as k_search.
__global__ void __launch_bounds__(256, 4) k_skin_filter(StepArgs a) {
    if (a.status->code) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    const int np = a.npad;
    const int cap = a.nstride;
    const int key = a.ckey[t];
    const int i = a.cell_list[t];
    const bool with_self = (a.prm.disctype == 1);
    const bool want_mind = (a.prm.tcrit_opt == 2 || a.prm.diag);
    const bool contact = a.prm.contact != 0;
    int nn = 0, gn = 0, nc = 0, gcn = 0;
    double mind = 1.0e20;
    if (key >= 0) {
        const int gl0 = a.grid->gridlim[0], gl1 = a.grid->gridlim[1], gl2 = a.grid->gridlim[2];
        const int bx = key % gl0 + 1, by = (key / gl0) % gl1 + 1, bz = key / (gl0 * gl1) + 1;
        const double4 xi = a.cpos[t];
        const float4 ui = a.cposf[t];
        const float cs[3] = {(float)(1.0 / a.grid->gridsize[0]), (float)(1.0 / a.grid->gridsize[1]),
                             (float)(1.0 / a.grid->gridsize[2])};
        const float csm = fmaxf(cs[0], fmaxf(cs[1], cs[2]));
        const float kb = 2.44140625e-4f * csm * csm;
        const float khi = 1.0f + 2.44140625e-4f, klo = 1.0f - 2.44140625e-4f;
        const int mati = a.cmat[t];
        unsigned *out = a.nidx + (size_t)t * cap;
        unsigned *cout = contact ? a.cidx + (size_t)t * a.cstride : nullptr;
        const int *cand = a.sup + (size_t)i * a.sstride;
        const int ns = a.supn[i];
        // with kernel contact the other materials follow the own material's neighbours
        const int passes = (a.nmat > 1 && a.prm.contacttype == 0) ? 2 : 1;
        for (int pass = 0; pass < passes; ++pass) {
            for (int k = 0; k < ns; ++k) {
                const int p = a.pos_of[cand[k]];
                const int kp = a.ckey[p];
                if (kp < 0) continue;
                const int ex = kp % gl0 + 1 - bx, ey = (kp / gl0) % gl1 + 1 - by, ez = kp / (gl0 * gl1) + 1 - bz;
                if (ex < -1 || ex > 1 || ey < -1 || ey > 1 || ez < -1 || ez > 1) continue;
                const float4 c = a.cposf[p];
                const float dx = (ui.x - (float)ex * cs[0]) - c.x;
                const float dy = (ui.y - (float)ey * cs[1]) - c.y;
                const float dz = (ui.z - (float)ez * cs[2]) - c.z;
                const float d2f = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                const float hsf = ui.w + c.w;
                const float r2f = hsf * hsf;
                if (d2f >= fmaf(r2f, khi, kb)) continue;
                double d2 = 0.0;
                if (d2f > fmaf(r2f, klo, -kb) || want_mind) {
                    const double4 cd = a.cpos[p];
                    d2 = exact_d2(xi, cd);
                    const double hs = __dadd_rn(cd.w, xi.w);
                    if (!(d2 < __dmul_rn(hs, hs))) continue;
                }
                const unsigned code = (unsigned)((ex + 1) + 3 * (ey + 1) + 9 * (ez + 1)) << 26;
                if (contact) {
                    if (a.cmat[p] != mati) {
                        if (nc < a.cstride) cout[nc] = (unsigned)p | code;
                        ++nc;
                        continue;
                    }
                } else if (a.nmat > 1 && (a.cmat[p] == mati) != (pass == 0)) {
                    continue;
                }
                if (want_mind) mind = fmin(mind, d2);
                if (nn < cap) out[nn] = (unsigned)p | code;
                ++nn;
            }
        }
        if (nn > cap) {
            atomicMax(&a.status->req_stride, nn);
            raise_status(a.status, MCM_ENBR_OVERFLOW, i);
        }
        if (contact && nc > a.cstride) {
            atomicMax(&a.status->req_cstride, nc);
            raise_status(a.status, MCM_ENBR_OVERFLOW, i);
        }
        // ghosts: as k_search, from the current grid's ghost cells
        if (a.prm.boundary) {
            const int lo0 = bx > 1 ? bx - 1 : 1, hi0 = bx < gl0 ? bx + 1 : gl0;
            const int lo1 = by > 1 ? by - 1 : 1, hi1 = by < gl1 ? by + 1 : gl1;
            const int lo2 = bz > 1 ? bz - 1 : 1, hi2 = bz < gl2 ? bz + 1 : gl2;
            const DevPlanes &pl = a.prm.planes;
            const bool near = (lo0 == 1 && pl.code[0][0]) || (hi0 == gl0 && pl.code[1][0]) ||
                              (lo1 == 1 && pl.code[0][1]) || (hi1 == gl1 && pl.code[1][1]) ||
                              (lo2 == 1 && pl.code[0][2]) || (hi2 == gl2 && pl.code[1][2]);
            if (near) {
                const int gpasses = (a.nmat > 1 && a.prm.contacttype == 0) ? 2 : 1;
                for (int pass = 0; pass < gpasses; ++pass) {
                    for (int nz = lo2; nz <= hi2; ++nz)
                        for (int my = lo1; my <= hi1; ++my)
                            for (int lx = lo0; lx <= hi0; ++lx) {
                                const int2 gcl = a.gcell[(lx - 1) + gl0 * ((my - 1) + gl1 * (nz - 1))];
                                for (int r = 0; r < gcl.y; ++r) {
                                    const int q = gcl.x + gcl.y - 1 - r;
                                    const double4 gq = make_double4(a.gx[q], a.gy[q], a.gz[q], a.gh[q]);
                                    const double d2 = exact_d2(xi, gq);
                                    const double hs = __dadd_rn(gq.w, xi.w);
                                    if (d2 < __dmul_rn(hs, hs)) {
                                        if (contact) {
                                            if (a.gmat[q] != mati) {
                                                if (gcn < a.gcstride) a.gcont[(size_t)gcn * np + t] = q;
                                                ++gcn;
                                                continue;
                                            }
                                        } else if (a.nmat > 1 && (a.gmat[q] == mati) != (pass == 0)) {
                                            continue;
                                        }
                                        mind = fmin(mind, d2);
                                        if (gn < a.gstride) a.gnbr[(size_t)gn * np + t] = q;
                                        ++gn;
                                    }
                                }
                            }
                }
                if (gn > a.gstride) {
                    atomicMax(&a.status->req_gstride, gn);
                    raise_status(a.status, MCM_ENBR_OVERFLOW, i);
                }
                if (gcn > a.gcstride) {
                    atomicMax(&a.status->req_gcstride, gcn);
                    raise_status(a.status, MCM_ENBR_OVERFLOW, i);
                }
            }
        }
        mind = sqrt(mind);
    }
    if (with_self) nn += 1;   // MCM/mcm_ll_neighbours.f90:288-299 (for every particle)
    a.nnbr[t] = nn;
    a.gnnbr[t] = gn;
    if (contact) { a.ncont[t] = nc; a.gncont[t] = gcn; }
    if (want_mind) a.F.f[FMINDIST][i] = mind;
    atomicMax(&a.status->max_nbr, nn);
    atomicMax(&a.status->max_gnbr, gn);
}

__global__ void k_skin_force(StepArgs a) {
    if (threadIdx.x == 0 && blockIdx.x == 0) a.skin_flags[0] = 1;
}

void launch_skin_force(const StepArgs &a, cudaStream_t s) { k_skin_force<<<1, 32, 0, s>>>(a); }

void launch_skin_search(const StepArgs &a, cudaStream_t s) {
    const int nb = (a.n + 255) / 256;
    k_skin_disp<<<nb < 148 * 8 ? nb : 148 * 8, 256, 0, s>>>(a);
    k_skin_decide<<<1, 32, 0, s>>>(a);
    k_skin_build<<<nb, 256, 0, s>>>(a);
    k_skin_filter<<<nb, 256, 0, s>>>(a);
}

void launch_search(const StepArgs &a, cudaStream_t s) {
    const int threads = search_threads_of(a);
    if (a.search_kind == 3) {
        // grid-stride over the cells (ncells is on the device): up to 16 blocks per SM
        long long b = (a.cell_cap + kCellWarps - 1) / kCellWarps;
        if (b > 148LL * 16) b = 148LL * 16;
        k_search_cell<<<(unsigned)(b < 1 ? 1 : b), kCellWarps * 32, 0, s>>>(a);
    } else if (a.search_kind == 2) {
        const long long lanes = 32LL * a.n;
        k_search_warp<<<(unsigned)((lanes + threads - 1) / threads), threads, 0, s>>>(a);
    } else {
        const bool mind = a.prm.tcrit_opt == 2 || a.prm.diag;
        const int v = (a.prm.contact ? kSrchContact : 0) | ((a.nmat > 1 && a.prm.contacttype == 0) ? kSrchTwoPass : 0) |
                      (mind ? kSrchMind : 0);
        const unsigned nb = (unsigned)((a.n + threads - 1) / threads);
        if (a.prm.xsort) {
            switch (v) {
                case 0: k_search<kSrchXWin><<<nb, threads, 0, s>>>(a); break;
                case kSrchContact: k_search<kSrchXWin | kSrchContact><<<nb, threads, 0, s>>>(a); break;
                case kSrchTwoPass: k_search<kSrchXWin | kSrchTwoPass><<<nb, threads, 0, s>>>(a); break;
                case kSrchMind: k_search<kSrchXWin | kSrchMind><<<nb, threads, 0, s>>>(a); break;
                case kSrchContact | kSrchMind: k_search<kSrchXWin | kSrchContact | kSrchMind><<<nb, threads, 0, s>>>(a); break;
                default: k_search<kSrchXWin | kSrchTwoPass | kSrchMind><<<nb, threads, 0, s>>>(a); break;
            }
        } else {
            switch (v) {
                case 0: k_search<0><<<nb, threads, 0, s>>>(a); break;
                case kSrchContact: k_search<kSrchContact><<<nb, threads, 0, s>>>(a); break;
                case kSrchTwoPass: k_search<kSrchTwoPass><<<nb, threads, 0, s>>>(a); break;
                case kSrchMind: k_search<kSrchMind><<<nb, threads, 0, s>>>(a); break;
                case kSrchContact | kSrchMind: k_search<kSrchContact | kSrchMind><<<nb, threads, 0, s>>>(a); break;
                default: k_search<kSrchTwoPass | kSrchMind><<<nb, threads, 0, s>>>(a); break;
            }
        }
    }
}

}  // namespace mcm

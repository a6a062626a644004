// noalloc.cu -- allocation-free variant of the per-material energy sums.
//
// mcm_gpu_calctotale_noalloc computes the per-material kinetic energy,
// internal energy and momentum sums that mcm_gpu_step_b computes (over every
// particle, with no active-particle filter, as step_b does), from device
// arrays the caller already owns, without allocating device memory.  It
// exists for callers that cannot call cudaMalloc: host codes that hand all
// device memory to their own pool or map the particle arrays to the device
// once and forbid further allocations, and drivers that must not add the
// device-wide synchronisation of cudaMalloc/cudaFree inside a time step.
//
// Scratch: the block partial sums live in g_noalloc_partials, a file-scope
// __device__ array of kNoAllocBlocks x 5 x MCM_GPU_MAX_MATERIALS doubles
// (296 x 80 x 8 B = 189 440 B).  Every GPU that loads the library holds it
// until the process exits.  All calls share it: each call overwrites every
// slot it later reads, so nothing has to start at zero, but calls whose
// kernels overlap on the GPU (different streams or devices sharing it) race.
#include <mutex>

#include "kernels.h"

namespace {

constexpr int kNoAllocBlocks = 296;   // 2 blocks per SM on a 148-SM B200
constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocValues = 5 * MCM_GPU_MAX_MATERIALS;

__device__ __align__(256) double g_noalloc_partials[kNoAllocBlocks * kNoAllocValues];

// Per-block sums: slot [block][5*(m-1) + {ke, ie, mom_x, mom_y, mom_z}] of
// 0.5 m |v|^2, e and m |v_d| over the particles of material m.  Particles with
// a material id outside 1..nmat are not counted.
__global__ void __launch_bounds__(kNoAllocThreads)
k_calctotale_partials(const double *mass, const double *vabs, const double *v, const double *e, const int *mat,
                      int np, int nmat, double *partials) {
    __shared__ double sm[kNoAllocThreads / 32];
    for (int m = 1; m <= nmat; ++m) {
        double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
            if (mat[i] != m) continue;
            const double mi = mass[i], va = vabs[i];
            acc[0] += 0.5 * mi * (va * va);
            acc[1] += e[i];
            acc[2] += mi * fabs(v[3 * (size_t)i + 0]);
            acc[3] += mi * fabs(v[3 * (size_t)i + 1]);
            acc[4] += mi * fabs(v[3 * (size_t)i + 2]);
        }
        for (int k = 0; k < 5; ++k) {
            double x = acc[k];
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            __syncthreads();
            if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = x;
            __syncthreads();
            if (threadIdx.x == 0) {
                double r = 0.0;
                for (int w = 0; w < kNoAllocThreads / 32; ++w) r += sm[w];
                partials[(size_t)blockIdx.x * kNoAllocValues + 5 * (m - 1) + k] = r;
            }
        }
    }
}

// One block: fixed-order sum of the block partials, then the totals (sums of
// ke and ie over the materials, and their sum), as step_b returns them.
__global__ void k_calctotale_finish(const double *partials, int nmat, double *out) {
    __shared__ double sm[32];
    for (int v = 0; v < 5 * nmat; ++v) {
        double x = 0.0;
        for (int b = threadIdx.x; b < kNoAllocBlocks; b += blockDim.x) x += partials[(size_t)b * kNoAllocValues + v];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        __syncthreads();
        if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = x;
        __syncthreads();
        if (threadIdx.x == 0) {
            double r = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += sm[w];
            out[v] = r;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ke = 0.0, ie = 0.0;
        for (int m = 0; m < nmat; ++m) { ke = ke + out[5 * m]; ie = ie + out[5 * m + 1]; }
        out[5 * nmat] = ke;
        out[5 * nmat + 1] = ie;
        out[5 * nmat + 2] = ke + ie;
    }
}

// Device address of g_noalloc_partials, looked up once per device (with that
// device current) by the first call on it and kept for the process.  The
// address belongs to the device's primary context: a process that resets the
// device (cudaDeviceReset) must not call the entry point afterwards.
std::mutex g_scratch_mu;
void *g_scratch_ptr[64] = {};

int scratch_address(double **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return MCM_ECUDA;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p) return MCM_ECUDA;
        g_scratch_ptr[dev] = p;
    }
    *out = static_cast<double *>(g_scratch_ptr[dev]);
    return MCM_OK;
}

}  // namespace

extern "C" int mcm_gpu_calctotale_noalloc(const double *mass, const double *vabs, const double *v, const double *e,
                                          const int *mat, int np, int nmat, double *energies, void *stream) {
    if (!mass || !vabs || !v || !e || !mat || !energies || np < 0) return MCM_EINVAL;
    if (nmat < 1 || nmat > MCM_GPU_MAX_MATERIALS) return MCM_EINVAL;   // scratch holds 16 materials
    // an error left pending by the caller's earlier CUDA calls is not this call's
    if (cudaPeekAtLastError() != cudaSuccess) return MCM_ECUDA;
    double *partials = nullptr;
    int st = scratch_address(&partials);
    if (st != MCM_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_calctotale_partials<<<kNoAllocBlocks, kNoAllocThreads, 0, s>>>(mass, vabs, v, e, mat, np, nmat, partials);
    if (cudaGetLastError() != cudaSuccess) return MCM_ECUDA;
    k_calctotale_finish<<<1, 256, 0, s>>>(partials, nmat, energies);
    if (cudaGetLastError() != cudaSuccess) return MCM_ECUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return MCM_ECUDA;
    return MCM_OK;
}

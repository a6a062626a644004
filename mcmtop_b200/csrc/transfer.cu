// transfer.cu -- layout conversion between the host arrays of the C ABI
// (Fortran order: vectors (3,np), tensors (3,3,np), particle index = the
// reference index) and the device's per-field arrays in storage order.
// A host array crosses PCIe in one contiguous copy into a device staging
// buffer; these kernels scatter it into the fields (upload) or gather the
// fields into it (download, undoing the storage permutation).
#include "kernels.h"

namespace mcm {

// Upload: record i of the staging buffer (width doubles) goes to particle i
// (storage order equals the reference order right after an upload).
__global__ void k_unpack(StepArgs a, PackSpec s, const double *__restrict__ stage) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const double *rec = stage + (size_t)s.width * i;
#pragma unroll 9
        for (int k = 0; k < s.width; ++k)
            if (s.field[k] >= 0) a.F.f[s.field[k]][i] = rec[k];
    }
}

// Download: the particle at storage position p is reference particle orig[p];
// its record gets each entry from a field (times its sign) or zero.
__global__ void k_pack(StepArgs a, PackSpec s, double *__restrict__ stage) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += gridDim.x * blockDim.x) {
        double *rec = stage + (size_t)s.width * a.F.orig[p];
#pragma unroll 9
        for (int k = 0; k < s.width; ++k)
            rec[k] = s.field[k] >= 0 ? s.sign[k] * a.F.f[s.field[k]][p] : 0.0;
    }
}

static int transfer_blocks(int n) {
    int b = (n + 255) / 256;
    return b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b);
}

void launch_unpack(const StepArgs &a, const PackSpec &s, const double *stage, cudaStream_t st) {
    k_unpack<<<transfer_blocks(a.n), 256, 0, st>>>(a, s, stage);
}

void launch_pack(const StepArgs &a, const PackSpec &s, double *stage, cudaStream_t st) {
    k_pack<<<transfer_blocks(a.n), 256, 0, st>>>(a, s, stage);
}

}  // namespace mcm

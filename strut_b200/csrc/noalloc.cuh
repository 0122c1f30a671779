// Factor-solve of one band system with no device allocation (included once, by strut_cuda.cu).
//
// strut_gpu_band_solve_noalloc runs the BandGeneral / BandSPD factor and solve of the Newton
// kernel (band_lu_smem / band_chol_smem and the same substitutions) on one system the caller
// already holds in device memory.  The dense partial-pivot fallback of BandGeneral
// (linear_solver_backend.mojo:175-240, 650-657) needs an n x n work matrix and n pivots; here
// they live in file-scope static device arrays sized for kNoAllocMaxN, whose device addresses
// are looked up once per device, so a call never allocates.
#pragma once

#include <mutex>

namespace strut {

constexpr int kNoAllocMaxN = 512;               // largest system order accepted
constexpr size_t kNoAllocSmemMax = 220 * 1024;  // band + 4 vectors in shared memory

// Shared by every call on a device and kept between calls.  Nothing in them has to start at
// zero: a call writes every entry of the n x n work matrix and the n pivots before reading them.
static __device__ __align__(256) double g_noalloc_dense[kNoAllocMaxN * kNoAllocMaxN];  // 2 MiB
static __device__ __align__(256) int g_noalloc_piv[kNoAllocMaxN];

// One CTA: load the band (BandGeneral n x (2bw+1) as stored; BandSPD n x (bw+1) with slot
// row*(bw+1) + (row-col), expanded into the lower half of the general layout), factor, fall back
// to the dense LU in `dense` / `piv` when a row swap is needed, solve, write x and *status
// (0 ok, 2 singular or not positive definite).
__global__ void __launch_bounds__(256) band_solve_one_kernel(const double* __restrict__ band, int n,
                                                             int bw, int spd,
                                                             const double* __restrict__ rhs,
                                                             double* __restrict__ x,
                                                             int* __restrict__ status,
                                                             double* __restrict__ dense,
                                                             int* __restrict__ piv) {
    extern __shared__ __align__(16) double smem_one[];
    __shared__ double red[32];
    __shared__ int red_r[32];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int rw = 2 * bw + 1;
    double* Kb = smem_one;
    double* R = Kb + (size_t)n * rw;
    double* w = R + n;
    double* xs = w + n;
    double* fac = xs + n;
    for (int t = tid; t < n * rw; t += nt) {
        const int i = t / rw, j = i + t % rw - bw;
        double v = 0.0;
        if (j >= 0 && j < n) {
            if (!spd)
                v = band[t];
            else if (j <= i)
                v = band[(size_t)i * (bw + 1) + (i - j)];
        }
        Kb[t] = v;
    }
    for (int i = tid; i < n; i += nt) R[i] = rhs[i];
    __syncthreads();
    int rc = spd ? band_chol_smem(Kb, n, bw, rw, fac) : band_lu_smem(Kb, n, bw, rw, fac);
    bool use_dense = false;
    if (rc == 6) {
        // the whole n x n work matrix is rewritten from the caller's band before the dense LU
        __syncthreads();
        for (long long t = tid; t < (long long)n * n; t += nt) {
            const int i = (int)(t / n), j = (int)(t % n);
            const int o = j - i + bw;
            dense[t] = (o >= 0 && o < rw) ? band[(size_t)i * rw + o] : 0.0;
        }
        __syncthreads();
        rc = dense_lu_global(dense, piv, n, fac, red, red_r);
        use_dense = true;
    }
    if (rc != 0) {
        if (tid == 0) *status = rc;
        return;
    }
    __syncthreads();
    if (tid < 32) {
        if (use_dense)
            dense_solve_warp(dense, piv, n, R, w, xs);
        else if (spd)
            band_solve_chol_warp(Kb, n, bw, rw, R, w, xs);
        else
            band_solve_lu_warp(Kb, n, bw, rw, R, w, xs);
    }
    __syncthreads();
    for (int i = tid; i < n; i += nt) x[i] = xs[i];
    if (tid == 0) *status = 0;
}

}  // namespace strut

namespace {

struct NoAllocDevice {
    double* dense = nullptr;  // device address of g_noalloc_dense on this device
    int* piv = nullptr;       // device address of g_noalloc_piv on this device
    size_t smem_limit = 0;    // dynamic shared memory the kernel may use on this device
    bool ready = false;
};
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc[kNoAllocMaxDevices];

}  // namespace

extern "C" int strut_gpu_band_solve_noalloc(const double* band_dev, int32_t n, int32_t half_bw,
                                            int32_t system, const double* rhs_dev, double* x_dev,
                                            int32_t* status_dev, void* stream) {
    if (system != STRUT_SYSTEM_BAND_GENERAL && system != STRUT_SYSTEM_BAND_SPD)
        return fail(STRUT_BAD_ARG, "system must be BandGeneral (1) or BandSPD (2)");
    if (n < 1 || n > strut::kNoAllocMaxN)
        return fail(STRUT_BAD_ARG, "n = " + std::to_string(n) + " is outside 1.." +
                                       std::to_string(strut::kNoAllocMaxN) +
                                       " (the static scratch of strut_gpu_band_solve_noalloc)");
    if (half_bw < 0 || half_bw > n - 1) return fail(STRUT_BAD_ARG, "half_bw must be in 0..n-1");
    if (!band_dev || !rhs_dev || !x_dev || !status_dev) return fail(STRUT_BAD_ARG, "null pointer");
    const int rw = 2 * half_bw + 1;
    const size_t smem = ((size_t)n * rw + 4 * (size_t)n) * sizeof(double);
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(STRUT_UNSUPPORTED, "device index too large");
    NoAllocDevice& D = g_noalloc[dev];
    {
        // first call on this device (its context current): look up the scratch's device
        // addresses and raise the kernel's shared-memory limit to what the device allows next
        // to the kernel's static shared memory; later calls reuse them
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!D.ready) {
            CK(cudaGetSymbolAddress((void**)&D.dense, strut::g_noalloc_dense));
            CK(cudaGetSymbolAddress((void**)&D.piv, strut::g_noalloc_piv));
            int optin = 0;
            CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
            cudaFuncAttributes fa;
            CK(cudaFuncGetAttributes(&fa, strut::band_solve_one_kernel));
            const size_t room = (size_t)optin > fa.sharedSizeBytes ? (size_t)optin - fa.sharedSizeBytes : 0;
            D.smem_limit = std::min(strut::kNoAllocSmemMax, room);
            CK(cudaFuncSetAttribute(strut::band_solve_one_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)D.smem_limit));
            D.ready = true;
        }
    }
    if (smem > D.smem_limit)
        return fail(STRUT_UNSUPPORTED, "n x (2*half_bw+1) band does not fit in shared memory");
    strut::band_solve_one_kernel<<<1, 256, smem, (cudaStream_t)stream>>>(
        band_dev, n, half_bw, system == STRUT_SYSTEM_BAND_SPD ? 1 : 0, rhs_dev, x_dev, status_dev, D.dense,
        D.piv);
    CK(cudaGetLastError());
    return STRUT_OK;
}

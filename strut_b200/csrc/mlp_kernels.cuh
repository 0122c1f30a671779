// Learned Newton predictor on the 5th-generation tensor cores (sm_100a).
//
// A per-node MLP, n_in -> 128 GELU -> 128 GELU -> n_out, applied to one 128-node tile per CTA:
// every layer is tcgen05.mma kind::f16 with bf16 operands in shared memory and fp32 accumulators
// in tensor memory (TMEM), issued by one thread and completed through tcgen05.commit on an
// mbarrier; the epilogues read the accumulators with tcgen05.ld (one warp per 32 TMEM lanes),
// add the bias, apply GELU in fp32 and write the next layer's bf16 operand back to shared memory.
// The weights and the feature tiles are stored in global memory already in the shared-memory
// operand layout, so they are staged with cp.async.bulk (the TMA unit's bulk copy, no multicast).
//
// Operand layout ("chunk-major", no swizzle): element (r, k) of an R-row operand whose rows are
// contiguous in K sits at byte ((k / 8) * R + r) * 16 + (k % 8) * 2.  Eight consecutive rows of
// one 8-element K chunk form one 128-byte core matrix; the MMA descriptor of K step s (16
// elements) starts at chunk 2s with leading-dimension offset R * 16 bytes (chunk 2s -> 2s + 1)
// and stride-dimension offset 128 bytes (8-row group -> next).
//
// Training (one fused forward + backward per tile, gradients of the tile written as partials,
// then reduced in tile order and applied with Adam) uses the same primitives.  The network and
// its roundings are restated on the CPU by the oracle the tests compare against.  Strut has no
// learned predictor; this is the network of the north-star configuration.
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

namespace strut {

constexpr int kMlpH = 128;     // hidden width
constexpr int kMlpKin = 48;    // input features, padded (a multiple of 16; 41 for a 3D node)
constexpr int kMlpNout = 16;   // outputs, padded (N of the last MMA)
constexpr int kMlpTile = 128;  // rows (nodes) per CTA = MMA M

// ---- shared-memory / mbarrier / bulk-copy primitives (element_kernels.cuh has the same) ----
__device__ __forceinline__ uint32_t mlp_smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mlp_mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mlp_smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mlp_mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mlp_smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mlp_bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            mlp_smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(mlp_smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mlp_mbar_wait(uint64_t* bar, uint32_t parity) {
    for (int i = 0; i < (1 << 20); ++i) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, "
            "p;\n}\n"
            : "=r"(ok)
            : "r"(mlp_smem_u32(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// ---- tcgen05 / TMEM primitives ----
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(mlp_smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes made visible to the tensor cores (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Shared-memory matrix descriptor, K-major, no swizzle (layout type 0), descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc(const void* smem, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    const uint32_t a = mlp_smem_u32(smem);
    uint64_t d = 0;
    d |= (uint64_t)((a >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::f16: bf16 A and B (both K-major), fp32 accumulator, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

// Arrives on the mbarrier once every MMA this thread issued before has completed.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     mlp_smem_u32(bar))
                 : "memory");
}

// 16 consecutive fp32 columns of this thread's TMEM lane (the warp's 32-lane quarter).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Byte offset of element (r, k) in a chunk-major operand of R rows.
__host__ __device__ __forceinline__ uint32_t chunk_off(int r, int k, int R) {
    return (uint32_t)(((k >> 3) * R + r) * 16 + (k & 7) * 2);
}

// D (TMEM) = A (128 x K) B^T (N x K), both chunk-major in shared memory.  One thread.
__device__ __forceinline__ void umma_gemm(uint32_t d_tmem, const void* A, const void* B, int K, int N,
                                          bool accumulate) {
    const uint32_t idesc = umma_idesc_bf16(128, N);
    for (int s = 0; s < K / 16; ++s) {
        const uint64_t a = umma_desc((const char*)A + (size_t)2 * s * 128 * 16, 128 * 16, 128);
        const uint64_t b = umma_desc((const char*)B + (size_t)2 * s * N * 16, N * 16, 128);
        umma_bf16(d_tmem, a, b, idesc, (accumulate || s > 0) ? 1u : 0u);
    }
}

__device__ __forceinline__ float gelu_tanh(float z) {
    const float t = tanhf(0.7978845608028654f * (z + 0.044715f * z * z * z));
    return 0.5f * z * (1.0f + t);
}
__device__ __forceinline__ float gelu_tanh_grad(float z) {
    const float t = tanhf(0.7978845608028654f * (z + 0.044715f * z * z * z));
    const float dt = (1.0f - t * t) * 0.7978845608028654f * (1.0f + 3.0f * 0.044715f * z * z);
    return 0.5f * (1.0f + t) + 0.5f * z * dt;
}

// Writes 16 consecutive columns [c, c + 16) of row r as bf16 into a chunk-major operand of R rows
// (two 16-byte stores; consecutive rows go to consecutive 16-byte slots).
__device__ __forceinline__ void store_row16(char* base, int r, int c, int R, const float* v) {
    uint32_t w[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const __nv_bfloat162 p = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
        w[i] = *reinterpret_cast<const uint32_t*>(&p);
    }
    *reinterpret_cast<uint4*>(base + chunk_off(r, c, R)) = make_uint4(w[0], w[1], w[2], w[3]);
    *reinterpret_cast<uint4*>(base + chunk_off(r, c + 8, R)) = make_uint4(w[4], w[5], w[6], w[7]);
}

struct MlpDev {
    const __nv_bfloat16* w1t;  // chunk-major, kMlpH rows x kMlpKin  (layer-1 B operand)
    const __nv_bfloat16* w2t;  // chunk-major, kMlpH rows x kMlpH
    const __nv_bfloat16* w3t;  // chunk-major, kMlpNout rows x kMlpH
    const float* b1;           // kMlpH
    const float* b2;           // kMlpH
    const float* b3;           // kMlpNout
};

constexpr uint32_t kMlpBytesX = kMlpTile * kMlpKin * 2;   // 12 KiB
constexpr uint32_t kMlpBytesW1 = kMlpH * kMlpKin * 2;     // 12 KiB
constexpr uint32_t kMlpBytesH = kMlpTile * kMlpH * 2;     // 32 KiB
constexpr uint32_t kMlpBytesW2 = kMlpH * kMlpH * 2;       // 32 KiB
constexpr uint32_t kMlpBytesW3 = kMlpNout * kMlpH * 2;    // 4 KiB
constexpr uint32_t kMlpFwdSmem = kMlpBytesX + kMlpBytesW1 + 2 * kMlpBytesH + kMlpBytesW2 + kMlpBytesW3 + 1024;

// Forward pass of tile blockIdx.x: xt holds the feature tiles (chunk-major, kMlpTile rows each,
// rows beyond n_rows zero), y receives n_out fp32 outputs per row.  128 threads.
__global__ void __launch_bounds__(128) mlp_forward_kernel(MlpDev w, const __nv_bfloat16* __restrict__ xt,
                                                          int n_rows, float* __restrict__ y, int n_out,
                                                          int* __restrict__ err) {
    extern __shared__ __align__(1024) char smem_mlp[];
    char* X = smem_mlp;
    char* W1 = X + kMlpBytesX;
    char* H1 = W1 + kMlpBytesW1;
    char* H2 = H1 + kMlpBytesH;
    char* W2 = H2 + kMlpBytesH;
    char* W3 = W2 + kMlpBytesW2;
    __shared__ __align__(8) uint64_t bar_ld, bar_mma;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int tile = blockIdx.x;
    if (warp == 0) {
        tmem_alloc(&tmem_base, 256);
        tmem_relinquish();
    }
    if (tid == 0) {
        mlp_mbar_init(&bar_ld, 1);
        mlp_mbar_init(&bar_mma, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tb = tmem_base;
    if (tid == 0) {
        mlp_mbar_expect_tx(&bar_ld, kMlpBytesX + kMlpBytesW1 + kMlpBytesW2 + kMlpBytesW3);
        mlp_bulk_g2s(X, (const char*)xt + (size_t)tile * kMlpBytesX, kMlpBytesX, &bar_ld);
        mlp_bulk_g2s(W1, w.w1t, kMlpBytesW1, &bar_ld);
        mlp_bulk_g2s(W2, w.w2t, kMlpBytesW2, &bar_ld);
        mlp_bulk_g2s(W3, w.w3t, kMlpBytesW3, &bar_ld);
    }
    // every thread takes the same branch; on a timeout nothing more is issued
    bool ok = __syncthreads_and(mlp_mbar_wait(&bar_ld, 0) ? 1 : 0) != 0;
    // layer 1: D[0,128) = X W1t^T
    if (tid == 0 && ok) {
        tc_fence_after();
        umma_gemm(tb + 0, X, W1, kMlpKin, kMlpH, false);
        umma_commit(&bar_mma);
    }
    ok = ok && __syncthreads_and(mlp_mbar_wait(&bar_mma, 0) ? 1 : 0) != 0;
    tc_fence_after();
    const uint32_t lane_off = (uint32_t)(32 * warp) << 16;
    float v[16];
    if (ok) {
        for (int c = 0; c < kMlpH; c += 16) {
            tmem_ld16(tb + lane_off + c, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = gelu_tanh(v[i] + w.b1[c + i]);
            store_row16(H1, tid, c, kMlpTile, v);
        }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    // layer 2: D[128,256) = H1 W2t^T
    if (tid == 0 && ok) {
        tc_fence_after();
        umma_gemm(tb + 128, H1, W2, kMlpH, kMlpH, false);
        umma_commit(&bar_mma);
    }
    ok = ok && __syncthreads_and(mlp_mbar_wait(&bar_mma, 1) ? 1 : 0) != 0;
    tc_fence_after();
    if (ok) {
        for (int c = 0; c < kMlpH; c += 16) {
            tmem_ld16(tb + lane_off + 128 + c, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = gelu_tanh(v[i] + w.b2[c + i]);
            store_row16(H2, tid, c, kMlpTile, v);
        }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    // layer 3: D[0,16) = H2 W3t^T
    if (tid == 0 && ok) {
        tc_fence_after();
        umma_gemm(tb + 0, H2, W3, kMlpH, kMlpNout, false);
        umma_commit(&bar_mma);
    }
    ok = ok && __syncthreads_and(mlp_mbar_wait(&bar_mma, 0) ? 1 : 0) != 0;
    tc_fence_after();
    if (ok) {
        tmem_ld16(tb + lane_off + 0, v);
        const int row = tile * kMlpTile + tid;
        if (row < n_rows)
            for (int i = 0; i < n_out; ++i) y[(size_t)row * n_out + i] = v[i] + w.b3[i];
    } else {
        // a wait ran out: let the copies and MMAs in flight finish (bounded) before the TMEM
        // columns are released
        if (tid == 0) atomicExch(err, 1);
        mlp_mbar_wait(&bar_ld, 0);
        mlp_mbar_wait(&bar_mma, 0);
        mlp_mbar_wait(&bar_mma, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tb, 256);
}

// ---- training: fused forward + backward of one tile ------------------------------------------

struct MlpTrainDev {
    MlpDev f;                  // forward operands
    const __nv_bfloat16* w2;   // chunk-major, kMlpH rows (inputs) x kMlpH (outputs): dH1 = dZ2 W2^T
    const __nv_bfloat16* w3;   // chunk-major, kMlpH rows (inputs) x kMlpNout (outputs): dH2 = dY W3^T
};

constexpr uint32_t kMlpBytesXT = kMlpKin * kMlpTile * 2;   // X^T: kMlpKin rows x kMlpTile   12 KiB
constexpr uint32_t kMlpBytesDY = kMlpTile * kMlpNout * 2;  // dY: 128 rows x 16                4 KiB
// region offsets (bytes) of the training kernel's shared memory
constexpr uint32_t kTrX = 0;
constexpr uint32_t kTrXT = kTrX + kMlpBytesX;
constexpr uint32_t kTrW1 = kTrXT + kMlpBytesXT;
constexpr uint32_t kTrW3t = kTrW1 + kMlpBytesW1;
constexpr uint32_t kTrW3 = kTrW3t + kMlpBytesW3;
constexpr uint32_t kTrDY = kTrW3 + kMlpBytesW3;
constexpr uint32_t kTrDYT = kTrDY + kMlpBytesDY;
constexpr uint32_t kTrH1T = kTrDYT + kMlpBytesDY;          // H1^T (dW2's A)
constexpr uint32_t kTrR1 = kTrH1T + kMlpBytesH;            // H2^T (dW3's A), then W2 (dH1's B)
constexpr uint32_t kTrR2 = kTrR1 + kMlpBytesH;             // W2t (layer-2 B), then dZ2 (dH1's A)
constexpr uint32_t kTrR3 = kTrR2 + kMlpBytesH;             // H1 (layer-2 A), then dZ2^T (dW2's B)
constexpr uint32_t kTrR4 = kTrR3 + kMlpBytesH;             // H2 (layer-3 A), then dZ1^T (dW1t's A)
constexpr uint32_t kTrRed = kTrR4 + kMlpBytesH;            // 4 warps x 128 floats (column sums)
constexpr uint32_t kMlpTrainSmem = kTrRed + 4 * kMlpH * 4 + 1024;  // 215 KiB
static_assert(kMlpTrainSmem <= 227 * 1024, "training tile exceeds the opt-in shared memory");

// Writes element (r, k) = v as bf16 into a chunk-major operand of R rows.
__device__ __forceinline__ void store_bf16(char* base, int r, int k, int R, float v) {
    *reinterpret_cast<__nv_bfloat16*>(base + chunk_off(r, k, R)) = __float2bfloat16_rn(v);
}

// Column sums of 16 values per thread over the 128 rows of the tile: warp shuffles, then the 4
// warps' partials in warp order (red: 4 x kMlpH floats).  Call with all 128 threads.
__device__ __forceinline__ void colsum16(const float* v, int c, float* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        float x = v[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[warp * kMlpH + c + i] = x;
    }
}

// One tile: forward (layers 1-3), mean-squared-error gradient dY = inv_count (Y - T) (rows
// >= n_rows and outputs >= n_out contribute nothing), backward; writes the tile's parameter
// gradients in the packed master layout (W1 n_in x H, b1, W2 H x H, b2, W3 H x n_out, b3) to
// part[tile * n_params ...] and its sum of squared errors to sse[tile].  128 threads.
__global__ void __launch_bounds__(128) mlp_train_tile_kernel(MlpTrainDev w, const __nv_bfloat16* __restrict__ xt,
                                                             const float* __restrict__ tgt, int n_rows, int n_in,
                                                             int n_out, float inv_count, float* __restrict__ part,
                                                             int n_params, double* __restrict__ sse,
                                                             int* __restrict__ err) {
    extern __shared__ __align__(1024) char smem_tr[];
    char* X = smem_tr + kTrX;
    char* XT = smem_tr + kTrXT;
    char* W1 = smem_tr + kTrW1;
    char* W3t = smem_tr + kTrW3t;
    char* W3 = smem_tr + kTrW3;
    char* DY = smem_tr + kTrDY;
    char* DYT = smem_tr + kTrDYT;
    char* H1T = smem_tr + kTrH1T;
    char* R1 = smem_tr + kTrR1;
    char* R2 = smem_tr + kTrR2;
    char* R3 = smem_tr + kTrR3;
    char* R4 = smem_tr + kTrR4;
    float* red = reinterpret_cast<float*>(smem_tr + kTrRed);
    __shared__ __align__(8) uint64_t bar_ld, bar_w2, bar_mma;
    __shared__ uint32_t tmem_base;
    __shared__ double sse_w[4];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tile = blockIdx.x;
    const int row = tile * kMlpTile + tid;
    float* gp = part + (size_t)tile * n_params;
    float* gW1 = gp;
    float* gb1 = gW1 + n_in * kMlpH;
    float* gW2 = gb1 + kMlpH;
    float* gb2 = gW2 + kMlpH * kMlpH;
    float* gW3 = gb2 + kMlpH;
    float* gb3 = gW3 + kMlpH * n_out;
    if (warp == 0) {
        tmem_alloc(&tmem_base, 512);
        tmem_relinquish();
    }
    if (tid == 0) {
        mlp_mbar_init(&bar_ld, 1);
        mlp_mbar_init(&bar_w2, 1);
        mlp_mbar_init(&bar_mma, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tb = tmem_base;
    const uint32_t lo = (uint32_t)(32 * warp) << 16;  // this warp's TMEM lanes
    if (tid == 0) {
        mlp_mbar_expect_tx(&bar_ld, kMlpBytesX + kMlpBytesW1 + kMlpBytesW2 + 2 * kMlpBytesW3);
        mlp_bulk_g2s(X, (const char*)xt + (size_t)tile * kMlpBytesX, kMlpBytesX, &bar_ld);
        mlp_bulk_g2s(W1, w.f.w1t, kMlpBytesW1, &bar_ld);
        mlp_bulk_g2s(R2, w.f.w2t, kMlpBytesW2, &bar_ld);
        mlp_bulk_g2s(W3t, w.f.w3t, kMlpBytesW3, &bar_ld);
        mlp_bulk_g2s(W3, w.w3, kMlpBytesW3, &bar_ld);
    }
    bool ok = __syncthreads_and(mlp_mbar_wait(&bar_ld, 0) ? 1 : 0) != 0;
    uint32_t mma_phase = 0;
    auto mma_wait = [&]() {
        ok = ok && __syncthreads_and(mlp_mbar_wait(&bar_mma, mma_phase) ? 1 : 0) != 0;
        mma_phase ^= 1u;
        tc_fence_after();
    };
    auto mma_begin = [&]() {
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
    };
    // X^T (dW1t's B operand): element (k, r) = X(r, k)
    if (ok) {
        for (int k = 0; k < kMlpKin; ++k) {
            const __nv_bfloat16 v = *reinterpret_cast<const __nv_bfloat16*>(X + chunk_off(tid, k, kMlpTile));
            *reinterpret_cast<__nv_bfloat16*>(XT + chunk_off(k, tid, kMlpKin)) = v;
        }
    }
    // ---- forward
    if (tid == 0 && ok) {
        tc_fence_after();
        umma_gemm(tb + 0, X, W1, kMlpKin, kMlpH, false);
        umma_commit(&bar_mma);
    }
    mma_wait();
    float v[16];
    if (ok) {
        for (int c = 0; c < kMlpH; c += 16) {
            tmem_ld16(tb + lo + c, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                v[i] = gelu_tanh(v[i] + w.f.b1[c + i]);
                store_bf16(H1T, c + i, tid, kMlpH, v[i]);
            }
            store_row16(R3, tid, c, kMlpTile, v);
        }
    }
    mma_begin();
    if (tid == 0 && ok) {
        tc_fence_after();
        umma_gemm(tb + 128, R3, R2, kMlpH, kMlpH, false);
        umma_commit(&bar_mma);
    }
    mma_wait();
    if (ok) {
        for (int c = 0; c < kMlpH; c += 16) {
            tmem_ld16(tb + lo + 128 + c, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                v[i] = gelu_tanh(v[i] + w.f.b2[c + i]);
                store_bf16(R1, c + i, tid, kMlpH, v[i]);  // H2^T
            }
            store_row16(R4, tid, c, kMlpTile, v);         // H2
        }
    }
    mma_begin();
    if (tid == 0 && ok) {
        tc_fence_after();
        umma_gemm(tb + 256, R4, W3t, kMlpH, kMlpNout, false);
        umma_commit(&bar_mma);
    }
    mma_wait();
    // ---- output error: dY, its transpose, db3, squared error
    double se = 0.0;
    if (ok) {
        tmem_ld16(tb + lo + 256, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            float d = 0.0f;
            if (row < n_rows && i < n_out) {
                const float yv = v[i] + w.f.b3[i];
                d = yv - tgt[(size_t)row * n_out + i];
                se += (double)d * (double)d;
            }
            v[i] = inv_count * d;
            store_bf16(DYT, i, tid, kMlpNout, v[i]);
        }
        store_row16(DY, tid, 0, kMlpTile, v);
        colsum16(v, 0, red);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
    if (lane == 0) sse_w[warp] = se;
    mma_begin();
    if (tid == 0) sse[tile] = ((sse_w[0] + sse_w[1]) + sse_w[2]) + sse_w[3];
    if (tid < n_out && ok) gb3[tid] = ((red[tid] + red[kMlpH + tid]) + red[2 * kMlpH + tid]) + red[3 * kMlpH + tid];
    // ---- layer 3 backward: dW3 = H2^T dY (cols 272..287), dH2 = dY W3^T (cols 384..511)
    if (tid == 0 && ok) {
        tc_fence_after();
        umma_gemm(tb + 272, R1, DYT, kMlpTile, kMlpNout, false);
        umma_gemm(tb + 384, DY, W3, kMlpNout, kMlpH, false);
        umma_commit(&bar_mma);
    }
    mma_wait();
    // W2 (dH1's B) into the H2^T region, now free
    if (tid == 0 && ok) {
        fence_async_smem();
        mlp_mbar_expect_tx(&bar_w2, kMlpBytesW2);
        mlp_bulk_g2s(R1, w.w2, kMlpBytesW2, &bar_w2);
    }
    if (ok) {
        tmem_ld16(tb + lo + 272, v);  // dW3 row = input tid
        for (int i = 0; i < n_out; ++i) gW3[tid * n_out + i] = v[i];
        for (int c = 0; c < kMlpH; c += 16) {
            float z[16];
            tmem_ld16(tb + lo + 384 + c, v);   // dH2
            tmem_ld16(tb + lo + 128 + c, z);   // layer-2 accumulator
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                v[i] = v[i] * gelu_tanh_grad(z[i] + w.f.b2[c + i]);  // dZ2
                store_bf16(R3, c + i, tid, kMlpH, v[i]);           // dZ2^T (dW2's B)
            }
            store_row16(R2, tid, c, kMlpTile, v);                  // dZ2 (dH1's A)
            colsum16(v, c, red);
        }
    }
    ok = ok && __syncthreads_and(mlp_mbar_wait(&bar_w2, 0) ? 1 : 0) != 0;
    mma_begin();
    if (ok) gb2[tid] = ((red[tid] + red[kMlpH + tid]) + red[2 * kMlpH + tid]) + red[3 * kMlpH + tid];
    // ---- layer 2 backward: dW2 = H1^T dZ2 (cols 256..383), dH1 = dZ2 W2^T (cols 384..511)
    if (tid == 0 && ok) {
        tc_fence_after();
        umma_gemm(tb + 256, H1T, R3, kMlpTile, kMlpH, false);
        umma_gemm(tb + 384, R2, R1, kMlpH, kMlpH, false);
        umma_commit(&bar_mma);
    }
    mma_wait();
    if (ok) {
        for (int c = 0; c < kMlpH; c += 16) {
            tmem_ld16(tb + lo + 256 + c, v);  // dW2 row = input tid
#pragma unroll
            for (int i = 0; i < 16; ++i) gW2[tid * kMlpH + c + i] = v[i];
        }
        for (int c = 0; c < kMlpH; c += 16) {
            float z[16];
            tmem_ld16(tb + lo + 384 + c, v);  // dH1
            tmem_ld16(tb + lo + 0 + c, z);    // layer-1 accumulator
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                v[i] = v[i] * gelu_tanh_grad(z[i] + w.f.b1[c + i]);  // dZ1
                store_bf16(R4, c + i, tid, kMlpH, v[i]);           // dZ1^T (dW1t's A)
            }
            colsum16(v, c, red);
        }
    }
    mma_begin();
    if (ok) gb1[tid] = ((red[tid] + red[kMlpH + tid]) + red[2 * kMlpH + tid]) + red[3 * kMlpH + tid];
    // ---- layer 1 backward: dW1t = dZ1^T X (rows: outputs, cols 128..175: inputs)
    if (tid == 0 && ok) {
        tc_fence_after();
        umma_gemm(tb + 128, R4, XT, kMlpTile, kMlpKin, false);
        umma_commit(&bar_mma);
    }
    mma_wait();
    if (ok) {
        for (int c = 0; c < kMlpKin; c += 16) {
            tmem_ld16(tb + lo + 128 + c, v);  // row = output tid, cols = inputs c..c+15
#pragma unroll
            for (int i = 0; i < 16; ++i)
                if (c + i < n_in) gW1[(c + i) * kMlpH + tid] = v[i];
        }
    } else {
        // a wait ran out: let the copies and MMAs in flight finish (bounded) before the TMEM
        // columns are released
        if (tid == 0) atomicExch(err, 1);
        mlp_mbar_wait(&bar_ld, 0);
        mlp_mbar_wait(&bar_w2, 0);
        mlp_mbar_wait(&bar_mma, 0);
        mlp_mbar_wait(&bar_mma, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tb, 512);
}

// Sums the tiles' gradients in tile order and applies one Adam step to the fp32 masters
// (c1 = 1 - beta1^t, c2 = 1 - beta2^t).  With lr == 0 only the summed gradient is written to
// grad_out (when not null).
__global__ void mlp_adam_kernel(float* __restrict__ params, float* __restrict__ m, float* __restrict__ v,
                                const float* __restrict__ part, int n_tiles, int n_params, float lr, float b1,
                                float b2, float c1, float c2, float eps, float* __restrict__ grad_out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_params) return;
    float g = 0.0f;
    for (int t = 0; t < n_tiles; ++t) g += part[(size_t)t * n_params + p];
    if (grad_out) grad_out[p] = g;
    if (lr == 0.0f) return;
    const float mp = b1 * m[p] + (1.0f - b1) * g;
    const float vp = b2 * v[p] + (1.0f - b2) * g * g;
    m[p] = mp;
    v[p] = vp;
    params[p] = params[p] - lr * (mp / c1) / (sqrtf(vp / c2) + eps);
}

}  // namespace strut

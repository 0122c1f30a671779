// Host side of the learned Newton predictor's network (included once, by strut_cuda.cu).
#pragma once

#include "mlp_kernels.cuh"

namespace strut {

// fp32 masters (packed: W1 n_in x H, b1 H, W2 H x H, b2 H, W3 H x n_out, b3 n_out; W[k][j] maps
// input k to output j) -> bf16 chunk-major B operands (rows = outputs) and padded biases.
__global__ void mlp_pack_params_kernel(const float* __restrict__ p, int n_in, int n_out,
                                       __nv_bfloat16* __restrict__ w1t, __nv_bfloat16* __restrict__ w2t,
                                       __nv_bfloat16* __restrict__ w3t, __nv_bfloat16* __restrict__ w2,
                                       __nv_bfloat16* __restrict__ w3, float* __restrict__ b1,
                                       float* __restrict__ b2, float* __restrict__ b3) {
    const float* W1 = p;
    const float* B1 = W1 + n_in * kMlpH;
    const float* W2 = B1 + kMlpH;
    const float* B2 = W2 + kMlpH * kMlpH;
    const float* W3 = B2 + kMlpH;
    const float* B3 = W3 + kMlpH * n_out;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < kMlpH * kMlpKin) {  // W1t: row h, col k
        const int h = t / kMlpKin, k = t % kMlpKin;
        const float v = k < n_in ? W1[k * kMlpH + h] : 0.0f;
        *reinterpret_cast<__nv_bfloat16*>((char*)w1t + chunk_off(h, k, kMlpH)) = __float2bfloat16_rn(v);
    }
    if (t < kMlpH * kMlpH) {  // W2t: row h (out), col k (in)
        const int h = t / kMlpH, k = t % kMlpH;
        *reinterpret_cast<__nv_bfloat16*>((char*)w2t + chunk_off(h, k, kMlpH)) =
            __float2bfloat16_rn(W2[k * kMlpH + h]);
    }
    if (t < kMlpH * kMlpH) {  // W2 (backward B operand): row k (in), col h (out)
        const int k = t / kMlpH, h = t % kMlpH;
        *reinterpret_cast<__nv_bfloat16*>((char*)w2 + chunk_off(k, h, kMlpH)) =
            __float2bfloat16_rn(W2[k * kMlpH + h]);
    }
    if (t < kMlpH * kMlpNout) {  // W3 (backward B operand): row k (in), col o (out)
        const int k = t / kMlpNout, o = t % kMlpNout;
        const float v = o < n_out ? W3[k * n_out + o] : 0.0f;
        *reinterpret_cast<__nv_bfloat16*>((char*)w3 + chunk_off(k, o, kMlpH)) = __float2bfloat16_rn(v);
    }
    if (t < kMlpNout * kMlpH) {  // W3t: row o, col k
        const int o = t / kMlpH, k = t % kMlpH;
        const float v = o < n_out ? W3[k * n_out + o] : 0.0f;
        *reinterpret_cast<__nv_bfloat16*>((char*)w3t + chunk_off(o, k, kMlpNout)) = __float2bfloat16_rn(v);
    }
    if (t < kMlpH) {
        b1[t] = B1[t];
        b2[t] = B2[t];
    }
    if (t < kMlpNout) b3[t] = t < n_out ? B3[t] : 0.0f;
}

// Row-major fp32 features (n x n_in) -> bf16 chunk-major tiles of kMlpTile rows (zero padded).
__global__ void mlp_pack_x_kernel(const float* __restrict__ x, int n, int n_in, __nv_bfloat16* __restrict__ xt,
                                  int n_tiles) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n_tiles * kMlpTile * kMlpKin) return;
    const int k = (int)(t % kMlpKin);
    const long long row = t / kMlpKin;
    const int tile = (int)(row / kMlpTile), r = (int)(row % kMlpTile);
    const float v = (row < n && k < n_in) ? x[row * n_in + k] : 0.0f;
    *reinterpret_cast<__nv_bfloat16*>((char*)xt + (size_t)tile * kMlpBytesX + chunk_off(r, k, kMlpTile)) =
        __float2bfloat16_rn(v);
}

// Minibatch rows idx[0..n) of x (n_rows_src x n_in) and t (.. x n_out) -> bf16 chunk-major
// feature tiles and contiguous fp32 targets.
__global__ void mlp_gather_kernel(const float* __restrict__ x, const float* __restrict__ t,
                                  const int* __restrict__ idx, int n, int n_in, int n_out,
                                  __nv_bfloat16* __restrict__ xt, float* __restrict__ tb, int n_tiles) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long long)n_tiles * kMlpTile * kMlpKin) return;
    const int k = (int)(q % kMlpKin);
    const long long row = q / kMlpKin;
    const int tile = (int)(row / kMlpTile), r = (int)(row % kMlpTile);
    const long long src = row < n ? idx[row] : -1;
    const float v = (src >= 0 && k < n_in) ? x[src * n_in + k] : 0.0f;
    *reinterpret_cast<__nv_bfloat16*>((char*)xt + (size_t)tile * kMlpBytesX + chunk_off(r, k, kMlpTile)) =
        __float2bfloat16_rn(v);
    if (src >= 0 && k < n_out) tb[row * n_out + k] = t[src * n_out + k];
}

}  // namespace strut

struct StrutMlp {
    int n_in = 0, n_out = 0;
    int device = 0;
    float* d_params = nullptr;  // fp32 masters
    float* d_m = nullptr;       // Adam moments
    float* d_v = nullptr;
    __nv_bfloat16 *d_w1t = nullptr, *d_w2t = nullptr, *d_w3t = nullptr, *d_w2 = nullptr, *d_w3 = nullptr;
    float *d_b1 = nullptr, *d_b2 = nullptr, *d_b3 = nullptr;
    int* d_err = nullptr;
    long long adam_step = 0;
    ~StrutMlp() {
        for (void* p : {(void*)d_params, (void*)d_m, (void*)d_v, (void*)d_w1t, (void*)d_w2t, (void*)d_w3t,
                        (void*)d_w2, (void*)d_w3,
                        (void*)d_b1, (void*)d_b2, (void*)d_b3, (void*)d_err})
            if (p) cudaFree(p);
    }
    int n_params() const { return n_in * kMlpH + kMlpH + kMlpH * kMlpH + kMlpH + kMlpH * n_out + n_out; }
    strut::MlpDev dev() const { return strut::MlpDev{d_w1t, d_w2t, d_w3t, d_b1, d_b2, d_b3}; }
    strut::MlpTrainDev train_dev() const { return strut::MlpTrainDev{dev(), d_w2, d_w3}; }
};

namespace {

int mlp_pack(StrutMlp* m, cudaStream_t s) {
    const int n = strut::kMlpH * strut::kMlpH;
    strut::mlp_pack_params_kernel<<<(n + 255) / 256, 256, 0, s>>>(m->d_params, m->n_in, m->n_out, m->d_w1t,
                                                                   m->d_w2t, m->d_w3t, m->d_w2, m->d_w3,
                                                                   m->d_b1, m->d_b2, m->d_b3);
    CK(cudaGetLastError());
    return STRUT_OK;
}

// Runs the forward kernel over n rows of device features (fp32 row-major) into device y.
int mlp_forward_dev(StrutMlp* m, const float* d_x, int n, float* d_y, cudaStream_t s) {
    const int n_tiles = (n + strut::kMlpTile - 1) / strut::kMlpTile;
    __nv_bfloat16* d_xt = nullptr;
    CK(cudaMallocAsync((void**)&d_xt, (size_t)n_tiles * strut::kMlpBytesX, s));
    const long long tot = (long long)n_tiles * strut::kMlpTile * strut::kMlpKin;
    strut::mlp_pack_x_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(d_x, n, m->n_in, d_xt, n_tiles);
    CK(cudaGetLastError());
    strut::mlp_forward_kernel<<<n_tiles, 128, strut::kMlpFwdSmem, s>>>(m->dev(), d_xt, n, d_y, m->n_out, m->d_err);
    CK(cudaGetLastError());
    CK(cudaFreeAsync(d_xt, s));
    return STRUT_OK;
}

// One minibatch on device buffers: x_tiles (n_tiles tiles), targets tb (n x n_out).  Writes
// the tile gradients to part and squared errors to sse; lr > 0 also applies Adam and repacks.
int mlp_step(StrutMlp* m, const __nv_bfloat16* d_xt, const float* d_tb, int n, float lr, float* d_part,
             double* d_sse, float* d_grad, cudaStream_t s) {
    const int n_tiles = (n + strut::kMlpTile - 1) / strut::kMlpTile;
    const int np = m->n_params();
    strut::mlp_train_tile_kernel<<<n_tiles, 128, strut::kMlpTrainSmem, s>>>(
        m->train_dev(), d_xt, d_tb, n, m->n_in, m->n_out, 2.0f / (float)((double)n * m->n_out), d_part, np, d_sse,
        m->d_err);
    CK(cudaGetLastError());
    float c1 = 1.0f, c2 = 1.0f;
    if (lr > 0.0f) {
        m->adam_step += 1;
        c1 = (float)(1.0 - std::pow(0.9, (double)m->adam_step));
        c2 = (float)(1.0 - std::pow(0.999, (double)m->adam_step));
    }
    strut::mlp_adam_kernel<<<(np + 255) / 256, 256, 0, s>>>(m->d_params, m->d_m, m->d_v, d_part, n_tiles, np, lr,
                                                            0.9f, 0.999f, c1, c2, 1.0e-8f, d_grad);
    CK(cudaGetLastError());
    if (lr > 0.0f) TRY(mlp_pack(m, s));
    return STRUT_OK;
}

}  // namespace

extern "C" {

int strut_gpu_mlp_create(int32_t n_in, int32_t n_out, StrutMlp** out) {
    if (!out || n_in < 1 || n_in > strut::kMlpKin || n_out < 1 || n_out > strut::kMlpNout)
        return fail(STRUT_BAD_ARG, "the predictor network takes 1..48 features and 1..16 outputs");
    *out = nullptr;
    StrutMlp* m = new StrutMlp();
    m->n_in = n_in;
    m->n_out = n_out;
    auto bail = [&](int rc) {
        delete m;
        return rc;
    };
    if (cudaGetDevice(&m->device) != cudaSuccess) return bail(fail(STRUT_CUDA_ERROR, "no device"));
    const size_t np = (size_t)m->n_params();
    if (cudaMalloc((void**)&m->d_params, np * 4) != cudaSuccess || cudaMalloc((void**)&m->d_m, np * 4) != cudaSuccess ||
        cudaMalloc((void**)&m->d_v, np * 4) != cudaSuccess ||
        cudaMalloc((void**)&m->d_w1t, strut::kMlpBytesW1) != cudaSuccess ||
        cudaMalloc((void**)&m->d_w2t, strut::kMlpBytesW2) != cudaSuccess ||
        cudaMalloc((void**)&m->d_w3t, strut::kMlpBytesW3) != cudaSuccess ||
        cudaMalloc((void**)&m->d_w2, strut::kMlpBytesW2) != cudaSuccess ||
        cudaMalloc((void**)&m->d_w3, strut::kMlpBytesW3) != cudaSuccess ||
        cudaMalloc((void**)&m->d_b1, strut::kMlpH * 4) != cudaSuccess ||
        cudaMalloc((void**)&m->d_b2, strut::kMlpH * 4) != cudaSuccess ||
        cudaMalloc((void**)&m->d_b3, strut::kMlpNout * 4) != cudaSuccess ||
        cudaMalloc((void**)&m->d_err, sizeof(int)) != cudaSuccess)
        return bail(fail(STRUT_CUDA_ERROR, "device allocation failed"));
    cudaMemset(m->d_params, 0, np * 4);
    cudaMemset(m->d_m, 0, np * 4);
    cudaMemset(m->d_v, 0, np * 4);
    cudaMemset(m->d_err, 0, sizeof(int));
    if (cudaFuncSetAttribute(strut::mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)strut::kMlpFwdSmem) != cudaSuccess ||
        cudaFuncSetAttribute(strut::mlp_train_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)strut::kMlpTrainSmem) != cudaSuccess)
        return bail(fail(STRUT_CUDA_ERROR, "cannot set the network kernel's shared memory"));
    *out = m;
    return STRUT_OK;
}

int strut_gpu_mlp_destroy(StrutMlp* m) {
    delete m;
    return STRUT_OK;
}

int32_t strut_gpu_mlp_param_count(const StrutMlp* m) { return m ? m->n_params() : -1; }

int strut_gpu_mlp_set_params(StrutMlp* m, const float* params) {
    if (!m || !params) return fail(STRUT_BAD_ARG, "bad arguments");
    CK(cudaMemcpy(m->d_params, params, (size_t)m->n_params() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemset(m->d_m, 0, (size_t)m->n_params() * 4));
    CK(cudaMemset(m->d_v, 0, (size_t)m->n_params() * 4));
    m->adam_step = 0;
    TRY(mlp_pack(m, 0));
    CK(cudaDeviceSynchronize());
    return STRUT_OK;
}

int strut_gpu_mlp_get_params(const StrutMlp* m, float* params) {
    if (!m || !params) return fail(STRUT_BAD_ARG, "bad arguments");
    CK(cudaMemcpy(params, m->d_params, (size_t)m->n_params() * 4, cudaMemcpyDeviceToHost));
    return STRUT_OK;
}

int strut_gpu_mlp_loss_grad(StrutMlp* m, const float* x, const float* t, int32_t n, float* loss, float* grads) {
    if (!m || !x || !t || n < 1) return fail(STRUT_BAD_ARG, "bad arguments");
    const int n_tiles = (n + strut::kMlpTile - 1) / strut::kMlpTile, np = m->n_params();
    float *d_x = nullptr, *d_t = nullptr, *d_tb = nullptr, *d_part = nullptr, *d_g = nullptr;
    int* d_idx = nullptr;
    double* d_sse = nullptr;
    __nv_bfloat16* d_xt = nullptr;
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    int rc = STRUT_OK;
    auto run = [&]() -> int {
        CK(cudaMalloc((void**)&d_x, (size_t)n * m->n_in * 4));
        CK(cudaMalloc((void**)&d_t, (size_t)n * m->n_out * 4));
        CK(cudaMalloc((void**)&d_tb, (size_t)n * m->n_out * 4));
        CK(cudaMalloc((void**)&d_idx, (size_t)n * 4));
        CK(cudaMalloc((void**)&d_xt, (size_t)n_tiles * strut::kMlpBytesX));
        CK(cudaMalloc((void**)&d_part, (size_t)n_tiles * np * 4));
        CK(cudaMalloc((void**)&d_sse, (size_t)n_tiles * 8));
        CK(cudaMalloc((void**)&d_g, (size_t)np * 4));
        CK(cudaMemcpy(d_x, x, (size_t)n * m->n_in * 4, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d_t, t, (size_t)n * m->n_out * 4, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d_idx, idx.data(), (size_t)n * 4, cudaMemcpyHostToDevice));
        CK(cudaMemset(m->d_err, 0, sizeof(int)));
        const long long tot = (long long)n_tiles * strut::kMlpTile * strut::kMlpKin;
        strut::mlp_gather_kernel<<<(unsigned)((tot + 255) / 256), 256>>>(d_x, d_t, d_idx, n, m->n_in, m->n_out, d_xt,
                                                                         d_tb, n_tiles);
        CK(cudaGetLastError());
        TRY(mlp_step(m, d_xt, d_tb, n, 0.0f, d_part, d_sse, d_g, 0));
        CK(cudaDeviceSynchronize());
        int err = 0;
        CK(cudaMemcpy(&err, m->d_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (err) return fail(STRUT_CUDA_ERROR, "network kernel wait ran out");
        std::vector<double> sse(n_tiles);
        CK(cudaMemcpy(sse.data(), d_sse, (size_t)n_tiles * 8, cudaMemcpyDeviceToHost));
        double tot_se = 0.0;
        for (double v : sse) tot_se += v;
        if (loss) *loss = (float)(tot_se / ((double)n * m->n_out));
        if (grads) CK(cudaMemcpy(grads, d_g, (size_t)np * 4, cudaMemcpyDeviceToHost));
        return STRUT_OK;
    };
    rc = run();
    for (void* p : {(void*)d_x, (void*)d_t, (void*)d_tb, (void*)d_idx, (void*)d_xt, (void*)d_part, (void*)d_sse,
                    (void*)d_g})
        if (p) cudaFree(p);
    return rc;
}

int strut_gpu_mlp_train(StrutMlp* m, const float* x, const float* t, int32_t n, int32_t epochs, int32_t batch,
                        float lr, uint64_t seed, float* loss_out) {
    if (!m || !x || !t || n < 1 || epochs < 1 || batch < 1 || !(lr > 0.0f)) return fail(STRUT_BAD_ARG, "bad arguments");
    batch = std::min(batch, n);
    const int max_tiles = (batch + strut::kMlpTile - 1) / strut::kMlpTile, np = m->n_params();
    float *d_x = nullptr, *d_t = nullptr, *d_tb = nullptr, *d_part = nullptr;
    int* d_idx = nullptr;
    double* d_sse = nullptr;
    __nv_bfloat16* d_xt = nullptr;
    auto run = [&]() -> int {
        CK(cudaMalloc((void**)&d_x, (size_t)n * m->n_in * 4));
        CK(cudaMalloc((void**)&d_t, (size_t)n * m->n_out * 4));
        CK(cudaMalloc((void**)&d_tb, (size_t)batch * m->n_out * 4));
        CK(cudaMalloc((void**)&d_idx, (size_t)n * 4));
        CK(cudaMalloc((void**)&d_xt, (size_t)max_tiles * strut::kMlpBytesX));
        CK(cudaMalloc((void**)&d_part, (size_t)max_tiles * np * 4));
        CK(cudaMalloc((void**)&d_sse, (size_t)max_tiles * 8));
        CK(cudaMemcpy(d_x, x, (size_t)n * m->n_in * 4, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d_t, t, (size_t)n * m->n_out * 4, cudaMemcpyHostToDevice));
        CK(cudaMemset(m->d_err, 0, sizeof(int)));
        std::vector<int> perm(n);
        uint64_t st = seed * 6364136223846793005ULL + 1442695040888963407ULL;
        double last = 0.0;
        for (int ep = 0; ep < epochs; ++ep) {
            for (int i = 0; i < n; ++i) perm[i] = i;
            for (int i = n - 1; i > 0; --i) {  // Fisher-Yates with a 64-bit LCG
                st = st * 6364136223846793005ULL + 1442695040888963407ULL;
                const int j = (int)((st >> 33) % (uint64_t)(i + 1));
                std::swap(perm[i], perm[j]);
            }
            CK(cudaMemcpy(d_idx, perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice));
            double ep_se = 0.0;
            std::vector<double> sse(max_tiles);
            for (int b0 = 0; b0 < n; b0 += batch) {
                const int nb = std::min(batch, n - b0), nt = (nb + strut::kMlpTile - 1) / strut::kMlpTile;
                const long long tot = (long long)nt * strut::kMlpTile * strut::kMlpKin;
                strut::mlp_gather_kernel<<<(unsigned)((tot + 255) / 256), 256>>>(d_x, d_t, d_idx + b0, nb, m->n_in,
                                                                                 m->n_out, d_xt, d_tb, nt);
                CK(cudaGetLastError());
                TRY(mlp_step(m, d_xt, d_tb, nb, lr, d_part, d_sse, nullptr, 0));
                CK(cudaMemcpy(sse.data(), d_sse, (size_t)nt * 8, cudaMemcpyDeviceToHost));
                for (int i = 0; i < nt; ++i) ep_se += sse[i];
            }
            last = ep_se / ((double)n * m->n_out);
        }
        CK(cudaDeviceSynchronize());
        int err = 0;
        CK(cudaMemcpy(&err, m->d_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (err) return fail(STRUT_CUDA_ERROR, "network kernel wait ran out");
        if (loss_out) *loss_out = (float)last;
        return STRUT_OK;
    };
    const int rc = run();
    for (void* p : {(void*)d_x, (void*)d_t, (void*)d_tb, (void*)d_idx, (void*)d_xt, (void*)d_part, (void*)d_sse})
        if (p) cudaFree(p);
    return rc;
}

int strut_gpu_mlp_forward(StrutMlp* m, const float* x, int32_t n, float* y) {
    if (!m || !x || !y || n < 1) return fail(STRUT_BAD_ARG, "bad arguments");
    float *d_x = nullptr, *d_y = nullptr;
    CK(cudaMalloc((void**)&d_x, (size_t)n * m->n_in * 4));
    CK(cudaMalloc((void**)&d_y, (size_t)n * m->n_out * 4));
    CK(cudaMemcpy(d_x, x, (size_t)n * m->n_in * 4, cudaMemcpyHostToDevice));
    CK(cudaMemset(m->d_err, 0, sizeof(int)));
    int rc = mlp_forward_dev(m, d_x, n, d_y, 0);
    if (rc == STRUT_OK) {
        CK(cudaDeviceSynchronize());
        int err = 0;
        CK(cudaMemcpy(&err, m->d_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (err) rc = fail(STRUT_CUDA_ERROR, "network kernel wait ran out");
        else CK(cudaMemcpy(y, d_y, (size_t)n * m->n_out * 4, cudaMemcpyDeviceToHost));
    }
    cudaFree(d_x);
    cudaFree(d_y);
    return rc;
}

}  // extern "C"

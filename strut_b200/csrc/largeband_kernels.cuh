// Newton iteration of instances whose effective band does not fit in shared memory (a 3D frame
// of a few thousand dofs and a bandwidth of a few hundred: ~10-30 MB, resident in the 126 MB L2).
//
//   large_assemble_kernel  one warp per band row: K gathered per slot in element order, C, the
//                          effective entries K + a1 C + a0 M written to the global band, the row's
//                          residual P - F_int - C v - M a (transient_nonlinear.mojo:2302-2356,
//                          linear_solver_backend.mojo:1877-1983)
//   large_factor_kernel    cooperative (all CTAs co-resident): blocked right-looking band LU
//                          without pivoting, panel width kPanel.  CTA 0 factors the panel
//                          (rows k0 .. k0+kb-1+bw) in shared memory with Strut's pivot test
//                          (a sub-diagonal entry larger than the pivot -> dense partial-pivot
//                          fallback, linear_solver_backend.mojo:631-680) and forms U12 =
//                          L11^-1 A12; every CTA then updates tiles of the trailing block
//                          A22 -= L21 U12.  Two bounded grid barriers per panel.
//   large_solve_kernel     one CTA per instance: blocked forward / back substitution
//                          (_solve_band_general, 735-770), then the displacement update and
//                          the convergence test shared with the shared-memory path.
//   large_dense_kernel     the dense partial-pivot fallback (175-240) of the instances whose
//                          band factorisation asked for it, one at a time in one n x n scratch.
//
// The entries are the reference's; only the order of the sums in the trailing updates and the
// substitutions differs (blocked), so the GPU agrees with the oracle to rounding.
#pragma once

#include "solver_kernels.cuh"

namespace strut {

constexpr int kPanel = 32;         // panel width of the blocked band LU
constexpr int kLargeThreads = 256; // threads of a factorisation CTA
constexpr int kSolveThreads = 1024;

enum { LSTAT_OK = 0, LSTAT_SINGULAR = 2, LSTAT_DENSE = 6, LSTAT_CONVERGED = 7, LSTAT_IDLE = -1 };

struct GridBarrier {
    unsigned int count;
    unsigned int gen;
    int err;
    int pad;
};

// Grid-wide barrier of a cooperative launch.  Thread 0 of each CTA arrives; the last arrival
// resets the count and advances the generation; the others wait for the generation to move,
// for a bounded number of polls, after which the barrier records an error and every CTA stops.
__device__ __forceinline__ bool grid_barrier(GridBarrier* gb, unsigned int& gen) {
    __syncthreads();
    int ok = 1;
    if (threadIdx.x == 0) {
        const unsigned int g = gen;
        __threadfence();
        const unsigned int arrived = atomicAdd(&gb->count, 1u) + 1u;
        if (arrived == gridDim.x) {
            atomicExch(&gb->count, 0u);
            __threadfence();
            atomicAdd(&gb->gen, 1u);
        } else {
            int polls = 0;
            while (atomicAdd(&gb->gen, 0u) == g) {
                if (++polls > (1 << 22) || atomicAdd(&gb->err, 0) != 0) {
                    atomicExch(&gb->err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        gen = g + 1u;
    }
    return __syncthreads_and(ok) != 0;
}

__device__ __forceinline__ long long lslot(int rw, int bw, int i, int j) {
    return (long long)i * rw + (j - i + bw);
}

// ---- assembly and residual ---------------------------------------------------------------

// grid.x: warps over the rows of all large instances (row r of the concatenation over
// large_list).  mode INST_MODE_NEWTON skips inactive instances; INST_MODE_EXPORT also writes the
// band and F_int to the export buffers.
__global__ void __launch_bounds__(256) large_assemble_kernel(const DevInst* __restrict__ insts,
                                                             InstArrays A, const int* __restrict__ large_list,
                                                             const int* __restrict__ row_base,
                                                             int n_large, int total_rows, int mode,
                                                             GridBarrier* gb) {
    const int warp_g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // the factorisation that follows starts from a clean barrier
        gb->count = 0u;
        gb->err = 0;
    }
    if (warp_g >= total_rows) return;
    int li = 0;
    while (li + 1 < n_large && row_base[li + 1] <= warp_g) ++li;
    const int inst = large_list[li];
    const DevInst& I = insts[inst];
    if (mode == INST_MODE_NEWTON && !A.active[inst]) return;
    const int i = warp_g - row_base[li];
    const int n = I.n, bw = I.bw, rw = I.rw, f0 = I.f_off;
    if (mode == INST_MODE_NEWTON && i == 0 && lane == 0) {
        A.iters[inst] += 1;
        if (A.bytes_counter) atomicAdd(A.bytes_counter, (unsigned long long)I.io_bytes);
    }
    const long long sp0 = I.slot_ptr_off;
    const double* Kinit = A.Kinit + I.band_off;
    double* B = A.lband + I.lband_off;
    double cv = 0.0;
    for (int o = lane; o < rw; o += 32) {
        const int j = i + o - bw;
        const long long slot = (long long)i * rw + o;
        if (j < 0 || j >= n) {
            B[slot] = 0.0;
            if (mode == INST_MODE_EXPORT) A.export_band[I.band_off + slot] = 0.0;
            continue;
        }
        const double K = gather_slot(A, sp0, (int)slot);
        double C = 0.0;
        if (I.has_damping) {
            C = I.alpha_m * (i == j ? A.Mrff[f0 + i] : 0.0);
            if (I.beta_k != 0.0) C += I.beta_k * K;
            if (I.beta_k_init != 0.0) C += I.beta_k_init * Kinit[slot];
            const int gj = f0 + j;
            const double an = I.a0 * (A.u_f[gj] - A.u_n[gj]) - I.a2 * A.v_n[gj] - I.a3 * A.a_n[gj];
            const double vt = A.v_n[gj] + I.dt * ((1.0 - I.gamma) * A.a_n[gj] + I.gamma * an);
            cv += C * vt;
        }
        double keff = K;
        if (I.has_damping && I.a1 != 0.0) keff += I.a1 * C;
        if (i == j) keff += I.a0 * A.Mff[f0 + i];
        B[slot] = keff;
        if (mode == INST_MODE_EXPORT) A.export_band[I.band_off + slot] = keff;
    }
    cv = warp_sum(cv);
    if (lane == 0) {
        const int gi = f0 + i;
        const double an = I.a0 * (A.u_f[gi] - A.u_n[gi]) - I.a2 * A.v_n[gi] - I.a3 * A.a_n[gi];
        const int q0 = A.fint_ptr[I.fint_ptr_off + i], q1 = A.fint_ptr[I.fint_ptr_off + i + 1];
        const double F = gather_fint(A, A.ef, q0, q1);
        const double ma = A.Mff[gi] * an;
        A.R[gi] = A.P_f[gi] - F - 0.0 - cv - ma;
        if (mode == INST_MODE_EXPORT) A.export_f[gi] = F;
    }
}

// ---- blocked band LU ------------------------------------------------------------------------

// Copies the exported band of every large instance into its factorisation buffer
// (strut_gpu_factor_solve on a band from strut_gpu_state_determination).
__global__ void large_load_exported_kernel(const DevInst* __restrict__ insts, InstArrays A,
                                           const int* __restrict__ large_list, int n_large,
                                           GridBarrier* gb) {
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
        gb->count = 0u;
        gb->err = 0;
    }
    const int li = blockIdx.y;
    if (li >= n_large) return;
    const DevInst& I = insts[large_list[li]];
    const long long total = (long long)I.n * I.rw;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x)
        A.lband[I.lband_off + t] = A.export_band[I.band_off + t];
}

// Cooperative.  Dynamic shared memory: panel (kPanel + bw) x kPanel, then two 32 x kPanel tiles.
__global__ void __launch_bounds__(kLargeThreads) large_factor_kernel(
    const DevInst* __restrict__ insts, InstArrays A, const int* __restrict__ large_list,
    int n_large, int mode, GridBarrier* gb) {
    extern __shared__ __align__(16) double smem_lf[];
    __shared__ int s_flag[2];
    __shared__ double red[32];
    const int tid = threadIdx.x, nt = blockDim.x;
    unsigned int gen = 0;
    if (tid == 0) gen = atomicAdd(&gb->gen, 0u);
    for (int li = 0; li < n_large; ++li) {
        const int inst = large_list[li];
        const DevInst& I = insts[inst];
        if (mode == INST_MODE_NEWTON && !A.active[inst]) {
            if (blockIdx.x == 0 && tid == 0) A.lstatus[li] = LSTAT_IDLE;
            continue;
        }
        const int n = I.n, bw = I.bw, rw = I.rw;
        double* B = A.lband + I.lband_off;
        if (mode == INST_MODE_NEWTON && I.test_type == 2) {
            // NormUnbalance is tested on the residual before the solve; every CTA reaches the
            // same decision from the same sums
            double s = 0.0;
            for (int i = tid; i < n; i += nt) s += A.R[I.f_off + i] * A.R[I.f_off + i];
            s = block_sum(s, red);
            if (sqrt(s) <= I.tol) {
                if (blockIdx.x == 0 && tid == 0) A.lstatus[li] = LSTAT_CONVERGED;
                continue;
            }
        }
        const int P = min(kPanel, max(bw, 1));
        int result = LSTAT_OK;
        for (int k0 = 0; k0 < n && result == LSTAT_OK; k0 += P) {
            const int kb = min(P, n - k0);
            const int r1 = min(n - 1, k0 + kb - 1 + bw);  // last row touched by the panel
            const int pr = r1 - k0 + 1;
            const int c1 = min(n - 1, k0 + kb - 1 + bw);  // last column of U12
            if (blockIdx.x == 0) {
                // ---- panel: rows k0..r1, columns k0..k0+kb-1 (row-major, stride kb)
                double* Pm = smem_lf;
                for (int t = tid; t < pr * kb; t += nt) {
                    const int r = t / kb, c = t % kb;
                    const int i = k0 + r, j = k0 + c;
                    Pm[t] = (i - j <= bw && j - i <= bw) ? B[lslot(rw, bw, i, j)] : 0.0;
                }
                if (tid == 0) s_flag[0] = LSTAT_OK;
                __syncthreads();
                for (int c = 0; c < kb; ++c) {
                    const int k = k0 + c;
                    const int last = min(pr - 1, c + bw);  // rows of column k inside the band
                    const double akk = Pm[c * kb + c];
                    const double aabs = fabs(akk);
                    int swap = 0, big = 0;
                    for (int r = c + 1 + tid; r <= last; r += nt) {
                        const double v = fabs(Pm[r * kb + c]);
                        swap |= v > aabs ? 1 : 0;
                        big |= v > 1.0e-14 ? 1 : 0;
                    }
                    const int any_swap = __syncthreads_or(swap);
                    const int any_big = __syncthreads_or(big);
                    if (any_swap || aabs <= 1.0e-14) {
                        if (tid == 0) s_flag[0] = (any_swap && any_big) ? LSTAT_DENSE : LSTAT_SINGULAR;
                        break;
                    }
                    (void)k;
                    for (int r = c + 1 + tid; r <= last; r += nt) Pm[r * kb + c] = Pm[r * kb + c] / akk;
                    __syncthreads();
                    const int rows = last - c, cols = kb - 1 - c;
                    for (int t = tid; t < rows * cols; t += nt) {
                        const int r = c + 1 + t / cols, cc = c + 1 + t % cols;
                        Pm[r * kb + cc] -= Pm[r * kb + c] * Pm[c * kb + cc];
                    }
                    __syncthreads();
                }
                __syncthreads();
                if (s_flag[0] == LSTAT_OK) {
                    for (int t = tid; t < pr * kb; t += nt) {
                        const int r = t / kb, c = t % kb;
                        const int i = k0 + r, j = k0 + c;
                        if (i - j <= bw && j - i <= bw) B[lslot(rw, bw, i, j)] = Pm[t];
                    }
                    // U12 = L11^-1 A12: one thread per column j of k0+kb..c1, rows in order
                    for (int j = k0 + kb + tid; j <= c1; j += nt) {
                        double u[kPanel];
                        for (int r = 0; r < kb; ++r) {
                            const int i = k0 + r;
                            double v = (j - i <= bw) ? B[lslot(rw, bw, i, j)] : 0.0;
                            for (int s = 0; s < r; ++s) v -= Pm[r * kb + s] * u[s];
                            u[r] = v;
                            if (j - i <= bw) B[lslot(rw, bw, i, j)] = v;
                        }
                    }
                }
                if (tid == 0) s_flag[1] = s_flag[0];
                __syncthreads();
                if (tid == 0) A.lstatus[li] = s_flag[0];
                // publish the panel result to the other CTAs through gb->pad
                if (tid == 0) atomicExch(&gb->pad, s_flag[0]);
            }
            if (!grid_barrier(gb, gen)) return;
            if (tid == 0) s_flag[1] = atomicAdd(&gb->pad, 0);
            __syncthreads();
            result = s_flag[1];
            if (result != LSTAT_OK) break;
            // ---- trailing update A22 -= L21 U12 over rows / columns k0+kb .. r1
            const int m = r1 - (k0 + kb) + 1;
            if (m > 0) {
                const int nbt = (m + 31) / 32;
                double* Lt = smem_lf;                 // 32 x kb
                double* Ut = smem_lf + 32 * kPanel;   // kb x 32
                for (int tile = blockIdx.x; tile < nbt * nbt; tile += gridDim.x) {
                    const int ti = tile / nbt, tj = tile % nbt;
                    const int i0 = k0 + kb + 32 * ti, j0 = k0 + kb + 32 * tj;
                    __syncthreads();
                    for (int t = tid; t < 32 * kb; t += nt) {
                        const int r = t / kb, s = t % kb;
                        const int i = i0 + r, kk = k0 + s;
                        Lt[t] = (i <= r1 && i - kk <= bw) ? B[lslot(rw, bw, i, kk)] : 0.0;
                        const int s2 = t / 32, cc = t % 32;
                        const int j = j0 + cc, k2 = k0 + s2;
                        Ut[t] = (j <= r1 && j - k2 <= bw) ? B[lslot(rw, bw, k2, j)] : 0.0;
                    }
                    __syncthreads();
                    for (int t = tid; t < 32 * 32; t += nt) {
                        const int r = t / 32, cc = t % 32;
                        const int i = i0 + r, j = j0 + cc;
                        if (i > r1 || j > r1) continue;
                        double acc = 0.0;
                        for (int s = 0; s < kb; ++s) acc += Lt[r * kb + s] * Ut[s * 32 + cc];
                        B[lslot(rw, bw, i, j)] -= acc;
                    }
                }
            }
            if (!grid_barrier(gb, gen)) return;
        }
    }
}

// ---- substitution, update and test ---------------------------------------------------------

// One CTA per large instance.  Forward: L (unit lower) in blocks of 32 rows, each block solved
// by warp 0 then pushed into the next bw rows; back: U in blocks of 32 rows from the end.
__global__ void __launch_bounds__(kSolveThreads) large_solve_kernel(
    const DevInst* __restrict__ insts, InstArrays A, const int* __restrict__ large_list, int n_large,
    int mode, double* __restrict__ wbuf, const GridBarrier* __restrict__ gb) {
    __shared__ double red[32];
    __shared__ int red_r[32];
    __shared__ double xb[32];
    const int li = blockIdx.x;
    if (li >= n_large) return;
    const int inst = large_list[li];
    const DevInst& I = insts[inst];
    const int st = A.lstatus[li];
    if (mode == INST_MODE_NEWTON && (st == LSTAT_IDLE || !A.active[inst])) return;
    if (gb->err) {
        // a barrier of the factorisation gave up: the factors are incomplete
        if (threadIdx.x == 0) {
            A.status[inst] = STRUT_CUDA_ERROR;
            if (mode == INST_MODE_NEWTON && A.active[inst]) {
                A.active[inst] = 0;
                atomicSub(A.nactive, 1);
            }
        }
        return;
    }
    if (st == LSTAT_DENSE) return;  // large_dense_kernel
    const int tid = threadIdx.x, nt = blockDim.x;
    const int n = I.n, bw = I.bw, rw = I.rw, f0 = I.f_off;
    int* hrow = (mode == INST_MODE_NEWTON && A.hist_iters && A.ctl)
                    ? A.hist_iters + (size_t)A.ctl->step * A.n_inst : nullptr;
    if (st == LSTAT_CONVERGED) {
        if (tid == 0) {
            A.active[inst] = 0;
            atomicSub(A.nactive, 1);
            if (hrow) hrow[inst] = A.iters[inst];
        }
        return;
    }
    if (st == LSTAT_SINGULAR) {
        if (tid == 0) {
            A.status[inst] = LSTAT_SINGULAR;
            if (mode == INST_MODE_NEWTON && A.active[inst]) {
                A.active[inst] = 0;
                atomicSub(A.nactive, 1);
            }
        }
        return;
    }
    const double* B = A.lband + I.lband_off;
    double* w = wbuf + f0;             // forward result, then x
    const double* rhs = (mode == INST_MODE_SOLVE_EXPORTED) ? A.rhs_in + f0 : A.R + f0;
    for (int i = tid; i < n; i += nt) w[i] = rhs[i];
    __syncthreads();
    const int lane = tid & 31;
    for (int r0 = 0; r0 < n; r0 += 32) {
        const int rb = min(32, n - r0);
        if (tid < 32) {
            double v = lane < rb ? w[r0 + lane] : 0.0;
            for (int s = 0; s < rb; ++s) {
                const double ws = __shfl_sync(0xffffffffu, v, s);
                if (lane > s && lane < rb && (lane - s) <= bw) v -= B[lslot(rw, bw, r0 + lane, r0 + s)] * ws;
            }
            if (lane < rb) {
                w[r0 + lane] = v;
                xb[lane] = v;
            }
        }
        __syncthreads();
        const int i_last = min(n - 1, r0 + rb - 1 + bw);
        for (int i = r0 + rb + tid; i <= i_last; i += nt) {
            double acc = 0.0;
            for (int s = 0; s < rb; ++s) {
                const int j = r0 + s;
                if (i - j <= bw) acc += B[lslot(rw, bw, i, j)] * xb[s];
            }
            w[i] -= acc;
        }
        __syncthreads();
    }
    for (int r1 = n; r1 > 0; r1 -= 32) {
        const int r0 = max(0, r1 - 32), rb = r1 - r0;
        if (tid < 32) {
            double v = lane < rb ? w[r0 + lane] : 0.0;
            for (int s = rb - 1; s >= 0; --s) {
                if (lane == s) v = v / B[lslot(rw, bw, r0 + s, r0 + s)];
                const double xs = __shfl_sync(0xffffffffu, v, s);
                if (lane < s && (s - lane) <= bw) v -= B[lslot(rw, bw, r0 + lane, r0 + s)] * xs;
            }
            if (lane < rb) {
                w[r0 + lane] = v;
                xb[lane] = v;
            }
        }
        __syncthreads();
        const int i_first = max(0, r0 - bw);
        for (int i = i_first + tid; i < r0; i += nt) {
            double acc = 0.0;
            for (int s = 0; s < rb; ++s) {
                const int j = r0 + s;
                if (j - i <= bw) acc += B[lslot(rw, bw, i, j)] * xb[s];
            }
            w[i] -= acc;
        }
        __syncthreads();
    }
    if (mode == INST_MODE_SOLVE_EXPORTED) {
        for (int i = tid; i < n; i += nt) A.du[f0 + i] = w[i];
        return;
    }
    InstArrays Ar = A;
    newton_tail(I, Ar, inst, w, A.R + f0, hrow, red, red_r);
}

// Dense partial-pivot fallback of the large instances that asked for it, one at a time (one
// CTA, one n x n scratch): D from the assembled effective entries, LU, solve, update, test.
__global__ void __launch_bounds__(256) large_dense_kernel(const DevInst* __restrict__ insts,
                                                          InstArrays A, const int* __restrict__ large_list,
                                                          int n_large, int mode, double* __restrict__ D,
                                                          int* __restrict__ piv, double* __restrict__ wbuf) {
    extern __shared__ __align__(16) double smem_ld[];  // fac (max n)
    __shared__ double red[32];
    __shared__ int red_r[32];
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int li = 0; li < n_large; ++li) {
        if (A.lstatus[li] != LSTAT_DENSE) continue;
        const int inst = large_list[li];
        const DevInst& I = insts[inst];
        if (mode == INST_MODE_NEWTON && !A.active[inst]) continue;
        const int n = I.n, bw = I.bw, rw = I.rw, f0 = I.f_off;
        for (long long t = tid; t < (long long)n * n; t += nt) D[t] = 0.0;
        __syncthreads();
        const double* Kinit = A.Kinit + I.band_off;
        for (long long t = tid; t < (long long)n * rw; t += nt) {
            const int i = (int)(t / rw), j = i + (int)(t % rw) - bw;
            if (j < 0 || j >= n) continue;
            D[(size_t)i * n + j] = (mode == INST_MODE_SOLVE_EXPORTED)
                                       ? A.export_band[I.band_off + t]
                                       : keff_slot(I, A, I.slot_ptr_off, Kinit, i, j, (int)t);
        }
        __syncthreads();
        const int rc = dense_lu_global(D, piv, n, smem_ld, red, red_r);
        if (tid == 0 && A.fallbacks) A.fallbacks[inst] += 1;
        if (rc != 0) {
            if (tid == 0) {
                A.status[inst] = rc;
                if (mode == INST_MODE_NEWTON && A.active[inst]) {
                    A.active[inst] = 0;
                    atomicSub(A.nactive, 1);
                }
            }
            __syncthreads();
            continue;
        }
        __syncthreads();
        double* w = wbuf + f0;
        double* x = A.du + f0;
        const double* rhs = (mode == INST_MODE_SOLVE_EXPORTED) ? A.rhs_in + f0 : A.R + f0;
        if (tid < 32) dense_solve_warp(D, piv, n, rhs, w, x);
        __syncthreads();
        if (mode == INST_MODE_SOLVE_EXPORTED) continue;
        int* hrow = (A.hist_iters && A.ctl) ? A.hist_iters + (size_t)A.ctl->step * A.n_inst : nullptr;
        for (int i = tid; i < n; i += nt) w[i] = x[i];
        __syncthreads();
        InstArrays Ar = A;
        newton_tail(I, Ar, inst, w, A.R + f0, hrow, red, red_r);
        __syncthreads();
    }
}

}  // namespace strut

// Per-instance Newton kernels: assembly gather, Rayleigh damping, residual, band factor/solve,
// displacement update and the convergence test, fused into one CTA per instance with the
// effective band matrix resident in shared memory.  Plus the Newmark predictor and post-step
// update over all free dofs.
//
// Algorithm (paths relative to the Strut project root):
//   element scatter order     src/mojo/solver/assembly/stiffness_internal_frame2d.mojo:594-619
//                             (contributions are gathered per band slot in element order, so
//                             every K entry is summed exactly as Strut's scatter sums it)
//   C_ff and residual         src/mojo/solver/run_case/analysis/transient_nonlinear.mojo:
//                             2302-2356
//   effective matrix          linear_solver_backend.mojo:1877-1983 (K + a1 C + a0 M)
//   BandGeneral factor/solve  linear_solver_backend.mojo:631-680, 735-770 (unpivoted Doolittle;
//                             when a row swap would be needed, the dense partial-pivot LU of
//                             175-240 on the assembled values, in global scratch)
//   BandSPD factor/solve      linear_solver_backend.mojo:689-726, 772-812
//   Newmark                   transient_nonlinear.mojo:496-648, 1052-1055
//   tests                     nonlinear_convergence.mojo:8-20, transient_nonlinear.mojo:2798-2811
#pragma once

#include "kernels.cuh"

namespace strut {

enum { INST_MODE_NEWTON = 0, INST_MODE_EXPORT = 1, INST_MODE_SOLVE_EXPORTED = 2 };

struct InstArrays {
    double *u_f, *v_f, *a_f, *u_n, *v_n, *a_n, *P_f, *du, *R;
    const double *Mff, *Mrff, *fconst;
    double* u_full;
    const int* free_dof;  // absolute index of each free dof in u_full
    const double* Kinit;  // band, per instance at band_off
    const long long* slot_ptr;
    const int* slot_contrib;
    const int* fint_ptr;
    const int* fint_contrib;
    const double* ek;
    const double* ef;
    int* active;
    int* status;
    int* iters;
    int* nactive;
    int* hist_iters;  // iteration-count history (steps x n_inst) or null
    const DevCtl* ctl;
    double* export_band;  // band per instance (BandGeneral rw / BandSPD bw+1 layout)
    double* export_f;     // F_int at free dofs
    const double* rhs_in; // INST_MODE_SOLVE_EXPORTED
    unsigned long long* bytes_counter;
    double* dense;        // per instance n x n scratch for the partial-pivot fallback
    int* piv;             // per free dof
    int* fallbacks;       // per instance count of dense fallbacks
    ElemList el;          // elements of the instances still iterating
    // learned predictor: the step starts from the learned guess (dual 1), whose first iteration
    // checks it against the Newmark predictor's (u_base); rejected: per instance, the step went
    // back to the predictor
    int dual;
    int* rejected;
    int* skip;              // global-memory band path: skip the factorisation this iteration
    double* estate;
    long long* pred_stats;  // per instance: first iterations offered, learned guess chosen
    double* hist_du;        // 4 x n_free ring of converged increments (slot = step % 4)
    int n_free_total;
    int n_inst;
    // multi-point constraints: per-contribution coefficients of the gathers (null without
    // constraints) and the slave dofs u_s = sum_k coef_k u_{master_k} (absolute u_full indices)
    const double* slot_coef;
    const double* fint_coef;
    const int* sl_dof;
    const int* sl_ptr;
    const int* sl_master;
    const double* sl_coef;
    // instances whose band lives in global memory
    // ModifiedNewton / ModifiedNewtonInitial: the step's tangent (band_off layout), its factored
    // effective band, and whether the factors are the dense fallback's (A.dense, A.piv)
    double* kfrz;
    double* lufrz;
    int* lu_dense;
    // solver chain: current attempt and the iterations of earlier attempts of the step, per
    // instance; the predictor's displacements and the element state at the step's start
    int* attempt;
    int* iters_prev;
    double* u_base;
    double* estate_base;
    double* lband;          // effective band (factored in place), at DevInst::lband_off
    int* lstatus;           // per large instance: 0 factored, 2 singular, 6 dense fallback,
                            // 7 converged before the solve (NormUnbalance), -1 not active
};

__device__ __forceinline__ Attempt attempt_of(const DevInst& I, const InstArrays& A, int inst) {
    const int k = A.attempt ? A.attempt[inst] : 0;
    Attempt a;
    a.alg = I.att_alg[k];
    a.test = I.att_test[k];
    a.max_iters = I.att_maxit[k];
    a.tol = I.att_tol[k];
    return a;
}

__device__ __forceinline__ double block_sum(double v, double* red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
    const int nw = (blockDim.x + 31) >> 5;
    for (int w = 0; w < nw; ++w) s += red[w];
    return s;
}

__device__ __forceinline__ double block_max(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
    const int nw = (blockDim.x + 31) >> 5;
    for (int w = 0; w < nw; ++w) s = fmax(s, red[w]);
    return s;
}

// Right-looking band LU without pivoting (Doolittle, unit-lower multipliers stored in place)
// on the n x (2bw+1) band in shared memory.  Step k computes the multiplier a_ik / a_kk of each
// row below the pivot once (fac, at least bw entries), checks the column for a row swap, then
// updates the trailing block one warp per row.  Every entry receives the same single update
// per step as in the reference's row loop.  Returns 0 ok, 2 singular, 6 a row swap would be
// needed (the caller then factors the assembled matrix densely with partial pivoting).
__device__ int band_lu_smem(double* B, int n, int bw, int rw, double* fac) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    for (int k = 0; k < n; ++k) {
        const int m = min(bw, n - 1 - k);
        const double akk = B[k * rw + bw];
        const double aabs = fabs(akk);
        int swap = 0, big = 0;
        for (int t = tid; t < m; t += nt) {
            const int i = k + 1 + t;
            const double v = B[i * rw + (k - i + bw)];
            const double c = fabs(v);
            swap |= (c > aabs) ? 1 : 0;
            big |= (c > 1.0e-14) ? 1 : 0;
            fac[t] = v / akk;
        }
        // pivot search of linear_solver_backend.mojo:640-657: an entry strictly larger than
        // the diagonal selects another row; the largest candidate decides singularity
        if (__syncthreads_or(swap)) return __syncthreads_or(big) ? 6 : 2;
        if (aabs <= 1.0e-14) return 2;
        for (int r = warp; r < m; r += nw) {
            const int i = k + 1 + r;
            const double f = fac[r];
            if (lane == 0) B[i * rw + (k - i + bw)] = f;
            if (f == 0.0) continue;
            const double* rowk = B + k * rw + (bw - k);
            double* rowi = B + i * rw + (bw - i);
            for (int c = lane; c < m; c += 32) {
                const int j = k + 1 + c;
                rowi[j] -= f * rowk[j];
            }
        }
        __syncthreads();
    }
    return 0;
}

// Right-looking band Cholesky (L L^T) on the lower band stored in general layout: column k of
// L is computed once per step (fac), then the trailing lower block is updated one warp per row.
// Same arithmetic per entry as the row-oriented reference up to summation order.  Returns 0
// ok, 2 not positive definite.
__device__ int band_chol_smem(double* B, int n, int bw, int rw, double* fac) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    for (int k = 0; k < n; ++k) {
        const int m = min(bw, n - 1 - k);
        const double dkk = B[k * rw + bw];
        if (!(dkk > 0.0)) return 2;
        const double lkk = sqrt(dkk);
        for (int t = tid; t < m; t += nt) {
            const int i = k + 1 + t;
            fac[t] = B[i * rw + (k - i + bw)] / lkk;
        }
        __syncthreads();
        for (int r = warp; r < m; r += nw) {
            const int i = k + 1 + r;
            const double li = fac[r];
            if (lane == 0) B[i * rw + (k - i + bw)] = li;
            double* rowi = B + i * rw + (bw - i);
            for (int c = lane; c <= r; c += 32) rowi[k + 1 + c] -= li * fac[c];
        }
        if (tid == 0) B[k * rw + bw] = lkk;
        __syncthreads();
    }
    return 0;
}

// BandGeneral forward/back substitution with one warp (_solve_band_general,
// linear_solver_backend.mojo:735-770).  Forward: column-oriented, so row i receives
// rhs_i - L_i,j0 w_j0 - L_i,j0+1 w_j0+1 - ... in increasing j, the order of the reference's row
// loop.  Back: lane 0 runs each row's sum in the reference's order.  w may not alias rhs.
__device__ void band_solve_lu_warp(const double* __restrict__ B, int n, int bw, int rw,
                                   const double* __restrict__ rhs, double* __restrict__ w,
                                   double* __restrict__ x) {
    const int lane = threadIdx.x & 31;
    for (int i = lane; i < n; i += 32) w[i] = rhs[i];
    __syncwarp();
    for (int j = 0; j < n; ++j) {
        const double wj = w[j];
        const int m = min(bw, n - 1 - j);
        for (int t = lane; t < m; t += 32) {
            const int i = j + 1 + t;
            w[i] -= B[i * rw + (j - i + bw)] * wj;
        }
        __syncwarp();
    }
    if (lane == 0) {
        for (int i = n - 1; i >= 0; --i) {
            const double* rowi = B + i * rw + (bw - i);
            double s = w[i];
            const int j1 = min(n - 1, i + bw);
            for (int j = i + 1; j <= j1; ++j) s -= rowi[j] * x[j];
            x[i] = s / rowi[i];
        }
    }
    __syncwarp();
}

// BandSPD substitution with one warp (_solve_band_spd, linear_solver_backend.mojo:772-812):
// both sweeps are column-oriented, which is the reference's own order for each entry.
__device__ void band_solve_chol_warp(const double* B, int n, int bw, int rw, const double* rhs,
                                     double* w, double* x) {
    const int lane = threadIdx.x & 31;
    for (int i = lane; i < n; i += 32) w[i] = rhs[i];
    __syncwarp();
    for (int j = 0; j < n; ++j) {
        // w_j = (rhs_j - sum_{k<j} L_jk w_k) / L_jj, then push w_j into the rows below
        if (lane == 0) w[j] = w[j] / B[j * rw + bw];
        __syncwarp();
        const double wj = w[j];
        const int m = min(bw, n - 1 - j);
        for (int t = lane; t < m; t += 32) {
            const int i = j + 1 + t;
            w[i] -= B[i * rw + (j - i + bw)] * wj;
        }
        __syncwarp();
    }
    for (int i = lane; i < n; i += 32) x[i] = w[i];
    __syncwarp();
    // L^T x = w: x_row /= L_row,row, then x_col -= L_row,col x_row for the columns of that row
    for (int row = n - 1; row >= 0; --row) {
        if (lane == 0) x[row] = x[row] / B[row * rw + bw];
        __syncwarp();
        const double xr = x[row];
        const int first = max(0, row - bw);
        for (int col = first + lane; col < row; col += 32) x[col] -= B[row * rw + (col - row + bw)] * xr;
        __syncwarp();
    }
}

__device__ __forceinline__ double gather_slot(const InstArrays& A, long long sp0, int slot) {
    const long long c0 = A.slot_ptr[sp0 + slot], c1 = A.slot_ptr[sp0 + slot + 1];
    double K = 0.0;
    if (A.slot_coef) {
        // collapsed through multi-point constraints: c_i k c_j
        for (long long c = c0; c < c1; ++c) K += A.slot_coef[c] * A.ek[A.slot_contrib[c]];
    } else {
        for (long long c = c0; c < c1; ++c) K += A.ek[A.slot_contrib[c]];
    }
    return K;
}

// The whole band of an instance (n x rw slots, entries outside the matrix zero): gather_slot of
// every slot, four slots per thread interleaved so that their dependent loads (list bounds,
// contribution indices, element entries) are in flight together.  Each slot adds its own
// contributions in list order, as gather_slot does.  The whole CTA.
__device__ __forceinline__ void gather_band4(const InstArrays& A, long long sp0, int n, int bw, int rw,
                                             double* __restrict__ Kb) {
    const int nt = blockDim.x, n_slots = n * rw;
    const long long* __restrict__ ptr = A.slot_ptr + sp0;
    const int* __restrict__ con = A.slot_contrib;
    const double* __restrict__ coef = A.slot_coef;
    const double* __restrict__ ek = A.ek;
    for (int s0 = threadIdx.x; s0 < n_slots; s0 += 4 * nt) {
        long long c[4], e[4];
        double K[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int slot = s0 + u * nt;
            c[u] = e[u] = 0;
            K[u] = 0.0;
            if (slot < n_slots) {
                const int i = slot / rw, j = i + (slot - i * rw) - bw;
                if (j >= 0 && j < n) {
                    c[u] = ptr[slot];
                    e[u] = ptr[slot + 1];
                }
            }
        }
        for (;;) {
            int idx[4];
            bool any = false;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                idx[u] = c[u] < e[u] ? con[c[u]] : -1;
                any |= idx[u] >= 0;
            }
            if (!any) break;
            if (coef) {
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (idx[u] >= 0) K[u] += coef[c[u]] * ek[idx[u]];
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (idx[u] >= 0) K[u] += ek[idx[u]];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) c[u] += c[u] < e[u] ? 1 : 0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (s0 + u * nt < n_slots) Kb[s0 + u * nt] = K[u];
    }
}

// F_int of free dof i of an instance: its element end forces in element order (times the
// collapse coefficient under multi-point constraints).
__device__ __forceinline__ double gather_fint(const InstArrays& A, const double* ef, int q0, int q1) {
    double F = 0.0;
    if (A.fint_coef) {
        for (int q = q0; q < q1; ++q) F += A.fint_coef[q] * ef[A.fint_contrib[q]];
    } else {
        for (int q = q0; q < q1; ++q) F += ef[A.fint_contrib[q]];
    }
    return F;
}

// Slave dofs of an instance from their retained dofs (_enforce_mpc_values,
// helpers.mojo:3380-3400), collectively over the CTA.
__device__ __forceinline__ void enforce_slaves(const DevInst& I, const InstArrays& A) {
    for (int s = threadIdx.x; s < I.n_sl; s += blockDim.x) {
        const int k = I.sl_off + s;
        double value = 0.0;
        for (int t = A.sl_ptr[k]; t < A.sl_ptr[k + 1]; ++t) value += A.sl_coef[t] * A.u_full[A.sl_master[t]];
        A.u_full[A.sl_dof[k]] = value;
    }
}

// ||R||_2 of the Newmark residual R = P - F_int - C v - M a at the free displacements uf with
// element results ek / ef (the residual of the first Newton iteration,
// transient_nonlinear.mojo:2302-2356).  Collective; vs, as: n-entry shared scratch.
__device__ double residual_norm(const DevInst& I, const InstArrays& A, const double* uf, const double* ek,
                               const double* ef, double* vs, double* as, double* red) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int n = I.n, bw = I.bw, rw = I.rw, f0 = I.f_off;
    for (int i = tid; i < n; i += nt) {
        const int gi = f0 + i;
        const double an = I.a0 * (uf[gi] - A.u_n[gi]) - I.a2 * A.v_n[gi] - I.a3 * A.a_n[gi];
        vs[i] = A.v_n[gi] + I.dt * ((1.0 - I.gamma) * A.a_n[gi] + I.gamma * an);
        as[i] = an;
    }
    __syncthreads();
    const long long sp0 = I.slot_ptr_off;
    const double* Kinit = A.Kinit + I.band_off;
    double ss = 0.0;
    for (int i = tid; i < n; i += nt) {
        double cv = 0.0;
        if (I.has_damping) {
            for (int o = 0; o < rw; ++o) {
                const int j = i + o - bw;
                if (j < 0 || j >= n) continue;
                const int slot = i * rw + o;
                double C = I.alpha_m * (i == j ? A.Mrff[f0 + i] : 0.0);
                if (I.beta_k != 0.0) {
                    const long long c0 = A.slot_ptr[sp0 + slot], c1 = A.slot_ptr[sp0 + slot + 1];
                    double K = 0.0;
                    for (long long c = c0; c < c1; ++c)
                        K += (A.slot_coef ? A.slot_coef[c] : 1.0) * ek[A.slot_contrib[c]];
                    C += I.beta_k * K;
                }
                if (I.beta_k_init != 0.0) C += I.beta_k_init * Kinit[slot];
                cv += C * vs[j];
            }
        }
        const int q0 = A.fint_ptr[I.fint_ptr_off + i], q1 = A.fint_ptr[I.fint_ptr_off + i + 1];
        const double F = gather_fint(A, ef, q0, q1);
        const double r = A.P_f[f0 + i] - F - 0.0 - cv - A.Mff[f0 + i] * as[i];
        ss += r * r;
    }
    const double tot = block_sum(ss, red);
    __syncthreads();
    return sqrt(tot);
}

// Effective-matrix entry of band slot (i, j) exactly as the row assembly computes it
// (load K, add a1 C, add a0 M).
__device__ __forceinline__ double keff_of(const DevInst& I, const InstArrays& A, const double* Kinit, int i,
                                          int j, int slot, double K) {
    double C = 0.0;
    if (I.has_damping) {
        C = I.alpha_m * (i == j ? A.Mrff[I.f_off + i] : 0.0);
        if (I.beta_k != 0.0) C += I.beta_k * K;
        if (I.beta_k_init != 0.0) C += I.beta_k_init * Kinit[slot];
    }
    double keff = K;
    if (I.has_damping && I.a1 != 0.0) keff += I.a1 * C;
    if (i == j) keff += I.a0 * A.Mff[I.f_off + i];
    return keff;
}

__device__ __forceinline__ double keff_slot(const DevInst& I, const InstArrays& A, long long sp0,
                                            const double* Kinit, int i, int j, int slot) {
    const double K = gather_slot(A, sp0, slot);
    double C = 0.0;
    if (I.has_damping) {
        C = I.alpha_m * (i == j ? A.Mrff[I.f_off + i] : 0.0);
        if (I.beta_k != 0.0) C += I.beta_k * K;
        if (I.beta_k_init != 0.0) C += I.beta_k_init * Kinit[slot];
    }
    double keff = K;
    if (I.has_damping && I.a1 != 0.0) keff += I.a1 * C;
    if (i == j) keff += I.a0 * A.Mff[I.f_off + i];
    return keff;
}

// Block argmax of |column| with the reference's tie rule (first row wins).
__device__ __forceinline__ void block_argmax(double& v, int& r, double* red_v, int* red_r) {
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int orr = __shfl_xor_sync(0xffffffffu, r, o);
        if (ov > v || (ov == v && orr < r)) {
            v = ov;
            r = orr;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) {
        red_v[warp] = v;
        red_r[warp] = r;
    }
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = red_v[0];
    r = red_r[0];
    for (int w = 1; w < nw; ++w) {
        if (red_v[w] > v || (red_v[w] == v && red_r[w] < r)) {
            v = red_v[w];
            r = red_r[w];
        }
    }
}

// Dense LU with partial pivoting on an n x n row-major matrix in global memory
// (_try_factorize_dense_unsymmetric_loaded, linear_solver_backend.mojo:175-215).  fac is an
// n-entry shared scratch.  Returns 0 ok, 2 singular.
__device__ int dense_lu_global(double* D, int* piv, int n, double* fac, double* red_v, int* red_r) {
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int i = tid; i < n; i += nt) piv[i] = i;
    __syncthreads();
    for (int col = 0; col < n; ++col) {
        double v = -1.0;
        int r = n;
        for (int row = col + tid; row < n; row += nt) {
            const double c = fabs(D[(size_t)row * n + col]);
            if (c > v) {
                v = c;
                r = row;
            }
        }
        block_argmax(v, r, red_v, red_r);
        if (v <= 1.0e-14) return 2;
        if (r != col) {
            for (int j = tid; j < n; j += nt) {
                const double t = D[(size_t)col * n + j];
                D[(size_t)col * n + j] = D[(size_t)r * n + j];
                D[(size_t)r * n + j] = t;
            }
            if (tid == 0) {
                const int t = piv[col];
                piv[col] = piv[r];
                piv[r] = t;
            }
        }
        __syncthreads();
        const double diag = D[(size_t)col * n + col];
        if (fabs(diag) <= 1.0e-14) return 2;
        for (int row = col + 1 + tid; row < n; row += nt) fac[row] = D[(size_t)row * n + col] / diag;
        __syncthreads();
        const int m = n - col - 1;
        for (long long t = tid; t < (long long)m * m; t += nt) {
            const int row = col + 1 + (int)(t / m);
            const int j = col + 1 + (int)(t % m);
            const double f = fac[row];
            if (f != 0.0) D[(size_t)row * n + j] -= f * D[(size_t)col * n + j];
        }
        for (int row = col + 1 + tid; row < n; row += nt) D[(size_t)row * n + col] = fac[row];
        __syncthreads();
    }
    return 0;
}

// _solve_dense_unsymmetric (linear_solver_backend.mojo:218-240) with one warp.
__device__ void dense_solve_warp(const double* D, const int* piv, int n, const double* rhs,
                                 double* w, double* x) {
    const int lane = threadIdx.x & 31;
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int j = lane; j < i; j += 32) s += D[(size_t)i * n + j] * w[j];
        s = warp_sum(s);
        if (lane == 0) w[i] = rhs[piv[i]] - s;
        __syncwarp();
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = 0.0;
        for (int j = i + 1 + lane; j < n; j += 32) s += D[(size_t)i * n + j] * x[j];
        s = warp_sum(s);
        if (lane == 0) x[i] = (w[i] - s) / D[(size_t)i * n + i];
        __syncwarp();
    }
}

__device__ void newton_tail(const DevInst& I, InstArrays& A, int inst, const double* du,
                            const double* R, int* hrow, double* red, int* red_r);

__global__ void __launch_bounds__(256) instance_newton_kernel(const DevInst* __restrict__ insts,
                                                              InstArrays A0, int mode, int step) {
    InstArrays A = A0;
    extern __shared__ __align__(16) double smem_inst[];
    __shared__ DevInst I;
    __shared__ double red[32];
    __shared__ int red_r[32];
    __shared__ int s_it;  // this instance's Newton iterations of the step so far
    const int inst = blockIdx.x;
    const int tid = threadIdx.x, nt = blockDim.x;
    {
        const uint32_t* s = reinterpret_cast<const uint32_t*>(insts + inst);
        uint32_t* d = reinterpret_cast<uint32_t*>(&I);
        for (int i = tid; i < (int)(sizeof(DevInst) / 4); i += nt) d[i] = s[i];
        if (tid == 0) s_it = mode == INST_MODE_NEWTON ? A.iters[inst] : 0;
    }
    __syncthreads();
    if (I.large) return;  // global-memory band path (largeband_kernels.cuh)
    if (mode == INST_MODE_NEWTON && !A.active[inst]) return;
    int* hrow = (A.hist_iters && A.ctl) ? A.hist_iters + (size_t)A.ctl->step * gridDim.x : nullptr;
    const int n = I.n, bw = I.bw, rw = I.rw;
    double* Kb = smem_inst;        // n * rw
    double* vt = Kb + (size_t)n * rw;
    double* R = vt + n;
    double* w = R + n;
    double* du = w + n;
    double* fac = du + n;
    const int f0 = I.f_off;
    int rc = 0;
    // ModifiedNewton(Initial): the first iteration of the step freezes the tangent (the current
    // one, or K_init) and factors; later iterations reuse both (transient_nonlinear.mojo:
    // 2072-2085, 2236-2268, 2302-2335, 2421-2440)
    const Attempt at = attempt_of(I, A, inst);
    const bool modified = mode == INST_MODE_NEWTON && at.alg != 0;
    const bool refresh = !modified || s_it == 0;
    double* Kfz = modified ? A.kfrz + I.band_off : nullptr;
    if (mode == INST_MODE_SOLVE_EXPORTED) {
        for (int t = tid; t < n * rw; t += nt) Kb[t] = A.export_band[I.band_off + t];
        for (int i = tid; i < n; i += nt) R[i] = A.rhs_in[f0 + i];
        __syncthreads();
    } else {
        if (mode == INST_MODE_NEWTON && tid == 0) {
            A.iters[inst] += 1;
            if (A.bytes_counter) atomicAdd(A.bytes_counter, (unsigned long long)I.io_bytes);
        }
        // v_trial, a_trial (transient_nonlinear.mojo:496-531)
        for (int i = tid; i < n; i += nt) {
            const int gi = f0 + i;
            const double an =
                I.a0 * (A.u_f[gi] - A.u_n[gi]) - I.a2 * A.v_n[gi] - I.a3 * A.a_n[gi];
            vt[i] = A.v_n[gi] + I.dt * ((1.0 - I.gamma) * A.a_n[gi] + I.gamma * an);
            w[i] = an;
        }
        __syncthreads();
        // K: every band slot gathers its element contributions in element order (one lane
        // per slot, so the dependent index loads of many slots are in flight at once)
        const long long sp0 = I.slot_ptr_off;
        const double* Kinit = A.Kinit + I.band_off;
        const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
        if (!modified) {
            // four slots per thread at a time, their contribution lists walked side by side
            // (each slot still sums its own contributions in element order)
            gather_band4(A, sp0, n, bw, rw, Kb);
        } else
        for (int i = warp; i < n; i += nw)
            for (int o = lane; o < rw; o += 32) {
                const int j = i + o - bw;
                const int slot = i * rw + o;
                double K = 0.0;
                if (j >= 0 && j < n) {
                    if (!modified) {
                        K = gather_slot(A, sp0, slot);
                    } else if (refresh) {
                        K = at.alg == 2 ? Kinit[slot] : gather_slot(A, sp0, slot);
                        Kfz[slot] = K;
                    } else {
                        K = Kfz[slot];
                    }
                }
                Kb[slot] = K;
            }
        __syncthreads();
        int bad_sym = 0;
        if (I.spd) {
            // BandSPD takes the lower triangle after checking symmetry to 1e-10
            // (linear_solver_backend.mojo:266-271, 1936-1948)
            for (int i = warp; i < n; i += nw)
                for (int o = lane; o < bw; o += 32) {
                    const int j = i + o - bw;
                    if (j < 0) continue;
                    const int slot = i * rw + o, mslot = j * rw + (i - j + bw);
                    const double K = Kb[slot], Kt = Kb[mslot];
                    if (fabs(K - Kt) > 1.0e-10) bad_sym = 1;
                    if (I.has_damping && I.a1 != 0.0) {
                        double C = I.alpha_m * 0.0, Ct = 0.0;
                        if (I.beta_k != 0.0) {
                            C += I.beta_k * K;
                            Ct += I.beta_k * Kt;
                        }
                        if (I.beta_k_init != 0.0) {
                            C += I.beta_k_init * Kinit[slot];
                            Ct += I.beta_k_init * Kinit[mslot];
                        }
                        if (fabs(C - Ct) > 1.0e-10) bad_sym = 1;
                    }
                }
        }
        if (__syncthreads_or(bad_sym)) {
            if (tid == 0) {
                A.status[inst] = 4;
                if (mode == INST_MODE_NEWTON && A.active[inst]) {
                    A.active[inst] = 0;
                    atomicSub(A.nactive, 1);
                }
            }
            return;
        }
        // rows: C, effective band entries in place, C v in column order, residual
        for (int i = tid; i < n; i += nt) {
            double cv = 0.0;
            for (int o = 0; o < rw; ++o) {
                const int j = i + o - bw;
                if (j < 0 || j >= n) continue;
                const int slot = i * rw + o;
                const double K = Kb[slot];
                double C = 0.0;
                if (I.has_damping) {
                    C = I.alpha_m * (i == j ? A.Mrff[f0 + i] : 0.0);
                    if (I.beta_k != 0.0) C += I.beta_k * K;
                    if (I.beta_k_init != 0.0) C += I.beta_k_init * Kinit[slot];
                    cv += C * vt[j];
                }
                double keff = K;
                if (I.has_damping && I.a1 != 0.0) keff += I.a1 * C;
                if (i == j) keff += I.a0 * A.Mff[f0 + i];
                Kb[slot] = keff;
            }
            const int q0 = A.fint_ptr[I.fint_ptr_off + i], q1 = A.fint_ptr[I.fint_ptr_off + i + 1];
            const double F = gather_fint(A, A.ef, q0, q1);
            const double ma = A.Mff[f0 + i] * w[i];
            R[i] = A.P_f[f0 + i] - F - 0.0 - cv - ma;
            A.R[f0 + i] = R[i];
            if (mode == INST_MODE_EXPORT) A.export_f[f0 + i] = F;
        }
        __syncthreads();
        if (mode == INST_MODE_EXPORT) {
            for (int t = tid; t < n * rw; t += nt) A.export_band[I.band_off + t] = Kb[t];
            return;
        }
        if (at.test == 2) {  // NormUnbalance before the solve
            double s = 0.0;
            for (int i = tid; i < n; i += nt) s += R[i] * R[i];
            s = block_sum(s, red);
            if (sqrt(s) <= at.tol) {
                if (tid == 0) {
                    A.active[inst] = 0;
                    atomicSub(A.nactive, 1);
                    if (hrow) hrow[inst] = A.iters[inst] + (A.iters_prev ? A.iters_prev[inst] : 0);
                }
                return;
            }
        }
        if (mode == INST_MODE_NEWTON && A.dual && A.rejected && s_it == 0 && !A.rejected[inst] &&
            (!A.attempt || A.attempt[inst] == 0)) {
            // The step started from the learned guess u_l.  The Newmark predictor's u_p would
            // have the residual R(u_p) = R(u_l) + K_eff (u_l - u_p) to first order, K_eff being
            // the effective tangent just assembled at u_l; keep u_l unless its residual is the
            // larger, else go back to u_p (the plain predictor is the fallback).
            for (int i = tid; i < n; i += nt) du[i] = A.u_f[f0 + i] - A.u_base[f0 + i];
            __syncthreads();
            double sl = 0.0, sp = 0.0;
            for (int i = tid; i < n; i += nt) {
                double kd = 0.0;
                for (int o = 0; o < rw; ++o) {
                    const int j = i + o - bw;
                    if (j >= 0 && j < n) kd += Kb[i * rw + o] * du[j];
                }
                if (I.spd)  // BandSPD holds the lower band: the upper half from the rows below
                    for (int j = i + 1; j <= min(n - 1, i + bw); ++j) kd += Kb[j * rw + (i - j + bw)] * du[j];
                const double rp = R[i] + kd;
                sl += R[i] * R[i];
                sp += rp * rp;
            }
            sl = block_sum(sl, red);
            sp = block_sum(sp, red);
            const bool keep = isfinite(sl) && sl <= sp;
            if (tid == 0 && A.pred_stats) {
                A.pred_stats[2 * inst] += 1;
                if (keep) A.pred_stats[2 * inst + 1] += 1;
            }
            if (!keep) {
                for (int i = tid; i < n; i += nt) {
                    const int gi = f0 + i;
                    const double u = A.u_base[gi];
                    A.u_f[gi] = u;
                    A.u_full[A.free_dof[gi]] = u;
                }
                const size_t e0 = (size_t)I.elem_off * kEStride;
                for (size_t t = tid; t < (size_t)I.n_elem * kEStride; t += nt) A.estate[e0 + t] = A.estate_base[e0 + t];
                if (I.n_sl > 0) {
                    __syncthreads();
                    enforce_slaves(I, A);
                }
                if (tid == 0) {
                    // the rejected evaluation is not a Newton iteration of the step
                    A.iters[inst] -= 1;
                    A.rejected[inst] = 1;
                    red_r[0] = A.ctl ? atomicAdd(&A.el.count[(A.ctl->iter + 1) & 1], I.n_elem) : -1;
                }
                __syncthreads();
                const int base = red_r[0];
                if (base >= 0) {
                    const int buf = (A.ctl->iter + 1) & 1;
                    for (int k = tid; k < I.n_elem; k += nt)
                        A.el.list[buf][base + k] = list_entry(A.el, buf, I.elem_off + k);
                }
                return;
            }
            __syncthreads();
        }
    }
    bool dense = false;
    double* D = A.dense + I.dense_off;
    int* piv = A.piv + f0;
    if (!refresh) {
        // the step's factors
        dense = A.lu_dense[inst] != 0;
        if (!dense) {
            const double* LU = A.lufrz + I.band_off;
            for (int t = tid; t < n * rw; t += nt) Kb[t] = LU[t];
        }
        __syncthreads();
    } else if (I.spd) {
        rc = band_chol_smem(Kb, n, bw, rw, fac);
    } else {
        rc = band_lu_smem(Kb, n, bw, rw, fac);
    }
    if (refresh && rc == 6) {
        // BandGeneral: a row swap would be needed, so the whole effective matrix is factored
        // densely with partial pivoting (linear_solver_backend.mojo:650-657, 612-629), starting
        // again from the assembled values.
        __syncthreads();
        for (long long t = tid; t < (long long)n * n; t += nt) D[t] = 0.0;
        __syncthreads();
        if (mode == INST_MODE_SOLVE_EXPORTED) {
            for (int t = tid; t < n * rw; t += nt) {
                const int i = t / rw, j = i + t % rw - bw;
                if (j >= 0 && j < n) D[(size_t)i * n + j] = A.export_band[I.band_off + t];
            }
        } else {
            const double* Kinit = A.Kinit + I.band_off;
            for (int t = tid; t < n * rw; t += nt) {
                const int i = t / rw, j = i + t % rw - bw;
                if (j >= 0 && j < n)
                    D[(size_t)i * n + j] = modified ? keff_of(I, A, Kinit, i, j, t, Kfz[t])
                                                    : keff_slot(I, A, I.slot_ptr_off, Kinit, i, j, t);
            }
        }
        __syncthreads();
        rc = dense_lu_global(D, piv, n, fac, red, red_r);
        dense = true;
        if (tid == 0 && A.fallbacks) A.fallbacks[inst] += 1;
    }
    if (modified && refresh && rc == 0) {
        __syncthreads();
        if (!dense) {
            double* LU = A.lufrz + I.band_off;
            for (int t = tid; t < n * rw; t += nt) LU[t] = Kb[t];
        }
        if (tid == 0) A.lu_dense[inst] = dense ? 1 : 0;
    }
    if (rc != 0) {
        if (tid == 0) {
            A.status[inst] = rc;
            if (mode == INST_MODE_NEWTON && A.active[inst]) {
                A.active[inst] = 0;
                atomicSub(A.nactive, 1);
            }
        }
        return;
    }
    // multipliers of the last column were written in the loop except column n-1 (none below)
    __syncthreads();
    if (tid < 32) {
        if (dense)
            dense_solve_warp(D, piv, n, R, w, du);
        else if (I.spd)
            band_solve_chol_warp(Kb, n, bw, rw, R, w, du);
        else
            band_solve_lu_warp(Kb, n, bw, rw, R, w, du);
    }
    __syncthreads();
    if (mode == INST_MODE_SOLVE_EXPORTED) {
        for (int i = tid; i < n; i += nt) A.du[f0 + i] = du[i];
        return;
    }
    newton_tail(I, A, inst, du, R, hrow, red, red_r);
}

// Displacement update, convergence test (NormDispIncr after the update,
// transient_nonlinear.mojo:2539, 2798-2811; EnergyIncr, MaxDispIncr) and, for an instance that
// keeps iterating, its elements appended to the next element list.  Collective over the CTA.
__device__ void newton_tail(const DevInst& I, InstArrays& A, int inst, const double* du,
                            const double* R, int* hrow, double* red, int* red_r) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int n = I.n, f0 = I.f_off;
    double ss = 0.0, en = 0.0, mx = 0.0;
    for (int i = tid; i < n; i += nt) {
        const int gi = f0 + i;
        const double d = du[i];
        ss += d * d;
        en += d * R[i];
        mx = fmax(mx, fabs(d));
        A.du[gi] = d;
        const double un = A.u_f[gi] + d;
        A.u_f[gi] = un;
        A.u_full[A.free_dof[gi]] = un;
    }
    if (I.n_sl > 0) {
        __syncthreads();
        enforce_slaves(I, A);
    }
    const double norm = sqrt(block_sum(ss, red));
    const double energy = fabs(block_sum(en, red));
    const double maxd = block_max(mx, red);
    const Attempt at = attempt_of(I, A, inst);
    if (tid == 0) {
        bool conv = false;
        if (at.test == 1) conv = norm <= at.tol;
        else if (at.test == 3) conv = energy <= at.tol;
        else if (at.test == 0) conv = maxd <= at.tol;
        if (!isfinite(norm)) {
            A.status[inst] = 3;
            conv = true;
        }
        const int prev = A.iters_prev ? A.iters_prev[inst] : 0;
        int base = -1, retry = 0, failed = 0;
        if (conv) {
            A.active[inst] = 0;
            atomicSub(A.nactive, 1);
            if (hrow) hrow[inst] = A.iters[inst] + prev;
        } else if (A.iters[inst] >= at.max_iters) {
            if (A.attempt && A.attempt[inst] + 1 < I.n_att) {
                // the next attempt of the chain, from the step's start
                A.attempt[inst] += 1;
                A.iters_prev[inst] = prev + A.iters[inst];
                A.iters[inst] = 0;
                retry = 1;
            } else {
                A.status[inst] = 1;
                A.active[inst] = 0;
                atomicSub(A.nactive, 1);
                if (hrow) hrow[inst] = A.iters[inst] + prev;
                failed = 1;
            }
        }
        if (!conv && !failed && A.ctl)
            base = atomicAdd(&A.el.count[(A.ctl->iter + 1) & 1], I.n_elem);
        red_r[0] = base;
        red_r[1] = retry;
    }
    __syncthreads();
    if (red_r[1]) {
        // back to the step's start (transient_nonlinear.mojo:1925-1942): the predictor's
        // displacements, the elements' basic state; fiber trial state is recomputed from the
        // committed state and needs nothing
        for (int i = tid; i < n; i += nt) {
            const int gi = f0 + i;
            const double u = A.u_base[gi];
            A.u_f[gi] = u;
            A.u_full[A.free_dof[gi]] = u;
        }
        const size_t e0 = (size_t)I.elem_off * kEStride;
        for (size_t t = tid; t < (size_t)I.n_elem * kEStride; t += nt) A.estate[e0 + t] = A.estate_base[e0 + t];
        if (I.n_sl > 0) {
            __syncthreads();
            enforce_slaves(I, A);
        }
    }
    // still iterating: list this instance's elements for the next element kernel
    const int base = red_r[0];
    if (base >= 0) {
        const int buf = (A.ctl->iter + 1) & 1;
        int* list = A.el.list[buf];
        for (int k = tid; k < I.n_elem; k += nt) list[base + k] = list_entry(A.el, buf, I.elem_off + k);
    }
}

// Newmark predictor over every free dof (transient_nonlinear.mojo:553-590), the excitation
// load P_f = F_const + (-M ag) on the excitation direction (1823-1852), and per-instance
// activation for the Newton loop.
__global__ void predictor_kernel(const DevInst* __restrict__ insts, InstArrays A,
                                 const int* __restrict__ free_inst,
                                 const int* __restrict__ free_dir, const double* __restrict__ ag_base,
                                 int n_free_total, int n_inst, DevCtl* ctl,
                                 cudaGraphConditionalHandle inner, int use_cond) {
    const int gi = blockIdx.x * blockDim.x + threadIdx.x;
    const double* ag = ag_base + (size_t)(ctl->step - ctl->step0) * 4 * n_inst;
    if (gi == 0) {
        ctl->iter = 0;
        if (use_cond) cudaGraphSetConditional(inner, 1);
    }
    if (gi < n_inst) {
        const bool ok = A.status[gi] == 0;
        A.active[gi] = ok ? 1 : 0;
        A.iters[gi] = 0;
        if (A.attempt) {
            A.attempt[gi] = 0;
            A.iters_prev[gi] = 0;
        }
        if (A.rejected) A.rejected[gi] = 0;
        if (ok) {
            atomicAdd(A.nactive, 1);
            const DevInst& I = insts[gi];
            const int base = atomicAdd(&A.el.count[0], I.n_elem);
            for (int k = 0; k < I.n_elem; ++k) A.el.list[0][base + k] = list_entry(A.el, 0, I.elem_off + k);
        }
    }
    if (gi >= n_free_total) return;
    const int inst = free_inst[gi];
    const DevInst& I = insts[inst];
    const double un = A.u_f[gi], vn = A.v_f[gi], an = A.a_f[gi];
    A.u_n[gi] = un;
    A.v_n[gi] = vn;
    A.a_n[gi] = an;
    const double up = un + I.dt * vn + I.coeff * an;
    A.u_f[gi] = up;
    if (A.u_base) A.u_base[gi] = up;
    A.u_full[A.free_dof[gi]] = up;
    double p = A.fconst[gi];
    // ag holds, per instance, the ground acceleration of each excitation direction at this
    // step followed by a has-excitation flag per direction.  Strut adds -M*ag onto a zero load
    // vector first (uniform_inertia_load), then onto F_const.
    const int dir = free_dir[gi];
    if (dir == 1 || dir == 2) {
        const double agv = ag[4 * inst + (dir - 1)];
        if (ag[4 * inst + 2 + (dir - 1)] != 0.0) {
            double load = 0.0;
            load += -A.Mff[gi] * agv;
            p += load;
        }
    }
    A.P_f[gi] = p;
}

// Newmark update after convergence (transient_nonlinear.mojo:594-647).
__global__ void post_step_kernel(const DevInst* __restrict__ insts, InstArrays A,
                                 const int* __restrict__ free_inst, int n_free_total) {
    const int gi = blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= n_free_total) return;
    const int inst = free_inst[gi];
    if (A.status[inst] != 0) return;
    const DevInst& I = insts[inst];
    const double an = I.a0 * (A.u_f[gi] - A.u_n[gi]) - I.a2 * A.v_n[gi] - I.a3 * A.a_n[gi];
    const double vn = A.v_n[gi] + I.dt * ((1.0 - I.gamma) * A.a_n[gi] + I.gamma * an);
    A.a_f[gi] = an;
    A.v_f[gi] = vn;
    // converged increment of this step for the learned predictor's features
    if (A.hist_du && A.ctl) A.hist_du[(size_t)(A.ctl->step & 3) * A.n_free_total + gi] = A.u_f[gi] - A.u_n[gi];
}

__global__ void record_disp_kernel(const double* __restrict__ u_full,
                                   const int* __restrict__ rec_dof, int n_rec_total,
                                   double* __restrict__ out_base, const DevCtl* __restrict__ ctl) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n_rec_total) out_base[(size_t)ctl->step * n_rec_total + t] = u_full[rec_dof[t]];
}

// End of a Newton iteration: continue while some instance is still iterating.
__global__ void newton_check_kernel(DevCtl* ctl, const int* __restrict__ nactive,
                                    cudaGraphConditionalHandle inner, int use_cond) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    ctl->iter += 1;
    const int more = (*nactive > 0 && ctl->iter < ctl->max_iters) ? 1 : 0;
    if (use_cond) cudaGraphSetConditional(inner, more);
}

// End of a step: note the step at which each instance failed, advance the step counter, reset
// the active count, and continue while steps remain (a single-instance handle stops at its
// failing step).
__global__ void step_end_kernel(DevCtl* ctl, const int* __restrict__ status,
                                int* __restrict__ fail_step, int n_inst, int* nactive,
                                ElemList el, cudaGraphConditionalHandle outer, int use_cond) {
    const int step = ctl->step;
    for (int i = threadIdx.x; i < n_inst; i += blockDim.x)
        if (status[i] != 0 && fail_step[i] < 0) fail_step[i] = step;
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->step = step + 1;
        *nactive = 0;
        el.count[0] = 0;
        el.count[1] = 0;
        el.next[0] = 0;
        el.next[1] = 0;
        el.hard_count[0] = 0;
        el.hard_count[1] = 0;
        if (el.rq) {
            el.rq_tail[0] = 0;
            el.rq_tail[1] = 0;
            el.fan_finished[0] = 0;
            el.fan_finished[1] = 0;
        }
        const bool stop = ctl->single && status[0] != 0;
        if (use_cond) cudaGraphSetConditional(outer, (step + 1 < ctl->n_end && !stop) ? 1 : 0);
    }
}

__global__ void scatter_free_kernel(const double* __restrict__ u_f, const int* __restrict__ free_dof,
                                    double* __restrict__ u_full, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) u_full[free_dof[t]] = u_f[t];
}

// Every slave dof of every instance from its retained dofs (after the Newmark predictor or a
// host-side displacement write; transient_nonlinear.mojo:1768-1790).
__global__ void slave_enforce_kernel(InstArrays A, int n_slaves) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_slaves) return;
    double value = 0.0;
    for (int t = A.sl_ptr[k]; t < A.sl_ptr[k + 1]; ++t) value += A.sl_coef[t] * A.u_full[A.sl_master[t]];
    A.u_full[A.sl_dof[k]] = value;
}

}  // namespace strut

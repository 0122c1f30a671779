// Newton iteration of instances whose effective band does not fit in shared memory (a 3D frame
// of a few thousand dofs and a bandwidth of a few hundred: ~10-30 MB, resident in the 126 MB L2).
//
//   large_assemble_kernel  one warp per band row: K gathered per slot in element order, C, the
//                          effective entries K + a1 C + a0 M written to the global band, the row's
//                          residual P - F_int - C v - M a (transient_nonlinear.mojo:2302-2356,
//                          linear_solver_backend.mojo:1877-1983)
//   large_factor_kernel    cooperative (all CTAs co-resident): blocked right-looking band LU with
//                          partial pivoting, panel width kPanel, the right-hand side carried as
//                          one more column.  CTA 0 factors the panel in shared memory; every CTA
//                          then takes column tiles of the trailing block (the panel's row
//                          interchanges, then the eliminations in column order).  Two bounded
//                          grid barriers per panel.
//   large_solve_kernel     one CTA per instance: blocked back substitution through U, then the
//                          displacement update and the convergence test shared with the
//                          shared-memory path.
//
// Strut's BandGeneral factorises without pivoting and, at the first column whose pivot test
// fails (a sub-diagonal entry larger than the pivot, linear_solver_backend.mojo:631-680),
// restarts from the original matrix with a dense partial-pivot LU (175-240).  The columns
// before that one choose no interchange under partial pivoting either (the same strict test,
// the first largest entry wins), so one partial-pivot factorisation performs the reference's
// interchanges and eliminations on every entry; it needs only the band, because below the
// band the dense matrix's columns are zero (rows never come from further than bw below) and
// the pivot rows' fill stays within 2 bw of the diagonal (storage: columns i - bw .. i + 2 bw
// of row i, 3 bw + 1 slots).  A factorisation that interchanged rows counts as a dense
// fallback in the statistics.  The order of the subtractions on an entry is the reference's
// (column by column); the substitution through U is blocked, so the GPU agrees with the
// oracle to rounding.
#pragma once

#include "solver_kernels.cuh"

namespace strut {

constexpr int kPanel = 32;         // panel width of the blocked band LU
constexpr int kLargeThreads = 384; // threads of a factorisation CTA (one per panel row)
// The variant for wider bands: 16-column panels and 640 threads (the panel rows' registers halve,
// so more rows fit a CTA).  Every entry receives the same subtractions in the same column order
// with either variant, so their results are the same bit for bit.
constexpr int kPanelWide = 16;
constexpr int kLargeThreadsWide = 640;
constexpr int kSolveThreads = 1024;

constexpr int kColTile = 16;       // trailing-update columns per tile
enum { LSTAT_OK = 0, LSTAT_SINGULAR = 2, LSTAT_CONVERGED = 7, LSTAT_IDLE = -1 };

struct GridBarrier {
    unsigned int count;
    unsigned int gen;
    int err;
    int pad;
    int limit;  // polls a waiting CTA makes before it gives up (strut_gpu_set_wait_limit)
    int pad2;
};

constexpr int kBarrierPolls = 1 << 22;

// Grid-wide barrier of a cooperative launch.  Thread 0 of each CTA arrives; the last arrival
// resets the count and advances the generation; the others wait for the generation to move,
// for a bounded number of polls (gb->limit), after which the barrier records an error and every
// CTA stops.
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
            const int limit = *(volatile int*)&gb->limit;
            while (atomicAdd(&gb->gen, 0u) == g) {
                if (++polls > limit || atomicAdd(&gb->err, 0) != 0) {
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

// Slot of (i, j) in the factorisation band: row i holds columns i - bw .. i + 2 bw.
__device__ __forceinline__ long long lslot(int lrw, int bw, int i, int j) {
    return (long long)i * lrw + (j - i + bw);
}

// ---- assembly and residual ---------------------------------------------------------------

// grid.x: warps over the rows of all large instances (row r of the concatenation over
// large_list).  mode INST_MODE_NEWTON skips inactive instances; INST_MODE_EXPORT also writes the
// band and F_int to the export buffers.  The residual is also written to wbuf, the column the
// factorisation carries along.
__global__ void __launch_bounds__(256) large_assemble_kernel(const DevInst* __restrict__ insts,
                                                             InstArrays A, const int* __restrict__ large_list,
                                                             const int* __restrict__ row_base,
                                                             int n_large, int total_rows, int mode,
                                                             GridBarrier* gb, double* __restrict__ wbuf) {
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
    double* B = A.lband + I.lband_off + (long long)i * I.lrw;
    for (int o = rw + lane; o < I.lrw; o += 32) B[o] = 0.0;  // fill slots
    double cv = 0.0;
    for (int o = lane; o < rw; o += 32) {
        const int j = i + o - bw;
        const long long slot = (long long)i * rw + o;
        if (j < 0 || j >= n) {
            B[o] = 0.0;
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
        B[o] = keff;
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
        wbuf[gi] = A.R[gi];
        if (mode == INST_MODE_EXPORT) A.export_f[gi] = F;
    }
}

// The learned guess's check on the global-memory band path, between the assembly and the
// factorisation (the instance kernel's check, the same arithmetic): one CTA per large instance.
// At the step's first iteration from a learned guess u_l, compare |R(u_l)| with the first-order
// residual of the Newmark predictor u_p, |R(u_l) + K_eff (u_l - u_p)|, K_eff being the band just
// assembled (row i: columns i - bw .. i + bw at slots 0 .. 2 bw); when the learned one is the
// larger, go back to u_p, skip this iteration's factorisation and list the elements again.
__global__ void __launch_bounds__(256) large_learned_check_kernel(const DevInst* __restrict__ insts, InstArrays A,
                                                                  const int* __restrict__ large_list,
                                                                  int n_large) {
    __shared__ double red[32];
    __shared__ int red_r[2];
    const int li = blockIdx.x;
    if (li >= n_large) return;
    const int inst = large_list[li];
    const DevInst& I = insts[inst];
    const int tid = threadIdx.x, nt = blockDim.x;
    if (tid == 0) A.skip[inst] = 0;
    if (!A.active[inst] || A.iters[inst] != 1 || A.rejected[inst] || (A.attempt && A.attempt[inst] != 0)) return;
    const int n = I.n, bw = I.bw, f0 = I.f_off;
    const double* B = A.lband + I.lband_off;
    double sl = 0.0, sp = 0.0;
    for (int i = tid; i < n; i += nt) {
        double kd = 0.0;
        for (int o = 0; o <= 2 * bw; ++o) {
            const int j = i + o - bw;
            if (j >= 0 && j < n) kd += B[(long long)i * I.lrw + o] * (A.u_f[f0 + j] - A.u_base[f0 + j]);
        }
        const double r = A.R[f0 + i];
        const double rp = r + kd;
        sl += r * r;
        sp += rp * rp;
    }
    sl = block_sum(sl, red);
    sp = block_sum(sp, red);
    const bool keep = isfinite(sl) && sl <= sp;
    if (tid == 0 && A.pred_stats) {
        A.pred_stats[2 * inst] += 1;
        if (keep) A.pred_stats[2 * inst + 1] += 1;
    }
    if (keep) return;
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
        A.iters[inst] -= 1;  // the rejected evaluation is not a Newton iteration of the step
        A.rejected[inst] = 1;
        A.skip[inst] = 1;
        red_r[0] = A.ctl ? atomicAdd(&A.el.count[(A.ctl->iter + 1) & 1], I.n_elem) : -1;
    }
    __syncthreads();
    const int base = red_r[0];
    if (base >= 0) {
        const int buf = (A.ctl->iter + 1) & 1;
        for (int k = tid; k < I.n_elem; k += nt) A.el.list[buf][base + k] = list_entry(A.el, buf, I.elem_off + k);
    }
}

// ---- blocked band LU with partial pivoting -------------------------------------------------

// Copies the exported band of every large instance into its factorisation band (fill slots
// zero) and the right-hand side into wbuf (strut_gpu_factor_solve on a band from
// strut_gpu_state_determination).
__global__ void large_load_exported_kernel(const DevInst* __restrict__ insts, InstArrays A,
                                           const int* __restrict__ large_list, int n_large,
                                           GridBarrier* gb, double* __restrict__ wbuf) {
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
        gb->count = 0u;
        gb->err = 0;
    }
    const int li = blockIdx.y;
    if (li >= n_large) return;
    const DevInst& I = insts[large_list[li]];
    const long long total = (long long)I.n * I.lrw;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long first = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (long long t = first; t < total; t += stride) {
        const long long i = t / I.lrw;
        const int o = (int)(t - i * I.lrw);
        A.lband[I.lband_off + t] = o < I.rw ? A.export_band[I.band_off + i * I.rw + o] : 0.0;
    }
    for (long long i = first; i < I.n; i += stride) wbuf[I.f_off + i] = A.rhs_in[I.f_off + i];
}

// Shared memory of large_factor_kernel: the panel's unit lower triangle L11
// (kPanel x (kPanel + 1)); CTA 0's panel rows (kLargeThreads x (kPanel + 1)), whose space the
// column slab of the trailing phase ((kPanel + bw) x (kColTile + 2)) reuses; the row at the
// diagonal (two, by column parity) and the row that replaces it; the panel's row permutation.
// Row stride of the panel-row buffer, which the slab (stride kColTile + 2) reuses.
__host__ __device__ constexpr int large_row_stride(int panel) {
    return panel + 1 > kColTile + 2 ? panel + 1 : kColTile + 2;
}
__host__ __device__ inline size_t large_factor_smem(int panel, int threads) {
    return sizeof(double) * ((size_t)panel * (panel + 1) + (size_t)threads * large_row_stride(panel) + 3 * panel) +
           sizeof(int) * (size_t)threads;
}

// Column tiles of the trailing update of one panel (+1: the right-hand side): the CTAs a
// factorisation can keep busy.
__host__ __device__ inline int large_factor_tiles(int bw) {
    return (2 * bw + kColTile - 1) / kColTile + 1;
}

// Largest half-band each variant takes: one thread per panel row.
constexpr int kLargeMaxBw = kLargeThreads - kPanel;
constexpr int kLargeMaxBwWide = kLargeThreadsWide - kPanelWide;

// Argmax over a warp, the first (smallest index) of equal values winning.
__device__ __forceinline__ void warp_argmax_first(double& v, int& idx) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, off);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, off);
        if (ov > v || (ov == v && oi < idx)) {
            v = ov;
            idx = oi;
        }
    }
}

// Cooperative.  wbuf holds the right-hand side on entry and L^-1 P b on exit; the band holds U
// on exit (its strictly lower part is left stale: the substitution reads U only).  lpan
// (column-major, leading dimension kLargeThreads) / lperm: the factored panel and the row
// permutation of its interchanges, from CTA 0 to the others.
//
// Per panel: CTA 0 factors the panel columns with one thread per panel row, the row in
// registers, four columns per rolled step (the finished columns go to shared memory and the
// row shifts left).  Per column the row at the diagonal publishes itself as the pivot row and
// one block vote asks whether any row below beats it strictly; only then the full search for the
// first largest entry runs and the two rows are exchanged whole (multipliers included).  Grid
// barrier; every CTA takes column tiles of the trailing block: loads them with the panel's row
// permutation applied, solves the panel rows against the unit lower L11 on the warps (lane =
// row), subtracts L21 U12 from the rows below entry by entry in column order (one thread per
// row, the row's multipliers in registers); grid barrier.
template <int PANEL, int THREADS>
__global__ void __launch_bounds__(THREADS) large_factor_kernel(
    const DevInst* __restrict__ insts, InstArrays A, const int* __restrict__ large_list,
    int n_large, int mode, GridBarrier* gb, double* wbuf, double* lpan, int* lperm) {
    extern __shared__ __align__(16) double smem_lf[];
    __shared__ int s_flag[2];
    __shared__ int s_piv[PANEL];
    __shared__ double red[32];
    __shared__ int red_r[32];
    constexpr int kPs = PANEL + 1;     // row stride of L11
    constexpr int kRs = large_row_stride(PANEL);  // row stride of the panel rows and the slab
    constexpr int kSs = kColTile + 2;   // row stride of the slab (even: 16-byte rows)
    constexpr int kLd = THREADS;  // leading dimension of lpan
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, wid = tid >> 5;
    const int nwarps = nt >> 5;
    double* L11 = smem_lf;                              // PANEL x kPs
    double* Pout = L11 + PANEL * kPs;                  // panel rows (CTA 0), THREADS x kRs
    double* S = Pout;                                   // slab of the trailing phase, pr x kSs
    double* prow2 = Pout + (size_t)THREADS * kRs;       // row at the diagonal, by column parity
    double* crow = prow2 + 2 * PANEL;                  // the row that replaces it
    int* s_perm = (int*)(crow + PANEL);                // panel row -> original row
    unsigned int gen = 0;
    if (tid == 0) gen = atomicAdd(&gb->gen, 0u);
    for (int li = 0; li < n_large; ++li) {
        const int inst = large_list[li];
        const DevInst& I = insts[inst];
        if (mode == INST_MODE_NEWTON && (!A.active[inst] || (A.skip && A.skip[inst]))) {
            if (blockIdx.x == 0 && tid == 0) A.lstatus[li] = LSTAT_IDLE;
            continue;
        }
        const int n = I.n, bw = I.bw, lrw = I.lrw;
        double* B = A.lband + I.lband_off;
        double* w = wbuf + I.f_off;
        const Attempt at = attempt_of(I, A, inst);
        if (mode == INST_MODE_NEWTON && at.test == 2) {
            // NormUnbalance is tested on the residual before the solve; every CTA reaches the
            // same decision from the same sums
            double s = 0.0;
            for (int i = tid; i < n; i += nt) s += A.R[I.f_off + i] * A.R[I.f_off + i];
            s = block_sum(s, red);
            if (sqrt(s) <= at.tol) {
                if (blockIdx.x == 0 && tid == 0) A.lstatus[li] = LSTAT_CONVERGED;
                continue;
            }
        }
        const int P = min(PANEL, max(bw, 1));
        int result = LSTAT_OK;
        int pivoted = 0;
        for (int k0 = 0; k0 < n && result == LSTAT_OK; k0 += P) {
            const int kb = min(P, n - k0);
            const int r1 = min(n - 1, k0 + kb - 1 + bw);      // last row with a nonzero in the panel
            const int pr = r1 - k0 + 1;
            const int c1 = min(n - 1, k0 + kb - 1 + 2 * bw);  // last column the panel's rows reach
            const int r = tid;                                // the panel row of this thread
            const bool own = r < pr;
            if (blockIdx.x == 0) {
                // ---- panel: rows k0..r1, columns k0..k0+kb-1 (rows loaded coalesced, lane = column)
                for (int rb = wid; rb < pr; rb += 4 * nwarps) {
                    double v[4];  // four rows in flight per warp
#pragma unroll
                    for (int m = 0; m < 4; ++m) {
                        const int rr = rb + m * nwarps;
                        const int d = lane - rr;
                        v[m] = (rr < pr && lane < kb && d >= -bw && d <= 2 * bw) ? B[lslot(lrw, bw, k0 + rr, k0 + lane)]
                                                                                 : 0.0;
                    }
#pragma unroll
                    for (int m = 0; m < 4; ++m)
                        if (rb + m * nwarps < pr && lane < PANEL) Pout[(rb + m * nwarps) * kRs + lane] = v[m];
                }
                if (own) s_perm[r] = r;
                if (tid == 0) s_flag[0] = LSTAT_OK;
                __syncthreads();
                double a[PANEL];  // a[q] = column c0 + q of this thread's row
#pragma unroll
                for (int q = 0; q < PANEL; ++q) a[q] = own ? Pout[r * kRs + q] : 0.0;
                bool failed = false;
                for (int c0 = 0; c0 < kb; c0 += 4) {
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) {
                        const int c = c0 + cc;
                        if (c < kb && !failed) {
                            const int last = min(pr - 1, c + bw);  // rows of column k0+c in the band
                            const bool act = own && r > c && r <= last;
                            // double buffered: a slow thread may still read the previous one
                            double* prow = prow2 + (c & 1) * PANEL;
                            if (r == c) {
#pragma unroll
                                for (int q = 0; q < PANEL; ++q) prow[q] = a[q];
                            }
                            __syncthreads();
                            // the reference's strict '>' scan keeps the diagonal unless a row
                            // below beats it
                            const double dabs = fabs(prow[cc]);
                            const int any = __syncthreads_or(act && fabs(a[cc]) > dabs);
                            const double* pivrow = prow;
                            int p = c;
                            if (any || dabs <= 1.0e-14) {
                                double bv = (own && r >= c && r <= last) ? fabs(a[cc]) : -1.0;
                                int br = r;
                                warp_argmax_first(bv, br);
                                if (lane == 0) {
                                    red[wid] = bv;
                                    red_r[wid] = br;
                                }
                                __syncthreads();
                                double pv = lane < nwarps ? red[lane] : -2.0;
                                p = lane < nwarps ? red_r[lane] : 0x7fffffff;
                                warp_argmax_first(pv, p);
                                if (pv <= 1.0e-14) {
                                    failed = true;
                                    if (tid == 0) s_flag[0] = LSTAT_SINGULAR;
                                } else if (p != c) {
                                    // whole rows, multipliers included, so that the trailing
                                    // columns can take all interchanges first and the
                                    // eliminations after
                                    pivoted = 1;
                                    if (r == p) {
#pragma unroll
                                        for (int q = 0; q < PANEL; ++q) crow[q] = a[q];
                                    }
                                    if (tid == 0) {
                                        const int o = s_perm[c];
                                        s_perm[c] = s_perm[p];
                                        s_perm[p] = o;
                                    }
                                    if (wid == 0 && lane < c0) {
                                        // finished columns of earlier steps
                                        const double t0 = Pout[c * kRs + lane];
                                        Pout[c * kRs + lane] = Pout[p * kRs + lane];
                                        Pout[p * kRs + lane] = t0;
                                    }
                                    __syncthreads();
                                    if (r == c) {
#pragma unroll
                                        for (int q = 0; q < PANEL; ++q) a[q] = crow[q];
                                    } else if (r == p) {
#pragma unroll
                                        for (int q = 0; q < PANEL; ++q) a[q] = prow[q];
                                    }
                                    pivrow = crow;
                                }
                            }
                            if (!failed) {
                                if (act) {
                                    const double f = a[cc] / pivrow[cc];
                                    a[cc] = f;
#pragma unroll
                                    for (int q = cc + 1; q < PANEL; ++q)
                                        if (c0 + q < kb) a[q] = fma(-f, pivrow[q], a[q]);
                                }
                                if (tid == 0) s_piv[c] = p;
                            }
                        }
                    }
                    // columns c0 .. c0+3 are final: keep them, shift the row left by four
                    if (own) {
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                            if (c0 + q < PANEL) Pout[r * kRs + c0 + q] = a[q];
                    }
#pragma unroll
                    for (int q = 0; q < PANEL; ++q) a[q] = q + 4 < PANEL ? a[q + 4] : 0.0;
                }
                __syncthreads();
                if (s_flag[0] == LSTAT_OK) {
                    for (int t = tid; t < kb * pr; t += nt) {
                        const int q = t / pr, rr = t - q * pr;
                        lpan[q * kLd + rr] = Pout[rr * kRs + q];
                    }
                    for (int rr = wid; rr < kb; rr += nwarps)
                        if (lane >= rr && lane < kb) B[lslot(lrw, bw, k0 + rr, k0 + lane)] = Pout[rr * kRs + lane];
                    if (own) lperm[r] = s_perm[r];
                }
                if (tid == 0) {
                    A.lstatus[li] = s_flag[0];
                    // publish the panel result to the other CTAs through gb->pad
                    atomicExch(&gb->pad, s_flag[0]);
                }
            }
            if (!grid_barrier(gb, gen)) return;
            if (tid == 0) s_flag[1] = atomicAdd(&gb->pad, 0);
            __syncthreads();
            result = s_flag[1];
            if (result != LSTAT_OK) break;
            // ---- trailing columns k0+kb .. c1 in tiles of kColTile, and the right-hand side
            const int j_first = k0 + kb;
            const int ncols = c1 - j_first + 1;
            const int ntiles = (ncols > 0 ? (ncols + kColTile - 1) / kColTile : 0) + 1;
            if (blockIdx.x >= ntiles) {
                if (!grid_barrier(gb, gen)) return;
                continue;
            }
            // this thread's panel row: its multipliers (L21, or L11 for the first kb rows)
            double lrow[PANEL];
#pragma unroll
            for (int q = 0; q < PANEL; ++q) lrow[q] = (own && q < kb) ? lpan[q * kLd + r] : 0.0;
            if (own) {
                s_perm[r] = lperm[r];
                if (r < kb) {
#pragma unroll
                    for (int q = 0; q < PANEL; ++q) L11[r * kPs + q] = lrow[q];
                }
            }
            for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
                const bool rhs = tile == ntiles - 1;
                const int j0 = j_first + tile * kColTile;
                const int ct = rhs ? 1 : min(kColTile, c1 - j0 + 1);
                __syncthreads();
                for (int t0 = tid; t0 < pr * ct; t0 += 4 * nt) {
                    double v[4];  // four loads in flight per thread
#pragma unroll
                    for (int m = 0; m < 4; ++m) {
                        const int t = t0 + m * nt;
                        v[m] = 0.0;
                        if (t < pr * ct) {
                            const int rr = t / ct, q = t - rr * ct;
                            const int src = k0 + s_perm[rr];
                            const int d = j0 + q - src;
                            if (rhs) v[m] = w[src];
                            else if (d >= -bw && d <= 2 * bw) v[m] = B[lslot(lrw, bw, src, j0 + q)];
                        }
                    }
#pragma unroll
                    for (int m = 0; m < 4; ++m) {
                        const int t = t0 + m * nt;
                        if (t < pr * ct) {
                            const int rr = t / ct;
                            S[rr * kSs + (t - rr * ct)] = v[m];
                        }
                    }
                }
                __syncthreads();
                // U12 = L11^-1 (P A12): one warp per column, lane = panel row
                for (int q = wid; q < ct; q += nwarps) {
                    double v = lane < kb ? S[lane * kSs + q] : 0.0;
                    for (int sc = 0; sc + 1 < kb; ++sc) {
                        const double u = __shfl_sync(0xffffffffu, v, sc);
                        if (lane > sc && lane < kb) v = fma(-L11[lane * kPs + sc], u, v);
                    }
                    if (lane < kb) S[lane * kSs + q] = v;
                }
                __syncthreads();
                // A22 -= L21 U12 entry by entry, column order; one thread per row
                double v[kColTile];
                if (own && r >= kb) {
#pragma unroll
                    for (int q = 0; q < kColTile; ++q) v[q] = S[r * kSs + q];
#pragma unroll
                    for (int sc = 0; sc < PANEL; ++sc) {
                        if (sc < kb) {
                            const double f = lrow[sc];
#pragma unroll
                            for (int q2 = 0; q2 < kColTile / 2; ++q2) {
                                const double2 u = reinterpret_cast<const double2*>(S + sc * kSs)[q2];
                                v[2 * q2] = fma(-f, u.x, v[2 * q2]);
                                v[2 * q2 + 1] = fma(-f, u.y, v[2 * q2 + 1]);
                            }
                        }
                    }
                }
                __syncthreads();
                if (own && r >= kb) {
#pragma unroll
                    for (int q = 0; q < kColTile; ++q) S[r * kSs + q] = v[q];
                }
                __syncthreads();
                for (int t = tid; t < pr * ct; t += nt) {
                    const int rr = t / ct, q = t - rr * ct;
                    const int i = k0 + rr;
                    if (rhs) {
                        w[i] = S[rr * kSs];
                    } else {
                        const int d = j0 + q - i;
                        if (d >= -bw && d <= 2 * bw) B[lslot(lrw, bw, i, j0 + q)] = S[rr * kSs + q];
                    }
                }
            }
            if (!grid_barrier(gb, gen)) return;
        }
        if (blockIdx.x == 0 && tid == 0 && pivoted && result == LSTAT_OK && A.fallbacks) A.fallbacks[inst] += 1;
    }
}

// ---- substitution, update and test ---------------------------------------------------------

// Dynamic shared memory of large_solve_kernel: x (n) and one 32 x 33 diagonal block of U.
__host__ __device__ inline size_t large_solve_smem(int n) {
    return sizeof(double) * ((size_t)n + 32 * 33);
}

// One CTA per large instance (32 warps): U x = L^-1 P b (left in wbuf by the factorisation) in
// blocks of 32 rows from the end.  Warp r of a block forms row r's sum over the columns below
// the block (the row's U entries are contiguous in the band), then warp 0 solves the block's
// triangle with shuffles.  x stays in shared memory.
__global__ void __launch_bounds__(kSolveThreads) large_solve_kernel(
    const DevInst* __restrict__ insts, InstArrays A, const int* __restrict__ large_list, int n_large,
    int mode, double* __restrict__ wbuf, const GridBarrier* __restrict__ gb) {
    extern __shared__ __align__(16) double smem_ls[];
    __shared__ double red[32];
    __shared__ int red_r[32];
    __shared__ double tb[32];
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
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, wid = tid >> 5;
    const int n = I.n, bw = I.bw, lrw = I.lrw, f0 = I.f_off;
    const int ub = 2 * bw;  // reach of U
    int* hrow = (mode == INST_MODE_NEWTON && A.hist_iters && A.ctl)
                    ? A.hist_iters + (size_t)A.ctl->step * A.n_inst : nullptr;
    if (st == LSTAT_CONVERGED) {
        if (tid == 0) {
            A.active[inst] = 0;
            atomicSub(A.nactive, 1);
            if (hrow) hrow[inst] = A.iters[inst] + (A.iters_prev ? A.iters_prev[inst] : 0);
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
    double* w = wbuf + f0;  // L^-1 P b, then x
    double* xs = smem_ls;         // n
    double* Ud = smem_ls + n;     // 32 x 33
    const int nwarps = nt >> 5;
    for (int r1 = n; r1 > 0; r1 -= 32) {
        const int r0 = max(0, r1 - 32), rb = r1 - r0;
        for (int r = wid; r < rb; r += nwarps) {
            const int i = r0 + r;
            const double* urow = B + (long long)i * lrw + bw;  // U(i, i + o), o = 0 .. 2 bw
            double acc = 0.0;
            const int jmax = min(n - 1, i + ub);
#pragma unroll 8
            for (int j = r1 + lane; j <= jmax; j += 32) acc = fma(urow[j - i], xs[j], acc);
            acc = warp_sum(acc);
            const int o = r0 + lane - i;
            if (lane < rb) Ud[r * 33 + lane] = (o >= 0 && o <= ub) ? urow[o] : 0.0;
            if (lane == 0) tb[r] = w[i] - acc;
        }
        __syncthreads();
        if (wid == 0) {
            double v = lane < rb ? tb[lane] : 0.0;
            // the block's reciprocal pivots at once, off the sequential chain
            const double rdiag = lane < rb ? 1.0 / Ud[lane * 33 + lane] : 0.0;
            for (int s = rb - 1; s >= 0; --s) {
                if (lane == s) v = v * rdiag;
                const double x = __shfl_sync(0xffffffffu, v, s);
                if (lane < s) v = fma(-Ud[lane * 33 + s], x, v);
            }
            if (lane < rb) xs[r0 + lane] = v;
        }
        __syncthreads();
    }
    for (int i = tid; i < n; i += nt) w[i] = xs[i];
    __syncthreads();
    if (mode == INST_MODE_SOLVE_EXPORTED) {
        for (int i = tid; i < n; i += nt) A.du[f0 + i] = w[i];
        return;
    }
    InstArrays Ar = A;
    newton_tail(I, Ar, inst, w, A.R + f0, hrow, red, red_r);
}

}  // namespace strut

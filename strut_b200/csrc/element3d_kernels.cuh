// Element state determination of forceBeamColumn3d / dispBeamColumn3d (12 dofs) on sm_100a.
//
// Same machinery as the 2D elements (one CTA per element, the element's committed fiber history
// staged into shared memory by cp.async.bulk, fiber phase then fixed-order section sums, warp 0
// running the element algebra with one lane per integration point); the section has a second
// bending axis, so a fiber's strain is eps0 + z kappa_y - y kappa_z and a section carries nine
// resultant / tangent terms, and the force-based element iterates on five basic forces with a
// 5x5 flexibility.
//
// Algorithm (paths relative to the Strut project root):
//   src/mojo/sections/fiber3d.mojo:191-256 (elastic family, uniform-modulus k12 = k13 = 0),
//   769-836 (nonlinear fibers);
//   src/mojo/elements/force_beam_column3d.mojo:679-728 (3x3 inverse), 788-834 (5x5
//   Gauss-Jordan), 1093-1118 (section flexibility), 1176-1201 (section basic deformation),
//   1203-1607 (_force_beam_column3d_try_increment; the flexibility at zero section deformation
//   of 1305-1322 depends on the committed state only and is evaluated once per launch),
//   1610-1622 (basic state), 2549-2990 (entry: subdivisions x schemes, abort when the element
//   does not converge, basic -> local -> global);
//   src/mojo/elements/beam_column3d_nonlinear.mojo:154-172, 357-575 (dispBeamColumn3d);
//   src/mojo/elements/utils.mojo:59-140 (local axes from vecxz).
#pragma once

namespace strut {

// element-level scratch of a 3D element (shares its shared memory with the 2D scratch)
struct ElemScratch3 {
    double q[5], acc_q[5], acc_v[5], v[5], rem[5], att[5], tv[5];
    double vs[kMaxIp][3];      // section deformations of the element state
    double svs[kMaxIp][3];     // accepted section deformations
    double pt[kMaxIp][3];      // points to evaluate
    double raw[kMaxIp][11];    // section sums of the last evaluation
    double scr[kMaxIp][32];    // per-point terms of the element algebra (warp 0)
    double init_f[kMaxIp][6];  // flexibility at zero section deformation
    double c_s[kMaxIp][3];     // cached N, My, Mz at vs
    double c_f[kMaxIp][6];     // cached flexibility at vs
    double resp[kMaxIp][9];    // dispBeamColumn3d section responses
    double kb[25];
    double ul[12], R[9];
    double k[144], wk[144];
    double f[12], fl[12];
    double torsion;
    int init_ok, c_valid, flag, loop_ctrl, local_iters, section_evals;
};

// Sums, over lanes 0..nip-1 of warp 0 in lane order, the NV values each lane put in
// scr[lane][0..NV-1]; every lane gets the same sums.  Warp 0 only.
template <int NV>
__device__ __forceinline__ void lane_ordered_sums_n(double (*scr)[32], int nip, double* out) {
    __syncwarp();
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v] = 0.0;
    for (int ip = 0; ip < nip; ++ip) {
#pragma unroll
        for (int v = 0; v < NV; ++v) out[v] += scr[ip][v];
    }
    __syncwarp();
}

// ---- sections --------------------------------------------------------------------------

// Phase 1 of a 3D evaluation: sig * A and tan * A of every fiber of every point at S.pt.
__device__ __forceinline__ void fiber_phase3(const Geo& g, const DevSection& sd,
                                             const StageView& sv, const DevElem& E,
                                             const double (*pt)[3], double* fo) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int nip = E.nip;
    const int n_tot = sd.n_s2 + sd.n_c2 + sd.n_s1 + sd.n_c1 + sd.n_el;
    const int n_s = nip * sd.n_s2;
    const int ws = steel_warps(n_s, nw);
    if (w < ws) {
        for (int i = w * 32 + lane; i < n_s; i += ws * 32) {
            const int ip = i / sd.n_s2, j = i - ip * sd.n_s2;
            S2State c;
            load_s2(sv, i, c);
            const int gi = sd.geo_off + j;
            const double y = __ldg(g.y + gi), z = __ldg(g.z + gi), A = __ldg(g.a + gi);
            const DevMat& mat = g.mats[__ldg(g.m + gi)];
            const double eps = steel02_strain(mat, pt[ip][0] + z * pt[ip][1] - y * pt[ip][2]);
            const double deps = eps - c.eps;
            double sig, tan;
            if (steel02_no_change(c, deps)) {
                tan = mat.p[1];
                sig = mat.p[10];
            } else {
                const int B = sv.s2_blk, k = steel02_up(c, deps) ? 0 : 6;
                S2Curve cv;
                cv.epsr = sv.s2d[(k + 0) * B + i];
                cv.sigr = sv.s2d[(k + 1) * B + i];
                cv.denom = sv.s2d[(k + 2) * B + i];
                cv.dsig = sv.s2d[(k + 3) * B + i];
                cv.R = sv.s2d[(k + 4) * B + i];
                cv.invR = sv.s2d[(k + 5) * B + i];
                steel02_curve_eval(mat, cv, eps, sig, tan);
            }
            double* o = fo + 2 * (ip * n_tot + j);
            o[0] = sig * A;
            o[1] = tan * A;
        }
        return;
    }
    const int n_o_sec = sd.n_c2 + sd.n_s1 + sd.n_c1 + sd.n_el;
    const int n_o = nip * n_o_sec;
    const int nwo = nw - ws;
    for (int k = (w - ws) * 32 + lane; k < n_o; k += nwo * 32) {
        const int ip = k / n_o_sec, jj = k - ip * n_o_sec;
        const int gi = sd.n_s2 + jj;
        const double y = __ldg(g.y + sd.geo_off + gi), z = __ldg(g.z + sd.geo_off + gi);
        const double A = __ldg(g.a + sd.geo_off + gi);
        const DevMat& mat = g.mats[__ldg(g.m + sd.geo_off + gi)];
        const double strain = pt[ip][0] + z * pt[ip][1] - y * pt[ip][2];
        double* o = fo + 2 * (ip * n_tot + gi);
        if (jj < sd.n_c2) {
            const int idx = ip * sd.n_c2 + jj;
            C2State c;
            load_c2(sv, idx, c);
            const int B = sv.c2_blk;
            C2Derived d;
            d.sigmm = sv.c2d[0 * B + idx];
            d.er = sv.c2d[1 * B + idx];
            d.ept = sv.c2d[2 * B + idx];
            d.epn = sv.c2d[3 * B + idx];
            d.etn = sv.c2d[4 * B + idx];
            double sig, tan;
            concrete02_sig_tan(mat, c, d, strain, sig, tan);
            o[0] = sig * A;
            o[1] = tan * A;
        } else if (jj < sd.n_c2 + sd.n_s1) {
            const int idx = ip * sd.n_s1 + (jj - sd.n_c2);
            const int B = sv.s1_blk;
            S1State c;
            c.eps = sv.s1[0 * B + idx];
            c.sig = sv.s1[1 * B + idx];
            c.tan = sv.s1[2 * B + idx];
            c.epsp = sv.s1[3 * B + idx];
            c.alpha = sv.s1[4 * B + idx];
            S1State t;
            steel01_trial(mat, c, strain, t);
            o[0] = t.sig * A;
            o[1] = t.tan * A;
        } else if (jj < sd.n_c2 + sd.n_s1 + sd.n_c1) {
            C1State c, t;
            load_c1(sv, ip * sd.n_c1 + (jj - sd.n_c2 - sd.n_s1), c);
            concrete01_trial(mat, c, strain, t);
            o[0] = t.sig * A;
            o[1] = t.tan * A;
        } else {
            const double ks = mat.p[0] * A;
            o[0] = ks * strain;
            o[1] = ks;
        }
    }
}

// Phase 2 of a 3D evaluation: eight contiguous chunks per point, each summed by one thread, the
// chunk sums combined by a fixed pairwise tree.  raw[ip] = N, My, Mz, k11, k12, k13 (non-elastic
// fibers), k22, k23, k33, k12, k13 (elastic fibers).
__device__ __forceinline__ void sum_phase3(const DevSection& sd, int nip, const double* ys,
                                           const double* zs, const double* fo,
                                           double (*raw)[11]) {
    const int t = threadIdx.x;
    const int n_sum = nip * 8;
    if ((t & ~31) >= n_sum) return;
    const int n_tot = sd.n_s2 + sd.n_c2 + sd.n_s1 + sd.n_c1 + sd.n_el;
    const int n_nl = n_tot - sd.n_el;
    const bool act = t < n_sum;
    const int ip = t >> 3, b = t & 7;
    double a[11];
#pragma unroll
    for (int c = 0; c < 11; ++c) a[c] = 0.0;
    if (act) {
        const int cs = (n_tot + 7) >> 3;
        const int g0 = b * cs, g1 = min(g0 + cs, n_tot);
        const double* f = fo + 2 * ip * n_tot;
        const int gm = min(g1, n_nl);
        for (int gg = g0; gg < gm; ++gg) {
            const double fs = f[2 * gg], ks = f[2 * gg + 1], y = ys[gg], z = zs[gg];
            a[0] += fs;
            a[1] += fs * z;
            a[2] += -fs * y;
            a[3] += ks;
            a[4] += ks * z;
            a[5] += -ks * y;
            a[6] += ks * z * z;
            a[7] += -ks * z * y;
            a[8] += ks * y * y;
        }
        for (int gg = max(g0, n_nl); gg < g1; ++gg) {
            const double fs = f[2 * gg], ks = f[2 * gg + 1], y = ys[gg], z = zs[gg];
            a[0] += fs;
            a[1] += fs * z;
            a[2] += -fs * y;
            a[3] += ks;
            a[9] += ks * z;
            a[10] += -ks * y;
            a[6] += ks * z * z;
            a[7] += -ks * z * y;
            a[8] += ks * y * y;
        }
    }
#pragma unroll
    for (int c = 0; c < 11; ++c) {
        double p = a[c];
        p += __shfl_down_sync(0xffffffffu, p, 1);
        p += __shfl_down_sync(0xffffffffu, p, 2);
        p += __shfl_down_sync(0xffffffffu, p, 4);
        if (act && b == 0) raw[ip][c] = p;
    }
}

__device__ __forceinline__ void eval_sections3(const Geo& g, const DevSection& sd,
                                               const StageView& sv, const DevElem& E,
                                               ElemScratch3& S, const double* ys,
                                               const double* zs, double* fo) {
    fiber_phase3(g, sd, sv, E, S.pt, fo);
    __syncthreads();
    sum_phase3(sd, E.nip, ys, zs, fo, S.raw);
    if (threadIdx.x == 0) S.section_evals += E.nip;
    __syncthreads();
}

// Resultants and tangent of a point from its raw sums; a section whose elastic fibers share one
// modulus reports no elastic k12 / k13 (fiber3d.mojo:243-253).
__device__ __forceinline__ void raw_resp3(const DevSection& sd, const double* raw, double* r) {
    r[0] = raw[0];
    r[1] = raw[1];
    r[2] = raw[2];
    r[3] = raw[3];
    r[4] = raw[4] + (sd.el_uniform ? 0.0 : raw[9]);
    r[5] = raw[5] + (sd.el_uniform ? 0.0 : raw[10]);
    r[6] = raw[6];
    r[7] = raw[7];
    r[8] = raw[8];
}

// _fiber_section3d_response_flexibility: f = {f11, f12, f13, f22, f23, f33} of the inverse of
// the symmetric tangent r[3..8]; false when |det| <= 1e-40.
__device__ __forceinline__ bool sec_flex3(const double* r, double* f) {
    const double F[9] = {r[3], r[4], r[5], r[4], r[6], r[7], r[5], r[7], r[8]};
    double k[9];
    if (!invert3(F, k)) return false;
    f[0] = k[0];
    f[1] = k[1];
    f[2] = k[2];
    f[3] = k[4];
    f[4] = k[5];
    f[5] = k[8];
    return true;
}

// ---- small dense algebra ------------------------------------------------------------------

// _invert_5x5_flat_into: Gauss-Jordan with partial pivoting on a (destroyed); false when a
// pivot column's largest magnitude is <= 1e-40.
__device__ __forceinline__ bool invert5(double* a, double* inv) {
#pragma unroll
    for (int i = 0; i < 25; ++i) inv[i] = 0.0;
#pragma unroll
    for (int i = 0; i < 5; ++i) inv[i * 5 + i] = 1.0;
    for (int i = 0; i < 5; ++i) {
        int pivot = i;
        double max_val = fabs(a[i * 5 + i]);
        for (int r = i + 1; r < 5; ++r) {
            const double v = fabs(a[r * 5 + i]);
            if (v > max_val) {
                max_val = v;
                pivot = r;
            }
        }
        if (max_val <= 1.0e-40) return false;
        if (pivot != i) {
            for (int c = 0; c < 5; ++c) {
                double t = a[i * 5 + c];
                a[i * 5 + c] = a[pivot * 5 + c];
                a[pivot * 5 + c] = t;
                t = inv[i * 5 + c];
                inv[i * 5 + c] = inv[pivot * 5 + c];
                inv[pivot * 5 + c] = t;
            }
        }
        const double piv = a[i * 5 + i];
        for (int c = 0; c < 5; ++c) {
            a[i * 5 + c] /= piv;
            inv[i * 5 + c] /= piv;
        }
        for (int r = 0; r < 5; ++r) {
            if (r == i) continue;
            const double factor = a[r * 5 + i];
            if (factor == 0.0) continue;
            for (int c = 0; c < 5; ++c) {
                a[r * 5 + c] -= factor * a[i * 5 + c];
                inv[r * 5 + c] -= factor * inv[i * 5 + c];
            }
        }
    }
    return true;
}

// Local axes (rows x, y, z) from the end coordinates and vecxz (utils.mojo:59-140): default
// vecxz is global x, or y, or z when the member is within |cos| >= 0.9 of the previous one.
__device__ __forceinline__ bool rotation3d(const double* x1, const double* x2, int has_vecxz,
                                           const double* vxz, double* R) {
    const double dx = x2[0] - x1[0], dy = x2[1] - x1[1], dz = x2[2] - x1[2];
    const double n = sqrt(dx * dx + dy * dy + dz * dz);
    if (n == 0.0) return false;
    const double lx = dx / n, ly = dy / n, lz = dz / n;
    double vx = 1.0, vy = 0.0, vz = 0.0;
    if (has_vecxz) {
        vx = vxz[0];
        vy = vxz[1];
        vz = vxz[2];
    } else if (fabs(lx) >= 0.9) {
        vx = 0.0;
        vy = 1.0;
        if (fabs(ly) >= 0.9) {
            vy = 0.0;
            vz = 1.0;
        }
    }
    double yx = vy * lz - vz * ly, yy = vz * lx - vx * lz, yz = vx * ly - vy * lx;
    const double yn = sqrt(yx * yx + yy * yy + yz * yz);
    if (yn == 0.0) return false;
    yx /= yn;
    yy /= yn;
    yz /= yn;
    R[0] = lx;
    R[1] = ly;
    R[2] = lz;
    R[3] = yx;
    R[4] = yy;
    R[5] = yz;
    R[6] = ly * yz - lz * yy;
    R[7] = lz * yx - lx * yz;
    R[8] = lx * yy - ly * yx;
    return true;
}

// Basic-force coefficients of the local dofs (_beam3d_local_basic_coeff,
// force_beam_column3d.mojo:419-464): q_row = sum_col c(row, col) u_col.
__device__ __forceinline__ double basic_coeff3(int row, int col, double inv_L) {
    switch (row) {
        case 0: return col == 0 ? -1.0 : (col == 6 ? 1.0 : 0.0);
        case 1: return col == 1 ? inv_L : (col == 5 ? 1.0 : (col == 7 ? -inv_L : 0.0));
        case 2: return col == 1 ? inv_L : (col == 7 ? -inv_L : (col == 11 ? 1.0 : 0.0));
        case 3: return col == 2 ? -inv_L : (col == 4 ? 1.0 : (col == 8 ? inv_L : 0.0));
        case 4: return col == 2 ? -inv_L : (col == 8 ? inv_L : (col == 10 ? 1.0 : 0.0));
        default: return col == 3 ? -1.0 : (col == 9 ? 1.0 : 0.0);
    }
}

// Which section resultant a basic force loads (0 N, 1 My, 2 Mz) and its interpolation
// factor: q0 -> N; q1, q2 -> Mz at b_mi, b_mj; q3, q4 -> My at b_mi, b_mj.
__device__ __forceinline__ int basic_comp3(int a) { return a == 0 ? 0 : (a <= 2 ? 2 : 1); }
__device__ __forceinline__ double basic_fac3(int a, double bmi, double bmj) {
    return a == 0 ? 1.0 : ((a == 1 || a == 3) ? bmi : bmj);
}
// flexibility entry of components (ca, cb) from f = {f11, f12, f13, f22, f23, f33}
__device__ __forceinline__ double flex_of(const double* f, int ca, int cb) {
    const int lo = ca < cb ? ca : cb, hi = ca < cb ? cb : ca;
    return lo == 0 ? f[hi] : (lo == 1 ? f[2 + hi] : f[5]);
}

// kg = T^T kl T, f_g = T^T f_l with T = diag(R, R, R, R): 144 threads of the CTA.
__device__ __forceinline__ void to_global3(ElemScratch3& S) {
    const int t = threadIdx.x;
    if (t < 144) {
        const int a = t / 12, b = t % 12, cb = 3 * (b / 3), j = b % 3;
        S.wk[t] = S.k[a * 12 + cb] * S.R[j] + S.k[a * 12 + cb + 1] * S.R[3 + j] +
                  S.k[a * 12 + cb + 2] * S.R[6 + j];
    }
    __syncthreads();
    if (t < 144) {
        const int a = t / 12, b = t % 12, ra = 3 * (a / 3), i = a % 3;
        S.k[t] = S.R[i] * S.wk[ra * 12 + b] + S.R[3 + i] * S.wk[(ra + 1) * 12 + b] +
                 S.R[6 + i] * S.wk[(ra + 2) * 12 + b];
    } else if (t < 156) {
        const int a = t - 144, ra = 3 * (a / 3), i = a % 3;
        S.f[a] = S.R[i] * S.fl[ra] + S.R[3 + i] * S.fl[ra + 1] + S.R[6 + i] * S.fl[ra + 2];
    }
    __syncthreads();
}

// Element displacements to local axes; R from the undeformed ends, or from the displaced ends
// for Corotational.  Thread 0.
__device__ __forceinline__ bool local_disp3(const DevElem& E, const double* u_full,
                                            ElemScratch3& S) {
    double ug[12];
    for (int a = 0; a < 12; ++a) ug[a] = u_full[E.dof[a]];
    bool ok = true;
    if (E.geom == 2) {
        const double a1[3] = {E.X1[0] + ug[0], E.X1[1] + ug[1], E.X1[2] + ug[2]};
        const double a2[3] = {E.X2[0] + ug[6], E.X2[1] + ug[7], E.X2[2] + ug[8]};
        ok = rotation3d(a1, a2, E.has_vecxz, E.vxz, S.R);
    } else {
        for (int i = 0; i < 9; ++i) S.R[i] = E.R[i];
    }
    for (int b = 0; b < 4; ++b)
        for (int i = 0; i < 3; ++i)
            S.ul[3 * b + i] = S.R[3 * i] * ug[3 * b] + S.R[3 * i + 1] * ug[3 * b + 1] +
                              S.R[3 * i + 2] * ug[3 * b + 2];
    return ok;
}

__device__ __forceinline__ double max_abs5(const double* r) {
    double m = fabs(r[0]);
    for (int i = 1; i < 5; ++i)
        if (fabs(r[i]) > m) m = fabs(r[i]);
    return m;
}

// ---- forceBeamColumn3d ------------------------------------------------------------------

// _force_beam_column3d_try_increment, executed collectively (warp 0: one lane per point).
// Start: S.q, S.vs; on success S.q / S.vs hold the converged state, S.kb the basic stiffness of
// the last flexibility, and the section-response cache describes S.vs.
__device__ bool fbc3_try_increment(const Geo& g, const DevSection& sd, const StageView& sv,
                                   const DevElem& E, ElemScratch3& S, const double* base,
                                   const double* dv, int scheme, const double* ys,
                                   const double* zs, double* fo) {
    const int tid = threadIdx.x, lane = tid & 31;
    const bool w0 = tid < 32;
    const int nip = E.nip;
    const bool act = w0 && lane < nip;
    if (!S.init_ok) return false;
    const double xi = act ? E.xi[lane] : 0.0, wL = act ? E.w[lane] * E.L : 0.0;
    const double bmi = xi - 1.0, bmj = xi;
    double sub[3] = {0.0, 0.0, 0.0}, ssr[3] = {0.0, 0.0, 0.0};
    double fl[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    double p[3] = {0.0, 0.0, 0.0};
    double q[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const int num_iters = scheme == 1 ? 100 : 10;
    const bool cached = S.c_valid != 0;
    if (w0) {
        for (int i = 0; i < 5; ++i) q[i] = S.q[i];
        if (act) {
            for (int c = 0; c < 3; ++c) sub[c] = S.vs[lane][c];
            if (!cached)
                for (int c = 0; c < 3; ++c) S.pt[lane][c] = sub[c];
        }
    }
    if (!cached) {
        __syncthreads();
        eval_sections3(g, sd, sv, E, S, ys, zs, fo);
    }
    // section targets of the current q (section_load terms are zero and still added)
    auto targets = [&](double* s) {
        s[0] = q[0] + 0.0;
        s[1] = bmi * q[3] + bmj * q[4] + 0.0;
        s[2] = bmi * q[1] + bmj * q[2] + 0.0;
    };
    auto next_points = [&](bool use_init) {
        double s[3];
        targets(s);
        const double d0 = s[0] - ssr[0], d1 = s[1] - ssr[1], d2 = s[2] - ssr[2];
        const double* a = use_init ? S.init_f[act ? lane : 0] : fl;
        p[0] = sub[0] + (a[0] * d0 + a[1] * d1 + a[2] * d2);
        p[1] = sub[1] + (a[1] * d0 + a[3] * d1 + a[4] * d2);
        p[2] = sub[2] + (a[2] * d0 + a[4] * d1 + a[5] * d2);
        if (act)
            for (int c = 0; c < 3; ++c) S.pt[lane][c] = p[c];
    };
    // flexibility integration terms of one point: F[a][b] = wL Ba f(ca, cb) Bb
    auto flex_terms5 = [&](double* o, const double* f) {
        for (int a = 0; a < 5; ++a) {
            const int ca = basic_comp3(a);
            const double ba = basic_fac3(a, bmi, bmj);
            for (int b = 0; b < 5; ++b)
                o[a * 5 + b] = wL * (ba * (flex_of(f, ca, basic_comp3(b)) * basic_fac3(b, bmi, bmj)));
        }
    };
    if (w0) {
        int ok = 1;
        if (cached) {
            if (act)
                for (int c = 0; c < 3; ++c) ssr[c] = S.c_s[lane][c];
            if (act)
                for (int c = 0; c < 6; ++c) fl[c] = S.c_f[lane][c];
        } else {
            bool good = true;
            if (act) {
                double r[9];
                raw_resp3(sd, S.raw[lane], r);
                ssr[0] = r[0];
                ssr[1] = r[1];
                ssr[2] = r[2];
                good = sec_flex3(r, fl);
            }
            ok = __all_sync(0xffffffffu, good) ? 1 : 0;
        }
        if (ok) {
            if (act) flex_terms5(S.scr[lane], fl);
            double P[25], kb[25];
            lane_ordered_sums_n<25>(S.scr, nip, P);
            if (invert5(P, kb)) {
                double dq[5];
                for (int i = 0; i < 5; ++i)
                    dq[i] = kb[i * 5] * dv[0] + kb[i * 5 + 1] * dv[1] + kb[i * 5 + 2] * dv[2] +
                            kb[i * 5 + 3] * dv[3] + kb[i * 5 + 4] * dv[4];
                for (int i = 0; i < 5; ++i) q[i] += dq[i];
            }
            next_points(scheme == 1 || scheme == 2);
        }
        if (lane == 0) S.flag = ok;
    }
    __syncthreads();
    if (!S.flag) return false;
    double tgt[5];
    for (int i = 0; i < 5; ++i) tgt[i] = base[i] + dv[i];
    for (int it = 0; it < num_iters; ++it) {
        eval_sections3(g, sd, sv, E, S, ys, zs, fo);
        if (w0) {
            bool good = true;
            double r[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            double nf[6] = {0, 0, 0, 0, 0, 0};
            if (act) {
                raw_resp3(sd, S.raw[lane], r);
                good = sec_flex3(r, nf);
            }
            int res = 0;
            if (__all_sync(0xffffffffu, good)) {
                double s[3];
                targets(s);
                for (int c = 0; c < 3; ++c) {
                    sub[c] = p[c];
                    ssr[c] = r[c];
                }
                for (int c = 0; c < 6; ++c) fl[c] = nf[c];
                const double d0 = s[0] - ssr[0], d1 = s[1] - ssr[1], d2 = s[2] - ssr[2];
                const double e0 = fl[0] * d0 + fl[1] * d1 + fl[2] * d2;
                const double e1 = fl[1] * d0 + fl[3] * d1 + fl[4] * d2;
                const double e2 = fl[2] * d0 + fl[4] * d1 + fl[5] * d2;
                if (act) {
                    flex_terms5(S.scr[lane], fl);
                    S.scr[lane][25] = wL * (p[0] + e0);
                    S.scr[lane][26] = wL * bmi * (p[2] + e2);
                    S.scr[lane][27] = wL * bmj * (p[2] + e2);
                    S.scr[lane][28] = wL * bmi * (p[1] + e1);
                    S.scr[lane][29] = wL * bmj * (p[1] + e1);
                }
                double F[30], kb[25];
                lane_ordered_sums_n<30>(S.scr, nip, F);
                if (invert5(F, kb)) {
                    double rr[5], dq[5];
                    for (int i = 0; i < 5; ++i) rr[i] = tgt[i] - F[25 + i];
                    for (int i = 0; i < 5; ++i)
                        dq[i] = kb[i * 5] * rr[0] + kb[i * 5 + 1] * rr[1] + kb[i * 5 + 2] * rr[2] +
                                kb[i * 5 + 3] * rr[3] + kb[i * 5 + 4] * rr[4];
                    const double work = fabs(rr[0] * dq[0] + rr[1] * dq[1] + rr[2] * dq[2] +
                                             rr[3] * dq[3] + rr[4] * dq[4]);
                    for (int i = 0; i < 5; ++i) q[i] += dq[i];
                    res = 1;
                    if (work < 1.0e-12) {
                        res = 2;
                        if (act) {
                            for (int c = 0; c < 3; ++c) {
                                S.vs[lane][c] = sub[c];
                                S.c_s[lane][c] = ssr[c];
                            }
                            for (int c = 0; c < 6; ++c) S.c_f[lane][c] = fl[c];
                        }
                        if (lane == 0) {
                            S.c_valid = 1;
                            for (int i = 0; i < 25; ++i) S.kb[i] = kb[i];
                        }
                    } else if (it + 1 < num_iters) {
                        next_points(scheme == 1);
                    }
                }
            }
            if (lane == 0) {
                S.local_iters++;
                S.flag = res;
                if (res)
                    for (int i = 0; i < 5; ++i) S.q[i] = q[i];
            }
        }
        __syncthreads();
        const int f = S.flag;
        if (f == 0) return false;
        if (f == 2) return true;
    }
    return false;
}

// ---- one 3D element -------------------------------------------------------------------------

// State determination of a 12-dof element, collectively by the CTA; E and sd are in shared
// memory.  Writes k (12x12 global) and f (12) at the element's offsets and its element state;
// returns false (status set) when the element fails.  rec_out (record pass) receives f.
__device__ void element3d_process(const Geo& g, const DevSection& sd, const DevElem& E, int e,
                                  FiberState& fs, const double* u_full, double* estate,
                                  double* ek, double* ef, int* status, int* elem_err,
                                  unsigned long long* counters, ElemScratch3& S, double* smem_fib,
                                  uint64_t* bar, uint32_t& phase, bool& stop, double* rec_out) {
    const int tid = threadIdx.x;
    const int nip = E.nip;
    double* es = estate + (size_t)e * kEStride;
    if (tid == 0) {
        S.local_iters = 0;
        S.section_evals = 0;
        S.flag = local_disp3(E, u_full, S) ? 1 : 0;
        for (int i = 0; i < 5; ++i) S.q[i] = es[kE3q + i];
        for (int ip = 0; ip < nip; ++ip) {
            S.vs[ip][0] = es[kE3e + ip];
            S.vs[ip][1] = es[kE3y + ip];
            S.vs[ip][2] = es[kE3z + ip];
            for (int c = 0; c < 3; ++c) S.c_s[ip][c] = es[kE3cs + 3 * ip + c];
            for (int c = 0; c < 6; ++c) S.c_f[ip][c] = es[kE3cf + 6 * ip + c];
        }
        S.c_valid = E.type == STRUT_ELEM_FORCE_BEAM_COLUMN_3D && es[kE3cv] != 0.0;
    }
    StageView sv;
    int err = ELEM_ERR_NONE;
    const bool staged = stage_element(E, fs, smem_fib, bar, phase, sv, &err);
    __syncthreads();
    if (!staged) {
        if (tid == 0) {
            elem_err[e] = err;
            status[E.inst] = STRUT_CUDA_ERROR;
        }
        stop = true;
        return;
    }
    if (!S.flag) {
        // degenerate Corotational axes: Strut aborts
        if (tid == 0) {
            elem_err[e] = ELEM_ERR_FAILED;
            status[E.inst] = STRUT_ELEMENT_FAILED;
        }
        return;
    }
    derive_element(g, sd, E, sv, fs.c2 + 4 * fs.c2_n + E.c2_off, const_cast<double*>(sv.c2d),
                   const_cast<double*>(sv.s2d));
    const int n_tot = sd.n_s2 + sd.n_c2 + sd.n_s1 + sd.n_c1 + sd.n_el;
    double* ys = const_cast<double*>(sv.s2d) + 12 * E.s2_blk;
    double* zs = ys + ((n_tot + 1) & ~1);
    double* fo = zs + ((n_tot + 1) & ~1);
    for (int gg = tid; gg < n_tot; gg += blockDim.x) {
        ys[gg] = __ldg(g.y + sd.geo_off + gg);
        zs[gg] = __ldg(g.z + sd.geo_off + gg);
    }
    __syncthreads();
    const double L = E.L, inv_L = E.inv_L;
    const bool has_torsion = E.G > 0.0 && E.J > 0.0;
    const bool pdelta = E.geom == 1 || E.geom == 2;
    if (E.type == STRUT_ELEM_DISP_BEAM_COLUMN_3D) {
        // ---------------- dispBeamColumn3d ----------------
        if (tid < nip) {
            const double xi = E.xi[tid];
            const double il = 1.0 / L;
            const double* ul = S.ul;
            const double e0 = (-il) * ul[0] + il * ul[6];
            const double ky = ((-6.0 + 12.0 * xi) / (L * L)) * ul[2] + ((4.0 - 6.0 * xi) / L) * ul[4] +
                              ((6.0 - 12.0 * xi) / (L * L)) * ul[8] + ((2.0 - 6.0 * xi) / L) * ul[10];
            const double kz = ((-6.0 + 12.0 * xi) / (L * L)) * ul[1] + ((-4.0 + 6.0 * xi) / L) * ul[5] +
                              ((6.0 - 12.0 * xi) / (L * L)) * ul[7] + ((-2.0 + 6.0 * xi) / L) * ul[11];
            S.pt[tid][0] = S.vs[tid][0] = e0;
            S.pt[tid][1] = S.vs[tid][1] = ky;
            S.pt[tid][2] = S.vs[tid][2] = kz;
        }
        __syncthreads();
        eval_sections3(g, sd, sv, E, S, ys, zs, fo);
        if (tid < nip) raw_resp3(sd, S.raw[tid], S.resp[tid]);
        __syncthreads();
        // B rows (N, My, Mz) of local dof a at xi (beam_column3d_nonlinear.mojo:449-488)
        auto bvec = [&](int a, double xi, double* b) {
            b[0] = a == 0 ? -1.0 / L : (a == 6 ? 1.0 / L : 0.0);
            b[1] = a == 2 ? (-6.0 + 12.0 * xi) / (L * L)
                 : a == 4 ? (4.0 - 6.0 * xi) / L
                 : a == 8 ? (6.0 - 12.0 * xi) / (L * L)
                 : a == 10 ? (2.0 - 6.0 * xi) / L : 0.0;
            b[2] = a == 1 ? (-6.0 + 12.0 * xi) / (L * L)
                 : a == 5 ? (-4.0 + 6.0 * xi) / L
                 : a == 7 ? (6.0 - 12.0 * xi) / (L * L)
                 : a == 11 ? (-2.0 + 6.0 * xi) / L : 0.0;
        };
        if (tid < 144) {
            const int a = tid / 12, b = tid % 12;
            double kab = 0.0;
            for (int ip = 0; ip < nip; ++ip) {
                const double xi = E.xi[ip], wL = E.w[ip] * L;
                const double* r = S.resp[ip];
                double ba[3], bb[3];
                bvec(a, xi, ba);
                bvec(b, xi, bb);
                const double dN = r[3] * bb[0] + r[4] * bb[1] + r[5] * bb[2];
                const double dMy = r[4] * bb[0] + r[6] * bb[1] + r[7] * bb[2];
                const double dMz = r[5] * bb[0] + r[7] * bb[1] + r[8] * bb[2];
                kab += wL * (ba[0] * dN + ba[1] * dMy + ba[2] * dMz);
            }
            S.k[tid] = kab;
        } else if (tid < 156) {
            const int a = tid - 144;
            double fa = 0.0;
            for (int ip = 0; ip < nip; ++ip) {
                const double xi = E.xi[ip], wL = E.w[ip] * L;
                const double* r = S.resp[ip];
                double ba[3];
                bvec(a, xi, ba);
                fa += wL * (ba[0] * r[0] + ba[1] * r[1] + ba[2] * r[2]);
            }
            S.fl[a] = fa;
        }
        __syncthreads();
        if (tid == 0) {
            if (has_torsion) {
                const double tk = E.G * E.J / L;
                S.k[3 * 12 + 3] += tk;
                S.k[3 * 12 + 9] -= tk;
                S.k[9 * 12 + 3] -= tk;
                S.k[9 * 12 + 9] += tk;
                const double q5 = tk * (S.ul[9] - S.ul[3]);
                S.fl[3] += -1.0 * q5;
                S.fl[9] += 1.0 * q5;
            }
            if (pdelta) {
                double avg = 0.0;
                for (int ip = 0; ip < nip; ++ip) avg += E.w[ip] * S.resp[ip][0];
                const double nl = avg / L;
                S.k[1 * 12 + 1] += nl;
                S.k[1 * 12 + 7] -= nl;
                S.k[7 * 12 + 1] -= nl;
                S.k[7 * 12 + 7] += nl;
                S.k[2 * 12 + 2] += nl;
                S.k[2 * 12 + 8] -= nl;
                S.k[8 * 12 + 2] -= nl;
                S.k[8 * 12 + 8] += nl;
            }
            for (int ip = 0; ip < nip; ++ip) {
                es[kE3e + ip] = S.vs[ip][0];
                es[kE3y + ip] = S.vs[ip][1];
                es[kE3z + ip] = S.vs[ip][2];
            }
            es[kE3cv] = 0.0;
            atomicAdd(&counters[3], (unsigned long long)E.io_bytes);
            atomicAdd(&counters[1], (unsigned long long)nip);
            atomicAdd(&counters[2], (unsigned long long)nip * n_tot);
            atomicAdd(&counters[7], (unsigned long long)nip * section_update_bytes(sd));
        }
        __syncthreads();
        to_global3(S);
        if (tid < 144) ek[E.ek_off + tid] = S.k[tid];
        else if (tid < 156) ef[E.ef_off + tid - 144] = S.f[tid - 144];
        if (rec_out && tid >= 160 && tid < 172) rec_out[tid - 160] = S.f[tid - 160];
        return;
    }
    // ---------------- forceBeamColumn3d ----------------
    // flexibility of every section at zero deformation from the committed state
    if (tid < nip)
        for (int c = 0; c < 3; ++c) S.pt[tid][c] = 0.0;
    __syncthreads();
    eval_sections3(g, sd, sv, E, S, ys, zs, fo);
    if (tid < 32) {
        bool good = true;
        if (tid < nip) {
            double r[9];
            raw_resp3(sd, S.raw[tid], r);
            good = sec_flex3(r, S.init_f[tid]);
        }
        const bool all = __all_sync(0xffffffffu, good);
        if (tid == 0) S.init_ok = all ? 1 : 0;
    }
    if (tid == 0) {
        const double* ul = S.ul;
        const double chord_z = (ul[7] - ul[1]) / L;
        const double chord_y = (ul[8] - ul[2]) / L;
        S.v[0] = ul[6] - ul[0];
        S.v[1] = ul[5] - chord_z;
        S.v[2] = ul[11] - chord_z;
        S.v[3] = ul[4] + chord_y;
        S.v[4] = ul[10] + chord_y;
        S.torsion = ul[9] - ul[3];
        // accepted basic deformation from the section deformations (1176-1201)
        for (int i = 0; i < 5; ++i) S.acc_v[i] = 0.0;
        for (int ip = 0; ip < nip; ++ip) {
            const double xi = E.xi[ip], wL = E.w[ip] * L;
            const double bmi = xi - 1.0, bmj = xi;
            S.acc_v[0] += wL * S.vs[ip][0];
            S.acc_v[1] += wL * bmi * S.vs[ip][2];
            S.acc_v[2] += wL * bmj * S.vs[ip][2];
            S.acc_v[3] += wL * bmi * S.vs[ip][1];
            S.acc_v[4] += wL * bmj * S.vs[ip][1];
        }
        for (int i = 0; i < 5; ++i) {
            S.acc_q[i] = S.q[i];
            S.rem[i] = S.v[i] - S.acc_v[i];
            S.att[i] = S.rem[i];
        }
        for (int ip = 0; ip < nip; ++ip)
            for (int c = 0; c < 3; ++c) S.svs[ip][c] = S.vs[ip][c];
        S.loop_ctrl = 0;
    }
    __syncthreads();
    int converged = 0;
    {
        int num_subdivide = 1;
        int guard = 0;
        while (num_subdivide <= 4 && guard < 10000) {
            ++guard;
            int scheme_success = 0;
            if (tid == 0)
                for (int i = 0; i < 5; ++i) S.tv[i] = S.acc_v[i] + S.att[i];
            __syncthreads();
            for (int scheme = 0; scheme < 3; ++scheme) {
                if (tid == 0) {
                    for (int i = 0; i < 5; ++i) S.q[i] = S.acc_q[i];
                    for (int ip = 0; ip < nip; ++ip)
                        for (int c = 0; c < 3; ++c) S.vs[ip][c] = S.svs[ip][c];
                }
                __syncthreads();
                if (!fbc3_try_increment(g, sd, sv, E, S, S.acc_v, S.att, scheme, ys, zs, fo)) continue;
                if (tid == 0) {
                    for (int i = 0; i < 5; ++i) {
                        S.acc_v[i] = S.tv[i];
                        S.acc_q[i] = S.q[i];
                    }
                    for (int ip = 0; ip < nip; ++ip)
                        for (int c = 0; c < 3; ++c) S.svs[ip][c] = S.vs[ip][c];
                    for (int i = 0; i < 5; ++i) S.rem[i] = S.v[i] - S.acc_v[i];
                    if (max_abs5(S.rem) <= 1.0e-12) {
                        S.loop_ctrl = 1;
                    } else {
                        for (int i = 0; i < 5; ++i) S.att[i] = S.rem[i];
                        S.loop_ctrl = 0;
                    }
                }
                __syncthreads();
                scheme_success = 1;
                if (S.loop_ctrl == 1) converged = 1;
                else num_subdivide = 1;
                break;
            }
            if (converged) break;
            if (scheme_success) continue;
            if (tid == 0)
                for (int i = 0; i < 5; ++i) S.att[i] /= 10.0;
            __syncthreads();
            num_subdivide += 1;
        }
    }
    if (tid == 0) {
        // the accepted state is what Strut keeps (and restores before aborting)
        for (int i = 0; i < 5; ++i) {
            S.q[i] = S.acc_q[i];
            es[kE3q + i] = S.acc_q[i];
        }
        for (int ip = 0; ip < nip; ++ip) {
            es[kE3e + ip] = S.svs[ip][0];
            es[kE3y + ip] = S.svs[ip][1];
            es[kE3z + ip] = S.svs[ip][2];
            for (int c = 0; c < 3; ++c) es[kE3cs + 3 * ip + c] = S.c_s[ip][c];
            for (int c = 0; c < 6; ++c) es[kE3cf + 6 * ip + c] = S.c_f[ip][c];
        }
        es[kE3cv] = S.c_valid ? 1.0 : 0.0;
        S.flag = converged ? 0 : 1;
        atomicAdd(&counters[3], (unsigned long long)E.io_bytes);
        atomicAdd(&counters[0], (unsigned long long)S.local_iters);
        atomicMax(&counters[5], (unsigned long long)S.local_iters);
        atomicAdd(&counters[1], (unsigned long long)S.section_evals);
        atomicAdd(&counters[2], (unsigned long long)S.section_evals * n_tot);
        atomicAdd(&counters[7], (unsigned long long)S.section_evals * section_update_bytes(sd));
    }
    __syncthreads();
    if (S.flag) {
        if (tid == 0) {
            elem_err[e] = ELEM_ERR_FAILED;
            status[E.inst] = STRUT_ELEMENT_FAILED;
        }
        return;
    }
    // basic -> local: k = a^T kb a (+ torsion, + PDelta), f = a^T q
    if (tid < 144) {
        const int a = tid / 12, b = tid % 12;
        double kab = 0.0;
        for (int i = 0; i < 5; ++i) {
            const double ai = basic_coeff3(i, a, inv_L);
            for (int j = 0; j < 5; ++j) kab += ai * S.kb[i * 5 + j] * basic_coeff3(j, b, inv_L);
        }
        if (has_torsion) kab += basic_coeff3(5, a, inv_L) * (E.G * E.J / L) * basic_coeff3(5, b, inv_L);
        S.k[tid] = kab;
    } else if (tid < 156) {
        const int a = tid - 144;
        const double q5b = has_torsion ? (E.G * E.J / L) * S.torsion : 0.0;
        double fa = 0.0;
        for (int i = 0; i < 5; ++i) fa += basic_coeff3(i, a, inv_L) * S.q[i];
        fa += basic_coeff3(5, a, inv_L) * q5b;
        S.fl[a] = fa;
    }
    __syncthreads();
    if (tid == 0 && pdelta) {
        const double ql = S.q[0] / L;
        S.k[1 * 12 + 1] += ql;
        S.k[1 * 12 + 7] -= ql;
        S.k[7 * 12 + 1] -= ql;
        S.k[7 * 12 + 7] += ql;
        S.k[2 * 12 + 2] += ql;
        S.k[2 * 12 + 8] -= ql;
        S.k[8 * 12 + 2] -= ql;
        S.k[8 * 12 + 8] += ql;
    }
    __syncthreads();
    to_global3(S);
    if (tid < 144) ek[E.ek_off + tid] = S.k[tid];
    else if (tid < 156) ef[E.ef_off + tid - 144] = S.f[tid - 144];
    if (rec_out && tid >= 160 && tid < 172) rec_out[tid - 160] = S.f[tid - 160];
}

}  // namespace strut

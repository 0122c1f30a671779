// Section recorders (section_force / section_deformation) after every step.
//
// Strut evaluates them in its recorder loop after the step (transient_nonlinear.mojo:3537-3605):
//   forceBeamColumn2d  from the basic state the step left: q0 and (xi - 1) q1 + xi q2, or the
//                      section deformations eps0, kappa (helpers.mojo:1974-2040);
//   dispBeamColumn2d   eps0, kappa of the displacements at the point (Hermite B, c and s from
//                      dx / L), and the section's N, Mz there (helpers.mojo:2043-2156);
//   forceBeamColumn3d  from the basic state of the recorder's own state determination at the
//                      step's displacements, which the 3D record pass has run for such an
//                      element: q0, (xi - 1) q1 + xi q2, (xi - 1) q3 + xi q4, G J twist, or eps0,
//                      kappa_z, kappa_y, twist (helpers.mojo:2158-2300);
//   dispBeamColumn3d   the section at the displacements' eps0, kappa_y, kappa_z: N, Mz, -My,
//                      G J twist, or eps0, kappa_z, -kappa_y, twist
//                      (beam_column3d_nonlinear.mojo:578-640).
// A section's resultants come from its fibers' trial state at that deformation, a function of the
// committed state only, so evaluating it changes nothing.  One warp per recorded section.
#pragma once

#include "element3d_kernels.cuh"

namespace strut {

// A recorded section: element (global index), point, kind, instance.
struct SecRec {
    int elem, ip, kind, inst;
};

// N, My, Mz of the element's section at point ip from the committed fiber state at
// eps0 + z ky - y kz (2D: z = 0, ky = 0, kz = kappa).  Whole warp; every lane gets the sums.
__device__ __forceinline__ void section_resultants(const Geo& g, const DevSection& sd, const FiberState& fs,
                                                   const DevElem& E, int ip, bool three_d, double eps0,
                                                   double ky, double kz, double& N, double& My, double& Mz) {
    const int lane = threadIdx.x & 31;
    double n = 0.0, my = 0.0, mz = 0.0;
    int base = sd.geo_off;
    auto acc = [&](int gi, double sig_times_a) {
        const double y = __ldg(g.y + gi), z = three_d ? __ldg(g.z + gi) : 0.0;
        n += sig_times_a;
        my += sig_times_a * z;
        mz += -sig_times_a * y;
    };
    auto strain = [&](int gi) {
        const double y = __ldg(g.y + gi), z = three_d ? __ldg(g.z + gi) : 0.0;
        return eps0 + z * ky - y * kz;
    };
    for (int j = lane; j < sd.n_s2; j += 32) {
        const long long x = E.s2_off + (long long)ip * sd.n_s2 + j;
        const double* F = fs.s2 + x;
        const long long S = fs.s2_n;
        S2State c, t;
        c.eps = F[0]; c.sig = F[S]; c.tan = F[2 * S]; c.epsmin = F[3 * S]; c.epsmax = F[4 * S];
        c.epspl = F[5 * S]; c.epss0 = F[6 * S]; c.sigs0 = F[7 * S]; c.epsr = F[8 * S]; c.sigr = F[9 * S];
        c.kon = fs.s2_kon[x];
        steel02_trial(g.mats[__ldg(g.m + base + j)], c, strain(base + j), t);
        acc(base + j, t.sig * __ldg(g.a + base + j));
    }
    base += sd.n_s2;
    for (int j = lane; j < sd.n_c2; j += 32) {
        const double* F = fs.c2 + E.c2_off + (long long)ip * sd.n_c2 + j;
        const long long S = fs.c2_n;
        C2State c, t;
        c.eps = F[0]; c.sig = F[S]; c.tan = F[2 * S]; c.ecmin = F[3 * S]; c.dept = F[4 * S];
        concrete02_trial(g.mats[__ldg(g.m + base + j)], c, strain(base + j), t);
        acc(base + j, t.sig * __ldg(g.a + base + j));
    }
    base += sd.n_c2;
    for (int j = lane; j < sd.n_s1; j += 32) {
        const double* F = fs.s1 + E.s1_off + (long long)ip * sd.n_s1 + j;
        const long long S = fs.s1_n;
        S1State c, t;
        c.eps = F[0]; c.sig = F[S]; c.tan = F[2 * S]; c.epsp = F[3 * S]; c.alpha = F[4 * S];
        steel01_trial(g.mats[__ldg(g.m + base + j)], c, strain(base + j), t);
        acc(base + j, t.sig * __ldg(g.a + base + j));
    }
    base += sd.n_s1;
    for (int j = lane; j < sd.n_c1; j += 32) {
        const double* F = fs.c1 + E.c1_off + (long long)ip * sd.n_c1 + j;
        const long long S = fs.c1_n;
        C1State c, t;
        c.eps = F[0]; c.sig = F[S]; c.tan = F[2 * S]; c.emin = F[3 * S]; c.eend = F[4 * S]; c.slope = F[5 * S];
        concrete01_trial(g.mats[__ldg(g.m + base + j)], c, strain(base + j), t);
        acc(base + j, t.sig * __ldg(g.a + base + j));
    }
    base += sd.n_c1;
    for (int j = lane; j < sd.n_el; j += 32) {
        const double ks = g.mats[__ldg(g.m + base + j)].p[0] * __ldg(g.a + base + j);
        acc(base + j, ks * strain(base + j));
    }
    N = warp_sum(n);
    My = warp_sum(my);
    Mz = warp_sum(mz);
}

// hist: [step][slot][W], W = 2 (2D) or 4 (3D).  n_slots records, one warp each.
__global__ void record_sections_kernel(const DevElem* __restrict__ elems, Geo g, FiberState fs,
                                       const double* __restrict__ u_full, const double* __restrict__ estate,
                                       const SecRec* __restrict__ recs, int n_slots, int W,
                                       double* __restrict__ hist, const DevCtl* __restrict__ ctl) {
    const int slot = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (slot >= n_slots) return;
    const SecRec r = recs[slot];
    const DevElem& E = elems[r.elem];
    const DevSection& sd = g.secs[E.sec];
    const int ip = r.ip;
    const bool defo = r.kind == 1;
    const double xi = E.xi[ip];
    double out[4] = {0.0, 0.0, 0.0, 0.0};
    if (E.type == STRUT_ELEM_FORCE_BEAM_COLUMN_2D) {
        const double* es = estate + (size_t)r.elem * kEStride;
        if (defo) {
            out[0] = es[kEe + ip];
            out[1] = es[kEk + ip];
        } else {
            out[0] = es[kEq] + 0.0;
            out[1] = (xi - 1.0) * es[kEq + 1] + xi * es[kEq + 2] + 0.0;
        }
    } else if (E.type == STRUT_ELEM_DISP_BEAM_COLUMN_2D) {
        double ug[6], ul[6];
        for (int a = 0; a < 6; ++a) ug[a] = u_full[E.dof[a]];
        u_to_local(E.c_div, E.s_div, ug, ul);
        const double L = E.L, inv_L = 1.0 / L;
        const double eps0 = (-inv_L) * ul[0] + inv_L * ul[3];
        const double kappa = ((-6.0 + 12.0 * xi) / (L * L)) * ul[1] + ((-4.0 + 6.0 * xi) / L) * ul[2] +
                             ((6.0 - 12.0 * xi) / (L * L)) * ul[4] + ((-2.0 + 6.0 * xi) / L) * ul[5];
        if (defo) {
            out[0] = eps0;
            out[1] = kappa;
        } else {
            double N, My, Mz;
            section_resultants(g, sd, fs, E, ip, false, eps0, 0.0, kappa, N, My, Mz);
            out[0] = N + 0.0;
            out[1] = Mz + 0.0;
        }
    } else if (E.type == STRUT_ELEM_FORCE_BEAM_COLUMN_3D) {
        const double* es = estate + (size_t)r.elem * kEStride;
        double ug[12];
        for (int a = 0; a < 12; ++a) ug[a] = u_full[E.dof[a]];
        const double dx = E.X2[0] - E.X1[0], dy = E.X2[1] - E.X1[1], dz = E.X2[2] - E.X1[2];
        const double L = sqrt(dx * dx + dy * dy + dz * dz);
        const double rot_i = (dx * ug[3] + dy * ug[4] + dz * ug[5]) / L;
        const double rot_j = (dx * ug[9] + dy * ug[10] + dz * ug[11]) / L;
        const double twist = (rot_j - rot_i) / L;
        if (defo) {
            out[0] = es[kE3e + ip];
            out[1] = es[kE3z + ip];
            out[2] = es[kE3y + ip];
            out[3] = twist;
        } else {
            out[0] = es[kE3q] + 0.0;
            out[1] = (xi - 1.0) * es[kE3q + 1] + xi * es[kE3q + 2] + 0.0;
            out[2] = (xi - 1.0) * es[kE3q + 3] + xi * es[kE3q + 4] + 0.0;
            out[3] = E.G * E.J * twist;
        }
    } else if (E.type == STRUT_ELEM_DISP_BEAM_COLUMN_3D) {
        double ug[12], R[9], ul[12];
        for (int a = 0; a < 12; ++a) ug[a] = u_full[E.dof[a]];
        if (E.geom == 2) {
            const double a1[3] = {E.X1[0] + ug[0], E.X1[1] + ug[1], E.X1[2] + ug[2]};
            const double a2[3] = {E.X2[0] + ug[6], E.X2[1] + ug[7], E.X2[2] + ug[8]};
            rotation3d(a1, a2, E.has_vecxz, E.vxz, R);
        } else {
            for (int i = 0; i < 9; ++i) R[i] = E.R[i];
        }
        for (int b = 0; b < 4; ++b)
            for (int i = 0; i < 3; ++i)
                ul[3 * b + i] = R[3 * i] * ug[3 * b] + R[3 * i + 1] * ug[3 * b + 1] + R[3 * i + 2] * ug[3 * b + 2];
        const double dx = E.X2[0] - E.X1[0], dy = E.X2[1] - E.X1[1], dz = E.X2[2] - E.X1[2];
        const double L = sqrt(dx * dx + dy * dy + dz * dz), inv_L = 1.0 / L;
        const double eps0 = (-inv_L) * ul[0] + inv_L * ul[6];
        const double ky = ((-6.0 + 12.0 * xi) / (L * L)) * ul[2] + ((4.0 - 6.0 * xi) / L) * ul[4] +
                          ((6.0 - 12.0 * xi) / (L * L)) * ul[8] + ((2.0 - 6.0 * xi) / L) * ul[10];
        const double kz = ((-6.0 + 12.0 * xi) / (L * L)) * ul[1] + ((-4.0 + 6.0 * xi) / L) * ul[5] +
                          ((6.0 - 12.0 * xi) / (L * L)) * ul[7] + ((-2.0 + 6.0 * xi) / L) * ul[11];
        const double twist = (ul[9] - ul[3]) / L;
        if (defo) {
            out[0] = eps0;
            out[1] = kz;
            out[2] = -ky;
            out[3] = twist;
        } else {
            double N, My, Mz;
            section_resultants(g, sd, fs, E, ip, true, eps0, ky, kz, N, My, Mz);
            out[0] = N;
            out[1] = Mz;
            out[2] = -My;
            out[3] = E.G * E.J * twist;
        }
    }
    if (lane == 0) {
        double* o = hist + ((size_t)ctl->step * n_slots + slot) * W;
        for (int c = 0; c < W; ++c) o[c] = out[c];
    }
}

}  // namespace strut

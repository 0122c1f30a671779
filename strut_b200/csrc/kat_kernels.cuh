// Known-answer drivers and the batched section kernel.
//
//   material_path_kernel   the scalar uniaxial path of Strut's material_path driver
//                          (src/mojo/material_path.mojo:233-262; ops.mojo:117-174: an unchanged
//                          trial strain returns the previous trial state)
//   section_path_kernel    Strut's section_path driver (src/mojo/section_path.mojo:354-470):
//                          evaluate the FiberSection2d at each (eps0, kappa), then commit
//   section3d_path_kernel  the same driver for a FiberSection3d (section_path.mojo:463-556):
//                          nine resultant / tangent terms per point
//   section_batch_kernel   many section instances, one warp each, reading committed history
//                          and writing trial (commit != 0: written over committed); the
//                          fiber-state throughput kernel
#pragma once

#include "kernels.cuh"

namespace strut {

__global__ void material_path_kernel(DevMat m, const double* __restrict__ strains, int n,
                                     double* __restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (m.type == 4) {
        C2State c{0.0, 0.0, m.k[C2K_EC0], 0.0, 0.0};
        C2State t = c;
        for (int i = 0; i < n; ++i) {
            const double eps = strains[i];
            if (eps != t.eps) concrete02_trial(m, c, eps, t);
            out[2 * i] = t.sig;
            out[2 * i + 1] = t.tan;
            c = t;
        }
    } else if (m.type == 3) {
        S2State c{};
        c.tan = m.p[1];
        c.epsmax = m.k[S2K_EPSY];
        c.epsmin = -m.k[S2K_EPSY];
        if (m.p[10] != 0.0) {
            c.eps = m.k[S2K_SIGINI_E0];
            c.sig = m.p[10];
        }
        S2State t = c;
        for (int i = 0; i < n; ++i) {
            const double eps = strains[i];
            if (eps != t.eps) steel02_trial(m, c, eps, t);
            out[2 * i] = t.sig;
            out[2 * i + 1] = t.tan;
            c = t;
        }
    } else if (m.type == 2) {
        C1State c{0.0, 0.0, m.k[C1K_EC0], 0.0, 0.0, m.k[C1K_EC0]};
        C1State t = c;
        for (int i = 0; i < n; ++i) {
            const double eps = strains[i];
            if (eps != t.eps) concrete01_trial(m, c, eps, t);
            out[2 * i] = t.sig;
            out[2 * i + 1] = t.tan;
            c = t;
        }
    } else if (m.type == 1) {
        S1State c{0.0, 0.0, m.p[1], 0.0, 0.0};
        S1State t = c;
        for (int i = 0; i < n; ++i) {
            const double eps = strains[i];
            if (eps != t.eps) steel01_trial(m, c, eps, t);
            out[2 * i] = t.sig;
            out[2 * i + 1] = t.tan;
            c = t;
        }
    } else {
        double teps = 0.0, tsig = 0.0;
        for (int i = 0; i < n; ++i) {
            const double eps = strains[i];
            if (eps != teps) {
                teps = eps;
                tsig = m.p[0] * eps;
            }
            out[2 * i] = tsig;
            out[2 * i + 1] = m.p[0];
        }
    }
}

// Batched section evaluation.  State of instance i, family field f, fiber j at
//   base_f + f * (n_inst * n_fam) + i * n_fam + j
// (field-major, then instance, then fiber) so a warp's loads are contiguous.
struct BatchState {
    double* c2;
    double* s2;
    int* kon;
    double* s1;
    double* c1;
    long long n_inst;  // instances with allocated state: a field's stride is n_inst x P
    int p_s2, p_c2, p_s1, p_c1;  // P: each instance's run per family, the family's length padded
                                 // to a multiple of 4
};

// One warp per instance (n_live instances), for sections whose stages do not fit the streaming
// kernel's shared memory.
__global__ void __launch_bounds__(256) section_batch_kernel(Geo g, DevSection sd, BatchState bs, long long n_live,
                                                            const double* __restrict__ ek,
                                                            double* __restrict__ resp,
                                                            int commit) {
    const long long warp_global = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp_global >= n_live) return;
    const long long i = warp_global;
    const double eps0 = ek[2 * i], kappa = ek[2 * i + 1];
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, a4 = 0.0, a3el = 0.0;
    int base = sd.geo_off;
    {
        const long long N = bs.n_inst * bs.p_s2;
        for (int j = lane; j < sd.n_s2; j += 32) {
            double* F = bs.s2 + i * bs.p_s2 + j;
            int* K = bs.kon + i * bs.p_s2 + j;
            S2State c, t;
            c.eps = F[0 * N]; c.sig = F[1 * N]; c.tan = F[2 * N]; c.epsmin = F[3 * N];
            c.epsmax = F[4 * N]; c.epspl = F[5 * N]; c.epss0 = F[6 * N]; c.sigs0 = F[7 * N];
            c.epsr = F[8 * N]; c.sigr = F[9 * N]; c.kon = *K;
            const double y = __ldg(g.y + base + j), A = __ldg(g.a + base + j);
            steel02_trial(g.mats[__ldg(g.m + base + j)], c, eps0 - y * kappa, t);
            if (commit) {
                F[0 * N] = t.eps; F[1 * N] = t.sig; F[2 * N] = t.tan; F[3 * N] = t.epsmin;
                F[4 * N] = t.epsmax; F[5 * N] = t.epspl; F[6 * N] = t.epss0;
                F[7 * N] = t.sigs0; F[8 * N] = t.epsr; F[9 * N] = t.sigr; *K = t.kon;
            }
            const double fs = t.sig * A, ks = t.tan * A;
            a0 += fs; a1 += -fs * y; a2 += ks; a3 += -ks * y; a4 += ks * y * y;
        }
    }
    base += sd.n_s2;
    {
        const long long N = bs.n_inst * bs.p_c2;
        for (int j = lane; j < sd.n_c2; j += 32) {
            double* F = bs.c2 + i * bs.p_c2 + j;
            C2State c, t;
            c.eps = F[0]; c.sig = F[N]; c.tan = F[2 * N]; c.ecmin = F[3 * N]; c.dept = F[4 * N];
            const double y = __ldg(g.y + base + j), A = __ldg(g.a + base + j);
            concrete02_trial(g.mats[__ldg(g.m + base + j)], c, eps0 - y * kappa, t);
            if (commit) {
                F[0] = t.eps; F[N] = t.sig; F[2 * N] = t.tan; F[3 * N] = t.ecmin;
                F[4 * N] = t.dept;
            }
            const double fs = t.sig * A, ks = t.tan * A;
            a0 += fs; a1 += -fs * y; a2 += ks; a3 += -ks * y; a4 += ks * y * y;
        }
    }
    base += sd.n_c2;
    {
        const long long N = bs.n_inst * bs.p_s1;
        for (int j = lane; j < sd.n_s1; j += 32) {
            double* F = bs.s1 + i * bs.p_s1 + j;
            S1State c, t;
            c.eps = F[0]; c.sig = F[N]; c.tan = F[2 * N]; c.epsp = F[3 * N]; c.alpha = F[4 * N];
            const double y = __ldg(g.y + base + j), A = __ldg(g.a + base + j);
            steel01_trial(g.mats[__ldg(g.m + base + j)], c, eps0 - y * kappa, t);
            if (commit) {
                F[0] = t.eps; F[N] = t.sig; F[2 * N] = t.tan; F[3 * N] = t.epsp;
                F[4 * N] = t.alpha;
            }
            const double fs = t.sig * A, ks = t.tan * A;
            a0 += fs; a1 += -fs * y; a2 += ks; a3 += -ks * y; a4 += ks * y * y;
        }
    }
    base += sd.n_s1;
    {
        const long long N = bs.n_inst * bs.p_c1;
        for (int j = lane; j < sd.n_c1; j += 32) {
            double* F = bs.c1 + i * bs.p_c1 + j;
            C1State c, t;
            c.eps = F[0]; c.sig = F[N]; c.tan = F[2 * N]; c.emin = F[3 * N]; c.eend = F[4 * N];
            c.slope = F[5 * N];
            const double y = __ldg(g.y + base + j), A = __ldg(g.a + base + j);
            concrete01_trial(g.mats[__ldg(g.m + base + j)], c, eps0 - y * kappa, t);
            if (commit) {
                F[0] = t.eps; F[N] = t.sig; F[2 * N] = t.tan; F[3 * N] = t.emin;
                F[4 * N] = t.eend; F[5 * N] = t.slope;
            }
            const double fs = t.sig * A, ks = t.tan * A;
            a0 += fs; a1 += -fs * y; a2 += ks; a3 += -ks * y; a4 += ks * y * y;
        }
    }
    base += sd.n_c1;
    for (int j = lane; j < sd.n_el; j += 32) {
        const double y = __ldg(g.y + base + j), A = __ldg(g.a + base + j);
        const double ks = g.mats[__ldg(g.m + base + j)].p[0] * A;
        const double fs = ks * (eps0 - y * kappa);
        a0 += fs; a1 += -fs * y; a2 += ks; a3el += -ks * y; a4 += ks * y * y;
    }
    a0 = warp_sum(a0);
    a1 = warp_sum(a1);
    a2 = warp_sum(a2);
    const double k12el = warp_sum(a3el);
    a3 = warp_sum(a3) + (sd.el_uniform ? 0.0 : k12el);
    a4 = warp_sum(a4);
    if (lane == 0) {
        double* r = resp + 5 * i;
        r[0] = a0; r[1] = a1; r[2] = a2; r[3] = a3; r[4] = a4;
    }
}

// One FiberSection3d along n points (eps0, kappa_y, kappa_z), committing after each point
// (fiber3d.mojo:769-836, section_path.mojo:463-556).  One warp; lane l owns fibers l, l + 32,
// ... of each family (their committed state in bs, one instance); the warp sums in a fixed
// butterfly order.  out: n x 9 = N, My, Mz, k11, k12, k13, k22, k23, k33.
__global__ void section3d_path_kernel(Geo g, DevSection sd, BatchState bs,
                                      const double* __restrict__ path, int n,
                                      double* __restrict__ out) {
    const int lane = threadIdx.x;
    if (blockIdx.x != 0 || lane >= 32) return;
    for (int p = 0; p < n; ++p) {
        const double e0 = path[3 * p], ky = path[3 * p + 1], kz = path[3 * p + 2];
        double a[11];
        for (int c = 0; c < 11; ++c) a[c] = 0.0;
        auto acc = [&](double fs, double ks, double y, double z, bool elastic) {
            a[0] += fs;
            a[1] += fs * z;
            a[2] += -fs * y;
            a[3] += ks;
            a[elastic ? 9 : 4] += ks * z;
            a[elastic ? 10 : 5] += -ks * y;
            a[6] += ks * z * z;
            a[7] += -ks * z * y;
            a[8] += ks * y * y;
        };
        int base = sd.geo_off;
        for (int j = lane; j < sd.n_s2; j += 32) {
            const long long N = bs.p_s2;
            double* F = bs.s2 + j;
            S2State c, t;
            c.eps = F[0 * N]; c.sig = F[1 * N]; c.tan = F[2 * N]; c.epsmin = F[3 * N];
            c.epsmax = F[4 * N]; c.epspl = F[5 * N]; c.epss0 = F[6 * N]; c.sigs0 = F[7 * N];
            c.epsr = F[8 * N]; c.sigr = F[9 * N]; c.kon = bs.kon[j];
            const double y = g.y[base + j], z = g.z[base + j], A = g.a[base + j];
            steel02_trial(g.mats[g.m[base + j]], c, e0 + z * ky - y * kz, t);
            F[0 * N] = t.eps; F[1 * N] = t.sig; F[2 * N] = t.tan; F[3 * N] = t.epsmin;
            F[4 * N] = t.epsmax; F[5 * N] = t.epspl; F[6 * N] = t.epss0; F[7 * N] = t.sigs0;
            F[8 * N] = t.epsr; F[9 * N] = t.sigr; bs.kon[j] = t.kon;
            acc(t.sig * A, t.tan * A, y, z, false);
        }
        base += sd.n_s2;
        for (int j = lane; j < sd.n_c2; j += 32) {
            const long long N = bs.p_c2;
            double* F = bs.c2 + j;
            C2State c, t;
            c.eps = F[0]; c.sig = F[N]; c.tan = F[2 * N]; c.ecmin = F[3 * N]; c.dept = F[4 * N];
            const double y = g.y[base + j], z = g.z[base + j], A = g.a[base + j];
            concrete02_trial(g.mats[g.m[base + j]], c, e0 + z * ky - y * kz, t);
            F[0] = t.eps; F[N] = t.sig; F[2 * N] = t.tan; F[3 * N] = t.ecmin; F[4 * N] = t.dept;
            acc(t.sig * A, t.tan * A, y, z, false);
        }
        base += sd.n_c2;
        for (int j = lane; j < sd.n_s1; j += 32) {
            const long long N = bs.p_s1;
            double* F = bs.s1 + j;
            S1State c, t;
            c.eps = F[0]; c.sig = F[N]; c.tan = F[2 * N]; c.epsp = F[3 * N]; c.alpha = F[4 * N];
            const double y = g.y[base + j], z = g.z[base + j], A = g.a[base + j];
            steel01_trial(g.mats[g.m[base + j]], c, e0 + z * ky - y * kz, t);
            F[0] = t.eps; F[N] = t.sig; F[2 * N] = t.tan; F[3 * N] = t.epsp; F[4 * N] = t.alpha;
            acc(t.sig * A, t.tan * A, y, z, false);
        }
        base += sd.n_s1;
        for (int j = lane; j < sd.n_c1; j += 32) {
            const long long N = bs.p_c1;
            double* F = bs.c1 + j;
            C1State c, t;
            c.eps = F[0]; c.sig = F[N]; c.tan = F[2 * N]; c.emin = F[3 * N]; c.eend = F[4 * N];
            c.slope = F[5 * N];
            const double y = g.y[base + j], z = g.z[base + j], A = g.a[base + j];
            concrete01_trial(g.mats[g.m[base + j]], c, e0 + z * ky - y * kz, t);
            F[0] = t.eps; F[N] = t.sig; F[2 * N] = t.tan; F[3 * N] = t.emin; F[4 * N] = t.eend;
            F[5 * N] = t.slope;
            acc(t.sig * A, t.tan * A, y, z, false);
        }
        base += sd.n_c1;
        for (int j = lane; j < sd.n_el; j += 32) {
            const double y = g.y[base + j], z = g.z[base + j], A = g.a[base + j];
            const double ks = g.mats[g.m[base + j]].p[0] * A;
            acc(ks * (e0 + z * ky - y * kz), ks, y, z, true);
        }
        for (int c = 0; c < 11; ++c) a[c] = warp_sum(a[c]);
        if (lane == 0) {
            double* o = out + 9 * p;
            o[0] = a[0];
            o[1] = a[1];
            o[2] = a[2];
            o[3] = a[3];
            o[4] = a[4] + (sd.el_uniform ? 0.0 : a[9]);
            o[5] = a[5] + (sd.el_uniform ? 0.0 : a[10]);
            o[6] = a[6];
            o[7] = a[7];
            o[8] = a[8];
        }
        __syncwarp();
    }
}

}  // namespace strut

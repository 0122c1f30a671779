// Device-side uniaxial fiber state determination (FP64) for the sm_100a hot path.
//
// Update rules follow Strut's 2D fiber runtime (paths relative to the Strut project root):
//   Steel02     src/mojo/sections/fiber2d.mojo:1103-1187 (SIMD form 2301-2516)
//   Concrete02  src/mojo/sections/fiber2d.mojo:1190-1244 (SIMD form 1785-1972), envelopes
//               src/mojo/materials/uniaxial/concrete02.mojo:3-31
//   Steel01     src/mojo/sections/fiber2d.mojo:1021-1045
//   Concrete01  src/mojo/sections/fiber2d.mojo:1049-1101, envelope / unloading / reloading
//               src/mojo/materials/uniaxial/concrete01.mojo:3-70
//   Elastic     src/mojo/materials/uniaxial/ops.mojo:10-21
// Every trial state is a pure function of the committed state and the strain; nothing is kept
// between calls.  That is what lets the element kernels keep trial fiber state out of HBM.
#pragma once

#include <cstdint>

namespace strut {

// Material record on the device: Strut's p0..p10 plus constants Strut recomputes per call
// with the same expression (so precomputing them on the host gives identical values).
struct DevMat {
    int type;
    int pad;
    double p[11];
    double k[8];
};

// derived-constant slots
enum {
    // Concrete02
    C2K_EC0 = 0,    // (2 fc) / epsc0
    C2K_EPSR = 1,   // (fcu - rat Ec0 epscu) / (Ec0 (1 - rat))
    C2K_SIGMR = 2,  // Ec0 epsr
    C2K_EPS0T = 3,  // ft / Ec0
    C2K_EPSUT = 4,  // ft (1/Ets + 1/Ec0)
    // Steel02
    S2K_ESH = 0,       // b E0
    S2K_EPSY = 1,      // Fy / E0
    S2K_SIGINI_E0 = 2, // sigini / E0
    S2K_DPOS = 3,      // 2 (a4 epsy)
    S2K_DNEG = 4,      // 2 (a2 epsy)
    S2K_E0MESH = 5,    // E0 - Esh
    S2K_ESHEPSY = 6,   // Esh epsy
    // Steel01
    S1K_H = 0,         // (b E0) / (1 - b)
    S1K_EH = 1,        // (E0 H) / (E0 + H)
    S1K_E0PH = 2,      // E0 + H
    // Concrete01
    C1K_EC0 = 0        // (2 fpc) / epsc0
};

// Committed history of one fiber, by family (structure-of-arrays in HBM, these are the
// per-thread register copies).
struct C2State {
    double eps, sig, tan, ecmin, dept;
};
struct S2State {
    double eps, sig, tan, epsmin, epsmax, epspl, epss0, sigs0, epsr, sigr;
    int kon;
};
struct S1State {
    double eps, sig, tan, epsp, alpha;
};
struct C1State {
    double eps, sig, tan, emin, eend, slope;  // min strain, end strain, unloading slope
};

// Concrete01 (Kent-Scott-Park without tension) trial from committed c.
__device__ __forceinline__ void concrete01_trial(const DevMat& m, const C1State& c, double eps,
                                                 C1State& t) {
    const double fpc = m.p[0], epsc0 = m.p[1], fpcu = m.p[2], epscu = m.p[3];
    const double Ec0 = m.k[C1K_EC0];
    t.eps = eps;
    const double d_strain = eps - c.eps;
    if (fabs(d_strain) < 1.0e-14) {
        t.sig = c.sig;
        t.tan = c.tan;
        t.emin = c.emin;
        t.eend = c.eend;
        t.slope = c.slope;
        return;
    }
    double emin = c.emin, eend = c.eend, slope = c.slope;
    if (eps > 0.0) {
        t.sig = 0.0;
        t.tan = 0.0;
        t.emin = emin;
        t.eend = eend;
        t.slope = slope;
        return;
    }
    const double temp_stress = c.sig + slope * eps - slope * c.eps;
    if (eps <= c.eps) {
        double rs, rt;
        if (eps <= emin) {
            // envelope, then the new unloading point (_concrete01_reload / _unload)
            emin = eps;
            if (eps > epsc0) {
                const double eta = eps / epsc0;
                rs = fpc * (2.0 * eta - eta * eta);
                rt = Ec0 * (1.0 - eta);
            } else if (eps > epscu) {
                rt = (fpc - fpcu) / (epsc0 - epscu);
                rs = fpc + rt * (eps - epsc0);
            } else {
                rs = fpcu;
                rt = 0.0;
            }
            double ts = emin < epscu ? epscu : emin;
            const double eta = ts / epsc0;
            double ratio = 0.707 * (eta - 2.0) + 0.834;
            if (eta < 2.0) ratio = 0.145 * eta * eta + 0.13 * eta;
            const double es = ratio * epsc0;
            const double temp1 = emin - es;
            const double temp2 = rs / Ec0;
            if (temp1 > -1.0e-14) {
                eend = es;
                slope = Ec0;
            } else if (temp1 <= temp2) {
                eend = emin - temp1;
                slope = rs / temp1;
            } else {
                eend = emin - temp2;
                slope = Ec0;
            }
        } else if (eps <= eend) {
            rt = slope;
            rs = rt * (eps - eend);
        } else {
            rs = 0.0;
            rt = 0.0;
        }
        t.sig = rs;
        t.tan = rt;
        if (temp_stress > t.sig) {
            t.sig = temp_stress;
            t.tan = slope;
        }
    } else if (temp_stress <= 0.0) {
        t.sig = temp_stress;
        t.tan = slope;
    } else {
        t.sig = 0.0;
        t.tan = 0.0;
    }
    t.emin = emin;
    t.eend = eend;
    t.slope = slope;
}

__device__ __forceinline__ void c2_compr_envlp(const DevMat& m, double strain, double& sig,
                                               double& tan) {
    const double fc = m.p[0], epsc0 = m.p[1], fcu = m.p[2], epscu = m.p[3];
    if (strain >= epsc0) {
        double rat = strain / epsc0;
        sig = fc * rat * (2.0 - rat);
        tan = m.k[C2K_EC0] * (1.0 - rat);
    } else if (strain > epscu) {
        sig = (fcu - fc) * (strain - epsc0) / (epscu - epsc0) + fc;
        tan = (fcu - fc) / (epscu - epsc0);
    } else {
        sig = fcu;
        tan = 1.0e-10;
    }
}

__device__ __forceinline__ void c2_tens_envlp(const DevMat& m, double strain, double& sig,
                                              double& tan) {
    const double ft = m.p[5], Ets = m.p[6], Ec0 = m.k[C2K_EC0];
    if (strain <= m.k[C2K_EPS0T]) {
        sig = strain * Ec0;
        tan = Ec0;
    } else if (strain <= m.k[C2K_EPSUT]) {
        sig = ft - Ets * (strain - m.k[C2K_EPS0T]);
        tan = -Ets;
    } else {
        sig = 0.0;
        tan = 1.0e-10;
    }
}

// Constants of a Concrete02 fiber that depend on its committed state only: every trial from
// that state evaluates them with these same expressions (fiber2d.mojo:1190-1244), so an
// element evaluating many trial strains against one committed state computes them once.
struct C2Derived {
    double sigmm;  // compression envelope stress at ecmin
    double er;     // unloading modulus
    double ept;    // strain at zero stress on the unloading branch
    double epn;    // ept + dept: end of the tension reloading branch
    double etn;    // tension reloading modulus
};

__device__ __forceinline__ void concrete02_derive(const DevMat& m, const C2State& c, C2Derived& d) {
    double tmm;
    c2_compr_envlp(m, c.ecmin, d.sigmm, tmm);
    d.er = (d.sigmm - m.k[C2K_SIGMR]) / (c.ecmin - m.k[C2K_EPSR]);
    d.ept = c.ecmin - d.sigmm / d.er;
    d.epn = d.ept + c.dept;
    double sicn, tcn;
    c2_tens_envlp(m, c.dept, sicn, tcn);
    d.etn = m.k[C2K_EC0];
    if (c.dept != 0.0) d.etn = sicn / c.dept;
}

// Stress and tangent for strain >= ecmin (unloading / reloading / tension branches).
__device__ __forceinline__ void concrete02_unload(const DevMat& m, const C2State& c,
                                                  const C2Derived& d, double strain, double deps,
                                                  double& sig, double& tan) {
    const double Ec0 = m.k[C2K_EC0];
    if (strain <= d.ept) {
        const double sigmin = d.sigmm + d.er * (strain - c.ecmin);
        const double sigmax = 0.5 * d.er * (strain - d.ept);
        double s = c.sig + Ec0 * deps;
        double e = Ec0;
        if (s <= sigmin) {
            s = sigmin;
            e = d.er;
        }
        if (s >= sigmax) {
            s = sigmax;
            e = 0.5 * d.er;
        }
        sig = s;
        tan = e;
    } else if (strain <= d.epn) {
        tan = d.etn;
        sig = d.etn * (strain - d.ept);
    } else {
        c2_tens_envlp(m, strain - d.ept, sig, tan);
    }
}

// Concrete02 trial from committed c at strain -> t.
__device__ __forceinline__ void concrete02_trial(const DevMat& m, const C2State& c,
                                                 double strain, C2State& t) {
    t.ecmin = c.ecmin;
    t.dept = c.dept;
    t.eps = strain;
    const double deps = strain - c.eps;
    if (fabs(deps) < 2.220446049250313e-16) {
        t.sig = c.sig;
        t.tan = c.tan;
        return;
    }
    if (strain < c.ecmin) {
        c2_compr_envlp(m, strain, t.sig, t.tan);
        t.ecmin = strain;
        return;
    }
    C2Derived d;
    concrete02_derive(m, c, d);
    concrete02_unload(m, c, d, strain, deps, t.sig, t.tan);
    if (strain > d.epn) t.dept = strain - d.ept;
}

// Stress and tangent of concrete02_trial, given the committed state's derived constants.
__device__ __forceinline__ void concrete02_sig_tan(const DevMat& m, const C2State& c,
                                                   const C2Derived& d, double strain,
                                                   double& sig, double& tan) {
    const double deps = strain - c.eps;
    if (fabs(deps) < 2.220446049250313e-16) {
        sig = c.sig;
        tan = c.tan;
        return;
    }
    if (strain < c.ecmin) {
        c2_compr_envlp(m, strain, sig, tan);
        return;
    }
    concrete02_unload(m, c, d, strain, deps, sig, tan);
}

// Steel02: given the committed state, the loading branch a trial follows depends only on the
// sign of the strain increment (first loading from kon 0/3, continued loading, or a reversal
// with the isotropic shift), so both possible branches can be formed once per committed state.
struct S2Curve {
    double epsr, sigr;
    double denom;  // epss0 - epsr
    double dsig;   // sigs0 - sigr
    double R, invR;
};
struct S2Derived {
    S2Curve up, dn;  // strain increasing / decreasing
};

// Branch state after an increment in direction `up` (fiber2d.mojo:1103-1187): everything of
// the trial state except eps, sig and tan.  Call only when the no-change test failed.
__device__ __forceinline__ void steel02_branch(const DevMat& m, const S2State& c, bool up,
                                               S2State& t) {
    const double Fy = m.p[0], E0 = m.p[1];
    const double a1 = m.p[6], a3 = m.p[8];
    const double Esh = m.k[S2K_ESH], epsy = m.k[S2K_EPSY];
    double epsmax = c.epsmax, epsmin = c.epsmin, epspl = c.epspl, epss0 = c.epss0;
    double sigs0 = c.sigs0, epsr = c.epsr, sigr = c.sigr;
    int kon = c.kon;
    if (kon == 0 || kon == 3) {
        epsmax = epsy;
        epsmin = -epsy;
        if (!up) {
            kon = 2;
            epss0 = epsmin;
            sigs0 = -Fy;
            epspl = epsmin;
        } else {
            kon = 1;
            epss0 = epsmax;
            sigs0 = Fy;
            epspl = epsmax;
        }
    }
    if (kon == 2 && up) {
        kon = 1;
        epsr = c.eps;
        sigr = c.sig;
        if (c.eps < epsmin) epsmin = c.eps;
        const double d1 = (epsmax - epsmin) / m.k[S2K_DPOS];
        const double shft = 1.0 + a3 * pow(d1, 0.8);
        epss0 = (Fy * shft - m.k[S2K_ESHEPSY] * shft - sigr + E0 * epsr) / m.k[S2K_E0MESH];
        sigs0 = Fy * shft + Esh * (epss0 - epsy * shft);
        epspl = epsmax;
    } else if (kon == 1 && !up) {
        kon = 2;
        epsr = c.eps;
        sigr = c.sig;
        if (c.eps > epsmax) epsmax = c.eps;
        const double d1 = (epsmax - epsmin) / m.k[S2K_DNEG];
        const double shft = 1.0 + a1 * pow(d1, 0.8);
        epss0 = (-Fy * shft + m.k[S2K_ESHEPSY] * shft - sigr + E0 * epsr) / m.k[S2K_E0MESH];
        sigs0 = -Fy * shft + Esh * (epss0 + epsy * shft);
        epspl = epsmin;
    }
    t.epsmin = epsmin;
    t.epsmax = epsmax;
    t.epspl = epspl;
    t.epss0 = epss0;
    t.sigs0 = sigs0;
    t.epsr = epsr;
    t.sigr = sigr;
    t.kon = kon;
}

__device__ __forceinline__ void steel02_curve_of(const DevMat& m, const S2State& t, S2Curve& cv) {
    const double R0 = m.p[3], cR1 = m.p[4], cR2 = m.p[5];
    const double epsy = m.k[S2K_EPSY];
    const double xi = fabs((t.epspl - t.epss0) / epsy);
    const double R = R0 * (1.0 - (cR1 * xi) / (cR2 + xi));
    cv.epsr = t.epsr;
    cv.sigr = t.sigr;
    cv.denom = t.epss0 - t.epsr;
    cv.dsig = t.sigs0 - t.sigr;
    cv.R = R;
    cv.invR = 1.0 / R;
}

// Menegotto-Pinto curve: stress and tangent at eps on the branch cv.
__device__ __forceinline__ void steel02_curve_eval(const DevMat& m, const S2Curve& cv, double eps,
                                                   double& sig, double& tan) {
    const double b = m.p[2];
    const double epsrat = (eps - cv.epsr) / cv.denom;
    const double dum1 = 1.0 + pow(fabs(epsrat), cv.R);
    const double dum2 = pow(dum1, cv.invR);
    double s = b * epsrat + (1.0 - b) * epsrat / dum2;
    s = s * cv.dsig + cv.sigr;
    double e = b + (1.0 - b) / (dum1 * dum2);
    e = e * cv.dsig / cv.denom;
    sig = s;
    tan = e;
}

__device__ __forceinline__ double steel02_strain(const DevMat& m, double trial_eps) {
    double eps = trial_eps;
    if (m.p[10] != 0.0) eps += m.k[S2K_SIGINI_E0];
    return eps;
}

// True when the trial leaves the fiber at its initial state (kon 0 / 3 and no strain change).
__device__ __forceinline__ bool steel02_no_change(const S2State& c, double deps) {
    return (c.kon == 0 || c.kon == 3) && fabs(deps) < 2.220446049250313e-15;
}

// Direction of the branch: increasing strain, or no change on an increasing branch.
__device__ __forceinline__ bool steel02_up(const S2State& c, double deps) {
    return deps > 0.0 || (deps == 0.0 && c.kon == 1);
}

// Steel02 (Giuffre-Menegotto-Pinto with isotropic shift) trial from committed c.
__device__ __forceinline__ void steel02_trial(const DevMat& m, const S2State& c,
                                              double trial_eps, S2State& t) {
    const double eps = steel02_strain(m, trial_eps);
    t.eps = eps;
    const double deps = eps - c.eps;
    if (steel02_no_change(c, deps)) {
        t.tan = m.p[1];
        t.sig = m.p[10];
        t.kon = 3;
        t.epsmin = c.epsmin;
        t.epsmax = c.epsmax;
        t.epspl = c.epspl;
        t.epss0 = c.epss0;
        t.sigs0 = c.sigs0;
        t.epsr = c.epsr;
        t.sigr = c.sigr;
        return;
    }
    steel02_branch(m, c, steel02_up(c, deps), t);
    S2Curve cv;
    steel02_curve_of(m, t, cv);
    steel02_curve_eval(m, cv, eps, t.sig, t.tan);
}

__device__ __forceinline__ void steel02_derive(const DevMat& m, const S2State& c, S2Derived& d) {
    S2State t;
    steel02_branch(m, c, true, t);
    steel02_curve_of(m, t, d.up);
    steel02_branch(m, c, false, t);
    steel02_curve_of(m, t, d.dn);
}

// Stress and tangent of steel02_trial, given the committed state's derived branches.
__device__ __forceinline__ void steel02_sig_tan(const DevMat& m, const S2State& c,
                                                const S2Derived& d, double trial_eps,
                                                double& sig, double& tan) {
    const double eps = steel02_strain(m, trial_eps);
    const double deps = eps - c.eps;
    if (steel02_no_change(c, deps)) {
        tan = m.p[1];
        sig = m.p[10];
        return;
    }
    steel02_curve_eval(m, steel02_up(c, deps) ? d.up : d.dn, eps, sig, tan);
}

// Steel01 bilinear kinematic return map.
__device__ __forceinline__ void steel01_trial(const DevMat& m, const S1State& c, double eps,
                                              S1State& t) {
    const double Fy = m.p[0], E0 = m.p[1];
    const double H = m.k[S1K_H];
    const double sigma_trial = E0 * (eps - c.epsp);
    const double xi = sigma_trial - c.alpha;
    const double f = fabs(xi) - Fy;
    t.eps = eps;
    if (f <= 0.0) {
        t.sig = sigma_trial;
        t.tan = E0;
        t.epsp = c.epsp;
        t.alpha = c.alpha;
        return;
    }
    const double dg = f / m.k[S1K_E0PH];
    const double sgn = xi < 0.0 ? -1.0 : 1.0;
    t.epsp = c.epsp + dg * sgn;
    t.alpha = c.alpha + H * dg * sgn;
    t.sig = sigma_trial - E0 * dg * sgn;
    t.tan = m.k[S1K_EH];
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace strut

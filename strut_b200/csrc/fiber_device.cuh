// Device-side uniaxial fiber state determination (FP64) for the sm_100a hot path.
//
// Update rules follow Strut's 2D fiber runtime (paths relative to the Strut project root):
//   Steel02     src/mojo/sections/fiber2d.mojo:1103-1187 (SIMD form 2301-2516)
//   Concrete02  src/mojo/sections/fiber2d.mojo:1190-1244 (SIMD form 1785-1972), envelopes
//               src/mojo/materials/uniaxial/concrete02.mojo:3-31
//   Steel01     src/mojo/sections/fiber2d.mojo:1021-1045
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
    S1K_E0PH = 2       // E0 + H
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

// Concrete02 trial from committed c at strain -> t.
__device__ __forceinline__ void concrete02_trial(const DevMat& m, const C2State& c,
                                                 double strain, C2State& t) {
    const double Ec0 = m.k[C2K_EC0];
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
    double sigmm, tmm;
    c2_compr_envlp(m, c.ecmin, sigmm, tmm);
    const double er = (sigmm - m.k[C2K_SIGMR]) / (c.ecmin - m.k[C2K_EPSR]);
    const double ept = c.ecmin - sigmm / er;
    if (strain <= ept) {
        const double sigmin = sigmm + er * (strain - c.ecmin);
        const double sigmax = 0.5 * er * (strain - ept);
        double s = c.sig + Ec0 * deps;
        double e = Ec0;
        if (s <= sigmin) {
            s = sigmin;
            e = er;
        }
        if (s >= sigmax) {
            s = sigmax;
            e = 0.5 * er;
        }
        t.sig = s;
        t.tan = e;
        return;
    }
    const double epn = ept + c.dept;
    if (strain <= epn) {
        double sicn, tcn;
        c2_tens_envlp(m, c.dept, sicn, tcn);
        double e = Ec0;
        if (c.dept != 0.0) e = sicn / c.dept;
        t.tan = e;
        t.sig = e * (strain - ept);
    } else {
        c2_tens_envlp(m, strain - ept, t.sig, t.tan);
        t.dept = strain - ept;
    }
}

// Steel02 (Giuffre-Menegotto-Pinto with isotropic shift) trial from committed c.
__device__ __forceinline__ void steel02_trial(const DevMat& m, const S2State& c,
                                              double trial_eps, S2State& t) {
    const double Fy = m.p[0], E0 = m.p[1], b = m.p[2], R0 = m.p[3], cR1 = m.p[4];
    const double cR2 = m.p[5], a1 = m.p[6], a3 = m.p[8], sigini = m.p[10];
    const double Esh = m.k[S2K_ESH], epsy = m.k[S2K_EPSY];
    double eps = trial_eps;
    if (sigini != 0.0) eps += m.k[S2K_SIGINI_E0];
    t.eps = eps;
    const double deps = eps - c.eps;
    double epsmax = c.epsmax, epsmin = c.epsmin, epspl = c.epspl, epss0 = c.epss0;
    double sigs0 = c.sigs0, epsr = c.epsr, sigr = c.sigr;
    int kon = c.kon;
    if (kon == 0 || kon == 3) {
        if (fabs(deps) < 2.220446049250313e-15) {
            t.tan = E0;
            t.sig = sigini;
            t.kon = 3;
            t.epsmin = epsmin;
            t.epsmax = epsmax;
            t.epspl = epspl;
            t.epss0 = epss0;
            t.sigs0 = sigs0;
            t.epsr = epsr;
            t.sigr = sigr;
            return;
        }
        epsmax = epsy;
        epsmin = -epsy;
        if (deps < 0.0) {
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
    if (kon == 2 && deps > 0.0) {
        kon = 1;
        epsr = c.eps;
        sigr = c.sig;
        if (c.eps < epsmin) epsmin = c.eps;
        const double d1 = (epsmax - epsmin) / m.k[S2K_DPOS];
        const double shft = 1.0 + a3 * pow(d1, 0.8);
        epss0 = (Fy * shft - m.k[S2K_ESHEPSY] * shft - sigr + E0 * epsr) / m.k[S2K_E0MESH];
        sigs0 = Fy * shft + Esh * (epss0 - epsy * shft);
        epspl = epsmax;
    } else if (kon == 1 && deps < 0.0) {
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
    const double xi = fabs((epspl - epss0) / epsy);
    const double R = R0 * (1.0 - (cR1 * xi) / (cR2 + xi));
    const double epsrat = (eps - epsr) / (epss0 - epsr);
    const double dum1 = 1.0 + pow(fabs(epsrat), R);
    const double dum2 = pow(dum1, 1.0 / R);
    double sig = b * epsrat + (1.0 - b) * epsrat / dum2;
    sig = sig * (sigs0 - sigr) + sigr;
    double e = b + (1.0 - b) / (dum1 * dum2);
    e = e * (sigs0 - sigr) / (epss0 - epsr);
    t.sig = sig;
    t.tan = e;
    t.epsmin = epsmin;
    t.epsmax = epsmax;
    t.epspl = epspl;
    t.epss0 = epss0;
    t.sigs0 = sigs0;
    t.epsr = epsr;
    t.sigr = sigr;
    t.kon = kon;
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

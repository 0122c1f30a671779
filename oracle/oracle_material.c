/*
 * ORACLE -- test infrastructure only.  A plain-C FP64 restatement of Strut's uniaxial
 * material state determination, used by tests/ and by bench.py's CPU-baseline leg as the
 * checker.  Nothing in the product library links or calls this code.
 *
 * Parity status: pinned against the reference's own known-answer tests (closed-form elastic
 * section sums, fiber-order invariance, element equilibrium); transient histories are
 * "parity unpinned" against Strut itself because the reference (Mojo) cannot run here.
 *
 * Followed line by line (paths relative to the Strut project root):
 *   Steel02     src/mojo/sections/fiber2d.mojo:1103-1187 (fiber runtime form; the SIMD
 *               homogeneous form 2301-2516 computes the same lane values)
 *               src/mojo/materials/uniaxial/steel02.mojo:3-114 (scalar form)
 *   Concrete02  src/mojo/sections/fiber2d.mojo:1190-1244 (runtime), 1785-1972 (SIMD)
 *               src/mojo/materials/uniaxial/concrete02.mojo:3-108 (scalar form, envelopes)
 *   Steel01     src/mojo/sections/fiber2d.mojo:1021-1045; materials/uniaxial/ops.mojo:24-53
 *   Elastic     src/mojo/materials/uniaxial/ops.mojo:10-21
 *   initial tangent / state ctor: src/mojo/materials/uniaxial/core.mojo:203-282
 */
#include "oracle.h"

#include <math.h>
#include <string.h>

double oracle_initial_tangent(const StrutUniMaterial* m) {
    /* core.mojo:270-282 */
    switch (m->type) {
        case STRUT_MAT_ELASTIC: return m->p[0];
        case STRUT_MAT_STEEL01: return m->p[1];
        case STRUT_MAT_CONCRETE01: return (2.0 * m->p[0]) / m->p[1];
        case STRUT_MAT_STEEL02: return m->p[1];
        case STRUT_MAT_CONCRETE02: return (2.0 * m->p[0]) / m->p[1];
        default: return 0.0;
    }
}

/* UniMaterialState(mat_def) committed == trial initial values (core.mojo:203-263),
 * restricted to the fields each family runtime stores. */
void oracle_fiber_init(const StrutUniMaterial* m, OFiberState* s) {
    memset(s, 0, sizeof(*s));
    double tangent = oracle_initial_tangent(m);
    s->tan = tangent;
    if (m->type == STRUT_MAT_STEEL02) {
        double Fy = m->p[0], E0 = m->p[1];
        double epsy = Fy / E0;
        s->h[S2_EPSMAX] = epsy;
        s->h[S2_EPSMIN] = -epsy;
        double sigini = m->p[10];
        if (sigini != 0.0) {
            s->eps = sigini / E0;
            s->sig = sigini;
        }
    }
    if (m->type == STRUT_MAT_CONCRETE01) s->h[C1_SLOPE] = tangent;
}

/* Concrete01 (Kent-Scott-Park, no tension): materials/uniaxial/concrete01.mojo:3-70, the trial
 * rule of ops.mojo:56-115 / fiber2d.mojo:1049-1101. */
static void c1_envelope(double fpc, double epsc0, double fpcu, double epscu, double strain,
                        double* sig, double* tan) {
    if (strain > epsc0) {
        double eta = strain / epsc0;
        *sig = fpc * (2.0 * eta - eta * eta);
        double Ec0 = (2.0 * fpc) / epsc0;
        *tan = Ec0 * (1.0 - eta);
    } else if (strain > epscu) {
        *tan = (fpc - fpcu) / (epsc0 - epscu);
        *sig = fpc + *tan * (strain - epsc0);
    } else {
        *sig = fpcu;
        *tan = 0.0;
    }
}

static void c1_unload(double fpc, double epsc0, double epscu, double min_strain, double stress,
                      double* end_strain, double* slope) {
    double temp_strain = min_strain;
    if (temp_strain < epscu) temp_strain = epscu;
    double eta = temp_strain / epsc0;
    double ratio = 0.707 * (eta - 2.0) + 0.834;
    if (eta < 2.0) ratio = 0.145 * eta * eta + 0.13 * eta;
    double es = ratio * epsc0;
    double temp1 = min_strain - es;
    double Ec0 = (2.0 * fpc) / epsc0;
    double temp2 = stress / Ec0;
    if (temp1 > -1.0e-14) {
        *end_strain = es;
        *slope = Ec0;
    } else if (temp1 <= temp2) {
        *end_strain = min_strain - temp1;
        *slope = stress / temp1;
    } else {
        *end_strain = min_strain - temp2;
        *slope = Ec0;
    }
}

void oracle_concrete01_trial(const StrutUniMaterial* m, const OFiberState* c, OFiberState* t,
                             double eps) {
    double fpc = m->p[0], epsc0 = m->p[1], fpcu = m->p[2], epscu = m->p[3];
    double d_strain = eps - c->eps;
    t->eps = eps;
    if (fabs(d_strain) < 1.0e-14) {
        t->sig = c->sig;
        t->tan = c->tan;
        t->h[C1_MIN] = c->h[C1_MIN];
        t->h[C1_END] = c->h[C1_END];
        t->h[C1_SLOPE] = c->h[C1_SLOPE];
        return;
    }
    double min_strain = c->h[C1_MIN], end_strain = c->h[C1_END], slope = c->h[C1_SLOPE];
    t->h[C1_MIN] = min_strain;
    t->h[C1_END] = end_strain;
    t->h[C1_SLOPE] = slope;
    if (eps > 0.0) {
        t->sig = 0.0;
        t->tan = 0.0;
        return;
    }
    double temp_stress = c->sig + slope * eps - slope * c->eps;
    if (eps <= c->eps) {
        /* _concrete01_reload: may move min_strain, end_strain and the unloading slope */
        double rs, rt;
        if (eps <= min_strain) {
            min_strain = eps;
            c1_envelope(fpc, epsc0, fpcu, epscu, eps, &rs, &rt);
            c1_unload(fpc, epsc0, epscu, min_strain, rs, &end_strain, &slope);
        } else if (eps <= end_strain) {
            rt = slope;
            rs = rt * (eps - end_strain);
        } else {
            rs = 0.0;
            rt = 0.0;
        }
        t->h[C1_MIN] = min_strain;
        t->h[C1_END] = end_strain;
        t->h[C1_SLOPE] = slope;
        t->sig = rs;
        t->tan = rt;
        if (temp_stress > t->sig) {
            t->sig = temp_stress;
            t->tan = slope;
        }
    } else if (temp_stress <= 0.0) {
        t->sig = temp_stress;
        t->tan = slope;
    } else {
        t->sig = 0.0;
        t->tan = 0.0;
    }
}

/* Concrete02 envelopes, concrete02.mojo:3-31. */
static void c2_tens_envlp(double fc, double epsc0, double ft, double Ets, double strain,
                          double* sig, double* tan) {
    double Ec0 = (2.0 * fc) / epsc0;
    double eps0 = ft / Ec0;
    double epsu = ft * (1.0 / Ets + 1.0 / Ec0);
    if (strain <= eps0) {
        *sig = strain * Ec0;
        *tan = Ec0;
    } else if (strain <= epsu) {
        *sig = ft - Ets * (strain - eps0);
        *tan = -Ets;
    } else {
        *sig = 0.0;
        *tan = 1.0e-10;
    }
}

static void c2_compr_envlp(double fc, double epsc0, double fcu, double epscu, double strain,
                           double* sig, double* tan) {
    double Ec0 = (2.0 * fc) / epsc0;
    double rat = strain / epsc0;
    if (strain >= epsc0) {
        *sig = fc * rat * (2.0 - rat);
        *tan = Ec0 * (1.0 - rat);
    } else if (strain > epscu) {
        *sig = (fcu - fc) * (strain - epsc0) / (epscu - epsc0) + fc;
        *tan = (fcu - fc) / (epscu - epsc0);
    } else {
        *sig = fcu;
        *tan = 1.0e-10;
    }
}

/* Steel02 trial update from committed state c into trial t (fiber2d.mojo:1103-1187). */
void oracle_steel02_trial(const StrutUniMaterial* m, const OFiberState* c, OFiberState* t,
                          double trial_eps) {
    const double* p = m->p;
    double Fy = p[0], E0 = p[1], b = p[2], R0 = p[3], cR1 = p[4], cR2 = p[5];
    double a1 = p[6], a2 = p[7], a3 = p[8], a4 = p[9], sigini = p[10];
    double Esh = b * E0;
    double epsy = Fy / E0;
    double eps = trial_eps;
    if (sigini != 0.0) eps += sigini / E0;
    t->eps = eps;
    double deps = eps - c->eps;
    double epsmax = c->h[S2_EPSMAX], epsmin = c->h[S2_EPSMIN], epspl = c->h[S2_EPSPL];
    double epss0 = c->h[S2_EPSS0], sigs0 = c->h[S2_SIGS0], epsr = c->h[S2_EPSR];
    double sigr = c->h[S2_SIGR];
    int kon = c->kon;
    if (kon == 0 || kon == 3) {
        if (fabs(deps) < 2.220446049250313e-15) {
            t->tan = E0;
            t->sig = sigini;
            t->kon = 3;
            t->h[S2_EPSMIN] = epsmin;
            t->h[S2_EPSMAX] = epsmax;
            t->h[S2_EPSPL] = epspl;
            t->h[S2_EPSS0] = epss0;
            t->h[S2_SIGS0] = sigs0;
            t->h[S2_EPSR] = epsr;
            t->h[S2_SIGR] = sigr;
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
        epsr = c->eps;
        sigr = c->sig;
        if (c->eps < epsmin) epsmin = c->eps;
        double d1 = (epsmax - epsmin) / (2.0 * (a4 * epsy));
        double shft = 1.0 + a3 * pow(d1, 0.8);
        epss0 = (Fy * shft - Esh * epsy * shft - sigr + E0 * epsr) / (E0 - Esh);
        sigs0 = Fy * shft + Esh * (epss0 - epsy * shft);
        epspl = epsmax;
    } else if (kon == 1 && deps < 0.0) {
        kon = 2;
        epsr = c->eps;
        sigr = c->sig;
        if (c->eps > epsmax) epsmax = c->eps;
        double d1 = (epsmax - epsmin) / (2.0 * (a2 * epsy));
        double shft = 1.0 + a1 * pow(d1, 0.8);
        epss0 = (-Fy * shft + Esh * epsy * shft - sigr + E0 * epsr) / (E0 - Esh);
        sigs0 = -Fy * shft + Esh * (epss0 + epsy * shft);
        epspl = epsmin;
    }
    double xi = fabs((epspl - epss0) / epsy);
    double R = R0 * (1.0 - (cR1 * xi) / (cR2 + xi));
    double epsrat = (eps - epsr) / (epss0 - epsr);
    double dum1 = 1.0 + pow(fabs(epsrat), R);
    double dum2 = pow(dum1, 1.0 / R);
    double sig = b * epsrat + (1.0 - b) * epsrat / dum2;
    sig = sig * (sigs0 - sigr) + sigr;
    double e = b + (1.0 - b) / (dum1 * dum2);
    e = e * (sigs0 - sigr) / (epss0 - epsr);
    t->sig = sig;
    t->tan = e;
    t->h[S2_EPSMIN] = epsmin;
    t->h[S2_EPSMAX] = epsmax;
    t->h[S2_EPSPL] = epspl;
    t->h[S2_EPSS0] = epss0;
    t->h[S2_SIGS0] = sigs0;
    t->h[S2_EPSR] = epsr;
    t->h[S2_SIGR] = sigr;
    t->kon = kon;
}

/* Concrete02 trial update (fiber2d.mojo:1190-1244). */
void oracle_concrete02_trial(const StrutUniMaterial* m, const OFiberState* c, OFiberState* t,
                             double strain) {
    const double* p = m->p;
    double fc = p[0], epsc0 = p[1], fcu = p[2], epscu = p[3], rat = p[4], ft = p[5];
    double Ets = p[6];
    double Ec0 = (2.0 * fc) / epsc0;
    double ecmin = c->h[C2_ECMIN];
    double dept = c->h[C2_DEPT];
    t->h[C2_ECMIN] = ecmin;
    t->h[C2_DEPT] = dept;
    t->eps = strain;
    double deps = strain - c->eps;
    if (fabs(deps) < 2.220446049250313e-16) {
        t->sig = c->sig;
        t->tan = c->tan;
        return;
    }
    if (strain < ecmin) {
        c2_compr_envlp(fc, epsc0, fcu, epscu, strain, &t->sig, &t->tan);
        t->h[C2_ECMIN] = strain;
        return;
    }
    double epsr = (fcu - rat * Ec0 * epscu) / (Ec0 * (1.0 - rat));
    double sigmr = Ec0 * epsr;
    double sigmm, tmm;
    c2_compr_envlp(fc, epsc0, fcu, epscu, ecmin, &sigmm, &tmm);
    double er = (sigmm - sigmr) / (ecmin - epsr);
    double ept = ecmin - sigmm / er;
    if (strain <= ept) {
        double sigmin = sigmm + er * (strain - ecmin);
        double sigmax = 0.5 * er * (strain - ept);
        t->sig = c->sig + Ec0 * deps;
        t->tan = Ec0;
        if (t->sig <= sigmin) {
            t->sig = sigmin;
            t->tan = er;
        }
        if (t->sig >= sigmax) {
            t->sig = sigmax;
            t->tan = 0.5 * er;
        }
        return;
    }
    double epn = ept + dept;
    if (strain <= epn) {
        double sicn, tcn;
        c2_tens_envlp(fc, epsc0, ft, Ets, dept, &sicn, &tcn);
        double e = Ec0;
        if (dept != 0.0) e = sicn / dept;
        t->tan = e;
        t->sig = e * (strain - ept);
    } else {
        c2_tens_envlp(fc, epsc0, ft, Ets, strain - ept, &t->sig, &t->tan);
        t->h[C2_DEPT] = strain - ept;
    }
}

/* Steel01 bilinear kinematic return map (fiber2d.mojo:1021-1045). */
void oracle_steel01_trial(const StrutUniMaterial* m, const OFiberState* c, OFiberState* t,
                          double eps) {
    double Fy = m->p[0], E0 = m->p[1], b = m->p[2];
    double H = (b * E0) / (1.0 - b);
    double eps_p = c->h[S1_EPSP];
    double alpha = c->h[S1_ALPHA];
    double sigma_trial = E0 * (eps - eps_p);
    double xi = sigma_trial - alpha;
    double f = fabs(xi) - Fy;
    t->eps = eps;
    if (f <= 0.0) {
        t->sig = sigma_trial;
        t->tan = E0;
        t->h[S1_EPSP] = eps_p;
        t->h[S1_ALPHA] = alpha;
        return;
    }
    double dg = f / (E0 + H);
    double sgn = xi < 0.0 ? -1.0 : 1.0;
    t->h[S1_EPSP] = eps_p + dg * sgn;
    t->h[S1_ALPHA] = alpha + H * dg * sgn;
    t->sig = sigma_trial - E0 * dg * sgn;
    t->tan = (E0 * H) / (E0 + H);
}

void oracle_elastic_trial(const StrutUniMaterial* m, const OFiberState* c, OFiberState* t,
                          double eps) {
    (void)c;
    t->eps = eps;
    t->sig = m->p[0] * eps;
    t->tan = m->p[0];
}

void oracle_fiber_trial(const StrutUniMaterial* m, const OFiberState* c, OFiberState* t,
                        double eps) {
    switch (m->type) {
        case STRUT_MAT_STEEL02: oracle_steel02_trial(m, c, t, eps); break;
        case STRUT_MAT_CONCRETE02: oracle_concrete02_trial(m, c, t, eps); break;
        case STRUT_MAT_STEEL01: oracle_steel01_trial(m, c, t, eps); break;
        case STRUT_MAT_CONCRETE01: oracle_concrete01_trial(m, c, t, eps); break;
        default: oracle_elastic_trial(m, c, t, eps); break;
    }
}

/* Scalar uniaxial path used by material_path.mojo (ops.mojo:117-174): identical update rules,
 * plus the "eps == eps_t" early return of the scalar dispatch.  state holds committed (c) and
 * trial (t) copies; returns the trial stress/tangent. */
void oracle_material_path(const StrutUniMaterial* m, const double* strains, int n,
                          double* out) {
    OFiberState c, t;
    oracle_fiber_init(m, &c);
    t = c;
    for (int i = 0; i < n; ++i) {
        double eps = strains[i];
        int skip = eps == t.eps;
        if (!skip) {
            OFiberState next = t;
            oracle_fiber_trial(m, &c, &next, eps);
            t = next;
        }
        out[2 * i + 0] = t.sig;
        out[2 * i + 1] = t.tan;
        c = t; /* uniaxial_commit */
    }
}

/*
 * ORACLE -- test infrastructure only.  forceBeamColumn2d and dispBeamColumn2d element state
 * determination restated from Strut:
 *   _invert_3x3_values                 src/mojo/elements/force_beam_column2d.mojo:223-272
 *   batch section eval + 2x2 flex      src/mojo/sections/fiber2d.mojo:3042-3086
 *   _force_beam_column2d_exact_elastic_state      force_beam_column2d.mojo:608-732
 *   _force_beam_column2d_initial_basic_tangent    force_beam_column2d.mojo:735-801
 *   _force_beam_column2d_try_increment            force_beam_column2d.mojo:804-1189
 *   force_beam_column2d_global_tangent_and_internal force_beam_column2d.mojo:1418-1920
 *   dispBeamColumn2d                   src/mojo/elements/disp_beam_column2d.mojo:24-254
 *   2D transforms                      src/mojo/elements/utils.mojo:142-238
 *   recorder force from basic state    src/mojo/solver/run_case/helpers.mojo:1500-1600
 * Element loads are not modelled (section load terms are 0.0 and are still added, as Strut
 * adds its zero load arrays).
 */
#include "oracle_internal.h"

#include <math.h>
#include <string.h>

/* Passes of forceBeamColumn2d's subdivision loop in which every scheme failed (the increment
 * was cut back), over all elements since the library was loaded. */
static long g_subdivisions = 0;
long oracle_subdivisions(void) { return g_subdivisions; }

static int invert3(double a, double b, double c, double d, double e, double f, double g,
                   double h, double i, double k[9]) {
    double co00 = e * i - f * h;
    double co01 = -(d * i - f * g);
    double co02 = d * h - e * g;
    double co10 = -(b * i - c * h);
    double co11 = a * i - c * g;
    double co12 = -(a * h - b * g);
    double co20 = b * f - c * e;
    double co21 = -(a * f - c * d);
    double co22 = a * e - b * d;
    double det = a * co00 + b * co01 + c * co02;
    if (fabs(det) <= 1.0e-40) return 0;
    double inv_det = 1.0 / det;
    k[0] = co00 * inv_det;
    k[1] = co10 * inv_det;
    k[2] = co20 * inv_det;
    k[3] = co01 * inv_det;
    k[4] = co11 * inv_det;
    k[5] = co21 * inv_det;
    k[6] = co02 * inv_det;
    k[7] = co12 * inv_det;
    k[8] = co22 * inv_det;
    return 1;
}

static double max_abs3(double a, double b, double c) {
    double m = fabs(a);
    if (fabs(b) > m) m = fabs(b);
    if (fabs(c) > m) m = fabs(c);
    return m;
}

/* fiber_section2d_batch_eval_same_def: evaluates points in order, stops at the first
 * singular section (remaining points are not evaluated). */
static int batch_eval(OElement* e, const double* eps0, const double* kappa, double* N,
                      double* M, double* f00, double* f01, double* f11) {
    for (int ip = 0; ip < e->nip; ++ip) {
        double r[5];
        oracle_section_response(e->sec, &e->sst[ip], eps0[ip], kappa[ip], r);
        e->section_evals++;
        N[ip] = r[0];
        M[ip] = r[1];
        double det = r[2] * r[4] - r[3] * r[3];
        if (fabs(det) <= 1.0e-40) return 0;
        double inv_det = 1.0 / det;
        f00[ip] = r[4] * inv_det;
        f01[ip] = -r[3] * inv_det;
        f11[ip] = r[2] * inv_det;
    }
    return 1;
}

#define FLEX_ACCUM(F, wL, bmi, bmj, sf00, sf01, sf11)          \
    do {                                                       \
        double sf10_ = (sf01);                                 \
        F[0] += (wL) * (sf00);                                 \
        F[1] += (wL) * (sf01) * (bmi);                         \
        F[2] += (wL) * (sf01) * (bmj);                         \
        F[3] += (wL) * (bmi) * sf10_;                          \
        F[4] += (wL) * (bmi) * (sf11) * (bmi);                 \
        F[5] += (wL) * (bmi) * (sf11) * (bmj);                 \
        F[6] += (wL) * (bmj) * sf10_;                          \
        F[7] += (wL) * (bmj) * (sf11) * (bmi);                 \
        F[8] += (wL) * (bmj) * (sf11) * (bmj);                 \
    } while (0)

/* returns 1 and res = {q0,q1,q2,k00,k01,k02,k10,k11,k12,k22} on convergence */
static int fbc_try_increment(OElement* e, const double base[3], const double dv[3],
                             int scheme, double res[10]) {
    const OSection* sd = e->sec;
    int nip = e->nip;
    double L = e->L;
    double q0 = e->q[0], q1 = e->q[1], q2 = e->q[2];
    double t0 = base[0] + dv[0], t1 = base[1] + dv[1], t2 = base[2] + dv[2];
    if (!sd->init_valid) return 0;
    double vs_e[STRUT_MAX_INT_PTS] = {0}, vs_k[STRUT_MAX_INT_PTS] = {0};
    double sub_e[STRUT_MAX_INT_PTS], sub_k[STRUT_MAX_INT_PTS];
    double ssr_n[STRUT_MAX_INT_PTS], ssr_m[STRUT_MAX_INT_PTS];
    double fs00[STRUT_MAX_INT_PTS], fs01[STRUT_MAX_INT_PTS], fs11[STRUT_MAX_INT_PTS];
    for (int ip = 0; ip < nip; ++ip) {
        vs_e[ip] = e->eps0[ip];
        vs_k[ip] = e->kappa[ip];
    }
    if (!batch_eval(e, vs_e, vs_k, ssr_n, ssr_m, fs00, fs01, fs11)) return 0;
    for (int ip = 0; ip < nip; ++ip) {
        sub_e[ip] = vs_e[ip];
        sub_k[ip] = vs_k[ip];
    }
    double P[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int ip = 0; ip < nip; ++ip) {
        double xi = e->xi[ip], wL = e->w[ip] * L;
        double bmi = xi - 1.0, bmj = xi;
        FLEX_ACCUM(P, wL, bmi, bmj, fs00[ip], fs01[ip], fs11[ip]);
    }
    double pk[9];
    if (invert3(P[0], P[1], P[2], P[3], P[4], P[5], P[6], P[7], P[8], pk)) {
        q0 += (pk[0] * dv[0] + pk[1] * dv[1] + pk[2] * dv[2]);
        q1 += (pk[3] * dv[0] + pk[4] * dv[1] + pk[5] * dv[2]);
        q2 += (pk[6] * dv[0] + pk[7] * dv[1] + pk[8] * dv[2]);
    }
    int num_iters = scheme == 1 ? 100 : 10;
    for (int it = 0; it < num_iters; ++it) {
        e->local_iters++;
        double F[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        double vr0 = 0.0, vr1 = 0.0, vr2 = 0.0;
        int use_init = scheme == 1 || (scheme == 2 && it == 0);
        double pe[STRUT_MAX_INT_PTS], pkp[STRUT_MAX_INT_PTS];
        for (int ip = 0; ip < nip; ++ip) {
            double xi = e->xi[ip];
            double bmi = xi - 1.0, bmj = xi;
            double ss0 = q0 + 0.0;
            double ss1 = bmi * q1 + bmj * q2 + 0.0;
            double dss0 = ss0 - ssr_n[ip];
            double dss1 = ss1 - ssr_m[ip];
            double a00, a01, a11;
            if (use_init) {
                a00 = sd->f00;
                a01 = sd->f01;
                a11 = sd->f11;
            } else {
                a00 = fs00[ip];
                a01 = fs01[ip];
                a11 = fs11[ip];
            }
            double dvs0 = a00 * dss0 + a01 * dss1;
            double dvs1 = a01 * dss0 + a11 * dss1;
            pe[ip] = sub_e[ip] + dvs0;
            pkp[ip] = sub_k[ip] + dvs1;
        }
        double nN[STRUT_MAX_INT_PTS], nM[STRUT_MAX_INT_PTS];
        double n00[STRUT_MAX_INT_PTS], n01[STRUT_MAX_INT_PTS], n11[STRUT_MAX_INT_PTS];
        if (!batch_eval(e, pe, pkp, nN, nM, n00, n01, n11)) return 0;
        for (int ip = 0; ip < nip; ++ip) {
            double xi = e->xi[ip], wL = e->w[ip] * L;
            double bmi = xi - 1.0, bmj = xi;
            double ss0 = q0 + 0.0;
            double ss1 = bmi * q1 + bmj * q2 + 0.0;
            sub_e[ip] = pe[ip];
            sub_k[ip] = pkp[ip];
            ssr_n[ip] = nN[ip];
            ssr_m[ip] = nM[ip];
            fs00[ip] = n00[ip];
            fs01[ip] = n01[ip];
            fs11[ip] = n11[ip];
            double dr0 = ss0 - ssr_n[ip];
            double dr1 = ss1 - ssr_m[ip];
            double dvr0 = n00[ip] * dr0 + n01[ip] * dr1;
            double dvr1 = n01[ip] * dr0 + n11[ip] * dr1;
            FLEX_ACCUM(F, wL, bmi, bmj, n00[ip], n01[ip], n11[ip]);
            vr0 += wL * (pe[ip] + dvr0);
            vr1 += wL * bmi * (pkp[ip] + dvr1);
            vr2 += wL * bmj * (pkp[ip] + dvr1);
        }
        double k[9];
        if (!invert3(F[0], F[1], F[2], F[3], F[4], F[5], F[6], F[7], F[8], k)) return 0;
        double r0 = t0 - vr0, r1 = t1 - vr1, r2 = t2 - vr2;
        double dq0 = k[0] * r0 + k[1] * r1 + k[2] * r2;
        double dq1 = k[3] * r0 + k[4] * r1 + k[5] * r2;
        double dq2 = k[6] * r0 + k[7] * r1 + k[8] * r2;
        double work = fabs(r0 * dq0 + r1 * dq1 + r2 * dq2);
        q0 += dq0;
        q1 += dq1;
        q2 += dq2;
        if (work < 1.0e-12) {
            e->q[0] = q0;
            e->q[1] = q1;
            e->q[2] = q2;
            for (int ip = 0; ip < nip; ++ip) {
                e->eps0[ip] = sub_e[ip];
                e->kappa[ip] = sub_k[ip];
            }
            res[0] = q0; res[1] = q1; res[2] = q2;
            res[3] = k[0]; res[4] = k[1]; res[5] = k[2];
            res[6] = k[3]; res[7] = k[4]; res[8] = k[5];
            res[9] = k[8];
            return 1;
        }
    }
    return 0;
}

static int fbc_exact_elastic(OElement* e, const double v[3], double res[10]) {
    const OSection* sd = e->sec;
    if (!sd->init_valid) return 0;
    double L = e->L;
    double F[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double vl0 = 0.0, vl1 = 0.0, vl2 = 0.0;
    for (int ip = 0; ip < e->nip; ++ip) {
        double xi = e->xi[ip], wL = e->w[ip] * L;
        double bmi = xi - 1.0, bmj = xi;
        FLEX_ACCUM(F, wL, bmi, bmj, sd->f00, sd->f01, sd->f11);
        vl0 += wL * (sd->f00 * 0.0 + sd->f01 * 0.0);
        vl1 += wL * bmi * (sd->f01 * 0.0 + sd->f11 * 0.0);
        vl2 += wL * bmj * (sd->f01 * 0.0 + sd->f11 * 0.0);
    }
    double k[9];
    if (!invert3(F[0], F[1], F[2], F[3], F[4], F[5], F[6], F[7], F[8], k)) return 0;
    double r0 = v[0] - vl0, r1 = v[1] - vl1, r2 = v[2] - vl2;
    double q0 = k[0] * r0 + k[1] * r1 + k[2] * r2;
    double q1 = k[3] * r0 + k[4] * r1 + k[5] * r2;
    double q2 = k[6] * r0 + k[7] * r1 + k[8] * r2;
    for (int ip = 0; ip < e->nip; ++ip) {
        double xi = e->xi[ip];
        double bmi = xi - 1.0, bmj = xi;
        double axial = q0 + 0.0;
        double moment = bmi * q1 + bmj * q2 + 0.0;
        double eps0 = sd->f00 * axial + sd->f01 * moment;
        double kappa = sd->f01 * axial + sd->f11 * moment;
        e->eps0[ip] = eps0;
        e->kappa[ip] = kappa;
        double r[5];
        oracle_section_response(sd, &e->sst[ip], eps0, kappa, r);
        e->section_evals++;
    }
    e->q[0] = q0;
    e->q[1] = q1;
    e->q[2] = q2;
    res[0] = q0; res[1] = q1; res[2] = q2;
    res[3] = k[0]; res[4] = k[1]; res[5] = k[2];
    res[6] = k[3]; res[7] = k[4]; res[8] = k[5];
    res[9] = k[8];
    return 1;
}

static int fbc_initial_basic_tangent(const OElement* e, double k8[8]) {
    const OSection* sd = e->sec;
    if (!sd->init_valid) return 0;
    double F[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int ip = 0; ip < e->nip; ++ip) {
        double xi = e->xi[ip], wL = e->w[ip] * e->L;
        double bmi = xi - 1.0, bmj = xi;
        FLEX_ACCUM(F, wL, bmi, bmj, sd->f00, sd->f01, sd->f11);
    }
    double k[9];
    if (!invert3(F[0], F[1], F[2], F[3], F[4], F[5], F[6], F[7], F[8], k)) return 0;
    for (int i = 0; i < 6; ++i) k8[i] = k[i];
    k8[6] = k[7];
    k8[7] = k[8];
    return 1;
}

static void u_global_to_local(double c, double s, const double* ug, double* ul) {
    ul[0] = c * ug[0] + s * ug[1];
    ul[1] = -s * ug[0] + c * ug[1];
    ul[2] = ug[2];
    ul[3] = c * ug[3] + s * ug[4];
    ul[4] = -s * ug[3] + c * ug[4];
    ul[5] = ug[5];
}

static void k_local_to_global(double* k, double c, double s) {
    /* utils.mojo:175-238: columns 0,1,3,4 first, then rows 0,1,3,4 */
    for (int i = 0; i < 6; ++i) {
        double k0 = k[i * 6 + 0], k1 = k[i * 6 + 1], k3 = k[i * 6 + 3], k4 = k[i * 6 + 4];
        k[i * 6 + 0] = c * k0 - s * k1;
        k[i * 6 + 1] = s * k0 + c * k1;
        k[i * 6 + 3] = c * k3 - s * k4;
        k[i * 6 + 4] = s * k3 + c * k4;
    }
    for (int pair = 0; pair < 2; ++pair) {
        int r0 = pair == 0 ? 0 : 3, r1 = r0 + 1;
        double a[6], b[6];
        for (int j = 0; j < 6; ++j) {
            a[j] = k[r0 * 6 + j];
            b[j] = k[r1 * 6 + j];
        }
        for (int j = 0; j < 6; ++j) {
            k[r0 * 6 + j] = c * a[j] - s * b[j];
            k[r1 * 6 + j] = s * a[j] + c * b[j];
        }
    }
}

static void f_local_to_global(double* f, double c, double s) {
    double f0 = f[0], f1 = f[1], f3 = f[3], f4 = f[4];
    f[0] = c * f0 - s * f1;
    f[1] = s * f0 + c * f1;
    f[3] = c * f3 - s * f4;
    f[4] = s * f3 + c * f4;
}

static void basic_map(int col, double inv_L, double* a) {
    a[0] = a[1] = a[2] = 0.0;
    switch (col) {
        case 0: a[0] = -1.0; break;
        case 1: a[1] = inv_L; a[2] = inv_L; break;
        case 2: a[1] = 1.0; break;
        case 3: a[0] = 1.0; break;
        case 4: a[1] = -inv_L; a[2] = -inv_L; break;
        default: a[2] = 1.0; break;
    }
}

int oracle_fbc2d(OElement* e, const double ug[6], double k[36], double f[6]) {
    const OSection* sd = e->sec;
    double L = e->L;
    double inv_L = 1.0 / L;
    double c = e->c, s = e->s;
    double ul[6];
    u_global_to_local(c, s, ug, ul);
    double chord = (ul[4] - ul[1]) / L;
    double v[3] = {ul[3] - ul[0], ul[2] - chord, ul[5] - chord};
    double acc_v[3] = {e->v[0], e->v[1], e->v[2]};
    double acc_q[3] = {e->q[0], e->q[1], e->q[2]};
    double svs_e[STRUT_MAX_INT_PTS], svs_k[STRUT_MAX_INT_PTS];
    for (int ip = 0; ip < e->nip; ++ip) {
        svs_e[ip] = e->eps0[ip];
        svs_k[ip] = e->kappa[ip];
    }
    double rem[3] = {v[0] - acc_v[0], v[1] - acc_v[1], v[2] - acc_v[2]};
    double att[3] = {rem[0], rem[1], rem[2]};
    int converged = 0;
    int best_ok = 0;
    double best[10];
    if (sd->nonlinear_count == 0) {
        double solved[10];
        if (fbc_exact_elastic(e, v, solved)) {
            acc_v[0] = v[0]; acc_v[1] = v[1]; acc_v[2] = v[2];
            e->v[0] = v[0]; e->v[1] = v[1]; e->v[2] = v[2];
            acc_q[0] = solved[0]; acc_q[1] = solved[1]; acc_q[2] = solved[2];
            for (int ip = 0; ip < e->nip; ++ip) {
                svs_e[ip] = e->eps0[ip];
                svs_k[ip] = e->kappa[ip];
            }
            converged = 1;
            rem[0] = rem[1] = rem[2] = 0.0;
            memcpy(best, solved, sizeof(best));
            best_ok = 1;
        }
    }
    const double zero[3] = {0.0, 0.0, 0.0};
    if (!converged && max_abs3(rem[0], rem[1], rem[2]) <= 1.0e-16) {
        for (int scheme = 0; scheme < 3; ++scheme) {
            e->q[0] = acc_q[0]; e->q[1] = acc_q[1]; e->q[2] = acc_q[2];
            for (int ip = 0; ip < e->nip; ++ip) {
                e->eps0[ip] = svs_e[ip];
                e->kappa[ip] = svs_k[ip];
            }
            e->v[0] = acc_v[0]; e->v[1] = acc_v[1]; e->v[2] = acc_v[2];
            double solved[10];
            if (!fbc_try_increment(e, acc_v, zero, scheme, solved)) continue;
            memcpy(best, solved, sizeof(best));
            best_ok = 1;
            converged = 1;
            break;
        }
    } else if (!converged) {
        int num_subdivide = 1;
        int guard = 0;
        while (num_subdivide <= 4 && guard < 10000) {
            ++guard;
            double tv[3] = {acc_v[0] + att[0], acc_v[1] + att[1], acc_v[2] + att[2]};
            int scheme_success = 0;
            for (int scheme = 0; scheme < 3; ++scheme) {
                e->q[0] = acc_q[0]; e->q[1] = acc_q[1]; e->q[2] = acc_q[2];
                for (int ip = 0; ip < e->nip; ++ip) {
                    e->eps0[ip] = svs_e[ip];
                    e->kappa[ip] = svs_k[ip];
                }
                e->v[0] = acc_v[0]; e->v[1] = acc_v[1]; e->v[2] = acc_v[2];
                double solved[10];
                if (!fbc_try_increment(e, acc_v, att, scheme, solved)) continue;
                acc_v[0] = tv[0]; acc_v[1] = tv[1]; acc_v[2] = tv[2];
                e->v[0] = tv[0]; e->v[1] = tv[1]; e->v[2] = tv[2];
                acc_q[0] = solved[0]; acc_q[1] = solved[1]; acc_q[2] = solved[2];
                for (int ip = 0; ip < e->nip; ++ip) {
                    svs_e[ip] = e->eps0[ip];
                    svs_k[ip] = e->kappa[ip];
                }
                memcpy(best, solved, sizeof(best));
                best_ok = 1;
                rem[0] = v[0] - acc_v[0];
                rem[1] = v[1] - acc_v[1];
                rem[2] = v[2] - acc_v[2];
                if (max_abs3(rem[0], rem[1], rem[2]) <= 1.0e-12) {
                    converged = 1;
                } else {
                    att[0] = rem[0]; att[1] = rem[1]; att[2] = rem[2];
                    num_subdivide = 1;
                }
                scheme_success = 1;
                break;
            }
            if (converged) break;
            if (scheme_success) continue;
            att[0] /= 10.0;
            att[1] /= 10.0;
            att[2] /= 10.0;
            num_subdivide += 1;
            __atomic_add_fetch(&g_subdivisions, 1, __ATOMIC_RELAXED);
        }
    }
    if (!converged) {
        e->q[0] = acc_q[0]; e->q[1] = acc_q[1]; e->q[2] = acc_q[2];
        for (int ip = 0; ip < e->nip; ++ip) {
            e->eps0[ip] = svs_e[ip];
            e->kappa[ip] = svs_k[ip];
        }
        e->v[0] = acc_v[0]; e->v[1] = acc_v[1]; e->v[2] = acc_v[2];
        for (int ip = 0; ip < e->nip; ++ip) {
            double r[5];
            oracle_section_response(sd, &e->sst[ip], svs_e[ip], svs_k[ip], r);
            e->section_evals++;
        }
    }
    if (!best_ok) {
        double k8[8];
        if (!fbc_initial_basic_tangent(e, k8)) return STRUT_ELEMENT_FAILED;
        best[0] = e->q[0]; best[1] = e->q[1]; best[2] = e->q[2];
        best[3] = k8[0]; best[4] = k8[1]; best[5] = k8[2];
        best[6] = k8[3]; best[7] = k8[4]; best[8] = k8[5];
        best[9] = k8[7];
    }
    double q0 = best[0], q1 = best[1], q2 = best[2];
    double kb[9] = {best[3], best[4], best[5], best[6], best[7], best[8], best[5], best[8],
                    best[9]};
    for (int a = 0; a < 6; ++a) {
        double av[3];
        basic_map(a, inv_L, av);
        for (int b = 0; b < 6; ++b) {
            double bv[3];
            basic_map(b, inv_L, bv);
            k[a * 6 + b] = av[0] * (kb[0] * bv[0] + kb[1] * bv[1] + kb[2] * bv[2]) +
                           av[1] * (kb[3] * bv[0] + kb[4] * bv[1] + kb[5] * bv[2]) +
                           av[2] * (kb[6] * bv[0] + kb[7] * bv[1] + kb[8] * bv[2]);
        }
    }
    if (e->desc->geom == STRUT_GEOM_PDELTA) {
        double ql = q0 * inv_L;
        k[1 * 6 + 1] += ql;
        k[4 * 6 + 4] += ql;
        k[1 * 6 + 4] -= ql;
        k[4 * 6 + 1] -= ql;
    }
    f[0] = -q0;
    f[1] = (q1 + q2) * inv_L;
    f[2] = q1;
    f[3] = q0;
    f[4] = -(q1 + q2) * inv_L;
    f[5] = q2;
    f[0] += 0.0;
    f[1] += 0.0;
    f[4] += 0.0;
    if (e->desc->geom == STRUT_GEOM_PDELTA) {
        double ps = (ul[1] - ul[4]) * q0 * inv_L;
        f[1] += ps;
        f[4] -= ps;
    }
    k_local_to_global(k, c, s);
    f_local_to_global(f, c, s);
    return STRUT_OK;
}

void oracle_fbc2d_force_from_basic(const OElement* e, const double ug[6], double f[6]) {
    /* helpers.mojo:1500-1600: L = sqrt(dx*dx+dy*dy), c = dx/L, s = dy/L */
    double L = e->L_sync;
    double c = e->c_sync, s = e->s_sync;
    double inv_L = 1.0 / L;
    double q0 = e->q[0], q1 = e->q[1], q2 = e->q[2];
    double shear = (q1 + q2) * inv_L;
    f[0] = -q0 + 0.0;
    f[1] = shear + 0.0;
    f[2] = q1;
    f[3] = q0;
    f[4] = -shear + 0.0;
    f[5] = q2;
    if (e->desc->geom == STRUT_GEOM_PDELTA) {
        double ul[6];
        u_global_to_local(c, s, ug, ul);
        double ps = (ul[1] - ul[4]) * q0 * inv_L;
        f[1] += ps;
        f[4] -= ps;
    }
    f_local_to_global(f, c, s);
}

static double curv_shape(int idx, double inv_L, double inv_L_sq, double xi) {
    switch (idx) {
        case 1: return (-6.0 + 12.0 * xi) * inv_L_sq;
        case 2: return (-4.0 + 6.0 * xi) * inv_L;
        case 4: return (6.0 - 12.0 * xi) * inv_L_sq;
        case 5: return (-2.0 + 6.0 * xi) * inv_L;
        default: return 0.0;
    }
}

static double axial_shape(int idx, double inv_L) {
    if (idx == 0) return -inv_L;
    if (idx == 3) return inv_L;
    return 0.0;
}

int oracle_dbc2d(OElement* e, const double ug[6], double k[36], double f[6]) {
    double L = e->L;
    double c = e->c_div, s = e->s_div;
    double inv_L = 1.0 / L;
    double inv_L_sq = inv_L * inv_L;
    double ul[6];
    u_global_to_local(c, s, ug, ul);
    memset(k, 0, sizeof(double) * 36);
    memset(f, 0, sizeof(double) * 6);
    double axial_avg = 0.0;
    for (int ip = 0; ip < e->nip; ++ip) {
        double xi = e->xi[ip], weight = e->w[ip];
        double b1 = curv_shape(1, inv_L, inv_L_sq, xi);
        double b2 = curv_shape(2, inv_L, inv_L_sq, xi);
        double b4 = curv_shape(4, inv_L, inv_L_sq, xi);
        double b5 = curv_shape(5, inv_L, inv_L_sq, xi);
        double eps0 = (-inv_L) * ul[0] + inv_L * ul[3];
        double kappa = b1 * ul[1] + b2 * ul[2] + b4 * ul[4] + b5 * ul[5];
        e->eps0[ip] = eps0;
        e->kappa[ip] = kappa;
        double r[5];
        oracle_section_response(e->sec, &e->sst[ip], eps0, kappa, r);
        e->section_evals++;
        double wL = weight * L;
        axial_avg += weight * r[0];
        for (int a = 0; a < 6; ++a) {
            double ban = axial_shape(a, inv_L);
            double bam = curv_shape(a, inv_L, inv_L_sq, xi);
            f[a] += wL * (ban * r[0] + bam * r[1]);
            for (int b = 0; b < 6; ++b) {
                double bbn = axial_shape(b, inv_L);
                double bbm = curv_shape(b, inv_L, inv_L_sq, xi);
                double dN = r[2] * bbn + r[3] * bbm;
                double dM = r[3] * bbn + r[4] * bbm;
                k[a * 6 + b] += wL * (ban * dN + bam * dM);
            }
        }
    }
    if (e->desc->geom == STRUT_GEOM_PDELTA) {
        double al = axial_avg / L;
        k[1 * 6 + 1] += al;
        k[4 * 6 + 4] += al;
        k[1 * 6 + 4] -= al;
        k[4 * 6 + 1] -= al;
        double ps = (ul[1] - ul[4]) * al;
        f[1] += ps;
        f[4] -= ps;
    }
    k_local_to_global(k, c, s);
    f_local_to_global(f, c, s);
    return STRUT_OK;
}

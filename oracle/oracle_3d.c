/*
 * ORACLE -- test infrastructure only.  FiberSection3d, dispBeamColumn3d and forceBeamColumn3d
 * restated from Strut (paths relative to the Strut project root):
 *   FiberSection3d definition     src/mojo/sections/fiber3d.mojo:156-188 (elastic and
 *                                 nonlinear fibers split, each in fiber order), centroid
 *                                 633-720 (area-weighted, accumulated in fiber order)
 *   elastic family response       fiber3d.mojo:191-256 (vectorize over W-wide chunks, each
 *                                 chunk reduced by a halving tree, scalar remainder; the
 *                                 uniform-modulus k12 = k13 = 0 quirk)
 *   set_trial_from_offset         fiber3d.mojo:769-836 (nonlinear fibers one by one through
 *                                 uniaxial_set_trial_strain, materials/uniaxial/ops.mojo:
 *                                 10-60, 117-150, with its eps == eps_t early return)
 *   local axes from vecxz         src/mojo/elements/utils.mojo:48-140,
 *                                 elements/force_beam_column3d.mojo:172-222, 510-547
 *   dispBeamColumn3d              src/mojo/elements/beam_column3d_nonlinear.mojo:81-172,
 *                                 357-575 (reached through disp_beam_column3d.mojo and the
 *                                 frame3d assembly, solver/assembly/
 *                                 stiffness_internal_frame3d.mojo:336-634), linalg.mojo:6-36
 *   forceBeamColumn3d             force_beam_column3d.mojo:340-386 (transforms), 419-464
 *                                 (basic coefficients), 679-728 (3x3 inverse), 788-868 (5x5
 *                                 Gauss-Jordan, stiffness transform), 1093-1118 (section
 *                                 flexibility), 1149-1201, 1203-1607 (try_increment),
 *                                 1610-1622 (basic state), 2549-2990 (element entry)
 * Element loads are not modelled: their zero terms are still added where Strut adds them.
 */
#include "oracle_internal.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- FiberSection3d ------------------------------------------------------------------ */

int oracle_section3d_build(OSection3d* sd, const StrutUniMaterial* mats, int nmat,
                           const StrutFiber* fibers, int off, int nfib) {
    memset(sd, 0, sizeof(*sd));
    sd->mats = mats;
    sd->W = oracle_get_simd_width();
    sd->nfib = nfib;
    if (nfib <= 0) return STRUT_BAD_ARG;
    double area_sum = 0.0, qy_sum = 0.0, qz_sum = 0.0;
    for (int i = 0; i < nfib; ++i) {
        const StrutFiber* f = &fibers[off + i];
        if (f->material < 0 || f->material >= nmat) return STRUT_BAD_ARG;
        int t = mats[f->material].type;
        if (t != STRUT_MAT_ELASTIC && t != STRUT_MAT_STEEL01 && t != STRUT_MAT_STEEL02 &&
            t != STRUT_MAT_CONCRETE02 && t != STRUT_MAT_CONCRETE01)
            return STRUT_UNSUPPORTED;
        area_sum += f->area;
        qy_sum += f->area * f->z;
        qz_sum += f->area * f->y;
    }
    if (area_sum <= 0.0) return STRUT_BAD_ARG;
    sd->y_bar = qz_sum / area_sum;
    sd->z_bar = qy_sum / area_sum;
    sd->el_y = (double*)calloc(nfib, sizeof(double));
    sd->el_z = (double*)calloc(nfib, sizeof(double));
    sd->el_a = (double*)calloc(nfib, sizeof(double));
    sd->el_e = (double*)calloc(nfib, sizeof(double));
    sd->nl_y = (double*)calloc(nfib, sizeof(double));
    sd->nl_z = (double*)calloc(nfib, sizeof(double));
    sd->nl_a = (double*)calloc(nfib, sizeof(double));
    sd->nl_mat = (int*)calloc(nfib, sizeof(int));
    for (int i = 0; i < nfib; ++i) {
        const StrutFiber* f = &fibers[off + i];
        const StrutUniMaterial* m = &mats[f->material];
        double y_rel = f->y - sd->y_bar;
        double z_rel = f->z - sd->z_bar;
        if (m->type == STRUT_MAT_ELASTIC) {
            sd->el_y[sd->n_el] = y_rel;
            sd->el_z[sd->n_el] = z_rel;
            sd->el_a[sd->n_el] = f->area;
            sd->el_e[sd->n_el] = oracle_initial_tangent(m);
            sd->n_el++;
        } else {
            sd->nl_y[sd->n_nl] = y_rel;
            sd->nl_z[sd->n_nl] = z_rel;
            sd->nl_a[sd->n_nl] = f->area;
            sd->nl_mat[sd->n_nl] = f->material;
            sd->n_nl++;
        }
    }
    return STRUT_OK;
}

void oracle_section3d_free(OSection3d* sd) {
    free(sd->el_y); free(sd->el_z); free(sd->el_a); free(sd->el_e);
    free(sd->nl_y); free(sd->nl_z); free(sd->nl_a); free(sd->nl_mat);
    memset(sd, 0, sizeof(*sd));
}

void oracle_section3d_state_alloc(const OSection3d* sd, OSecState* st) {
    /* only the nonlinear fibers carry history that the response reads */
    int n = sd->n_nl;
    st->n = n;
    st->c = (OFiberState*)calloc(n + 1, sizeof(OFiberState));
    st->t = (OFiberState*)calloc(n + 1, sizeof(OFiberState));
    for (int k = 0; k < n; ++k) oracle_fiber_init(&sd->mats[sd->nl_mat[k]], &st->c[k]);
    memcpy(st->t, st->c, sizeof(OFiberState) * (n + 1));
}

/* uniaxial_set_trial_strain (ops.mojo:117-150): a strain equal to the current trial strain
 * keeps the trial state. */
static void scalar_trial(const StrutUniMaterial* m, OFiberState* c, OFiberState* t, double eps) {
    if (eps == t->eps) return;
    OFiberState next = *t;
    oracle_fiber_trial(m, c, &next, eps);
    *t = next;
}

void oracle_section3d_response(const OSection3d* sd, OSecState* st, double eps0, double ky,
                               double kz, double out[9]) {
    int W = sd->W;
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double lane[9][16];
    int i = 0;
    for (; i + W <= sd->n_el; i += W) {
        for (int l = 0; l < W; ++l) {
            double y = sd->el_y[i + l], z = sd->el_z[i + l];
            double ks = sd->el_e[i + l] * sd->el_a[i + l];
            double fs = ks * (eps0 + z * ky - y * kz);
            lane[0][l] = fs;
            lane[1][l] = fs * z;
            lane[2][l] = -fs * y;
            lane[3][l] = ks;
            lane[4][l] = ks * z;
            lane[5][l] = -ks * y;
            lane[6][l] = ks * z * z;
            lane[7][l] = -ks * z * y;
            lane[8][l] = ks * y * y;
        }
        for (int c = 0; c < 9; ++c) acc[c] += oracle_tree_reduce(lane[c], W);
    }
    for (; i < sd->n_el; ++i) {
        double y = sd->el_y[i], z = sd->el_z[i];
        double ks = sd->el_e[i] * sd->el_a[i];
        double fs = ks * (eps0 + z * ky - y * kz);
        acc[0] += fs;
        acc[1] += fs * z;
        acc[2] += -fs * y;
        acc[3] += ks;
        acc[4] += ks * z;
        acc[5] += -ks * y;
        acc[6] += ks * z * z;
        acc[7] += -ks * z * y;
        acc[8] += ks * y * y;
    }
    if (sd->n_el > 0) {
        int uniform = 1;
        for (int j = 1; j < sd->n_el; ++j)
            if (sd->el_e[j] != sd->el_e[0]) {
                uniform = 0;
                break;
            }
        if (uniform) {
            acc[4] = 0.0;
            acc[5] = 0.0;
        }
    }
    for (int k = 0; k < sd->n_nl; ++k) {
        double y = sd->nl_y[k], z = sd->nl_z[k];
        double eps = eps0 + z * ky - y * kz;
        scalar_trial(&sd->mats[sd->nl_mat[k]], &st->c[k], &st->t[k], eps);
        double a = sd->nl_a[k];
        double fs = st->t[k].sig * a;
        double ks = st->t[k].tan * a;
        acc[0] += fs;
        acc[1] += fs * z;
        acc[2] += -fs * y;
        acc[3] += ks;
        acc[4] += ks * z;
        acc[5] += -ks * y;
        acc[6] += ks * z * z;
        acc[7] += -ks * z * y;
        acc[8] += ks * y * y;
    }
    for (int c = 0; c < 9; ++c) out[c] = acc[c];
}

/* section_path.mojo:463-556: one FiberSection3d along (eps0, ky, kz) points, commit after
 * each.  out: npts x 9. */
int oracle_section3d_path(const StrutUniMaterial* mats, int nmat, const StrutFiber* fibers,
                          int nfib, const double* path, int npts, double* out) {
    OSection3d sd;
    int rc = oracle_section3d_build(&sd, mats, nmat, fibers, 0, nfib);
    if (rc != STRUT_OK) {
        oracle_section3d_free(&sd);
        return rc;
    }
    OSecState st;
    oracle_section3d_state_alloc(&sd, &st);
    for (int p = 0; p < npts; ++p) {
        oracle_section3d_response(&sd, &st, path[3 * p], path[3 * p + 1], path[3 * p + 2],
                                  out + 9 * p);
        oracle_section_commit(&st);
    }
    oracle_section_state_free(&st);
    oracle_section3d_free(&sd);
    return STRUT_OK;
}

/* ---- geometry -------------------------------------------------------------------------- */

int oracle_rotation3d(const double x1[3], const double x2[3], int has_vecxz, const double* vxz,
                      double R[9]) {
    double dx = x2[0] - x1[0], dy = x2[1] - x1[1], dz = x2[2] - x1[2];
    double L = sqrt(dx * dx + dy * dy + dz * dz);
    if (L == 0.0) return STRUT_BAD_ARG;
    double n = sqrt(dx * dx + dy * dy + dz * dz);
    double lx = dx / n, ly = dy / n, lz = dz / n;
    double vx, vy, vz;
    if (has_vecxz) {
        vx = vxz[0];
        vy = vxz[1];
        vz = vxz[2];
    } else {
        vx = 1.0; vy = 0.0; vz = 0.0;
        if (fabs(lx * vx + ly * vy + lz * vz) >= 0.9) {
            vx = 0.0; vy = 1.0; vz = 0.0;
            if (fabs(lx * vx + ly * vy + lz * vz) >= 0.9) {
                vx = 0.0; vy = 0.0; vz = 1.0;
            }
        }
    }
    double yx = vy * lz - vz * ly;
    double yy = vz * lx - vx * lz;
    double yz = vx * ly - vy * lx;
    double yn = sqrt(yx * yx + yy * yy + yz * yz);
    if (yn == 0.0) return STRUT_BAD_ARG;
    yx /= yn;
    yy /= yn;
    yz /= yn;
    R[0] = lx; R[1] = ly; R[2] = lz;
    R[3] = yx; R[4] = yy; R[5] = yz;
    R[6] = ly * yz - lz * yy;
    R[7] = lz * yx - lx * yz;
    R[8] = lx * yy - ly * yx;
    return STRUT_OK;
}

/* rotation used by one element call: the displaced ends for Corotational */
static int element_rotation(const OElement* e, const double ug[12], double R[9]) {
    if (e->desc->geom == STRUT_GEOM_COROTATIONAL) {
        double a[3] = {e->x1[0] + ug[0], e->x1[1] + ug[1], e->x1[2] + ug[2]};
        double b[3] = {e->x2[0] + ug[6], e->x2[1] + ug[7], e->x2[2] + ug[8]};
        return oracle_rotation3d(a, b, e->desc->has_vecxz, e->desc->vecxz, R);
    }
    memcpy(R, e->R, sizeof(double) * 9);
    return STRUT_OK;
}

static void u_to_local(const double R[9], const double ug[12], double ul[12]) {
    for (int b = 0; b < 4; ++b) {
        int o = 3 * b;
        double g0 = ug[o], g1 = ug[o + 1], g2 = ug[o + 2];
        for (int i = 0; i < 3; ++i) ul[o + i] = R[3 * i] * g0 + R[3 * i + 1] * g1 + R[3 * i + 2] * g2;
    }
}

static void f_to_global(const double R[9], const double fl[12], double fg[12]) {
    for (int b = 0; b < 4; ++b) {
        int o = 3 * b;
        double l0 = fl[o], l1 = fl[o + 1], l2 = fl[o + 2];
        for (int i = 0; i < 3; ++i) fg[o + i] = R[i] * l0 + R[3 + i] * l1 + R[6 + i] * l2;
    }
}

/* _beam3d_transform_stiffness_local_to_global_flat (force_beam_column3d.mojo:836-868) */
static void k_to_global_flat(const double R[9], const double* kl, double* kg) {
    double work[144];
    for (int rb = 0; rb < 4; ++rb) {
        int ro = 3 * rb;
        for (int cb = 0; cb < 4; ++cb) {
            int co = 3 * cb;
            for (int i = 0; i < 3; ++i) {
                int base = (ro + i) * 12 + co;
                double s0 = kl[base], s1 = kl[base + 1], s2 = kl[base + 2];
                for (int j = 0; j < 3; ++j) work[base + j] = s0 * R[j] + s1 * R[3 + j] + s2 * R[6 + j];
            }
        }
    }
    for (int rb = 0; rb < 4; ++rb) {
        int ro = 3 * rb;
        for (int col = 0; col < 12; ++col)
            for (int i = 0; i < 3; ++i)
                kg[(ro + i) * 12 + col] = R[i] * work[ro * 12 + col] +
                                          R[3 + i] * work[(ro + 1) * 12 + col] +
                                          R[6 + i] * work[(ro + 2) * 12 + col];
    }
}

/* matmul(transpose(T), matmul(k, T)) with T = blockdiag(R, R, R, R) (linalg.mojo:20-36:
 * i-k-j order, zero a[i][k] skipped) */
static void k_to_global_matmul(const double R[9], const double* kl, double* kg) {
    double T[144], kt[144];
    memset(T, 0, sizeof(T));
    for (int b = 0; b < 4; ++b)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) T[(3 * b + i) * 12 + 3 * b + j] = R[3 * i + j];
    memset(kt, 0, sizeof(kt));
    for (int i = 0; i < 12; ++i)
        for (int k = 0; k < 12; ++k) {
            double aik = kl[i * 12 + k];
            if (aik == 0.0) continue;
            for (int j = 0; j < 12; ++j) kt[i * 12 + j] += aik * T[k * 12 + j];
        }
    memset(kg, 0, sizeof(double) * 144);
    for (int i = 0; i < 12; ++i)
        for (int k = 0; k < 12; ++k) {
            double aik = T[k * 12 + i];
            if (aik == 0.0) continue;
            for (int j = 0; j < 12; ++j) kg[i * 12 + j] += aik * kt[k * 12 + j];
        }
}

/* _beam3d_transform_f_local_to_global (beam_column3d_nonlinear.mojo:105-115) */
static void f_to_global_dense(const double R[9], const double fl[12], double fg[12]) {
    double T[144];
    memset(T, 0, sizeof(T));
    for (int b = 0; b < 4; ++b)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) T[(3 * b + i) * 12 + 3 * b + j] = R[3 * i + j];
    for (int i = 0; i < 12; ++i) {
        double sum = 0.0;
        for (int j = 0; j < 12; ++j) sum += T[j * 12 + i] * fl[j];
        fg[i] = sum;
    }
}

static void u_to_local_dense(const double R[9], const double ug[12], double ul[12]) {
    double T[144];
    memset(T, 0, sizeof(T));
    for (int b = 0; b < 4; ++b)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) T[(3 * b + i) * 12 + 3 * b + j] = R[3 * i + j];
    for (int i = 0; i < 12; ++i) {
        double sum = 0.0;
        for (int j = 0; j < 12; ++j) sum += T[i * 12 + j] * ug[j];
        ul[i] = sum;
    }
}

/* Section kinematics of a dispBeamColumn3d at integration point ip for the section recorders
 * (beam_column3d_nonlinear.mojo:578-640): out = eps0, kappa_y, kappa_z, twist. */
int oracle_dbc3d_section_kinematics(const OElement* e, const double ug[12], int ip, double out[4]) {
    double dx = e->x2[0] - e->x1[0], dy = e->x2[1] - e->x1[1], dz = e->x2[2] - e->x1[2];
    double L = sqrt(dx * dx + dy * dy + dz * dz);
    if (L == 0.0) return STRUT_BAD_ARG;
    double R[9];
    int rc = element_rotation(e, ug, R);
    if (rc != STRUT_OK) return rc;
    double ul[12];
    u_to_local_dense(R, ug, ul);
    double xi = e->xi[ip];
    double inv_L = 1.0 / L;
    out[0] = (-inv_L) * ul[0] + inv_L * ul[6];
    out[1] = ((-6.0 + 12.0 * xi) / (L * L)) * ul[2] + ((4.0 - 6.0 * xi) / L) * ul[4] +
             ((6.0 - 12.0 * xi) / (L * L)) * ul[8] + ((2.0 - 6.0 * xi) / L) * ul[10];
    out[2] = ((-6.0 + 12.0 * xi) / (L * L)) * ul[1] + ((-4.0 + 6.0 * xi) / L) * ul[5] +
             ((6.0 - 12.0 * xi) / (L * L)) * ul[7] + ((-2.0 + 6.0 * xi) / L) * ul[11];
    out[3] = (ul[9] - ul[3]) / L;
    return STRUT_OK;
}

/* ---- dispBeamColumn3d (beam_column3d_nonlinear.mojo:357-575) ---------------------------- */

int oracle_dbc3d(OElement* e, const double ug[12], double k[144], double f[12]) {
    double dx = e->x2[0] - e->x1[0], dy = e->x2[1] - e->x1[1], dz = e->x2[2] - e->x1[2];
    double L = sqrt(dx * dx + dy * dy + dz * dz);
    if (L == 0.0) return STRUT_BAD_ARG;
    double R[9];
    int rc = element_rotation(e, ug, R);
    if (rc != STRUT_OK) return rc;
    double ul[12];
    u_to_local_dense(R, ug, ul);
    double kl[144], fl[12];
    memset(kl, 0, sizeof(kl));
    memset(fl, 0, sizeof(fl));
    double q5 = 0.0;
    double axial_avg = 0.0;
    for (int ip = 0; ip < e->nip; ++ip) {
        double xi = e->xi[ip], weight = e->w[ip];
        double wL = weight * L;
        double inv_L = 1.0 / L;
        double eps0 = (-inv_L) * ul[0] + inv_L * ul[6];
        double ky = ((-6.0 + 12.0 * xi) / (L * L)) * ul[2] + ((4.0 - 6.0 * xi) / L) * ul[4] +
                    ((6.0 - 12.0 * xi) / (L * L)) * ul[8] + ((2.0 - 6.0 * xi) / L) * ul[10];
        double kz = ((-6.0 + 12.0 * xi) / (L * L)) * ul[1] + ((-4.0 + 6.0 * xi) / L) * ul[5] +
                    ((6.0 - 12.0 * xi) / (L * L)) * ul[7] + ((-2.0 + 6.0 * xi) / L) * ul[11];
        e->eps0[ip] = eps0;
        e->ky[ip] = ky;
        e->kz[ip] = kz;
        double r[9];
        oracle_section3d_response(e->sec3, &e->sst[ip], eps0, ky, kz, r);
        e->section_evals++;
        axial_avg += weight * r[0];
        double be[12] = {0}, by[12] = {0}, bz[12] = {0};
        be[0] = -1.0 / L;
        be[6] = 1.0 / L;
        by[2] = (-6.0 + 12.0 * xi) / (L * L);
        by[4] = (4.0 - 6.0 * xi) / L;
        by[8] = (6.0 - 12.0 * xi) / (L * L);
        by[10] = (2.0 - 6.0 * xi) / L;
        bz[1] = (-6.0 + 12.0 * xi) / (L * L);
        bz[5] = (-4.0 + 6.0 * xi) / L;
        bz[7] = (6.0 - 12.0 * xi) / (L * L);
        bz[11] = (-2.0 + 6.0 * xi) / L;
        for (int a = 0; a < 12; ++a) {
            fl[a] += wL * (be[a] * r[0] + by[a] * r[1] + bz[a] * r[2]);
            for (int b = 0; b < 12; ++b) {
                double dN = r[3] * be[b] + r[4] * by[b] + r[5] * bz[b];
                double dMy = r[4] * be[b] + r[6] * by[b] + r[7] * bz[b];
                double dMz = r[5] * be[b] + r[7] * by[b] + r[8] * bz[b];
                kl[a * 12 + b] += wL * (be[a] * dN + by[a] * dMy + bz[a] * dMz);
            }
        }
    }
    if (e->G > 0.0 && e->J > 0.0) {
        double tk = e->G * e->J / L;
        kl[3 * 12 + 3] += tk;
        kl[3 * 12 + 9] -= tk;
        kl[9 * 12 + 3] -= tk;
        kl[9 * 12 + 9] += tk;
        q5 = tk * (ul[9] - ul[3]);
    }
    if (e->desc->geom == STRUT_GEOM_PDELTA || e->desc->geom == STRUT_GEOM_COROTATIONAL) {
        double nl = axial_avg / L;
        kl[1 * 12 + 1] += nl;
        kl[1 * 12 + 7] -= nl;
        kl[7 * 12 + 1] -= nl;
        kl[7 * 12 + 7] += nl;
        kl[2 * 12 + 2] += nl;
        kl[2 * 12 + 8] -= nl;
        kl[8 * 12 + 2] -= nl;
        kl[8 * 12 + 8] += nl;
    }
    for (int a = 0; a < 12; ++a) {
        double c5 = a == 3 ? -1.0 : (a == 9 ? 1.0 : 0.0);
        fl[a] += c5 * q5;
    }
    k_to_global_matmul(R, kl, k);
    f_to_global_dense(R, fl, f);
    return STRUT_OK;
}

/* ---- forceBeamColumn3d -------------------------------------------------------------------- */

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

/* _fiber_section3d_response_flexibility (force_beam_column3d.mojo:1093-1118):
 * fs = {f11, f12, f13, f22, f23, f33} of the inverse of the symmetric section tangent */
static int section_flex(const double r[9], double fs[6]) {
    double k[9];
    if (!invert3(r[3], r[4], r[5], r[4], r[6], r[7], r[5], r[7], r[8], k)) return 0;
    fs[0] = k[0];
    fs[1] = k[1];
    fs[2] = k[2];
    fs[3] = k[4];
    fs[4] = k[5];
    fs[5] = k[8];
    return 1;
}

/* _invert_5x5_flat_into (force_beam_column3d.mojo:788-834) */
static int invert5(double* a, double* inv) {
    for (int i = 0; i < 25; ++i) inv[i] = 0.0;
    for (int i = 0; i < 5; ++i) inv[i * 5 + i] = 1.0;
    for (int i = 0; i < 5; ++i) {
        int pivot = i;
        double max_val = fabs(a[i * 5 + i]);
        for (int r = i + 1; r < 5; ++r) {
            double v = fabs(a[r * 5 + i]);
            if (v > max_val) {
                max_val = v;
                pivot = r;
            }
        }
        if (max_val <= 1.0e-40) return 0;
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
        double piv = a[i * 5 + i];
        for (int c = 0; c < 5; ++c) {
            a[i * 5 + c] /= piv;
            inv[i * 5 + c] /= piv;
        }
        for (int r = 0; r < 5; ++r) {
            if (r == i) continue;
            double factor = a[r * 5 + i];
            if (factor == 0.0) continue;
            for (int c = 0; c < 5; ++c) {
                a[r * 5 + c] -= factor * a[i * 5 + c];
                inv[r * 5 + c] -= factor * inv[i * 5 + c];
            }
        }
    }
    return 1;
}

/* _beam3d_local_basic_coeff (force_beam_column3d.mojo:419-464) */
static double basic_coeff(int row, int col, double inv_L) {
    switch (row) {
        case 0: return col == 0 ? -1.0 : (col == 6 ? 1.0 : 0.0);
        case 1: return col == 1 ? inv_L : (col == 5 ? 1.0 : (col == 7 ? -inv_L : 0.0));
        case 2: return col == 1 ? inv_L : (col == 7 ? -inv_L : (col == 11 ? 1.0 : 0.0));
        case 3: return col == 2 ? -inv_L : (col == 4 ? 1.0 : (col == 8 ? inv_L : 0.0));
        case 4: return col == 2 ? -inv_L : (col == 8 ? inv_L : (col == 10 ? 1.0 : 0.0));
        default: return col == 3 ? -1.0 : (col == 9 ? 1.0 : 0.0);
    }
}

/* Section-resultant component of basic force a: 0 = N, 1 = My, 2 = Mz (B rows of
 * force_beam_column3d.mojo:1461-1497), with its interpolation factor. */
static void basic_b(int a, double bmi, double bmj, double* bn, double* bmy, double* bmz) {
    *bn = 0.0;
    *bmy = 0.0;
    *bmz = 0.0;
    if (a == 0) *bn = 1.0;
    else if (a == 1) *bmz = bmi;
    else if (a == 2) *bmz = bmj;
    else if (a == 3) *bmy = bmi;
    else *bmy = bmj;
}

static void fbc3d_section_basic(const OElement* e, double L, double v[5]) {
    for (int i = 0; i < 5; ++i) v[i] = 0.0;
    for (int ip = 0; ip < e->nip; ++ip) {
        double xi = e->xi[ip], wL = e->w[ip] * L;
        double bmi = xi - 1.0, bmj = xi;
        v[0] += wL * e->eps0[ip];
        v[1] += wL * bmi * e->kz[ip];
        v[2] += wL * bmj * e->kz[ip];
        v[3] += wL * bmi * e->ky[ip];
        v[4] += wL * bmj * e->ky[ip];
    }
}

/* _force_beam_column3d_try_increment: on success e->q5 and the section deformations hold the
 * solved state and kb the basic stiffness of the last flexibility. */
static int fbc3d_try_increment(OElement* e, double L, const double base[5], const double dv[5],
                               int scheme, double kb[25]) {
    const OSection3d* sd = e->sec3;
    int nip = e->nip;
    double q[5];
    for (int i = 0; i < 5; ++i) q[i] = e->q5[i];
    double target[5];
    for (int i = 0; i < 5; ++i) target[i] = base[i] + dv[i];
    double sub_v[STRUT_MAX_INT_PTS][3], sub_s[STRUT_MAX_INT_PTS][3];
    double sub_f[STRUT_MAX_INT_PTS][6], init_f[STRUT_MAX_INT_PTS][6];
    for (int ip = 0; ip < nip; ++ip) {
        double r[9];
        sub_v[ip][0] = e->eps0[ip];
        sub_v[ip][1] = e->ky[ip];
        sub_v[ip][2] = e->kz[ip];
        oracle_section3d_response(sd, &e->sst[ip], sub_v[ip][0], sub_v[ip][1], sub_v[ip][2], r);
        e->section_evals++;
        sub_s[ip][0] = r[0];
        sub_s[ip][1] = r[1];
        sub_s[ip][2] = r[2];
        if (!section_flex(r, sub_f[ip])) return 0;
        /* the initial flexibility comes from the section at zero deformation, which also
         * overwrites the trial state (force_beam_column3d.mojo:1305-1322) */
        oracle_section3d_response(sd, &e->sst[ip], 0.0, 0.0, 0.0, r);
        e->section_evals++;
        if (!section_flex(r, init_f[ip])) return 0;
    }
    double P[25];
    for (int i = 0; i < 25; ++i) P[i] = 0.0;
    for (int ip = 0; ip < nip; ++ip) {
        double xi = e->xi[ip], wL = e->w[ip] * L;
        double bmi = xi - 1.0, bmj = xi;
        double f11 = sub_f[ip][0], f12 = sub_f[ip][1], f13 = sub_f[ip][2];
        double f22 = sub_f[ip][3], f23 = sub_f[ip][4], f33 = sub_f[ip][5];
        P[0] += wL * f11;
        P[1] += wL * f13 * bmi;
        P[2] += wL * f13 * bmj;
        P[3] += wL * f12 * bmi;
        P[4] += wL * f12 * bmj;
        P[5] += wL * bmi * f13;
        P[6] += wL * bmi * f33 * bmi;
        P[7] += wL * bmi * f33 * bmj;
        P[8] += wL * bmi * f23 * bmi;
        P[9] += wL * bmi * f23 * bmj;
        P[10] += wL * bmj * f13;
        P[11] += wL * bmj * f33 * bmi;
        P[12] += wL * bmj * f33 * bmj;
        P[13] += wL * bmj * f23 * bmi;
        P[14] += wL * bmj * f23 * bmj;
        P[15] += wL * bmi * f12;
        P[16] += wL * bmi * f23 * bmi;
        P[17] += wL * bmi * f23 * bmj;
        P[18] += wL * bmi * f22 * bmi;
        P[19] += wL * bmi * f22 * bmj;
        P[20] += wL * bmj * f12;
        P[21] += wL * bmj * f23 * bmi;
        P[22] += wL * bmj * f23 * bmj;
        P[23] += wL * bmj * f22 * bmi;
        P[24] += wL * bmj * f22 * bmj;
    }
    if (invert5(P, kb)) {
        for (int i = 0; i < 5; ++i)
            q[i] += (kb[i * 5] * dv[0] + kb[i * 5 + 1] * dv[1] + kb[i * 5 + 2] * dv[2] +
                     kb[i * 5 + 3] * dv[3] + kb[i * 5 + 4] * dv[4]);
    }
    int num_iters = scheme == 1 ? 100 : 10;
    for (int it = 0; it < num_iters; ++it) {
        e->local_iters++;
        double F[25], vf[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int i = 0; i < 25; ++i) F[i] = 0.0;
        int use_init = scheme == 1 || (scheme == 2 && it == 0);
        for (int ip = 0; ip < nip; ++ip) {
            double xi = e->xi[ip], wL = e->w[ip] * L;
            double bmi = xi - 1.0, bmj = xi;
            double axial_t = q[0] + 0.0;
            double mz_t = bmi * q[1] + bmj * q[2] + 0.0;
            double my_t = bmi * q[3] + bmj * q[4] + 0.0;
            double dss0 = axial_t - sub_s[ip][0];
            double dss1 = my_t - sub_s[ip][1];
            double dss2 = mz_t - sub_s[ip][2];
            const double* sf = use_init ? init_f[ip] : sub_f[ip];
            double dvs0 = sf[0] * dss0 + sf[1] * dss1 + sf[2] * dss2;
            double dvs1 = sf[1] * dss0 + sf[3] * dss1 + sf[4] * dss2;
            double dvs2 = sf[2] * dss0 + sf[4] * dss1 + sf[5] * dss2;
            double vs0 = sub_v[ip][0] + dvs0;
            double vs1 = sub_v[ip][1] + dvs1;
            double vs2 = sub_v[ip][2] + dvs2;
            double r[9];
            oracle_section3d_response(sd, &e->sst[ip], vs0, vs1, vs2, r);
            e->section_evals++;
            sub_v[ip][0] = vs0;
            sub_v[ip][1] = vs1;
            sub_v[ip][2] = vs2;
            sub_s[ip][0] = r[0];
            sub_s[ip][1] = r[1];
            sub_s[ip][2] = r[2];
            double fl[6];
            if (!section_flex(r, fl)) return 0;
            for (int c = 0; c < 6; ++c) sub_f[ip][c] = fl[c];
            double dr0 = axial_t - sub_s[ip][0];
            double dr1 = my_t - sub_s[ip][1];
            double dr2 = mz_t - sub_s[ip][2];
            double dvr0 = fl[0] * dr0 + fl[1] * dr1 + fl[2] * dr2;
            double dvr1 = fl[1] * dr0 + fl[3] * dr1 + fl[4] * dr2;
            double dvr2 = fl[2] * dr0 + fl[4] * dr1 + fl[5] * dr2;
            vf[0] += wL * (vs0 + dvr0);
            vf[1] += wL * bmi * (vs2 + dvr2);
            vf[2] += wL * bmj * (vs2 + dvr2);
            vf[3] += wL * bmi * (vs1 + dvr1);
            vf[4] += wL * bmj * (vs1 + dvr1);
            for (int a = 0; a < 5; ++a) {
                double an, amy, amz;
                basic_b(a, bmi, bmj, &an, &amy, &amz);
                for (int b = 0; b < 5; ++b) {
                    double bn, bmy, bmz;
                    basic_b(b, bmi, bmj, &bn, &bmy, &bmz);
                    double dE = fl[0] * bn + fl[1] * bmy + fl[2] * bmz;
                    double dKy = fl[1] * bn + fl[3] * bmy + fl[4] * bmz;
                    double dKz = fl[2] * bn + fl[4] * bmy + fl[5] * bmz;
                    F[a * 5 + b] += wL * (an * dE + amy * dKy + amz * dKz);
                }
            }
        }
        double Fc[25];
        memcpy(Fc, F, sizeof(Fc));
        if (!invert5(Fc, kb)) return 0;
        double res[5], dq[5];
        for (int i = 0; i < 5; ++i) res[i] = target[i] - vf[i];
        for (int i = 0; i < 5; ++i)
            dq[i] = kb[i * 5] * res[0] + kb[i * 5 + 1] * res[1] + kb[i * 5 + 2] * res[2] +
                    kb[i * 5 + 3] * res[3] + kb[i * 5 + 4] * res[4];
        double work = fabs(res[0] * dq[0] + res[1] * dq[1] + res[2] * dq[2] + res[3] * dq[3] +
                           res[4] * dq[4]);
        for (int i = 0; i < 5; ++i) q[i] += dq[i];
        if (work < 1.0e-12) {
            for (int i = 0; i < 5; ++i) e->q5[i] = q[i];
            for (int ip = 0; ip < nip; ++ip) {
                e->eps0[ip] = sub_v[ip][0];
                e->ky[ip] = sub_v[ip][1];
                e->kz[ip] = sub_v[ip][2];
            }
            return 1;
        }
    }
    return 0;
}

static double max_abs5(const double* r) {
    double a = fabs(r[0]) > fabs(r[1]) ? fabs(r[0]) : fabs(r[1]);
    double b = fabs(r[2]) > fabs(r[3]) ? fabs(r[2]) : fabs(r[3]);
    b = b > fabs(r[4]) ? b : fabs(r[4]);
    return a > b ? a : b;
}

int oracle_fbc3d(OElement* e, const double ug[12], double k[144], double f[12]) {
    int nip = e->nip;
    double L = e->L;
    double R[9];
    int rc = element_rotation(e, ug, R);
    if (rc != STRUT_OK) return rc;
    double ul[12];
    u_to_local(R, ug, ul);
    double chord_z = (ul[7] - ul[1]) / L;
    double chord_y = (ul[8] - ul[2]) / L;
    double v[5] = {ul[6] - ul[0], ul[5] - chord_z, ul[11] - chord_z, ul[4] + chord_y,
                   ul[10] + chord_y};
    double torsion = ul[9] - ul[3];
    double kb[25];
    for (int i = 0; i < 25; ++i) kb[i] = 0.0;
    double acc_v[5];
    fbc3d_section_basic(e, L, acc_v);
    double acc_q[5];
    for (int i = 0; i < 5; ++i) acc_q[i] = e->q5[i];
    double svs[STRUT_MAX_INT_PTS][3];
    for (int ip = 0; ip < nip; ++ip) {
        svs[ip][0] = e->eps0[ip];
        svs[ip][1] = e->ky[ip];
        svs[ip][2] = e->kz[ip];
    }
    double rem[5], att[5];
    for (int i = 0; i < 5; ++i) rem[i] = v[i] - acc_v[i];
    for (int i = 0; i < 5; ++i) att[i] = rem[i];
    int converged = 0;
    int num_subdivide = 1;
    int guard = 0;
    while (num_subdivide <= 4 && guard < 10000) {
        ++guard;
        double tv[5];
        for (int i = 0; i < 5; ++i) tv[i] = acc_v[i] + att[i];
        int scheme_success = 0;
        for (int scheme = 0; scheme < 3; ++scheme) {
            for (int i = 0; i < 5; ++i) e->q5[i] = acc_q[i];
            for (int ip = 0; ip < nip; ++ip) {
                e->eps0[ip] = svs[ip][0];
                e->ky[ip] = svs[ip][1];
                e->kz[ip] = svs[ip][2];
            }
            if (!fbc3d_try_increment(e, L, acc_v, att, scheme, kb)) continue;
            for (int i = 0; i < 5; ++i) acc_v[i] = tv[i];
            for (int i = 0; i < 5; ++i) acc_q[i] = e->q5[i];
            for (int ip = 0; ip < nip; ++ip) {
                svs[ip][0] = e->eps0[ip];
                svs[ip][1] = e->ky[ip];
                svs[ip][2] = e->kz[ip];
            }
            for (int i = 0; i < 5; ++i) rem[i] = v[i] - acc_v[i];
            if (max_abs5(rem) <= 1.0e-12) {
                converged = 1;
            } else {
                for (int i = 0; i < 5; ++i) att[i] = rem[i];
                num_subdivide = 1;
            }
            scheme_success = 1;
            break;
        }
        if (converged) break;
        if (scheme_success) continue;
        for (int i = 0; i < 5; ++i) att[i] /= 10.0;
        num_subdivide += 1;
    }
    if (!converged) {
        /* Strut restores the accepted state and aborts the analysis */
        for (int i = 0; i < 5; ++i) e->q5[i] = acc_q[i];
        for (int ip = 0; ip < nip; ++ip) {
            e->eps0[ip] = svs[ip][0];
            e->ky[ip] = svs[ip][1];
            e->kz[ip] = svs[ip][2];
        }
        return STRUT_ELEMENT_FAILED;
    }
    double q0 = acc_q[0], q1 = acc_q[1], q2 = acc_q[2], q3 = acc_q[3], q4 = acc_q[4];
    double inv_L = e->inv_L3;
    double kl[144];
    for (int i = 0; i < 144; ++i) kl[i] = 0.0;
    for (int a = 0; a < 12; ++a) {
        double ac[5], bc[5];
        for (int i = 0; i < 5; ++i) ac[i] = basic_coeff(i, a, inv_L);
        for (int b = 0; b < 12; ++b) {
            for (int j = 0; j < 5; ++j) bc[j] = basic_coeff(j, b, inv_L);
            for (int i = 0; i < 5; ++i)
                for (int j = 0; j < 5; ++j) kl[a * 12 + b] += ac[i] * kb[i * 5 + j] * bc[j];
        }
    }
    int has_torsion = e->G > 0.0 && e->J > 0.0;
    if (has_torsion) {
        double tk = e->G * e->J / L;
        for (int a = 0; a < 12; ++a)
            for (int b = 0; b < 12; ++b)
                kl[a * 12 + b] += basic_coeff(5, a, inv_L) * tk * basic_coeff(5, b, inv_L);
    }
    if (e->desc->geom == STRUT_GEOM_PDELTA || e->desc->geom == STRUT_GEOM_COROTATIONAL) {
        kl[1 * 12 + 1] += q0 / L;
        kl[1 * 12 + 7] -= q0 / L;
        kl[7 * 12 + 1] -= q0 / L;
        kl[7 * 12 + 7] += q0 / L;
        kl[2 * 12 + 2] += q0 / L;
        kl[2 * 12 + 8] -= q0 / L;
        kl[8 * 12 + 2] -= q0 / L;
        kl[8 * 12 + 8] += q0 / L;
    }
    double q5b = 0.0;
    if (has_torsion) q5b = (e->G * e->J / L) * torsion;
    double fl[12];
    for (int a = 0; a < 12; ++a) {
        fl[a] = 0.0;
        fl[a] += basic_coeff(0, a, inv_L) * q0;
        fl[a] += basic_coeff(1, a, inv_L) * q1;
        fl[a] += basic_coeff(2, a, inv_L) * q2;
        fl[a] += basic_coeff(3, a, inv_L) * q3;
        fl[a] += basic_coeff(4, a, inv_L) * q4;
        fl[a] += basic_coeff(5, a, inv_L) * q5b;
    }
    fl[0] += 0.0;
    fl[1] += 0.0;
    fl[2] += 0.0;
    fl[7] += 0.0;
    fl[8] += 0.0;
    k_to_global_flat(R, kl, k);
    f_to_global(R, fl, f);
    return STRUT_OK;
}

/* ---- ShellMITC4 on an ElasticMembranePlateSection (shell4.mojo:10-363) -------------------
 * 24 x 24 global stiffness of the linear four-node shell: MITC4 basis g1, g2, g3 from the
 * diagonals, local coordinates, membrane / bending / transverse-shear moduli, the assumed
 * transverse-shear strains through the edge interpolation (Gm, Ms, r1/r2 scaling, Rot), 2 x 2
 * Gauss points, B matrices projected through Gmem / Gshear, the drilling term with Ktt = G h;
 * the bending block of dd is negated and the bending rows of B flipped back, as the reference
 * does.  Row-major K[24 * a + b]. */
static void v_normalize(double* x, double* y, double* z) {
    const double n = sqrt(*x * *x + *y * *y + *z * *z);
    *x /= n;
    *y /= n;
    *z /= n;
}

int oracle_shell4_stiffness(double E, double nu, double h, const double* x, const double* y, const double* z,
                            double* K) {
    double v1x = (x[2] + x[1] - x[3] - x[0]) * 0.5, v1y = (y[2] + y[1] - y[3] - y[0]) * 0.5,
           v1z = (z[2] + z[1] - z[3] - z[0]) * 0.5;
    double v2x = (x[3] + x[2] - x[1] - x[0]) * 0.5, v2y = (y[3] + y[2] - y[1] - y[0]) * 0.5,
           v2z = (z[3] + z[2] - z[1] - z[0]) * 0.5;
    double g1x = v1x, g1y = v1y, g1z = v1z;
    v_normalize(&g1x, &g1y, &g1z);
    const double alpha = v2x * g1x + v2y * g1y + v2z * g1z;
    v2x -= alpha * g1x;
    v2y -= alpha * g1y;
    v2z -= alpha * g1z;
    double g2x = v2x, g2y = v2y, g2z = v2z;
    v_normalize(&g2x, &g2y, &g2z);
    const double g3x = g1y * g2z - g1z * g2y, g3y = g1z * g2x - g1x * g2z, g3z = g1x * g2y - g1y * g2x;
    double xl[2][4];
    for (int i = 0; i < 4; ++i) {
        xl[0][i] = x[i] * g1x + y[i] * g1y + z[i] * g1z;
        xl[1][i] = x[i] * g2x + y[i] * g2y + z[i] * g2z;
    }
    const double factor = E / (1.0 - nu * nu);
    const double Dm[3][3] = {{factor, factor * nu, 0.0}, {factor * nu, factor, 0.0}, {0.0, 0.0, factor * (1.0 - nu) / 2.0}};
    const double bf = E * h * h * h / (12.0 * (1.0 - nu * nu));
    const double Db[3][3] = {{bf, bf * nu, 0.0}, {bf * nu, bf, 0.0}, {0.0, 0.0, bf * (1.0 - nu) / 2.0}};
    const double G = E / (2.0 * (1.0 + nu));
    const double Ds = (5.0 / 6.0) * G * h;
    const double Ktt = G * h;
    double dd[8][8] = {{0}};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            dd[i][j] = Dm[i][j] * h;
            dd[i + 3][j + 3] = -Db[i][j];
        }
    dd[6][6] = Ds;
    dd[7][7] = Ds;
    const double dx34 = xl[0][2] - xl[0][3], dy34 = xl[1][2] - xl[1][3];
    const double dx21 = xl[0][1] - xl[0][0], dy21 = xl[1][1] - xl[1][0];
    const double dx32 = xl[0][2] - xl[0][1], dy32 = xl[1][2] - xl[1][1];
    const double dx41 = xl[0][3] - xl[0][0], dy41 = xl[1][3] - xl[1][0];
    double Gm[4][12] = {{0}};
    const double q4 = 0.25;
    Gm[0][0] = -0.5; Gm[0][1] = -dy41 * q4; Gm[0][2] = dx41 * q4;
    Gm[0][9] = 0.5;  Gm[0][10] = -dy41 * q4; Gm[0][11] = dx41 * q4;
    Gm[1][0] = -0.5; Gm[1][1] = -dy21 * q4; Gm[1][2] = dx21 * q4;
    Gm[1][3] = 0.5;  Gm[1][4] = -dy21 * q4; Gm[1][5] = dx21 * q4;
    Gm[2][3] = -0.5; Gm[2][4] = -dy32 * q4; Gm[2][5] = dx32 * q4;
    Gm[2][6] = 0.5;  Gm[2][7] = -dy32 * q4; Gm[2][8] = dx32 * q4;
    Gm[3][6] = 0.5;  Gm[3][7] = -dy34 * q4; Gm[3][8] = dx34 * q4;
    Gm[3][9] = -0.5; Gm[3][10] = -dy34 * q4; Gm[3][11] = dx34 * q4;
    const double Ax = -xl[0][0] + xl[0][1] + xl[0][2] - xl[0][3];
    const double Bx = xl[0][0] - xl[0][1] + xl[0][2] - xl[0][3];
    const double Cx = -xl[0][0] - xl[0][1] + xl[0][2] + xl[0][3];
    const double Ay = -xl[1][0] + xl[1][1] + xl[1][2] - xl[1][3];
    const double By = xl[1][0] - xl[1][1] + xl[1][2] - xl[1][3];
    const double Cy = -xl[1][0] - xl[1][1] + xl[1][2] + xl[1][3];
    const double alph = atan2(Ay, Ax);
    const double beta = 0.5 * 3.141592653589793 - atan2(Cx, Cy);
    const double Rot[2][2] = {{sin(beta), -sin(alph)}, {-cos(beta), cos(alph)}};
    const double r3i = 1.0 / sqrt(3.0);
    const double sg[4] = {-r3i, r3i, r3i, -r3i}, tg[4] = {-r3i, -r3i, r3i, r3i};
    const double sn[4] = {-0.5, 0.5, 0.5, -0.5}, tn[4] = {-0.5, -0.5, 0.5, 0.5};
    const double Gmem[2][3] = {{g1x, g1y, g1z}, {g2x, g2y, g2z}};
    const double Gshear[3][6] = {{g3x, g3y, g3z, 0, 0, 0}, {0, 0, 0, g1x, g1y, g1z}, {0, 0, 0, g2x, g2y, g2z}};
    for (int t = 0; t < 576; ++t) K[t] = 0.0;
    for (int gp = 0; gp < 4; ++gp) {
        const double ss = sg[gp], tt = tg[gp];
        double shp[3][4];
        for (int i = 0; i < 4; ++i) {
            shp[2][i] = (0.5 + sn[i] * ss) * (0.5 + tn[i] * tt);
            shp[0][i] = sn[i] * (0.5 + tn[i] * tt);
            shp[1][i] = tn[i] * (0.5 + sn[i] * ss);
        }
        double xs[2][2];
        for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 2; ++j) {
                xs[i][j] = 0.0;
                for (int k = 0; k < 4; ++k) xs[i][j] += xl[i][k] * shp[j][k];
            }
        const double xsj = xs[0][0] * xs[1][1] - xs[0][1] * xs[1][0];
        if (xsj == 0.0) return STRUT_BAD_ARG;
        const double jinv = 1.0 / xsj;
        const double sx00 = xs[1][1] * jinv, sx11 = xs[0][0] * jinv, sx01 = -xs[0][1] * jinv,
                     sx10 = -xs[1][0] * jinv;
        for (int i = 0; i < 4; ++i) {
            const double temp = shp[0][i] * sx00 + shp[1][i] * sx10;
            shp[1][i] = shp[0][i] * sx01 + shp[1][i] * sx11;
            shp[0][i] = temp;
        }
        const double dvol = 1.0 * xsj;
        double Ms[2][4] = {{0}};
        Ms[1][0] = 1.0 - ss;
        Ms[0][1] = 1.0 - tt;
        Ms[1][2] = 1.0 + ss;
        Ms[0][3] = 1.0 + tt;
        double Bsv[2][12];
        for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 12; ++j) {
                double sum = 0.0;
                for (int k = 0; k < 4; ++k) sum += Ms[i][k] * Gm[k][j];
                Bsv[i][j] = sum;
            }
        double r1 = Cx + ss * Bx, r3 = Cy + ss * By;
        r1 = sqrt(r1 * r1 + r3 * r3);
        double r2 = Ax + tt * Bx;
        r3 = Ay + tt * By;
        r2 = sqrt(r2 * r2 + r3 * r3);
        for (int j = 0; j < 12; ++j) {
            Bsv[0][j] = Bsv[0][j] * r1 / (8.0 * xsj);
            Bsv[1][j] = Bsv[1][j] * r2 / (8.0 * xsj);
        }
        double Bs[2][12];
        for (int j = 0; j < 12; ++j) {
            Bs[0][j] = Rot[0][0] * Bsv[0][j] + Rot[0][1] * Bsv[1][j];
            Bs[1][j] = Rot[1][0] * Bsv[0][j] + Rot[1][1] * Bsv[1][j];
        }
        double saveB[4][8][6];
        double Bdrill[4][6];
        for (int j = 0; j < 4; ++j) {
            double Bmem[3][2] = {{0}}, Bb[3][2] = {{0}};
            Bmem[0][0] = shp[0][j];
            Bmem[1][1] = shp[1][j];
            Bmem[2][0] = shp[1][j];
            Bmem[2][1] = shp[0][j];
            Bb[0][1] = -shp[0][j];
            Bb[1][0] = shp[1][j];
            Bb[2][0] = shp[0][j];
            Bb[2][1] = -shp[1][j];
            double Bsh[2][3];
            for (int p = 0; p < 3; ++p) {
                Bsh[0][p] = Bs[0][j * 3 + p];
                Bsh[1][p] = Bs[1][j * 3 + p];
            }
            for (int p = 0; p < 8; ++p)
                for (int q = 0; q < 6; ++q) saveB[j][p][q] = 0.0;
            for (int p = 0; p < 3; ++p)
                for (int q = 0; q < 3; ++q) {
                    double sm = 0.0, sb = 0.0;
                    for (int r = 0; r < 2; ++r) {
                        sm += Bmem[p][r] * Gmem[r][q];
                        sb += Bb[p][r] * Gmem[r][q];
                    }
                    saveB[j][p][q] = sm;
                    saveB[j][p + 3][q + 3] = sb;
                }
            for (int p = 0; p < 2; ++p)
                for (int q = 0; q < 6; ++q) {
                    double s_ = 0.0;
                    for (int r = 0; r < 3; ++r) s_ += Bsh[p][r] * Gshear[r][q];
                    saveB[j][p + 6][q] = s_;
                }
            const double B1 = -0.5 * shp[1][j], B2 = 0.5 * shp[0][j], B6 = -shp[2][j];
            Bdrill[j][0] = B1 * g1x + B2 * g2x;
            Bdrill[j][1] = B1 * g1y + B2 * g2y;
            Bdrill[j][2] = B1 * g1z + B2 * g2z;
            Bdrill[j][3] = B6 * g3x;
            Bdrill[j][4] = B6 * g3y;
            Bdrill[j][5] = B6 * g3z;
        }
        for (int j = 0; j < 4; ++j) {
            double BJ[8][6];
            for (int p = 0; p < 8; ++p)
                for (int q = 0; q < 6; ++q) BJ[p][q] = saveB[j][p][q];
            for (int p = 3; p < 6; ++p)
                for (int q = 3; q < 6; ++q) BJ[p][q] *= -1.0;
            double BJtD[6][8];
            for (int p = 0; p < 6; ++p)
                for (int q = 0; q < 8; ++q) {
                    double sum = 0.0;
                    for (int r = 0; r < 8; ++r) sum += BJ[r][p] * dd[r][q];
                    BJtD[p][q] = sum * dvol;
                }
            double BdJ[6];
            for (int p = 0; p < 6; ++p) BdJ[p] = Bdrill[j][p] * (Ktt * dvol);
            for (int k = 0; k < 4; ++k)
                for (int p = 0; p < 6; ++p)
                    for (int q = 0; q < 6; ++q) {
                        double sum = 0.0;
                        for (int r = 0; r < 8; ++r) sum += BJtD[p][r] * saveB[k][r][q];
                        K[(j * 6 + p) * 24 + k * 6 + q] += sum + BdJ[p] * Bdrill[k][q];
                    }
        }
    }
    return STRUT_OK;
}

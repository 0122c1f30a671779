/*
 * ORACLE -- test infrastructure only.  FiberSection2d restated from Strut:
 *   definition build      src/mojo/sections/fiber2d.mojo:3323-3455 (families, centroid,
 *                         initial flexibility), grouping 3167-3228, padding 31-35
 *   state allocation      fiber2d.mojo:961-1006
 *   set_trial_from_offset fiber2d.mojo:3982-4024: elastic family (3459-3501, including the
 *                         uniform-modulus k12 = 0 quirk), Steel02 groups (2301-2516),
 *                         Concrete02 groups (1785-1972), Steel01 (1297-1325)
 *   commit / revert       fiber2d.mojo:4191-4252
 *
 * Reduction order: Strut sums each family in SIMD chunks of FLOAT64_SIMD_WIDTH lanes
 * (solver/simd_contiguous.mojo:6), reducing each chunk with a halving tree and adding the chunk
 * sum to a running scalar.  The width is a parameter here (oracle_set_simd_width, default 8 =
 * AVX-512); families are padded to that width with zero-area fibers exactly as in Strut.
 */
#include "oracle_internal.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static int g_simd_width = 8;

void oracle_set_simd_width(int w) {
    if (w == 1 || w == 2 || w == 4 || w == 8 || w == 16) g_simd_width = w;
}
int oracle_get_simd_width(void) { return g_simd_width; }

double oracle_tree_reduce(double* v, int w) {
    for (int h = w / 2; h >= 1; h /= 2) {
        for (int i = 0; i < h; ++i) v[i] = v[i] + v[i + h];
    }
    return v[0];
}

double oracle_simd_dot(const double* a, const double* b, int n) {
    /* vectorize_contiguous_binary_map_reduce_float64_simd (simd_contiguous.mojo:197-225):
     * full chunks reduced by reduce_add, remainder one element at a time. */
    int W = g_simd_width;
    double sum = 0.0;
    double lane[16];
    int i = 0;
    for (; i + W <= n; i += W) {
        for (int l = 0; l < W; ++l) lane[l] = (a[i + l] * b[i + l]) * 1.0;
        sum += oracle_tree_reduce(lane, W);
    }
    for (; i < n; ++i) sum += (a[i] * b[i]) * 1.0;
    return sum;
}

static int padded(int count, int W) {
    if (count <= 0) return 0;
    return ((count + W - 1) / W) * W;
}

static void build_group_family(const StrutFiber* fibers, int off, int nfib,
                               const StrutUniMaterial* mats, int mtype, double y_bar, int W,
                               int* n_out, double** y_out, double** a_out, int** mat_out,
                               int* ngroups_out, int** goff_out, int** gpad_out) {
    /* unique definition indices in first-appearance order (fiber2d.mojo:3182-3192) */
    int* uniq = (int*)malloc(sizeof(int) * (nfib + 1));
    int nu = 0;
    int count = 0;
    for (int i = 0; i < nfib; ++i) {
        int m = fibers[off + i].material;
        if (mats[m].type != mtype) continue;
        ++count;
        int seen = 0;
        for (int j = 0; j < nu; ++j)
            if (uniq[j] == m) seen = 1;
        if (!seen) uniq[nu++] = m;
    }
    int total = 0;
    for (int g = 0; g < nu; ++g) {
        int c = 0;
        for (int i = 0; i < nfib; ++i)
            if (fibers[off + i].material == uniq[g]) ++c;
        total += padded(c, W);
    }
    double* y = (double*)calloc(total > 0 ? total : 1, sizeof(double));
    double* a = (double*)calloc(total > 0 ? total : 1, sizeof(double));
    int* mt = (int*)calloc(total > 0 ? total : 1, sizeof(int));
    int* goff = (int*)calloc(nu > 0 ? nu : 1, sizeof(int));
    int* gpad = (int*)calloc(nu > 0 ? nu : 1, sizeof(int));
    int pos = 0;
    for (int g = 0; g < nu; ++g) {
        goff[g] = pos;
        int c = 0;
        for (int i = 0; i < nfib; ++i) {
            const StrutFiber* f = &fibers[off + i];
            if (f->material != uniq[g]) continue;
            y[pos] = f->y - y_bar;
            a[pos] = f->area;
            mt[pos] = f->material;
            ++pos;
            ++c;
        }
        int pc = padded(c, W);
        for (int k = c; k < pc; ++k) {
            y[pos] = 0.0;
            a[pos] = 0.0;
            mt[pos] = uniq[g];
            ++pos;
        }
        gpad[g] = pc;
    }
    (void)count;
    free(uniq);
    *n_out = total;
    *y_out = y;
    *a_out = a;
    *mat_out = mt;
    *ngroups_out = nu;
    *goff_out = goff;
    *gpad_out = gpad;
}

int oracle_section_build(OSection* sd, const StrutUniMaterial* mats, int nmat,
                         const StrutFiber* fibers, int off, int nfib) {
    memset(sd, 0, sizeof(*sd));
    if (nfib <= 0) return STRUT_BAD_ARG;
    int W = g_simd_width;
    double area_sum = 0.0, qz_sum = 0.0;
    for (int i = 0; i < nfib; ++i) {
        const StrutFiber* f = &fibers[off + i];
        if (f->material < 0 || f->material >= nmat) return STRUT_BAD_ARG;
        area_sum += f->area;
        qz_sum += f->area * f->y;
    }
    if (area_sum <= 0.0) return STRUT_BAD_ARG;
    sd->nfib = nfib;
    sd->y_bar = qz_sum / area_sum;
    sd->mats = mats;
    double ik11 = 0.0, ik12 = 0.0, ik22 = 0.0;
    int n_el = 0, n_s1 = 0, n_c1 = 0;
    for (int i = 0; i < nfib; ++i) {
        const StrutFiber* f = &fibers[off + i];
        double y_rel = f->y - sd->y_bar;
        double ks = oracle_initial_tangent(&mats[f->material]) * f->area;
        ik11 += ks;
        ik12 += -ks * y_rel;
        ik22 += ks * y_rel * y_rel;
        if (mats[f->material].type == STRUT_MAT_ELASTIC) ++n_el;
        if (mats[f->material].type == STRUT_MAT_STEEL01) ++n_s1;
        if (mats[f->material].type == STRUT_MAT_CONCRETE01) ++n_c1;
    }
    sd->n_el = n_el;
    sd->el_y = (double*)calloc(n_el + 1, sizeof(double));
    sd->el_a = (double*)calloc(n_el + 1, sizeof(double));
    sd->el_e = (double*)calloc(n_el + 1, sizeof(double));
    sd->n_s1 = n_s1;
    sd->s1_y = (double*)calloc(n_s1 + 1, sizeof(double));
    sd->s1_a = (double*)calloc(n_s1 + 1, sizeof(double));
    sd->s1_mat = (int*)calloc(n_s1 + 1, sizeof(int));
    sd->n_c1 = n_c1;
    sd->c1_y = (double*)calloc(n_c1 + 1, sizeof(double));
    sd->c1_a = (double*)calloc(n_c1 + 1, sizeof(double));
    sd->c1_mat = (int*)calloc(n_c1 + 1, sizeof(int));
    int ie = 0, i1 = 0, ic1 = 0;
    for (int i = 0; i < nfib; ++i) {
        const StrutFiber* f = &fibers[off + i];
        double y_rel = f->y - sd->y_bar;
        if (mats[f->material].type == STRUT_MAT_ELASTIC) {
            sd->el_y[ie] = y_rel;
            sd->el_a[ie] = f->area;
            sd->el_e[ie] = oracle_initial_tangent(&mats[f->material]);
            ++ie;
        } else if (mats[f->material].type == STRUT_MAT_STEEL01) {
            sd->s1_y[i1] = y_rel;
            sd->s1_a[i1] = f->area;
            sd->s1_mat[i1] = f->material;
            ++i1;
        } else if (mats[f->material].type == STRUT_MAT_CONCRETE01) {
            sd->c1_y[ic1] = y_rel;
            sd->c1_a[ic1] = f->area;
            sd->c1_mat[ic1] = f->material;
            ++ic1;
        }
    }
    sd->nonlinear_count = nfib - n_el;
    build_group_family(fibers, off, nfib, mats, STRUT_MAT_STEEL02, sd->y_bar, W, &sd->n_s2,
                       &sd->s2_y, &sd->s2_a, &sd->s2_mat, &sd->s2_ngroups, &sd->s2_goff,
                       &sd->s2_gpad);
    build_group_family(fibers, off, nfib, mats, STRUT_MAT_CONCRETE02, sd->y_bar, W, &sd->n_c2,
                       &sd->c2_y, &sd->c2_a, &sd->c2_mat, &sd->c2_ngroups, &sd->c2_goff,
                       &sd->c2_gpad);
    double det = ik11 * ik22 - ik12 * ik12;
    if (fabs(det) > 1.0e-40) {
        double inv_det = 1.0 / det;
        sd->init_valid = 1;
        sd->f00 = ik22 * inv_det;
        sd->f01 = -ik12 * inv_det;
        sd->f11 = ik11 * inv_det;
    }
    sd->W = W;
    return STRUT_OK;
}

void oracle_section_free(OSection* sd) {
    free(sd->el_y); free(sd->el_a); free(sd->el_e);
    free(sd->s1_y); free(sd->s1_a); free(sd->s1_mat);
    free(sd->c1_y); free(sd->c1_a); free(sd->c1_mat);
    free(sd->s2_y); free(sd->s2_a); free(sd->s2_mat); free(sd->s2_goff); free(sd->s2_gpad);
    free(sd->c2_y); free(sd->c2_a); free(sd->c2_mat); free(sd->c2_goff); free(sd->c2_gpad);
    memset(sd, 0, sizeof(*sd));
}

void oracle_section_state_alloc(const OSection* sd, OSecState* st) {
    int n = sd->n_s2 + sd->n_c2 + sd->n_s1 + sd->n_c1;
    st->n = n;
    st->c = (OFiberState*)calloc(n + 1, sizeof(OFiberState));
    st->t = (OFiberState*)calloc(n + 1, sizeof(OFiberState));
    /* fiber2d_runtime_alloc_instances: only real fibers are initialised from their
     * definition; padding slots stay zero (fiber2d.mojo:987-1002). */
    for (int k = 0; k < sd->n_s2; ++k)
        if (sd->s2_a[k] != 0.0) oracle_fiber_init(&sd->mats[sd->s2_mat[k]], &st->c[k]);
    for (int k = 0; k < sd->n_c2; ++k)
        if (sd->c2_a[k] != 0.0)
            oracle_fiber_init(&sd->mats[sd->c2_mat[k]], &st->c[sd->n_s2 + k]);
    for (int k = 0; k < sd->n_s1; ++k)
        oracle_fiber_init(&sd->mats[sd->s1_mat[k]], &st->c[sd->n_s2 + sd->n_c2 + k]);
    for (int k = 0; k < sd->n_c1; ++k)
        oracle_fiber_init(&sd->mats[sd->c1_mat[k]], &st->c[sd->n_s2 + sd->n_c2 + sd->n_s1 + k]);
    memcpy(st->t, st->c, sizeof(OFiberState) * (n + 1));
}

void oracle_section_state_free(OSecState* st) {
    free(st->c);
    free(st->t);
    st->c = st->t = 0;
}

void oracle_section_commit(OSecState* st) { memcpy(st->c, st->t, sizeof(OFiberState) * st->n); }
void oracle_section_revert(OSecState* st) { memcpy(st->t, st->c, sizeof(OFiberState) * st->n); }

static void family_chunks(const OSection* sd, const double* yv, const double* av, const int* mt,
                          int base, int count, OSecState* st, double eps0, double kappa,
                          double* acc) {
    int W = sd->W;
    double f0[16], f1[16], f2[16], f3[16], f4[16];
    for (int i = 0; i < count; i += W) {
        for (int l = 0; l < W; ++l) {
            int k = i + l;
            double y = yv[k];
            double strain = eps0 - y * kappa;
            const StrutUniMaterial* m = &sd->mats[mt[k]];
            OFiberState* c = &st->c[base + k];
            OFiberState* t = &st->t[base + k];
            oracle_fiber_trial(m, c, t, strain);
            double fs = t->sig * av[k];
            double ks = t->tan * av[k];
            f0[l] = fs;
            f1[l] = -fs * y;
            f2[l] = ks;
            f3[l] = -ks * y;
            f4[l] = ks * y * y;
        }
        acc[0] += oracle_tree_reduce(f0, W);
        acc[1] += oracle_tree_reduce(f1, W);
        acc[2] += oracle_tree_reduce(f2, W);
        acc[3] += oracle_tree_reduce(f3, W);
        acc[4] += oracle_tree_reduce(f4, W);
    }
}

void oracle_section_response(const OSection* sd, OSecState* st, double eps0, double kappa,
                             double out[5]) {
    int W = sd->W;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    /* elastic family, unpadded: vectorize[.., W](count) with a scalar remainder */
    {
        double f0[16], f1[16], f2[16], f3[16], f4[16];
        int i = 0;
        for (; i + W <= sd->n_el; i += W) {
            for (int l = 0; l < W; ++l) {
                double y = sd->el_y[i + l];
                double ks = sd->el_e[i + l] * sd->el_a[i + l];
                double fs = ks * (eps0 - y * kappa);
                f0[l] = fs;
                f1[l] = -fs * y;
                f2[l] = ks;
                f3[l] = -ks * y;
                f4[l] = ks * y * y;
            }
            acc[0] += oracle_tree_reduce(f0, W);
            acc[1] += oracle_tree_reduce(f1, W);
            acc[2] += oracle_tree_reduce(f2, W);
            acc[3] += oracle_tree_reduce(f3, W);
            acc[4] += oracle_tree_reduce(f4, W);
        }
        for (; i < sd->n_el; ++i) {
            double y = sd->el_y[i];
            double ks = sd->el_e[i] * sd->el_a[i];
            double fs = ks * (eps0 - y * kappa);
            acc[0] += fs;
            acc[1] += -fs * y;
            acc[2] += ks;
            acc[3] += -ks * y;
            acc[4] += ks * y * y;
        }
        if (sd->n_el > 0) {
            int uniform = 1;
            for (int j = 1; j < sd->n_el; ++j)
                if (sd->el_e[j] != sd->el_e[0]) uniform = 0;
            if (uniform) acc[3] = 0.0;
        }
    }
    for (int g = 0; g < sd->s2_ngroups; ++g) {
        int o = sd->s2_goff[g];
        family_chunks(sd, sd->s2_y + o, sd->s2_a + o, sd->s2_mat + o, o, sd->s2_gpad[g], st,
                      eps0, kappa, acc);
    }
    for (int g = 0; g < sd->c2_ngroups; ++g) {
        int o = sd->c2_goff[g];
        family_chunks(sd, sd->c2_y + o, sd->c2_a + o, sd->c2_mat + o, sd->n_s2 + o,
                      sd->c2_gpad[g], st, eps0, kappa, acc);
    }
    for (int k = 0; k < sd->n_s1; ++k) {
        int slot = sd->n_s2 + sd->n_c2 + k;
        double y = sd->s1_y[k];
        oracle_steel01_trial(&sd->mats[sd->s1_mat[k]], &st->c[slot], &st->t[slot],
                             eps0 - y * kappa);
        double fs = st->t[slot].sig * sd->s1_a[k];
        double ks = st->t[slot].tan * sd->s1_a[k];
        acc[0] += fs;
        acc[1] += -fs * y;
        acc[2] += ks;
        acc[3] += -ks * y;
        acc[4] += ks * y * y;
    }
    /* Concrete01 fibers one by one after Steel01 (fiber2d.mojo:1388-1420) */
    for (int k = 0; k < sd->n_c1; ++k) {
        int slot = sd->n_s2 + sd->n_c2 + sd->n_s1 + k;
        double y = sd->c1_y[k];
        oracle_concrete01_trial(&sd->mats[sd->c1_mat[k]], &st->c[slot], &st->t[slot],
                                eps0 - y * kappa);
        double fs = st->t[slot].sig * sd->c1_a[k];
        double ks = st->t[slot].tan * sd->c1_a[k];
        acc[0] += fs;
        acc[1] += -fs * y;
        acc[2] += ks;
        acc[3] += -ks * y;
        acc[4] += ks * y * y;
    }
    (void)W;
    for (int i = 0; i < 5; ++i) out[i] = acc[i];
}

int oracle_section_path(const StrutUniMaterial* mats, int nmat, const StrutFiber* fibers,
                        int nfib, const double* eps0_kappa, int npts, double* out) {
    OSection sd;
    int rc = oracle_section_build(&sd, mats, nmat, fibers, 0, nfib);
    if (rc != STRUT_OK) return rc;
    OSecState st;
    oracle_section_state_alloc(&sd, &st);
    for (int p = 0; p < npts; ++p) {
        oracle_section_response(&sd, &st, eps0_kappa[2 * p], eps0_kappa[2 * p + 1], out + 5 * p);
        oracle_section_commit(&st);
    }
    oracle_section_state_free(&st);
    oracle_section_free(&sd);
    return STRUT_OK;
}

int oracle_section_batch_path(const StrutUniMaterial* mats, int nmat, const StrutFiber* fibers,
                              int nfib, int n_inst, const double* eps0_kappa, int npts,
                              double* out) {
    OSection sd;
    int rc = oracle_section_build(&sd, mats, nmat, fibers, 0, nfib);
    if (rc != STRUT_OK) return rc;
    OSecState* st = (OSecState*)calloc(n_inst, sizeof(OSecState));
    for (int i = 0; i < n_inst; ++i) oracle_section_state_alloc(&sd, &st[i]);
    for (int p = 0; p < npts; ++p) {
        for (int i = 0; i < n_inst; ++i) {
            const double* ek = eps0_kappa + 2 * ((size_t)p * n_inst + i);
            oracle_section_response(&sd, &st[i], ek[0], ek[1], out + 5 * ((size_t)p * n_inst + i));
            oracle_section_commit(&st[i]);
        }
    }
    for (int i = 0; i < n_inst; ++i) oracle_section_state_free(&st[i]);
    free(st);
    oracle_section_free(&sd);
    return STRUT_OK;
}

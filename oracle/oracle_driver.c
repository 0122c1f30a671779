/*
 * ORACLE -- test infrastructure only.  Newmark-Newton transient driver, assembly and band
 * linear systems restated from Strut (paths relative to the Strut project root):
 *   Newmark constants / kernels   src/mojo/solver/run_case/analysis/transient_nonlinear.mojo:
 *                                 496-648, 1052-1055
 *   initial assembly (K_init)     transient_nonlinear.mojo:1207-1453
 *   step loop                     transient_nonlinear.mojo:1698-3110 (predictor 1766,
 *                                 ground motion 1823-1852, Newton 1959-2847, residual with
 *                                 dense dot products 2341-2356, band load 2400-2411,
 *                                 NormDispIncr test 2539 / 2798-2811, commit 3081-3108)
 *   element scatter               src/mojo/solver/assembly/stiffness_internal_frame2d.mojo:
 *                                 594-619 (element order)
 *   band slots / load / add       src/mojo/solver/run_case/linear_solver_backend.mojo:363-440,
 *                                 1877-1983; bandwidth 1481-1507
 *   BandGeneral factor / solve    linear_solver_backend.mojo:631-680 (+ dense partial-pivot
 *                                 fallback 175-240, 612-629), 735-770
 *   BandSPD factor / solve        linear_solver_backend.mojo:689-726, 772-812
 *   basic-state sync at commit    src/mojo/solver/run_case/helpers.mojo:1832-1883
 *   Path time series (dt form)    src/mojo/solver/time_series.mojo:61-90
 */
#include "oracle_internal.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

static long g_dense_fallbacks = 0;
long oracle_dense_fallbacks(void) { return g_dense_fallbacks; }

typedef struct OModel {
    const StrutModelDesc* d;
    int n, bw, rw; /* free count, half band width, general row width 2bw+1 */
    int spd;
    int nd; /* element dofs: 6 (2D) or 12 (3D) */
    OSection* secs;
    OSection3d* secs3;
    OElement* elems;
    int* efree; /* num_elements x nd free equation numbers */
    double *K, *Kinit, *Kcomm, *C, *Keff, *Kspd;
    double *Mff, *Mrff;
    double *dense;
    int* piv;
    int dense_mode;
    double *u, *u_f, *v_f, *a_f, *u_n, *v_n, *a_n, *Fint, *Fext, *P_f, *R_f, *du, *at, *vt,
        *work;
    double a0, a1, a2, a3;
    int has_damping;
    long newton_iters, factorizations;
    /* multi-point constraints: full K in a CSR pattern (rows = full dofs, sorted columns),
     * per element the position of each of its nd x nd entries, the collapse rows of every
     * dof and the collapsed F_int (full size) */
    int has_mpc;
    int* mrow_ptr;     /* num_dofs + 1: collapse terms of each dof (none for a fixed dof) */
    int* mrow_dof;
    double* mrow_coef;
    int* kptr;         /* num_dofs + 1 */
    int* kcol;
    double* kval;
    int* epos;         /* num_elements x nd x nd */
    double* sec_hist;  /* section recorder values, steps x num_record_sections x (2 or 4), or NULL */
    int* epos_sh;      /* num_shells x 24 x 24 */
    double* shell_k;   /* num_shells x 576, constant */
    int* efree_sh;     /* num_shells x 24 */
    double* Fred;
} OModel;

static double path_eval(const StrutExcitation* x, double t) {
    /* eval_time_series_input, Path with dt (time_series.mojo:71-90) */
    int n = x->count;
    if (n == 0) return 0.0;
    if (t < x->start_time) return 0.0;
    double incr = (t - x->start_time) / x->dt;
    int incr1 = (int)floor(incr);
    int incr2 = incr1 + 1;
    if (incr2 >= n) {
        if (x->use_last) return x->factor * x->values[n - 1];
        return 0.0;
    }
    double v1 = x->values[incr1], v2 = x->values[incr2];
    return x->factor * (v1 + (v2 - v1) * (incr - (double)incr1));
}

static int gslot(const OModel* m, int row, int col) {
    int off = col - row + m->bw;
    if (off < 0 || off > 2 * m->bw) return -1;
    return row * m->rw + off;
}

static void model_free(OModel* m) {
    if (m->elems) {
        for (int e = 0; e < m->d->num_elements; ++e) {
            if (!m->elems[e].sst) continue;
            for (int ip = 0; ip < m->elems[e].nip; ++ip)
                oracle_section_state_free(&m->elems[e].sst[ip]);
            free(m->elems[e].sst);
        }
        free(m->elems);
    }
    if (m->secs) {
        for (int s = 0; s < m->d->num_sections; ++s) oracle_section_free(&m->secs[s]);
        free(m->secs);
    }
    if (m->secs3) {
        for (int s = 0; s < m->d->num_sections; ++s) oracle_section3d_free(&m->secs3[s]);
        free(m->secs3);
    }
    free(m->efree);
    free(m->K); free(m->Kinit); free(m->Kcomm); free(m->C); free(m->Keff); free(m->Kspd);
    free(m->Mff); free(m->Mrff); free(m->dense); free(m->piv);
    free(m->u); free(m->u_f); free(m->v_f); free(m->a_f); free(m->u_n); free(m->v_n);
    free(m->a_n); free(m->Fint); free(m->Fext); free(m->P_f); free(m->R_f); free(m->du);
    free(m->at); free(m->vt); free(m->work);
    free(m->mrow_ptr); free(m->mrow_dof); free(m->mrow_coef); free(m->kptr); free(m->kcol);
    free(m->kval); free(m->epos); free(m->Fred);
    free(m->epos_sh); free(m->shell_k); free(m->efree_sh);
    memset(m, 0, sizeof(*m));
}

static int cmp_int(const void* a, const void* b) {
    int x = *(const int*)a, y = *(const int*)b;
    return (x > y) - (x < y);
}

/* Collapse rows (loader.mojo:2239-2380): a free dof maps to itself with coefficient 1, a slave
 * to its retained dofs, a fixed dof to nothing.  Full K pattern from the elements' dof pairs.
 * A slave dof may carry no mass (the collapsed mass would not be diagonal). */
static int mpc_build(OModel* m) {
    const StrutModelDesc* d = m->d;
    int nd = d->num_dofs, ned = m->nd;
    int* slave_of = (int*)malloc(sizeof(int) * nd);
    for (int i = 0; i < nd; ++i) slave_of[i] = -1;
    for (int s = 0; s < d->num_slaves; ++s) {
        int dof = d->slave_dof[s];
        if (dof < 0 || dof >= nd) {
            free(slave_of);
            return STRUT_BAD_ARG;
        }
        slave_of[dof] = s;
        if (d->mass[dof] != 0.0 || (d->mass_rayleigh && d->mass_rayleigh[dof] != 0.0)) {
            free(slave_of);
            return STRUT_UNSUPPORTED;
        }
    }
    m->mrow_ptr = (int*)calloc(nd + 1, sizeof(int));
    int total = 0;
    for (int i = 0; i < nd; ++i) {
        m->mrow_ptr[i] = total;
        if (slave_of[i] >= 0) total += d->slave_ptr[slave_of[i] + 1] - d->slave_ptr[slave_of[i]];
        else if (d->free_index[i] >= 0) total += 1;
    }
    m->mrow_ptr[nd] = total;
    m->mrow_dof = (int*)malloc(sizeof(int) * (total + 1));
    m->mrow_coef = (double*)malloc(sizeof(double) * (total + 1));
    for (int i = 0; i < nd; ++i) {
        int o = m->mrow_ptr[i];
        if (slave_of[i] >= 0) {
            int s = slave_of[i];
            for (int t = d->slave_ptr[s]; t < d->slave_ptr[s + 1]; ++t) {
                m->mrow_dof[o] = d->slave_master[t];
                m->mrow_coef[o] = d->slave_coef[t];
                ++o;
            }
        } else if (d->free_index[i] >= 0) {
            m->mrow_dof[o] = i;
            m->mrow_coef[o] = 1.0;
        }
    }
    free(slave_of);
    /* full K pattern */
    int* cnt = (int*)calloc(nd, sizeof(int));
    for (int e = 0; e < d->num_elements; ++e)
        for (int a = 0; a < ned; ++a) cnt[d->elements[e].dof[a]] += ned;
    for (int s = 0; s < d->num_shells; ++s)
        for (int a = 0; a < 24; ++a) cnt[d->shells[s].dof[a]] += 24;
    m->kptr = (int*)calloc(nd + 1, sizeof(int));
    for (int i = 0; i < nd; ++i) m->kptr[i + 1] = m->kptr[i] + cnt[i];
    int* tmp = (int*)malloc(sizeof(int) * (m->kptr[nd] + 1));
    for (int i = 0; i < nd; ++i) cnt[i] = 0;
    for (int e = 0; e < d->num_elements; ++e)
        for (int a = 0; a < ned; ++a) {
            int r = d->elements[e].dof[a];
            for (int b = 0; b < ned; ++b) tmp[m->kptr[r] + cnt[r]++] = d->elements[e].dof[b];
        }
    for (int s = 0; s < d->num_shells; ++s)
        for (int a = 0; a < 24; ++a) {
            int r = d->shells[s].dof[a];
            for (int b = 0; b < 24; ++b) tmp[m->kptr[r] + cnt[r]++] = d->shells[s].dof[b];
        }
    /* sort and unique each row */
    int nnz = 0;
    int* nptr = (int*)calloc(nd + 1, sizeof(int));
    for (int i = 0; i < nd; ++i) {
        int* row = tmp + m->kptr[i];
        int len = m->kptr[i + 1] - m->kptr[i];
        qsort(row, len, sizeof(int), cmp_int);
        int u = 0;
        for (int k = 0; k < len; ++k)
            if (u == 0 || row[u - 1] != row[k]) row[u++] = row[k];
        nptr[i] = nnz;
        nnz += u;
        cnt[i] = u;
    }
    nptr[nd] = nnz;
    m->kcol = (int*)malloc(sizeof(int) * (nnz + 1));
    for (int i = 0; i < nd; ++i) memcpy(m->kcol + nptr[i], tmp + m->kptr[i], sizeof(int) * cnt[i]);
    free(m->kptr);
    m->kptr = nptr;
    free(tmp);
    free(cnt);
    m->kval = (double*)calloc(nnz + 1, sizeof(double));
    m->epos = (int*)malloc(sizeof(int) * (size_t)d->num_elements * ned * ned);
    for (int e = 0; e < d->num_elements; ++e)
        for (int a = 0; a < ned; ++a) {
            int r = d->elements[e].dof[a];
            for (int b = 0; b < ned; ++b) {
                int c = d->elements[e].dof[b];
                int lo = m->kptr[r], hi = m->kptr[r + 1] - 1, pos = -1;
                while (lo <= hi) {
                    int mid = (lo + hi) / 2;
                    if (m->kcol[mid] == c) {
                        pos = mid;
                        break;
                    }
                    if (m->kcol[mid] < c) lo = mid + 1;
                    else hi = mid - 1;
                }
                m->epos[((size_t)e * ned + a) * ned + b] = pos;
            }
        }
    m->epos_sh = (int*)malloc(sizeof(int) * ((size_t)d->num_shells * 576 + 1));
    for (int s = 0; s < d->num_shells; ++s)
        for (int a = 0; a < 24; ++a) {
            int r = d->shells[s].dof[a];
            for (int b = 0; b < 24; ++b) {
                int c = d->shells[s].dof[b];
                int lo = m->kptr[r], hi = m->kptr[r + 1] - 1, pos = -1;
                while (lo <= hi) {
                    int mid = (lo + hi) / 2;
                    if (m->kcol[mid] == c) {
                        pos = mid;
                        break;
                    }
                    if (m->kcol[mid] < c) lo = mid + 1;
                    else hi = mid - 1;
                }
                m->epos_sh[((size_t)s * 24 + a) * 24 + b] = pos;
            }
        }
    m->Fred = (double*)calloc(nd, sizeof(double));
    m->has_mpc = 1;
    return STRUT_OK;
}

/* _collapse_vector_by_mpc (helpers.mojo:3288-3301): out[r] += c * v[i], i ascending */
static void mpc_collapse_vector(const OModel* m, const double* v, double* out) {
    int nd = m->d->num_dofs;
    for (int i = 0; i < nd; ++i) out[i] = 0.0;
    for (int i = 0; i < nd; ++i)
        for (int t = m->mrow_ptr[i]; t < m->mrow_ptr[i + 1]; ++t)
            out[m->mrow_dof[t]] += m->mrow_coef[t] * v[i];
}

/* _enforce_mpc_values (helpers.mojo:3380-3400) on the full displacement vector */
static void mpc_enforce(const OModel* m, double* u) {
    const StrutModelDesc* d = m->d;
    for (int s = 0; s < d->num_slaves; ++s) {
        double value = 0.0;
        for (int t = d->slave_ptr[s]; t < d->slave_ptr[s + 1]; ++t)
            value += d->slave_coef[t] * u[d->slave_master[t]];
        u[d->slave_dof[s]] = value;
    }
}

static int model_build(OModel* m, const StrutModelDesc* d) {
    memset(m, 0, sizeof(*m));
    m->d = d;
    int three_d = d->ndm == 3 && d->ndf == 6;
    if (!three_d && (d->ndm != 2 || d->ndf != 3)) return STRUT_UNSUPPORTED;
    int ned = 2 * d->ndf;
    m->nd = ned;
    if (d->num_free <= 0 || d->num_elements <= 0) return STRUT_BAD_ARG;
    if (d->system != STRUT_SYSTEM_BAND_GENERAL && d->system != STRUT_SYSTEM_BAND_SPD)
        return STRUT_UNSUPPORTED;
    m->spd = d->system == STRUT_SYSTEM_BAND_SPD;
    m->n = d->num_free;
    if (three_d) {
        m->secs3 = (OSection3d*)calloc(d->num_sections, sizeof(OSection3d));
        for (int s = 0; s < d->num_sections; ++s) {
            int rc = oracle_section3d_build(&m->secs3[s], d->materials, d->num_materials,
                                            d->fibers, d->sections[s].fiber_offset,
                                            d->sections[s].fiber_count);
            if (rc != STRUT_OK) return rc;
        }
    } else {
        m->secs = (OSection*)calloc(d->num_sections, sizeof(OSection));
        for (int s = 0; s < d->num_sections; ++s) {
            int rc = oracle_section_build(&m->secs[s], d->materials, d->num_materials, d->fibers,
                                          d->sections[s].fiber_offset, d->sections[s].fiber_count);
            if (rc != STRUT_OK) return rc;
        }
    }
    m->elems = (OElement*)calloc(d->num_elements, sizeof(OElement));
    m->efree = (int*)malloc(sizeof(int) * ned * d->num_elements);
    int bw = 0;
    for (int e = 0; e < d->num_elements; ++e) {
        const StrutFrameElement* ed = &d->elements[e];
        OElement* el = &m->elems[e];
        int is3 = ed->type == STRUT_ELEM_FORCE_BEAM_COLUMN_3D ||
                  ed->type == STRUT_ELEM_DISP_BEAM_COLUMN_3D;
        int is2 = ed->type == STRUT_ELEM_FORCE_BEAM_COLUMN_2D ||
                  ed->type == STRUT_ELEM_DISP_BEAM_COLUMN_2D;
        if (three_d ? !is3 : !is2) return STRUT_UNSUPPORTED;
        if (!three_d && ed->geom == STRUT_GEOM_COROTATIONAL) return STRUT_UNSUPPORTED;
        el->desc = ed;
        const StrutBeamIntegration* r = &d->integrations[ed->integration];
        el->nip = r->num_int_pts;
        for (int ip = 0; ip < el->nip; ++ip) {
            el->xi[ip] = r->xi[ip];
            el->w[ip] = r->w[ip];
        }
        if (three_d) {
            el->sec3 = &m->secs3[ed->section];
            for (int c = 0; c < 3; ++c) {
                el->x1[c] = d->node_coords[3 * ed->node_i + c];
                el->x2[c] = d->node_coords[3 * ed->node_j + c];
            }
            double dx = el->x2[0] - el->x1[0], dy = el->x2[1] - el->x1[1];
            double dz = el->x2[2] - el->x1[2];
            el->L = sqrt(dx * dx + dy * dy + dz * dz);
            if (el->L == 0.0) return STRUT_BAD_ARG;
            el->inv_L3 = 1.0 / el->L;
            int rrc = oracle_rotation3d(el->x1, el->x2, ed->has_vecxz, ed->vecxz, el->R);
            if (rrc != STRUT_OK) return rrc;
            el->G = d->sections[ed->section].G;
            el->J = d->sections[ed->section].J;
            el->sst = (OSecState*)calloc(el->nip, sizeof(OSecState));
            for (int ip = 0; ip < el->nip; ++ip)
                oracle_section3d_state_alloc(el->sec3, &el->sst[ip]);
        } else {
        el->sec = &m->secs[ed->section];
        double x1 = d->node_coords[2 * ed->node_i], y1 = d->node_coords[2 * ed->node_i + 1];
        double x2 = d->node_coords[2 * ed->node_j], y2 = d->node_coords[2 * ed->node_j + 1];
        double dx = x2 - x1, dy = y2 - y1;
        el->L = hypot(dx, dy);
        if (el->L == 0.0) return STRUT_BAD_ARG;
        double inv_L = 1.0 / el->L;
        el->c = dx * inv_L;
        el->s = dy * inv_L;
        el->c_div = dx / el->L;
        el->s_div = dy / el->L;
        el->L_sync = sqrt(dx * dx + dy * dy);
        el->c_sync = dx / el->L_sync;
        el->s_sync = dy / el->L_sync;
        el->sst = (OSecState*)calloc(el->nip, sizeof(OSecState));
        for (int ip = 0; ip < el->nip; ++ip) oracle_section_state_alloc(el->sec, &el->sst[ip]);
        }
        for (int a = 0; a < ned; ++a) {
            int dof = ed->dof[a];
            m->efree[ned * e + a] = (dof >= 0 && dof < d->num_dofs) ? d->free_index[dof] : -1;
        }
        for (int a = 0; a < ned; ++a) {
            int ia = m->efree[ned * e + a];
            if (ia < 0) continue;
            for (int b = a + 1; b < ned; ++b) {
                int ib = m->efree[ned * e + b];
                if (ib < 0) continue;
                int diff = ia > ib ? ia - ib : ib - ia;
                if (diff > bw) bw = diff;
            }
        }
    }
    /* linear shells (shell4.mojo:10-363): constant stiffness, their free-dof pairs in the band */
    if (d->num_shells > 0 && (d->ndm != 3 || d->ndf != 6 || !d->shells)) return STRUT_BAD_ARG;
    m->shell_k = (double*)malloc(sizeof(double) * ((size_t)d->num_shells * 576 + 1));
    m->efree_sh = (int*)malloc(sizeof(int) * ((size_t)d->num_shells * 24 + 1));
    for (int s = 0; s < d->num_shells; ++s) {
        const StrutShellElement* sh = &d->shells[s];
        double xs[4], ys[4], zs[4];
        for (int k = 0; k < 4; ++k) {
            if (sh->nodes[k] < 0 || sh->nodes[k] >= d->num_nodes) return STRUT_BAD_ARG;
            xs[k] = d->node_coords[3 * sh->nodes[k]];
            ys[k] = d->node_coords[3 * sh->nodes[k] + 1];
            zs[k] = d->node_coords[3 * sh->nodes[k] + 2];
        }
        if (oracle_shell4_stiffness(sh->E, sh->nu, sh->h, xs, ys, zs, m->shell_k + (size_t)576 * s) != STRUT_OK)
            return STRUT_BAD_ARG;
        for (int a = 0; a < 24; ++a) {
            int dof = sh->dof[a];
            if (dof < 0 || dof >= d->num_dofs) return STRUT_BAD_ARG;
            m->efree_sh[24 * s + a] = d->free_index[dof];
        }
        for (int a = 0; a < 24; ++a) {
            int ia = m->efree_sh[24 * s + a];
            if (ia < 0) continue;
            for (int b = a + 1; b < 24; ++b) {
                int ib = m->efree_sh[24 * s + b];
                if (ib < 0) continue;
                int diff = ia > ib ? ia - ib : ib - ia;
                if (diff > bw) bw = diff;
            }
        }
    }
    m->bw = bw;
    m->rw = 2 * bw + 1;
    int n = m->n;
    size_t bsz = (size_t)n * m->rw;
    m->K = (double*)calloc(bsz, sizeof(double));
    m->Kinit = (double*)calloc(bsz, sizeof(double));
    m->Kcomm = (double*)calloc(bsz, sizeof(double));
    m->C = (double*)calloc(bsz, sizeof(double));
    m->Keff = (double*)calloc(bsz, sizeof(double));
    m->Kspd = (double*)calloc((size_t)n * (bw + 1), sizeof(double));
    m->Mff = (double*)calloc(n, sizeof(double));
    m->Mrff = (double*)calloc(n, sizeof(double));
    int nd = d->num_dofs;
    m->u = (double*)calloc(nd, sizeof(double));
    m->Fint = (double*)calloc(nd, sizeof(double));
    m->Fext = (double*)calloc(nd, sizeof(double));
    m->u_f = (double*)calloc(n, sizeof(double));
    m->v_f = (double*)calloc(n, sizeof(double));
    m->a_f = (double*)calloc(n, sizeof(double));
    m->u_n = (double*)calloc(n, sizeof(double));
    m->v_n = (double*)calloc(n, sizeof(double));
    m->a_n = (double*)calloc(n, sizeof(double));
    m->P_f = (double*)calloc(n, sizeof(double));
    m->R_f = (double*)calloc(n, sizeof(double));
    m->du = (double*)calloc(n, sizeof(double));
    m->at = (double*)calloc(n, sizeof(double));
    m->vt = (double*)calloc(n, sizeof(double));
    m->work = (double*)calloc(n, sizeof(double));
    int has_mass = 0;
    for (int dof = 0; dof < nd; ++dof) {
        int fi = d->free_index[dof];
        if (fi < 0) continue;
        if (d->mass[dof] != 0.0) {
            m->Mff[fi] += d->mass[dof] * 1.0 * 1.0;
            has_mass = 1;
        }
        if (d->mass_rayleigh && d->mass_rayleigh[dof] != 0.0)
            m->Mrff[fi] += d->mass_rayleigh[dof] * 1.0 * 1.0;
    }
    if (!has_mass) return STRUT_BAD_ARG;
    double beta = d->beta, gamma = d->gamma, dt = d->dt;
    if (beta <= 0.0 || dt <= 0.0) return STRUT_BAD_ARG;
    m->a0 = 1.0 / (beta * dt * dt);
    m->a1 = gamma / (beta * dt);
    m->a2 = 1.0 / (beta * dt);
    m->a3 = 1.0 / (2.0 * beta) - 1.0;
    m->has_damping = d->alpha_m != 0.0 || d->beta_k != 0.0 || d->beta_k_init != 0.0 ||
                     d->beta_k_comm != 0.0;
    if (d->num_slaves > 0) {
        int rc = mpc_build(m);
        if (rc != STRUT_OK) return rc;
    }
    return STRUT_OK;
}

/* assemble_global_stiffness_and_internal_soa: zero K and F_int, then every element in order */
/* one element's global tangent and resisting force (nd x nd, nd) */
static int element_state(OElement* el, const double* ug, double* k, double* f) {
    switch (el->desc->type) {
        case STRUT_ELEM_FORCE_BEAM_COLUMN_2D: return oracle_fbc2d(el, ug, k, f);
        case STRUT_ELEM_DISP_BEAM_COLUMN_2D: return oracle_dbc2d(el, ug, k, f);
        case STRUT_ELEM_FORCE_BEAM_COLUMN_3D: return oracle_fbc3d(el, ug, k, f);
        default: return oracle_dbc3d(el, ug, k, f);
    }
}

/* assemble_global_stiffness_and_internal_soa into the full K, then _collapse_matrix_by_mpc
 * (helpers.mojo:3345-3377: out[r_i][r_j] += c_i K[i][j] c_j over i, j ascending, zero entries
 * skipped) straight into the band, where an entry outside the detected half width is dropped
 * as _update_banded_general_values_from_dense drops it (linear_solver_backend.mojo:413-427);
 * F_int collapsed by _collapse_vector_by_mpc. */
static void mpc_collapse_K(OModel* m) {
    const StrutModelDesc* d = m->d;
    int nd = d->num_dofs;
    memset(m->K, 0, sizeof(double) * (size_t)m->n * m->rw);
    for (int i = 0; i < nd; ++i) {
        int ti0 = m->mrow_ptr[i], ti1 = m->mrow_ptr[i + 1];
        if (ti0 == ti1) continue;
        for (int k = m->kptr[i]; k < m->kptr[i + 1]; ++k) {
            double value = m->kval[k];
            if (value == 0.0) continue;
            int j = m->kcol[k];
            int tj0 = m->mrow_ptr[j], tj1 = m->mrow_ptr[j + 1];
            if (tj0 == tj1) continue;
            for (int ti = ti0; ti < ti1; ++ti) {
                int fi = d->free_index[m->mrow_dof[ti]];
                double ci = m->mrow_coef[ti];
                for (int tj = tj0; tj < tj1; ++tj) {
                    int fj = d->free_index[m->mrow_dof[tj]];
                    double contrib = ci * value * m->mrow_coef[tj];
                    if (fi < 0 || fj < 0) continue;
                    int sl = gslot(m, fi, fj);
                    if (sl >= 0) m->K[sl] += contrib;
                }
            }
        }
    }
    mpc_collapse_vector(m, m->Fint, m->Fred);
}

static int assemble(OModel* m, double* ek_out, double* ef_out) {
    const StrutModelDesc* d = m->d;
    int nd = m->nd;
    memset(m->K, 0, sizeof(double) * (size_t)m->n * m->rw);
    memset(m->Fint, 0, sizeof(double) * d->num_dofs);
    if (m->has_mpc) {
        int nnz = m->kptr[d->num_dofs];
        memset(m->kval, 0, sizeof(double) * (nnz + 1));
        for (int e = 0; e < d->num_elements; ++e) {
            OElement* el = &m->elems[e];
            double ug[12], k[144], f[12];
            for (int a = 0; a < nd; ++a) ug[a] = m->u[el->desc->dof[a]];
            int rc = element_state(el, ug, k, f);
            if (rc != STRUT_OK) return rc;
            if (ek_out) memcpy(ek_out + (size_t)nd * nd * e, k, sizeof(double) * nd * nd);
            if (ef_out) memcpy(ef_out + (size_t)nd * e, f, sizeof(double) * nd);
            const int* pos = m->epos + (size_t)e * nd * nd;
            for (int a = 0; a < nd; ++a) {
                for (int b = 0; b < nd; ++b) m->kval[pos[a * nd + b]] += k[a * nd + b];
                m->Fint[el->desc->dof[a]] += f[a];
            }
        }
        for (int s = 0; s < d->num_shells; ++s) {
            const double* k = m->shell_k + (size_t)576 * s;
            double ue[24];
            for (int b = 0; b < 24; ++b) ue[b] = m->u[d->shells[s].dof[b]];
            const int* pos = m->epos_sh + (size_t)s * 576;
            for (int a = 0; a < 24; ++a) {
                for (int b = 0; b < 24; ++b) m->kval[pos[a * 24 + b]] += k[a * 24 + b];
                m->Fint[d->shells[s].dof[a]] += oracle_simd_dot(k + 24 * a, ue, 24);
            }
        }
        mpc_collapse_K(m);
        return STRUT_OK;
    }
    for (int e = 0; e < d->num_elements; ++e) {
        OElement* el = &m->elems[e];
        double ug[12], k[144], f[12];
        for (int a = 0; a < nd; ++a) ug[a] = m->u[el->desc->dof[a]];
        int rc = element_state(el, ug, k, f);
        if (rc != STRUT_OK) return rc;
        if (ek_out) memcpy(ek_out + (size_t)nd * nd * e, k, sizeof(double) * nd * nd);
        if (ef_out) memcpy(ef_out + (size_t)nd * e, f, sizeof(double) * nd);
        for (int a = 0; a < nd; ++a) {
            int ia = m->efree[nd * e + a];
            if (ia >= 0) {
                for (int b = 0; b < nd; ++b) {
                    int ib = m->efree[nd * e + b];
                    if (ib < 0) continue;
                    int sl = gslot(m, ia, ib);
                    if (sl >= 0) m->K[sl] += k[a * nd + b];
                }
            }
            m->Fint[el->desc->dof[a]] += f[a];
        }
    }
    /* shells after the frames (stiffness_internal_surface.mojo:240-280): K rows scattered,
     * F_int the row dot the element displacements */
    for (int s = 0; s < d->num_shells; ++s) {
        const double* k = m->shell_k + (size_t)576 * s;
        double ue[24];
        for (int b = 0; b < 24; ++b) ue[b] = m->u[d->shells[s].dof[b]];
        for (int a = 0; a < 24; ++a) {
            int ia = m->efree_sh[24 * s + a];
            if (ia >= 0) {
                for (int b = 0; b < 24; ++b) {
                    int ib = m->efree_sh[24 * s + b];
                    if (ib < 0) continue;
                    int sl = gslot(m, ia, ib);
                    if (sl >= 0) m->K[sl] += k[a * 24 + b];
                }
            }
            m->Fint[d->shells[s].dof[a]] += oracle_simd_dot(k + 24 * a, ue, 24);
        }
    }
    return STRUT_OK;
}

/* dense dot of a band row against x with Strut's chunked reduction order */
static double band_row_dot(const OModel* m, const double* band, int i, const double* x) {
    int W = oracle_get_simd_width();
    int n = m->n;
    double sum = 0.0;
    double lane[16];
    int j0 = i - m->bw < 0 ? 0 : i - m->bw;
    int j1 = i + m->bw > n - 1 ? n - 1 : i + m->bw;
    int full_end = (n / W) * W;
    for (int c = (j0 / W) * W; c < full_end && c <= j1; c += W) {
        for (int l = 0; l < W; ++l) {
            int j = c + l;
            double aij = (j >= j0 && j <= j1) ? band[i * m->rw + (j - i + m->bw)] : 0.0;
            lane[l] = (aij * x[j]) * 1.0;
        }
        sum += oracle_tree_reduce(lane, W);
    }
    int start = full_end > j0 ? full_end : j0;
    for (int j = start; j <= j1; ++j) sum += (band[i * m->rw + (j - i + m->bw)] * x[j]) * 1.0;
    return sum;
}

static double diag_dot(const OModel* m, const double* diag, int i, const double* x) {
    /* M_ff rows are diagonal: every chunk but the one holding i reduces to zero */
    (void)m;
    return (diag[i] * x[i]) * 1.0;
}

static int dense_lu(OModel* m) {
    int n = m->n;
    double* A = m->dense;
    for (int i = 0; i < n; ++i) m->piv[i] = i;
    double eps = 1.0e-14;
    for (int col = 0; col < n; ++col) {
        int prow = col;
        double pabs = fabs(A[(size_t)col * n + col]);
        for (int row = col + 1; row < n; ++row) {
            double cand = fabs(A[(size_t)row * n + col]);
            if (cand > pabs) {
                pabs = cand;
                prow = row;
            }
        }
        if (pabs <= eps) return STRUT_SINGULAR;
        if (prow != col) {
            for (int j = 0; j < n; ++j) {
                double t = A[(size_t)col * n + j];
                A[(size_t)col * n + j] = A[(size_t)prow * n + j];
                A[(size_t)prow * n + j] = t;
            }
            int t = m->piv[col];
            m->piv[col] = m->piv[prow];
            m->piv[prow] = t;
        }
        double diag = A[(size_t)col * n + col];
        if (fabs(diag) <= eps) return STRUT_SINGULAR;
        for (int row = col + 1; row < n; ++row) {
            double factor = A[(size_t)row * n + col] / diag;
            A[(size_t)row * n + col] = factor;
            if (factor == 0.0) continue;
            for (int j = col + 1; j < n; ++j) A[(size_t)row * n + j] -= factor * A[(size_t)col * n + j];
        }
    }
    return STRUT_OK;
}

static int band_general_factor(OModel* m) {
    int n = m->n, bw = m->bw;
    double* B = m->Keff;
    double tol = 1.0e-14;
    double* orig = (double*)malloc(sizeof(double) * (size_t)n * m->rw);
    memcpy(orig, B, sizeof(double) * (size_t)n * m->rw);
    m->dense_mode = 0;
    int rc = STRUT_OK;
    for (int k = 0; k < n; ++k) {
        int i1 = k + bw > n - 1 ? n - 1 : k + bw;
        int prow = k;
        double pabs = 0.0;
        for (int row = k; row <= i1; ++row) {
            int sl = gslot(m, row, k);
            if (sl < 0) continue;
            double cand = fabs(B[sl]);
            if (cand > pabs) {
                pabs = cand;
                prow = row;
            }
        }
        if (pabs <= tol) {
            rc = STRUT_SINGULAR;
            break;
        }
        if (prow != k) {
            if (!m->dense) {
                m->dense = (double*)malloc(sizeof(double) * (size_t)n * n);
                m->piv = (int*)malloc(sizeof(int) * n);
            }
            memset(m->dense, 0, sizeof(double) * (size_t)n * n);
            for (int row = 0; row < n; ++row) {
                int c0 = row - bw < 0 ? 0 : row - bw;
                int c1 = row + bw > n - 1 ? n - 1 : row + bw;
                for (int col = c0; col <= c1; ++col) m->dense[(size_t)row * n + col] = orig[gslot(m, row, col)];
            }
            rc = dense_lu(m);
            m->dense_mode = 1;
            __atomic_add_fetch(&g_dense_fallbacks, 1, __ATOMIC_RELAXED);
            break;
        }
        double diag = B[gslot(m, k, k)];
        if (fabs(diag) <= tol) {
            rc = STRUT_SINGULAR;
            break;
        }
        int j1 = k + bw > n - 1 ? n - 1 : k + bw;
        for (int i = k + 1; i <= i1; ++i) {
            int ik = gslot(m, i, k);
            if (ik < 0) continue;
            double factor = B[ik] / diag;
            B[ik] = factor;
            if (factor == 0.0) continue;
            for (int j = k + 1; j <= j1; ++j) {
                int kj = gslot(m, k, j), ij = gslot(m, i, j);
                if (ij < 0 || kj < 0) continue;
                B[ij] -= factor * B[kj];
            }
        }
    }
    free(orig);
    return rc;
}

static int band_general_solve(OModel* m, const double* rhs, double* x) {
    int n = m->n, bw = m->bw;
    if (m->dense_mode) {
        double* A = m->dense;
        for (int i = 0; i < n; ++i) {
            double s = rhs[m->piv[i]];
            for (int j = 0; j < i; ++j) s -= A[(size_t)i * n + j] * m->work[j];
            m->work[i] = s;
        }
        for (int i = n - 1; i >= 0; --i) {
            double s = m->work[i];
            for (int j = i + 1; j < n; ++j) s -= A[(size_t)i * n + j] * x[j];
            x[i] = s / A[(size_t)i * n + i];
        }
        return STRUT_OK;
    }
    const double* B = m->Keff;
    for (int i = 0; i < n; ++i) {
        double sum = rhs[i];
        int j0 = i - bw < 0 ? 0 : i - bw;
        for (int j = j0; j < i; ++j) sum -= B[gslot(m, i, j)] * m->work[j];
        m->work[i] = sum;
    }
    for (int i = n - 1; i >= 0; --i) {
        double sum = m->work[i];
        int j1 = i + bw > n - 1 ? n - 1 : i + bw;
        for (int j = i + 1; j <= j1; ++j) sum -= B[gslot(m, i, j)] * x[j];
        double diag = B[gslot(m, i, i)];
        if (diag == 0.0) return STRUT_SINGULAR;
        x[i] = sum / diag;
    }
    return STRUT_OK;
}

#define SSLOT(bw, row, col) ((row) * ((bw) + 1) + ((row) - (col)))

static int band_spd_factor(OModel* m) {
    int n = m->n, bw = m->bw;
    double* S = m->Kspd;
    for (int row = 0; row < n; ++row) {
        int first = row - bw < 0 ? 0 : row - bw;
        for (int col = first; col < row; ++col) {
            double sum = S[SSLOT(bw, row, col)];
            int k0 = first;
            int cf = col - bw < 0 ? 0 : col - bw;
            if (cf > k0) k0 = cf;
            for (int k = k0; k < col; ++k) sum -= S[SSLOT(bw, row, k)] * S[SSLOT(bw, col, k)];
            double diag = S[SSLOT(bw, col, col)];
            if (diag == 0.0) return STRUT_SINGULAR;
            S[SSLOT(bw, row, col)] = sum / diag;
        }
        double ds = S[SSLOT(bw, row, row)];
        for (int k = first; k < row; ++k) {
            double v = S[SSLOT(bw, row, k)];
            ds -= v * v;
        }
        if (ds <= 0.0) return STRUT_SINGULAR;
        S[SSLOT(bw, row, row)] = sqrt(ds);
    }
    return STRUT_OK;
}

static int band_spd_solve(OModel* m, const double* rhs, double* x) {
    int n = m->n, bw = m->bw;
    const double* S = m->Kspd;
    for (int row = 0; row < n; ++row) {
        int first = row - bw < 0 ? 0 : row - bw;
        double sum = rhs[row];
        for (int col = first; col < row; ++col) sum -= S[SSLOT(bw, row, col)] * m->work[col];
        double diag = S[SSLOT(bw, row, row)];
        if (diag == 0.0) return STRUT_SINGULAR;
        m->work[row] = sum / diag;
    }
    for (int i = 0; i < n; ++i) x[i] = m->work[i];
    for (int row = n - 1; row >= 0; --row) {
        double diag = S[SSLOT(bw, row, row)];
        if (diag == 0.0) return STRUT_SINGULAR;
        x[row] /= diag;
        double xv = x[row];
        int first = row - bw < 0 ? 0 : row - bw;
        for (int col = first; col < row; ++col) x[col] -= S[SSLOT(bw, row, col)] * xv;
    }
    return STRUT_OK;
}

/* C_ff rebuild (transient_nonlinear.mojo:2302-2335) and the effective band
 * (load_reduced_matrix K_ff, add_reduced_matrix C_ff*a1, add_reduced_matrix M_ff*a0). */
static int build_keff(OModel* m) {
    const StrutModelDesc* d = m->d;
    int n = m->n, bw = m->bw;
    size_t bsz = (size_t)n * m->rw;
    if (m->has_damping) {
        for (size_t i = 0; i < bsz; ++i) m->C[i] = 0.0;
        if (d->alpha_m != 0.0) {
            for (int i = 0; i < n; ++i) {
                for (int j = i - bw; j <= i + bw; ++j) {
                    if (j < 0 || j >= n) continue;
                    m->C[gslot(m, i, j)] = d->alpha_m * (i == j ? m->Mrff[i] : 0.0);
                }
            }
        }
        for (size_t i = 0; i < bsz; ++i) {
            if (d->beta_k != 0.0) m->C[i] += d->beta_k * m->K[i];
            if (d->beta_k_init != 0.0) m->C[i] += d->beta_k_init * m->Kinit[i];
            if (d->beta_k_comm != 0.0) m->C[i] += d->beta_k_comm * m->Kcomm[i];
        }
    }
    if (!m->spd) {
        for (size_t i = 0; i < bsz; ++i) m->Keff[i] = m->K[i];
        if (m->has_damping && m->a1 != 0.0)
            for (size_t i = 0; i < bsz; ++i) m->Keff[i] += m->a1 * m->C[i];
        if (m->a0 != 0.0)
            for (int i = 0; i < n; ++i) m->Keff[gslot(m, i, i)] += m->a0 * m->Mff[i];
        /* off-diagonal entries of a0 * M_ff add 0.0 */
        return STRUT_OK;
    }
    /* BandSPD: lower triangle with the 1e-10 symmetry check (linear_solver_backend.mojo:
     * 266-271, 1936-1948) */
    for (int i = 0; i < n; ++i) {
        int j0 = i - bw < 0 ? 0 : i - bw;
        for (int j = j0; j <= i; ++j) {
            double lo = m->K[gslot(m, i, j)], up = m->K[gslot(m, j, i)];
            if (fabs(lo - up) > 1.0e-10) return STRUT_BAD_ARG;
            m->Kspd[SSLOT(bw, i, j)] = lo;
        }
    }
    if (m->has_damping && m->a1 != 0.0) {
        for (int i = 0; i < n; ++i) {
            int j0 = i - bw < 0 ? 0 : i - bw;
            for (int j = j0; j <= i; ++j) {
                double lo = m->C[gslot(m, i, j)], up = m->C[gslot(m, j, i)];
                if (fabs(lo - up) > 1.0e-10) return STRUT_BAD_ARG;
                m->Kspd[SSLOT(bw, i, j)] += m->a1 * lo;
            }
        }
    }
    for (int i = 0; i < n; ++i) m->Kspd[SSLOT(bw, i, i)] += m->a0 * m->Mff[i];
    return STRUT_OK;
}

static void scatter_u(OModel* m) {
    const StrutModelDesc* d = m->d;
    for (int dof = 0; dof < d->num_dofs; ++dof) {
        int fi = d->free_index[dof];
        if (fi >= 0) m->u[dof] = m->u_f[fi];
    }
    if (m->has_mpc) mpc_enforce(m, m->u);
}

static int initial_assembly(OModel* m) {
    int rc = assemble(m, 0, 0);
    if (rc != STRUT_OK) return rc;
    size_t bsz = (size_t)m->n * m->rw;
    int initial_tangent = m->d->algorithm == STRUT_ALGORITHM_MODIFIED_NEWTON_INITIAL;
    for (int k = 0; k < m->d->num_attempts; ++k)
        if (m->d->attempts[k].algorithm == STRUT_ALGORITHM_MODIFIED_NEWTON_INITIAL) initial_tangent = 1;
    if (m->d->beta_k_init != 0.0 || initial_tangent) memcpy(m->Kinit, m->K, sizeof(double) * bsz);
    if (m->d->beta_k_comm != 0.0) memcpy(m->Kcomm, m->K, sizeof(double) * bsz);
    for (int e = 0; e < m->d->num_elements; ++e)
        for (int ip = 0; ip < m->elems[e].nip; ++ip) oracle_section_revert(&m->elems[e].sst[ip]);
    return STRUT_OK;
}

static double simd_sumsq(const double* x, int n) { return oracle_simd_dot(x, x, n); }

/* Section recorders after the step (transient_nonlinear.mojo:3537-3605).  forceBeamColumn2d:
 * from the basic state the step left (helpers.mojo:1974-2040); dispBeamColumn2d: the section at
 * the deformation of the step's displacements (2043-2156); forceBeamColumn3d: from the basic
 * state of the recorder's state determination, which the element-force pass ran since such an
 * element is also recorded (2158-2300); dispBeamColumn3d: beam_column3d_nonlinear.mojo:578-640.
 * Evaluating a section sets its trial state from the committed one only. */
static int record_sections(OModel* m, int step) {
    const StrutModelDesc* d = m->d;
    if (!m->sec_hist || d->num_record_sections <= 0) return STRUT_OK;
    const int W = m->nd == 6 ? 2 : 4;
    for (int k = 0; k < d->num_record_sections; ++k) {
        const StrutSectionRecord* sr = &d->record_sections[k];
        OElement* el = &m->elems[sr->element];
        const int ip = sr->section;
        const int defo = sr->kind == STRUT_SECTION_DEFORMATION;
        const double xi = el->xi[ip];
        double* out = m->sec_hist + ((size_t)step * d->num_record_sections + k) * W;
        double ug[12];
        for (int a = 0; a < m->nd; ++a) ug[a] = m->u[el->desc->dof[a]];
        switch (el->desc->type) {
        case STRUT_ELEM_FORCE_BEAM_COLUMN_2D:
            if (defo) {
                out[0] = el->eps0[ip];
                out[1] = el->kappa[ip];
            } else {
                out[0] = el->q[0] + 0.0;
                out[1] = (xi - 1.0) * el->q[1] + xi * el->q[2] + 0.0;
            }
            break;
        case STRUT_ELEM_DISP_BEAM_COLUMN_2D: {
            const double c = el->c_div, s = el->s_div, L = el->L, inv_L = 1.0 / L;
            double ul[6];
            ul[0] = c * ug[0] + s * ug[1];
            ul[1] = -s * ug[0] + c * ug[1];
            ul[2] = ug[2];
            ul[3] = c * ug[3] + s * ug[4];
            ul[4] = -s * ug[3] + c * ug[4];
            ul[5] = ug[5];
            const double eps0 = (-inv_L) * ul[0] + inv_L * ul[3];
            const double kappa = ((-6.0 + 12.0 * xi) / (L * L)) * ul[1] + ((-4.0 + 6.0 * xi) / L) * ul[2] +
                                 ((6.0 - 12.0 * xi) / (L * L)) * ul[4] + ((-2.0 + 6.0 * xi) / L) * ul[5];
            if (defo) {
                out[0] = eps0;
                out[1] = kappa;
            } else {
                double r[5];
                oracle_section_response(el->sec, &el->sst[ip], eps0, kappa, r);
                out[0] = r[0] + 0.0;
                out[1] = r[1] + 0.0;
            }
            break;
        }
        case STRUT_ELEM_FORCE_BEAM_COLUMN_3D: {
            const double dx = el->x2[0] - el->x1[0], dy = el->x2[1] - el->x1[1], dz = el->x2[2] - el->x1[2];
            const double L = sqrt(dx * dx + dy * dy + dz * dz);
            const double rot_i = (dx * ug[3] + dy * ug[4] + dz * ug[5]) / L;
            const double rot_j = (dx * ug[9] + dy * ug[10] + dz * ug[11]) / L;
            const double twist = (rot_j - rot_i) / L;
            if (defo) {
                out[0] = el->eps0[ip];
                out[1] = el->kz[ip];
                out[2] = el->ky[ip];
                out[3] = twist;
            } else {
                out[0] = el->q5[0] + 0.0;
                out[1] = (xi - 1.0) * el->q5[1] + xi * el->q5[2] + 0.0;
                out[2] = (xi - 1.0) * el->q5[3] + xi * el->q5[4] + 0.0;
                out[3] = el->G * el->J * twist;
            }
            break;
        }
        case STRUT_ELEM_DISP_BEAM_COLUMN_3D: {
            double kin[4];
            int rc = oracle_dbc3d_section_kinematics(el, ug, ip, kin);
            if (rc != STRUT_OK) return rc;
            if (defo) {
                out[0] = kin[0];
                out[1] = kin[2];
                out[2] = -kin[1];
                out[3] = kin[3];
            } else {
                double r[9];
                oracle_section3d_response(el->sec3, &el->sst[ip], kin[0], kin[1], kin[2], r);
                out[0] = r[0];
                out[1] = r[2];
                out[2] = -r[1];
                out[3] = el->G * el->J * kin[3];
            }
            break;
        }
        default:
            return STRUT_UNSUPPORTED;
        }
    }
    return STRUT_OK;
}

/* Recorders after the step's commit (transient_nonlinear.mojo:3225-3300): node displacements,
 * and element forces computed once per element and step.  A 3D beam-column's force comes from
 * a full element state determination at the converged displacements
 * (helpers.mojo:544-775), which for forceBeamColumn3d also updates its trial basic forces and
 * section deformations, so recording an element is part of the trajectory. */
static int record_step(OModel* m, int step, double* disp_hist, double* eforce_hist) {
    const StrutModelDesc* d = m->d;
    int nd = m->nd;
    if (disp_hist)
        for (int j = 0; j < d->num_record_dofs; ++j)
            disp_hist[(size_t)step * d->num_record_dofs + j] = m->u[d->record_dofs[j]];
    for (int j = 0; j < d->num_record_elements; ++j) {
        int eidx = d->record_elements[j];
        int first = j;
        for (int i = 0; i < j; ++i)
            if (d->record_elements[i] == eidx) {
                first = i;
                break;
            }
        double* out = eforce_hist ? eforce_hist + ((size_t)step * d->num_record_elements + j) * nd : 0;
        if (first != j) {
            if (out) memcpy(out, eforce_hist + ((size_t)step * d->num_record_elements + first) * nd,
                            sizeof(double) * nd);
            continue;
        }
        OElement* el = &m->elems[eidx];
        double ug[12], f[12], k[144];
        for (int a = 0; a < nd; ++a) ug[a] = m->u[el->desc->dof[a]];
        if (el->desc->type == STRUT_ELEM_FORCE_BEAM_COLUMN_2D) {
            oracle_fbc2d_force_from_basic(el, ug, f);
        } else {
            int rc = element_state(el, ug, k, f);
            if (rc != STRUT_OK) return rc;
        }
        if (out) memcpy(out, f, sizeof(double) * nd);
    }
    return record_sections(m, step);
}

/* The step's solver chain (transient_nonlinear.mojo:758-830): the attempts as given, or the
 * primary settings followed by Newton when the primary algorithm is not Newton. */
static int resolve_chain(const StrutModelDesc* d, StrutSolverAttempt* at) {
    if (d->num_attempts > 0) {
        for (int k = 0; k < d->num_attempts; ++k) at[k] = d->attempts[k];
        return d->num_attempts;
    }
    at[0].algorithm = d->algorithm;
    at[0].test_type = d->test_type;
    at[0].max_iters = d->max_iters;
    at[0].tol = d->tol;
    if (d->algorithm == STRUT_ALGORITHM_NEWTON) return 1;
    at[1] = at[0];
    at[1].algorithm = STRUT_ALGORITHM_NEWTON;
    return 2;
}

/* The force_basic_q blocks of every element (2D: q, eps0, kappa, v; 3D: q5, eps0, ky, kz),
 * saved at a step's start and put back before a retry (transient_nonlinear.mojo:1925-1942). */
typedef struct {
    double q[3], eps0[STRUT_MAX_INT_PTS], kappa[STRUT_MAX_INT_PTS], v[3];
    double q5[5], ky[STRUT_MAX_INT_PTS], kz[STRUT_MAX_INT_PTS];
} OBasicState;

static void basic_save(const OElement* e, OBasicState* b) {
    memcpy(b->q, e->q, sizeof(b->q));
    memcpy(b->eps0, e->eps0, sizeof(b->eps0));
    memcpy(b->kappa, e->kappa, sizeof(b->kappa));
    memcpy(b->v, e->v, sizeof(b->v));
    memcpy(b->q5, e->q5, sizeof(b->q5));
    memcpy(b->ky, e->ky, sizeof(b->ky));
    memcpy(b->kz, e->kz, sizeof(b->kz));
}

static void basic_restore(OElement* e, const OBasicState* b) {
    memcpy(e->q, b->q, sizeof(b->q));
    memcpy(e->eps0, b->eps0, sizeof(b->eps0));
    memcpy(e->kappa, b->kappa, sizeof(b->kappa));
    memcpy(e->v, b->v, sizeof(b->v));
    memcpy(e->q5, b->q5, sizeof(b->q5));
    memcpy(e->ky, b->ky, sizeof(b->ky));
    memcpy(e->kz, b->kz, sizeof(b->kz));
}

static int run_steps_chain(OModel* m, int steps, double* disp_hist, double* eforce_hist,
                           int* iters_hist, int* failed_step, const StrutSolverAttempt* chain,
                           int n_att, OBasicState* base, double* u_base);

static int run_steps(OModel* m, int steps, double* disp_hist, double* eforce_hist,
                     int* iters_hist, int* failed_step) {
    const StrutModelDesc* d = m->d;
    StrutSolverAttempt chain[STRUT_MAX_ATTEMPTS];
    const int n_att = resolve_chain(d, chain);
    OBasicState* base = n_att > 1 ? (OBasicState*)calloc((size_t)(d->num_elements > 0 ? d->num_elements : 1),
                                                         sizeof(OBasicState)) : 0;
    double* u_base = n_att > 1 ? (double*)calloc((size_t)(m->n > 0 ? m->n : 1), sizeof(double)) : 0;
    int rc_out = run_steps_chain(m, steps, disp_hist, eforce_hist, iters_hist, failed_step, chain, n_att,
                                 base, u_base);
    free(base);
    free(u_base);
    return rc_out;
}

static int run_steps_chain(OModel* m, int steps, double* disp_hist, double* eforce_hist,
                           int* iters_hist, int* failed_step, const StrutSolverAttempt* chain,
                           int n_att, OBasicState* base, double* u_base) {
    const StrutModelDesc* d = m->d;
    int n = m->n;
    double dt = d->dt, beta = d->beta, gamma = d->gamma;
    double coeff = dt * dt * (0.5 - beta);
    if (failed_step) *failed_step = -1;
    for (int step = 0; step < steps; ++step) {
        memcpy(m->u_n, m->u_f, sizeof(double) * n);
        memcpy(m->v_n, m->v_f, sizeof(double) * n);
        memcpy(m->a_n, m->a_f, sizeof(double) * n);
        for (int i = 0; i < n; ++i) m->u_f[i] = m->u_n[i] + dt * m->v_n[i] + coeff * m->a_n[i];
        scatter_u(m);
        double t = (double)(step + 1) * dt;
        for (int dof = 0; dof < d->num_dofs; ++dof) m->Fext[dof] = d->f_const ? d->f_const[dof] : 0.0;
        for (int x = 0; x < d->num_excitations; ++x) {
            const StrutExcitation* ex = &d->excitation[x];
            if (ex->direction < 1) continue;
            double ag = path_eval(ex, t);
            for (int dof = 0; dof < d->num_dofs; ++dof) {
                if ((dof % d->ndf) + 1 == ex->direction) {
                    double load = 0.0;
                    load += -d->mass[dof] * ag;
                    m->Fext[dof] += load;
                }
            }
        }
        if (m->has_mpc) {
            /* F_const is collapsed once at load, the inertia load of each excitation every
             * step (loader.mojo:2344, transient_nonlinear.mojo:1836-1848) */
            int nd = d->num_dofs;
            double* acc = (double*)calloc((size_t)(nd > 0 ? nd : 1), sizeof(double));
            double* inert = (double*)calloc((size_t)(nd > 0 ? nd : 1), sizeof(double));
            double* red = (double*)calloc((size_t)(nd > 0 ? nd : 1), sizeof(double));
            for (int dof = 0; dof < nd; ++dof) inert[dof] = d->f_const ? d->f_const[dof] : 0.0;
            mpc_collapse_vector(m, inert, acc);
            for (int x = 0; x < d->num_excitations; ++x) {
                const StrutExcitation* ex = &d->excitation[x];
                if (ex->direction < 1) continue;
                double ag = path_eval(ex, t);
                for (int dof = 0; dof < nd; ++dof) {
                    inert[dof] = 0.0;
                    if ((dof % d->ndf) + 1 == ex->direction) inert[dof] += -d->mass[dof] * ag;
                }
                mpc_collapse_vector(m, inert, red);
                for (int dof = 0; dof < nd; ++dof) acc[dof] += red[dof];
            }
            for (int dof = 0; dof < nd; ++dof) {
                int fi = d->free_index[dof];
                if (fi >= 0) m->P_f[fi] = acc[dof];
            }
            free(acc);
            free(inert);
            free(red);
        } else {
            for (int dof = 0; dof < d->num_dofs; ++dof) {
                int fi = d->free_index[dof];
                if (fi >= 0) m->P_f[fi] = m->Fext[dof];
            }
        }
        int converged = 0;
        int it = 0, step_iters = 0;
        if (n_att > 1) {
            for (int e = 0; e < d->num_elements; ++e) basic_save(&m->elems[e], &base[e]);
            memcpy(u_base, m->u_f, sizeof(double) * n);
        }
        for (int att = 0; att < n_att && !converged; ++att) {
        const int alg = chain[att].algorithm, test = chain[att].test_type, max_iters = chain[att].max_iters;
        const double tol = chain[att].tol;
        if (att > 0) {
            /* back to the step's start: u at the predictor, basic states, fiber trial states */
            memcpy(m->u_f, u_base, sizeof(double) * n);
            scatter_u(m);
            for (int e = 0; e < d->num_elements; ++e) {
                OElement* el = &m->elems[e];
                basic_restore(el, &base[e]);
                for (int ip = 0; ip < el->nip; ++ip) oracle_section_revert(&el->sst[ip]);
            }
        }
        for (it = 0; it < max_iters; ++it) {
            m->newton_iters++;
            int rc = assemble(m, 0, 0);
            if (rc != STRUT_OK) {
                if (failed_step) *failed_step = step;
                return rc;
            }
            /* Newton refreshes K_ff, C_ff and the factors every iteration; ModifiedNewton keeps
             * the first iteration's for the step, ModifiedNewtonInitial takes K_init_ff
             * (transient_nonlinear.mojo:2072-2085, 2236-2268, 2302-2335, 2421-2440) */
            const int refresh = alg == STRUT_ALGORITHM_NEWTON || it == 0;
            if (refresh) {
                if (alg == STRUT_ALGORITHM_MODIFIED_NEWTON_INITIAL)
                    memcpy(m->K, m->Kinit, sizeof(double) * (size_t)n * m->rw);
                rc = build_keff(m);
                if (rc != STRUT_OK) {
                    if (failed_step) *failed_step = step;
                    return rc;
                }
            }
            for (int i = 0; i < n; ++i) {
                double an = m->a0 * (m->u_f[i] - m->u_n[i]) - m->a2 * m->v_n[i] - m->a3 * m->a_n[i];
                m->at[i] = an;
                m->vt[i] = m->v_n[i] + dt * ((1.0 - gamma) * m->a_n[i] + gamma * an);
            }
            int ndofs = d->num_dofs;
            (void)ndofs;
            for (int dof = 0; dof < d->num_dofs; ++dof) {
                int i = d->free_index[dof];
                if (i < 0) continue;
                double damping = 0.0;
                if (m->has_damping) damping = band_row_dot(m, m->C, i, m->vt);
                double inertia = diag_dot(m, m->Mff, i, m->at);
                const double fint = m->has_mpc ? m->Fred[dof] : m->Fint[dof];
                m->R_f[i] = m->P_f[i] - fint - 0.0 - damping - inertia;
            }
            if (test == STRUT_TEST_NORM_UNBALANCE) {
                if (sqrt(simd_sumsq(m->R_f, n)) <= tol) {
                    converged = 1;
                    break;
                }
            }
            if (refresh) {
                rc = m->spd ? band_spd_factor(m) : band_general_factor(m);
                if (rc != STRUT_OK) {
                    if (failed_step) *failed_step = step;
                    return rc;
                }
                m->factorizations++;
            }
            rc = m->spd ? band_spd_solve(m, m->R_f, m->du) : band_general_solve(m, m->R_f, m->du);
            if (rc != STRUT_OK) {
                if (failed_step) *failed_step = step;
                return rc;
            }
            double max_diff = 0.0;
            for (int i = 0; i < n; ++i)
                if (fabs(m->du[i]) > max_diff) max_diff = fabs(m->du[i]);
            double norm = sqrt(simd_sumsq(m->du, n));
            double energy = fabs(oracle_simd_dot(m->du, m->R_f, n));
            for (int i = 0; i < n; ++i) m->u_f[i] += m->du[i];
            scatter_u(m);
            if (!isfinite(norm)) {
                if (failed_step) *failed_step = step;
                return STRUT_NAN;
            }
            if (test == STRUT_TEST_NORM_DISP_INCR && norm <= tol) {
                converged = 1;
                break;
            }
            if (test == STRUT_TEST_ENERGY_INCR && energy <= tol) {
                converged = 1;
                break;
            }
            if (test == STRUT_TEST_MAX_DISP_INCR && max_diff <= tol) {
                converged = 1;
                break;
            }
        }
        step_iters += converged ? it + 1 : max_iters;
        }
        if (iters_hist) iters_hist[step] = step_iters;
        if (!converged) {
            if (failed_step) *failed_step = step;
            return STRUT_NONCONVERGED;
        }
        /* commit: fibers, then the forceBeamColumn2d basic deformation sync */
        for (int e = 0; e < d->num_elements; ++e) {
            OElement* el = &m->elems[e];
            for (int ip = 0; ip < el->nip; ++ip) oracle_section_commit(&el->sst[ip]);
            if (el->desc->type == STRUT_ELEM_FORCE_BEAM_COLUMN_2D) {
                double ug[6], ul[6];
                for (int a = 0; a < 6; ++a) ug[a] = m->u[el->desc->dof[a]];
                double c = el->c_sync, s = el->s_sync;
                ul[0] = c * ug[0] + s * ug[1];
                ul[1] = -s * ug[0] + c * ug[1];
                ul[2] = ug[2];
                ul[3] = c * ug[3] + s * ug[4];
                ul[4] = -s * ug[3] + c * ug[4];
                ul[5] = ug[5];
                double chord = (ul[4] - ul[1]) / el->L_sync;
                el->v[0] = ul[3] - ul[0];
                el->v[1] = ul[2] - chord;
                el->v[2] = ul[5] - chord;
            }
        }
        for (int i = 0; i < n; ++i) {
            double an = m->a0 * (m->u_f[i] - m->u_n[i]) - m->a2 * m->v_n[i] - m->a3 * m->a_n[i];
            double vn = m->v_n[i] + dt * ((1.0 - gamma) * m->a_n[i] + gamma * an);
            m->a_f[i] = an;
            m->v_f[i] = vn;
        }
        int rrc = record_step(m, step, disp_hist, eforce_hist);
        if (rrc != STRUT_OK) {
            if (failed_step) *failed_step = step;
            return rrc;
        }
    }
    return STRUT_OK;
}

int oracle_run_transient(const StrutModelDesc* d, int steps, double* disp_hist,
                         double* eforce_hist, int* iters_hist, int* failed_step) {
    return oracle_run_transient_sections(d, steps, disp_hist, eforce_hist, iters_hist, failed_step, 0);
}

int oracle_run_transient_sections(const StrutModelDesc* d, int steps, double* disp_hist,
                                  double* eforce_hist, int* iters_hist, int* failed_step,
                                  double* section_hist) {
    OModel m;
    int rc = model_build(&m, d);
    m.sec_hist = section_hist;
    if (rc == STRUT_OK) rc = initial_assembly(&m);
    if (rc == STRUT_OK) rc = run_steps(&m, steps, disp_hist, eforce_hist, iters_hist, failed_step);
    model_free(&m);
    return rc;
}

int oracle_state_determination(const StrutModelDesc* d, const double* u_free,
                               double* f_int_free, double* band_out, int* half_bw) {
    OModel m;
    int rc = model_build(&m, d);
    if (rc == STRUT_OK) rc = initial_assembly(&m);
    if (rc == STRUT_OK) {
        memcpy(m.u_f, u_free, sizeof(double) * m.n);
        scatter_u(&m);
        rc = assemble(&m, 0, 0);
    }
    if (rc == STRUT_OK) rc = build_keff(&m);
    if (rc == STRUT_OK) {
        if (half_bw) *half_bw = m.bw;
        if (f_int_free)
            for (int dof = 0; dof < d->num_dofs; ++dof)
                if (d->free_index[dof] >= 0)
                    f_int_free[d->free_index[dof]] = m.has_mpc ? m.Fred[dof] : m.Fint[dof];
        if (band_out) {
            if (m.spd)
                memcpy(band_out, m.Kspd, sizeof(double) * (size_t)m.n * (m.bw + 1));
            else
                memcpy(band_out, m.Keff, sizeof(double) * (size_t)m.n * m.rw);
        }
    }
    model_free(&m);
    return rc;
}

int oracle_element_state(const StrutModelDesc* d, int elem, const double* u_elem, double* k,
                         double* f) {
    OModel m;
    int rc = model_build(&m, d);
    if (rc == STRUT_OK && (elem < 0 || elem >= d->num_elements)) rc = STRUT_BAD_ARG;
    if (rc == STRUT_OK) rc = element_state(&m.elems[elem], u_elem, k, f);
    model_free(&m);
    return rc;
}

typedef struct {
    const StrutModelDesc* models;
    int n, steps, next, total_iters, rc;
    int* record_status;
    int* record_failed_step;   /* optional: failing step of each record, -1 if none */
    int* record_iters;         /* optional: Newton iterations of each record          */
    pthread_mutex_t lock;
} BatchJob;

static void* batch_worker(void* arg) {
    BatchJob* job = (BatchJob*)arg;
    for (;;) {
        pthread_mutex_lock(&job->lock);
        int i = job->next++;
        pthread_mutex_unlock(&job->lock);
        if (i >= job->n) break;
        const StrutModelDesc* d = &job->models[i];
        int* iters = (int*)calloc(job->steps, sizeof(int));
        int failed = -1;
        int rc = oracle_run_transient(d, job->steps, 0, 0, iters, &failed);
        int tot = 0;
        for (int s = 0; s < job->steps; ++s) tot += iters[s];
        free(iters);
        pthread_mutex_lock(&job->lock);
        job->total_iters += tot;
        if (job->record_status) job->record_status[i] = rc;
        if (job->record_failed_step) job->record_failed_step[i] = failed;
        if (job->record_iters) job->record_iters[i] = tot;
        if (rc != STRUT_OK && job->rc == STRUT_OK) job->rc = rc;
        pthread_mutex_unlock(&job->lock);
    }
    return 0;
}

int oracle_run_transient_batch(const StrutModelDesc* models, int n, int steps, int nthreads,
                               int* total_iters, int* record_status, int* record_failed_step,
                               int* record_iters) {
    BatchJob job;
    memset(&job, 0, sizeof(job));
    job.record_status = record_status;
    job.record_failed_step = record_failed_step;
    job.record_iters = record_iters;
    job.models = models;
    job.n = n;
    job.steps = steps;
    pthread_mutex_init(&job.lock, 0);
    if (nthreads < 1) nthreads = 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nthreads);
    for (int i = 0; i < nthreads; ++i) pthread_create(&th[i], 0, batch_worker, &job);
    for (int i = 0; i < nthreads; ++i) pthread_join(th[i], 0);
    free(th);
    pthread_mutex_destroy(&job.lock);
    if (total_iters) *total_iters = job.total_iters;
    return job.rc;
}

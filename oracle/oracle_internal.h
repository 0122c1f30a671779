/* ORACLE -- test infrastructure only.  Internal declarations shared by the oracle sources. */
#ifndef STRUT_ORACLE_INTERNAL_H
#define STRUT_ORACLE_INTERNAL_H

#include "oracle.h"

typedef struct OSection {
    const StrutUniMaterial* mats;
    int W;
    int nfib;
    int nonlinear_count;
    double y_bar;
    int init_valid;
    double f00, f01, f11;
    int n_el;
    double *el_y, *el_a, *el_e;
    int n_s2, s2_ngroups;
    double *s2_y, *s2_a;
    int *s2_mat, *s2_goff, *s2_gpad;
    int n_c2, c2_ngroups;
    double *c2_y, *c2_a;
    int *c2_mat, *c2_goff, *c2_gpad;
    int n_s1;
    double *s1_y, *s1_a;
    int* s1_mat;
    int n_c1;
    double *c1_y, *c1_a;
    int* c1_mat;
} OSection;

/* Committed and trial states of one section instance: Steel02 slots, then Concrete02, then
 * Steel01, then Concrete01 (each family in its padded runtime order). */
typedef struct OSecState {
    int n;
    OFiberState* c;
    OFiberState* t;
} OSecState;

double oracle_tree_reduce(double* v, int w);
double oracle_simd_dot(const double* a, const double* b, int n);
int oracle_section_build(OSection* sd, const StrutUniMaterial* mats, int nmat,
                         const StrutFiber* fibers, int off, int nfib);
void oracle_section_free(OSection* sd);
void oracle_section_state_alloc(const OSection* sd, OSecState* st);
void oracle_section_state_free(OSecState* st);
void oracle_section_commit(OSecState* st);
void oracle_section_revert(OSecState* st);
void oracle_section_response(const OSection* sd, OSecState* st, double eps0, double kappa,
                             double out[5]);

/* FiberSection3d definition (fiber3d.mojo:156-188): elastic fibers and nonlinear fibers, each
 * in fiber order, coordinates relative to the area centroid. */
typedef struct OSection3d {
    const StrutUniMaterial* mats;
    int W;
    int nfib;
    double y_bar, z_bar;
    int n_el;
    double *el_y, *el_z, *el_a, *el_e;
    int n_nl;
    double *nl_y, *nl_z, *nl_a;
    int* nl_mat;
} OSection3d;

int oracle_section3d_build(OSection3d* sd, const StrutUniMaterial* mats, int nmat,
                           const StrutFiber* fibers, int off, int nfib);
void oracle_section3d_free(OSection3d* sd);
void oracle_section3d_state_alloc(const OSection3d* sd, OSecState* st);
/* out = {N, My, Mz, k11, k12, k13, k22, k23, k33} */
void oracle_section3d_response(const OSection3d* sd, OSecState* st, double eps0, double ky,
                               double kz, double out[9]);

/* One frame element's persistent data. */
typedef struct OElement {
    const StrutFrameElement* desc;
    const OSection* sec;
    int nip;
    double xi[STRUT_MAX_INT_PTS], w[STRUT_MAX_INT_PTS];
    double L;        /* hypot(dx, dy) */
    double c, s;      /* dx * (1/L): forceBeamColumn2d cached geometry */
    double c_div, s_div; /* dx / L: dispBeamColumn2d */
    double L_sync;   /* sqrt(dx*dx + dy*dy) used by the commit-time basic-state sync */
    double c_sync, s_sync;
    /* force_basic_q block: q0..q2, eps0[nip], kappa[nip], v0..v2 (loader.mojo:1757-1771) */
    double q[3];
    double eps0[STRUT_MAX_INT_PTS], kappa[STRUT_MAX_INT_PTS];
    double v[3];
    OSecState* sst; /* nip section states */
    /* 3D elements (12 dofs) */
    const OSection3d* sec3;
    double R[9];            /* rows: local x, y, z axes (undeformed geometry)        */
    double x1[3], x2[3];    /* end coordinates (Corotational rotation)              */
    double inv_L3;          /* 1/L cached by forceBeamColumn3d                      */
    double G, J;
    /* forceBeamColumn3d force_basic_q block: q0..q4, eps0[nip], ky[nip], kz[nip]
     * (loader.mojo:1836-1840) */
    double q5[5];
    double ky[STRUT_MAX_INT_PTS], kz[STRUT_MAX_INT_PTS];
    /* counters */
    long local_iters;
    long section_evals;
} OElement;

int oracle_fbc2d(OElement* e, const double u_global[6], double k[36], double f[6]);
int oracle_dbc2d(OElement* e, const double u_global[6], double k[36], double f[6]);
void oracle_fbc2d_force_from_basic(const OElement* e, const double u_global[6], double f[6]);
int oracle_rotation3d(const double x1[3], const double x2[3], int has_vecxz, const double* vecxz,
                      double R[9]);
int oracle_fbc3d(OElement* e, const double u_global[12], double k[144], double f[12]);
int oracle_dbc3d(OElement* e, const double u_global[12], double k[144], double f[12]);
int oracle_dbc3d_section_kinematics(const OElement* e, const double u_global[12], int ip, double out[4]);

#endif

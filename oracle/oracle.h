/*
 * ORACLE -- test infrastructure only (CPU FP64 restatement of Strut's hot path).  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load liboracle.so.
 */
#ifndef STRUT_ORACLE_H
#define STRUT_ORACLE_H

#include "strut_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* History slots of one fiber (subset of UniMaterialState, core.mojo:121-201). */
enum { S2_EPSMIN = 0, S2_EPSMAX, S2_EPSPL, S2_EPSS0, S2_SIGS0, S2_EPSR, S2_SIGR };
enum { C2_ECMIN = 0, C2_DEPT = 1 };
enum { S1_EPSP = 0, S1_ALPHA = 1 };
enum { C1_MIN = 0, C1_END = 1, C1_SLOPE = 2 };

typedef struct OFiberState {
    double eps, sig, tan;
    double h[7];
    int kon;
} OFiberState;

double oracle_initial_tangent(const StrutUniMaterial* m);
void oracle_fiber_init(const StrutUniMaterial* m, OFiberState* s);
void oracle_steel02_trial(const StrutUniMaterial* m, const OFiberState* c, OFiberState* t,
                          double eps);
void oracle_concrete02_trial(const StrutUniMaterial* m, const OFiberState* c, OFiberState* t,
                             double eps);
void oracle_steel01_trial(const StrutUniMaterial* m, const OFiberState* c, OFiberState* t,
                          double eps);
void oracle_concrete01_trial(const StrutUniMaterial* m, const OFiberState* c, OFiberState* t,
                             double eps);
void oracle_elastic_trial(const StrutUniMaterial* m, const OFiberState* c, OFiberState* t,
                          double eps);
void oracle_fiber_trial(const StrutUniMaterial* m, const OFiberState* c, OFiberState* t,
                        double eps);

/* ---- exported entry points (ctypes) ------------------------------------------------ */
void oracle_set_simd_width(int w);
int oracle_get_simd_width(void);
void oracle_material_path(const StrutUniMaterial* m, const double* strains, int n,
                          double* out);
int oracle_section_path(const StrutUniMaterial* mats, int nmat, const StrutFiber* fibers,
                        int nfib, const double* eps0_kappa, int npts, double* out);
/* Batched section micro-benchmark: n_inst independent copies of one section, each driven
 * along its own path (eps0_kappa: npts x n_inst x 2), commit after each point.
 * out: npts x n_inst x 5.  Used to cross-check the GPU section kernel. */
int oracle_section_batch_path(const StrutUniMaterial* mats, int nmat, const StrutFiber* fibers,
                              int nfib, int n_inst, const double* eps0_kappa, int npts,
                              double* out);
/* One FiberSection3d along npts (eps0, kappa_y, kappa_z) points (path: npts x 3), committing
 * after each; out: npts x 9 = N, My, Mz, k11, k12, k13, k22, k23, k33. */
int oracle_shell4_stiffness(double E, double nu, double h, const double* x, const double* y, const double* z,
                            double* K);
int oracle_section3d_path(const StrutUniMaterial* mats, int nmat, const StrutFiber* fibers,
                          int nfib, const double* path, int npts, double* out);
/* Single-instance transient run (the reference's plain CPU path).  eforce_hist holds
 * 2*ndf values per recorded element and step. */
int oracle_run_transient(const StrutModelDesc* m, int steps, double* disp_hist,
                         double* eforce_hist, int* iters_hist, int* failed_step);
/* The same with the section recorders' values: steps x num_record_sections x (2 or 4). */
int oracle_run_transient_sections(const StrutModelDesc* m, int steps, double* disp_hist,
                                  double* eforce_hist, int* iters_hist, int* failed_step,
                                  double* section_hist);
/* One element state determination + assembly at u_free (parity entry). */
int oracle_state_determination(const StrutModelDesc* m, const double* u_free,
                               double* f_int_free, double* band_out, int* half_bw);
/* One element's global tangent (nd x nd) and resisting force (nd) at element displacements
 * u_elem (nd = 2 * ndf), from the element's initial state. */
int oracle_element_state(const StrutModelDesc* m, int elem, const double* u_elem, double* k,
                         double* f);
/* Number of BandGeneral factorisations that fell back to dense partial-pivot LU. */
long oracle_dense_fallbacks(void);
/* Number of forceBeamColumn2d subdivision passes in which every scheme failed. */
long oracle_subdivisions(void);
/* Multi-instance run over nthreads host threads (CPU baseline leg, batch parity).  Optional
 * n-entry outputs: record_status (each record's status), record_failed_step (its failing step
 * or -1) and record_iters (its Newton iterations); the return value is the first failure seen. */
int oracle_run_transient_batch(const StrutModelDesc* models, int n, int steps, int nthreads,
                               int* total_iters, int* record_status, int* record_failed_step,
                               int* record_iters);

#ifdef __cplusplus
}
#endif

#endif

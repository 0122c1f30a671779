/*
 * strut_cuda.h -- C ABI of the B200 (sm_100a) nonlinear-transient hot path of Strut.
 *
 * Everything here is plain C11: integer status codes, plain pointers and sizes, FP64
 * mechanics.  The caller owns every host buffer it passes; the library copies what it needs
 * into device memory and never keeps a caller pointer past the call.
 *
 * The entry points replace the per-Newton-iteration block and the step-level calls of Strut's
 * transient nonlinear driver (reference paths are relative to the Strut project root):
 *
 *   strut_gpu_create          <- model set-up done by src/mojo/solver/run_case/loader.mojo
 *                                (material defs 963-1100, per-element state 1700-1830,
 *                                DOF numbering 2393-2450) and
 *                                analysis/transient_nonlinear.mojo:830-1160
 *   strut_gpu_run_steps       <- analysis/transient_nonlinear.mojo:1698-3110 (step loop:
 *                                Newmark predictor, Newton loop, commit, post-step update)
 *   strut_gpu_state_determination
 *                             <- assemble_global_stiffness_and_internal_soa
 *                                (solver/assembly/stiffness_internal.mojo:1293-1460) followed
 *                                by load_reduced_matrix/add_reduced_matrix
 *                                (solver/run_case/linear_solver_backend.mojo:1877-1983)
 *   strut_gpu_factor_solve    <- factorize_loaded + solve
 *                                (linear_solver_backend.mojo:2174-2199, 2277-2305)
 *   strut_gpu_commit / revert <- fiber_section2d_commit_runtime_all /
 *                                fiber_section2d_revert_trial_runtime_all
 *                                (sections/fiber2d.mojo:4191-4252) and
 *                                _sync_force_beam_column2d_committed_basic_states
 *                                (solver/run_case/helpers.mojo:1832-1883)
 *   strut_gpu_section_path    <- src/mojo/section_path.mojo:354-560 (known-answer driver)
 *   strut_gpu_material_path   <- src/mojo/material_path.mojo:233-262 (known-answer driver)
 *   strut_gpu_section_eval_batch
 *                             <- fiber_section2d_set_trial_from_offset
 *                                (sections/fiber2d.mojo:3982-4024) over many section
 *                                instances at once (the fiber-state micro-benchmark path of
 *                                src/mojo/benchmarks_micro.mojo:234)
 *
 * Tag values follow src/mojo/tag_types.mojo so a Strut host can pass its own tags through.
 */
#ifndef STRUT_CUDA_H
#define STRUT_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define STRUT_ABI_VERSION 7
#define STRUT_MAX_INT_PTS 10

/* Status codes.  No entry point aborts the process. */
enum {
    STRUT_OK = 0,
    STRUT_NONCONVERGED = 1,   /* Newton (global) ran out of iterations at some step      */
    STRUT_SINGULAR = 2,       /* zero / tiny pivot, or a non-positive Cholesky diagonal  */
    STRUT_NAN = 3,            /* non-finite value in the state                           */
    STRUT_BAD_ARG = 4,        /* invalid input, sizes out of range                       */
    STRUT_CUDA_ERROR = 5,     /* a CUDA runtime call failed                              */
    STRUT_UNSUPPORTED = 6,    /* valid Strut input that this library does not implement  */
    STRUT_ELEMENT_FAILED = 7  /* forceBeamColumn final tangent recovery failed           */
};

/* UniMaterialTypeTag (tag_types.mojo:136-141). */
enum { STRUT_MAT_ELASTIC = 0, STRUT_MAT_STEEL01 = 1, STRUT_MAT_CONCRETE01 = 2,
       STRUT_MAT_STEEL02 = 3, STRUT_MAT_CONCRETE02 = 4 };

/* ElementTypeTag (tag_types.mojo:1-14). */
enum { STRUT_ELEM_FORCE_BEAM_COLUMN_2D = 2, STRUT_ELEM_DISP_BEAM_COLUMN_2D = 3,
       STRUT_ELEM_FORCE_BEAM_COLUMN_3D = 11, STRUT_ELEM_DISP_BEAM_COLUMN_3D = 12 };

/* geomTransf.  Corotational applies to the 3D beam-columns only: their local axes follow the
 * displaced end positions and they add the PDelta axial term (force_beam_column3d.mojo:
 * 510-547, beam_column3d_nonlinear.mojo:200-238). */
enum { STRUT_GEOM_LINEAR = 0, STRUT_GEOM_PDELTA = 1, STRUT_GEOM_COROTATIONAL = 2 };

/* AnalysisSystemTag (tag_types.mojo:43-51). */
enum { STRUT_SYSTEM_BAND_GENERAL = 1, STRUT_SYSTEM_BAND_SPD = 2 };

/* Transient test modes (transient_nonlinear.mojo:671-684). */
/* Newton variants (transient_nonlinear.mojo:650-668, 2072-2085, 2236-2268, 2421-2440): Newton
 * refreshes the tangent every iteration; ModifiedNewton takes the first iteration's tangent (and
 * the Rayleigh C built from it) for the whole step and factors once per step; ModifiedNewtonInitial
 * does the same with the initial tangent. */
enum { STRUT_ALGORITHM_NEWTON = 0, STRUT_ALGORITHM_MODIFIED_NEWTON = 1,
       STRUT_ALGORITHM_MODIFIED_NEWTON_INITIAL = 2 };

enum { STRUT_TEST_MAX_DISP_INCR = 0, STRUT_TEST_NORM_DISP_INCR = 1,
       STRUT_TEST_NORM_UNBALANCE = 2, STRUT_TEST_ENERGY_INCR = 3 };

/* Uniaxial material definition: UniMaterialDef (materials/uniaxial/core.mojo:48-118).
 * p[] holds p0..p10 exactly as Strut's loader fills them (loader.mojo:913-1100):
 *   Elastic    p0=E
 *   Steel01    p0=Fy p1=E0 p2=b
 *   Steel02    p0=Fy p1=E0 p2=b p3=R0 p4=cR1 p5=cR2 p6=a1 p7=a2 p8=a3 p9=a4 p10=sigInit
 *   Concrete02 p0=fc p1=epsc0 p2=fcu p3=epscu p4=rat p5=ft p6=Ets  (compression negative) */
typedef struct StrutUniMaterial {
    int32_t type;
    int32_t reserved;
    double p[11];
} StrutUniMaterial;

/* One fiber cell as discretised from patches / layers / direct fibers (fiber2d.mojo:37-56):
 * raw coordinates (not centroid-relative), area and an index into the material table. */
typedef struct StrutFiber {
    double y;
    double z;
    double area;
    int32_t material;
    int32_t reserved;
} StrutFiber;

/* A FiberSection2d / FiberSection3d: a contiguous run of fibers[]
 * (append_fiber_section2d_from_input, fiber2d.mojo:3881-3944; append_fiber_section3d_from_input,
 * fiber3d.mojo:654-720).  G and J (FiberSection3d params) give the torsional stiffness GJ/L of
 * 3D beam-columns. */
typedef struct StrutFiberSection {
    int32_t fiber_offset;
    int32_t fiber_count;
    int32_t dim;           /* 2 or 3                                            */
    int32_t reserved;
    double G;
    double J;
} StrutFiberSection;

/* Beam integration rule, already mapped to xi in [0,1] and weights x0.5
 * (beam_integration_rule, elements/beam_integration.mojo:224-243). */
typedef struct StrutBeamIntegration {
    int32_t num_int_pts;
    int32_t reserved;
    double xi[STRUT_MAX_INT_PTS];
    double w[STRUT_MAX_INT_PTS];
} StrutBeamIntegration;

/* A frame element: forceBeamColumn2d / dispBeamColumn2d (6 dofs) or forceBeamColumn3d /
 * dispBeamColumn3d (12 dofs, local axes from vecxz as in elements/utils.mojo:96-140). */
typedef struct StrutFrameElement {
    int32_t type;          /* STRUT_ELEM_*                                      */
    int32_t node_i;        /* node indices, 0-based                             */
    int32_t node_j;
    int32_t section;       /* index into sections[]                             */
    int32_t geom;          /* STRUT_GEOM_*                                      */
    int32_t integration;   /* index into integrations[]                         */
    int32_t dof[12];       /* global dof indices node*ndf + (d-1)               */
    double vecxz[3];       /* 3D only                                           */
    int32_t has_vecxz;
    int32_t reserved;
} StrutFrameElement;

/* A uniform excitation (pattern UniformExcitation + Path time series with dt,
 * time_series.mojo:61-90; transient_nonlinear.mojo:1823-1852).  direction is 1-based; a model
 * may carry up to two (the second one is an extension beyond Strut's single pattern). */
typedef struct StrutExcitation {
    int32_t direction;     /* 0 = unused                                        */
    int32_t count;         /* number of samples in values                       */
    const double* values;
    double dt;             /* Path dt                                           */
    double factor;
    double start_time;
    int32_t use_last;
    int32_t reserved;
} StrutExcitation;

/* ShellMITC4 on an ElasticMembranePlateSection (elements/shell4.mojo:10-363): a linear
 * four-node shell whose 24 x 24 global stiffness is computed once from the node coordinates,
 * E, nu and the thickness h; its internal force is that stiffness times the element
 * displacements.  Requires ndm 3, ndf 6.  Its section's rho enters the lumped translational
 * masses through StrutModelDesc.mass (loader.mojo:2060-2100), not here. */
typedef struct StrutShellElement {
    int32_t nodes[4];      /* node indices, counter-clockwise                         */
    int32_t dof[24];       /* global dof indices node*6 + (d-1), nodes in order       */
    double E, nu, h;
} StrutShellElement;

/* One attempt of a step's solver chain (SolverAttemptInput, input_types.mojo; the retry loop of
 * transient_nonlinear.mojo:1925-1942).  algorithm STRUT_ALGORITHM_*, test_type STRUT_TEST_*. */
#define STRUT_MAX_ATTEMPTS 4
typedef struct StrutSolverAttempt {
    int32_t algorithm;
    int32_t test_type;
    int32_t max_iters;
    int32_t reserved;
    double tol;
} StrutSolverAttempt;

/* A section recorder entry (section_force / section_deformation recorders,
 * transient_nonlinear.mojo:1631-1655, 3537-3605): integration point `section` (0-based) of
 * element `element`.  Values per step (2D: 2, 3D: 4):
 *   forceBeamColumn2d  force  q0, (xi - 1) q1 + xi q2          deformation  eps0, kappa
 *                      (from the element's basic state after the step, helpers.mojo:1974-2040)
 *   dispBeamColumn2d   force  N, Mz of the section at          deformation  eps0, kappa
 *                      the displacements' deformation          (helpers.mojo:2043-2156)
 *   forceBeamColumn3d  force  q0, (xi-1) q1 + xi q2,           deformation  eps0, kappa_z,
 *                      (xi-1) q3 + xi q4, GJ twist                          kappa_y, twist
 *                      (after the recorder's state determination at the step's displacements,
 *                      helpers.mojo:2158-2300; the element is then also a recorded element)
 *   dispBeamColumn3d   force  N, Mz, -My, GJ twist             deformation  eps0, kappa_z,
 *                                                                           -kappa_y, twist
 *                      (beam_column3d_nonlinear.mojo:578-640) */
#define STRUT_SECTION_FORCE 0
#define STRUT_SECTION_DEFORMATION 1
typedef struct StrutSectionRecord {
    int32_t element;
    int32_t section;
    int32_t kind;     /* STRUT_SECTION_FORCE or STRUT_SECTION_DEFORMATION */
    int32_t reserved;
} StrutSectionRecord;

/* One analysis instance (one frame + one record). */
typedef struct StrutModelDesc {
    int32_t ndm;                 /* 2 (ndf 3) or 3 (ndf 6)                               */
    int32_t ndf;
    int32_t num_nodes;
    int32_t num_dofs;            /* num_nodes * ndf                                      */
    const double* node_coords;   /* num_nodes * ndm : x, y (, z)                         */
    int32_t num_materials;
    int32_t num_fibers;
    const StrutUniMaterial* materials;
    const StrutFiber* fibers;
    int32_t num_sections;
    int32_t num_integrations;
    const StrutFiberSection* sections;
    const StrutBeamIntegration* integrations;
    int32_t num_elements;
    int32_t num_free;
    const StrutFrameElement* elements;
    const int32_t* free_index;   /* num_dofs : free equation number or -1                */
    const double* mass;          /* num_dofs : M_total (lumped)                          */
    const double* mass_rayleigh; /* num_dofs : M_rayleigh_total                          */
    const double* f_const;       /* num_dofs : constant nodal loads (may be NULL)        */
    double alpha_m, beta_k, beta_k_init, beta_k_comm;   /* rayleigh                      */
    double dt, gamma, beta;      /* Newmark                                              */
    double tol;
    int32_t max_iters;
    int32_t test_type;           /* STRUT_TEST_*                                         */
    int32_t system;              /* STRUT_SYSTEM_*                                       */
    int32_t num_excitations;     /* 0..2                                                 */
    StrutExcitation excitation[2];
    /* recorders: displacement history of these dofs, global end forces of these elements */
    int32_t num_record_dofs;
    int32_t num_record_elements;
    const int32_t* record_dofs;
    const int32_t* record_elements;
    /* multi-point constraints, Transformation handler (loader.mojo:2239-2380): slave dof s
     * follows its retained dofs, u_s = sum_k coef_k u_{master_k} (equalDOF: one term with
     * coefficient 1; rigidDiaphragm: the constraint matrix row).  Slave dofs are neither free
     * nor fixed; K, F_int and loads are collapsed onto the retained dofs, and the band keeps
     * the half width detected from the elements' free dofs (slaves excluded), dropping coupled
     * entries outside it as Strut does (linear_solver_backend.mojo:413-427, 1481-1507).  A slave
     * dof may carry no mass.  num_slaves 0: none. */
    int32_t num_slaves;
    int32_t algorithm;             /* STRUT_ALGORITHM_* (0, Newton, when left zero)        */
    const int32_t* slave_dof;      /* num_slaves full dof indices                          */
    const int32_t* slave_ptr;      /* num_slaves + 1 offsets into the term arrays          */
    const int32_t* slave_master;   /* retained full dof of each term                       */
    const double* slave_coef;      /* coefficient of each term                             */
    /* linear shells, assembled after the frame elements as Strut's assembly groups them
     * (stiffness_internal.mojo: frames, then surfaces) */
    int32_t num_shells;
    int32_t reserved_shell;
    const StrutShellElement* shells;
    /* solver chain (analysis.solver_chain; transient_nonlinear.mojo:758-830, 1925-1942): when a
     * step does not converge with attempt k, u, the elements' basic state and the fibers' trial
     * state go back to the step's start (its Newmark predictor) and attempt k + 1 runs; the step
     * fails when the last attempt does.  num_attempts 0: the chain is the primary settings
     * (algorithm, test_type, max_iters, tol) followed, when the algorithm is not Newton, by Newton
     * with the same test, iterations and tolerance (Strut's automatic fallback, 804-829). */
    int32_t num_attempts;          /* 0 .. STRUT_MAX_ATTEMPTS                              */
    int32_t reserved_attempts;
    StrutSolverAttempt attempts[STRUT_MAX_ATTEMPTS];
    /* section recorders: their values every step (strut_gpu_get_section_history) */
    int32_t num_record_sections;
    int32_t reserved_sections;
    const StrutSectionRecord* record_sections;
} StrutModelDesc;

/* Per-run statistics (RuntimeProfileMetrics counters, solver/profile.mojo:37-74). */
typedef struct StrutStepStats {
    int64_t global_newton_iterations;  /* summed over instances                      */
    int64_t local_element_iterations;  /* forceBeamColumn corrector iterations       */
    int64_t section_evaluations;       /* section (integration point) evaluations    */
    int64_t fiber_updates;             /* fiber trial-state updates                  */
    int64_t factorizations;
    int32_t steps_done;
    int32_t failed_instance;           /* first instance with a non-OK status, or -1 */
    int32_t failed_step;
    int32_t status;
    int64_t fanned_out;                /* forceBeamColumn2d determinations whose attempts ran
                                          fanned out (StrutTuning.fan_out)               */
} StrutStepStats;

typedef struct StrutHandle StrutHandle;

/* Per-kernel timing of a handle's launches, measured with CUDA events on the handle's own
 * stream while profiling is enabled (no counterpart in the reference; used for rooflines).
 * Index: 0 element state, 1 instance Newton, 2 commit, 3 predictor, 4 post-step;
 * 5 the element critical path: bytes[5] sums, over element launches, the largest number of
 * forceBeamColumn local iterations one element ran in that launch (ms[5] = ms[0]).
 * bytes[0] counts, per section evaluation, one fiber-state update of every fiber: its committed
 * history read and its trial history written (Concrete02 80 B, Steel02 168 B, Steel01 56 B,
 * Concrete01 96 B per fiber), whether or not those bytes reach HBM; bytes[2] the commit's
 * reads and writes of the same histories. */
#define STRUT_PROF_KERNELS 8
typedef struct StrutKernelProfile {
    int64_t launches[STRUT_PROF_KERNELS];
    double ms[STRUT_PROF_KERNELS];
    double bytes[STRUT_PROF_KERNELS];   /* algorithmic HBM bytes moved by those launches */
} StrutKernelProfile;

/* ---- library ----------------------------------------------------------------------- */
int strut_gpu_abi_version(void);
/* Human readable text of the last error on this thread (never NULL). */
const char* strut_gpu_last_error(void);

/* ---- batched transient analysis ---------------------------------------------------- */
/* Copies num_instances model descriptions into device memory, performs the initial
 * assembly (K_init for betaKInit) and leaves every instance at step 0.  device < 0 keeps the
 * current device. */
int strut_gpu_create(const StrutModelDesc* models, int32_t num_instances, int32_t device,
                     StrutHandle** out);
int strut_gpu_destroy(StrutHandle* h);
int strut_gpu_num_instances(const StrutHandle* h);
/* Runs n_steps Newmark steps for every instance (predictor, Newton to the test tolerance,
 * commit, Newmark update).  An instance that fails (non-convergence, singular matrix, ...) is
 * masked out of the remaining steps while the others carry on; the first failure (instance,
 * step, status) is returned.  A single-instance handle stops at its failing step. */
int strut_gpu_run_steps(StrutHandle* h, int32_t n_steps, StrutStepStats* stats);
/* Copies recorder histories of one instance for steps [0, steps_done):
 * disp: steps x num_record_dofs, eforce: steps x num_record_elements x (2 ndf) global end
 * forces, iters: Newton iterations per step.  Any pointer may be NULL.  A handle holds either
 * 2D (ndf 3) or 3D (ndf 6) instances. */
int strut_gpu_get_history(StrutHandle* h, int32_t instance, double* disp, double* eforce,
                          int32_t* iters);
/* Same for all instances at once, instance-major, each block sized as for one instance
 * with that instance's recorder counts; offsets are the prefix sums of those sizes. */
int strut_gpu_get_history_all(StrutHandle* h, double* disp, double* eforce, int32_t* iters);
/* Section recorder values of one instance for steps [0, steps_done): steps x
 * num_record_sections x (2 for a 2D handle, 4 for a 3D one), in the order of the instance's
 * record_sections (see StrutSectionRecord).  Replaces the section recorder branch of Strut's
 * transient recorder loop (transient_nonlinear.mojo:3537-3605). */
int strut_gpu_get_section_history(StrutHandle* h, int32_t instance, double* out);
/* Status of every instance (STRUT_OK or the code it failed with), n_inst entries. */
int strut_gpu_instance_status(const StrutHandle* h, int32_t* status);
/* Current free displacement / velocity / acceleration vectors of one instance. */
int strut_gpu_get_state(StrutHandle* h, int32_t instance, double* u_free, double* v_free,
                        double* a_free);

/* Enables / disables per-launch event timing; enabling clears the accumulated profile. */
int strut_gpu_set_profiling(StrutHandle* h, int32_t enabled);
int strut_gpu_get_profile(const StrutHandle* h, StrutKernelProfile* out);
/* The cudaStream_t every kernel of this handle is launched on (for callers' own events). */
void* strut_gpu_stream(const StrutHandle* h);

/* Launch-shape choices of a handle.  No counterpart in the reference (Strut runs one CPU
 * thread); every choice gives the same results bit for bit and changes only the speed.
 *   fan_out      1: a forceBeamColumn2d element whose last state determination needed a
 *                subdivided increment runs the twelve attempts of its next first pass (three
 *                schemes x four subdivision levels, force_beam_column2d.mojo:1669-1763, each
 *                from the accepted state) on twelve CTAs at once, and the first success in
 *                Strut's order is kept; 0: the attempts run one after another.  Default 1.
 *   commit_team  threads per integration point in the commit kernel, 64 or 128 (default 128
 *                for up to 5 points, else 64; 128 needs at most 5 points).
 *   factor_ctas  CTAs of the cooperative wide-band factorisation (1 .. its resident limit;
 *                0: the default, as many as one panel has trailing tiles).
 *   element_threads  threads of an element CTA: 640 (default, one CTA per SM: the shortest
 *                per-element iteration), 320, 224 or 160 (2D only): as many CTAs per SM as
 *                registers and shared memory allow, more elements in flight.
 * strut_gpu_set_tuning with t = NULL restores the defaults. */
typedef struct StrutTuning {
    int32_t fan_out;
    int32_t commit_team;
    int32_t factor_ctas;
    int32_t element_threads;
    int32_t reserved[4];
} StrutTuning;
int strut_gpu_set_tuning(StrutHandle* h, const StrutTuning* t);
int strut_gpu_get_tuning(const StrutHandle* h, StrutTuning* out);
/* How many times a CTA of the cooperative wide-band factorisation polls a grid barrier before it
 * gives up (default 4194304); when one gives up, every CTA of the launch returns and the
 * instance ends with STRUT_CUDA_ERROR instead of the GPU waiting for good.  No counterpart in the
 * reference: failure-detection tests set it to 0 to make the wait run out on purpose.  A handle
 * without a wide band ignores it. */
int strut_gpu_set_wait_limit(StrutHandle* h, int32_t polls);

/* ---- single-iteration entries (parity tests) --------------------------------------- */
/* Sets the trial free displacements of every instance (concatenated in instance order),
 * runs element state determination + assembly and returns, concatenated per instance,
 * F_int at the free dofs and the effective band matrix (K + a1*C + a0*M in band storage,
 * n_free x (2*bw+1) for BandGeneral, n_free x (bw+1) for BandSPD).  Outputs may be NULL. */
int strut_gpu_state_determination(StrutHandle* h, const double* u_free, double* f_int_free,
                                  double* band_out);
/* Band width / storage width of one instance (so the caller can size band_out). */
int strut_gpu_band_info(const StrutHandle* h, int32_t instance, int32_t* half_bw,
                        int32_t* row_width);
/* Factors the effective matrix from the last state determination and solves K du = rhs
 * (rhs / du concatenated per instance). */
int strut_gpu_factor_solve(StrutHandle* h, const double* rhs, double* du);
/* trial -> committed for every fiber and element (fiber2d.mojo:4191; helpers.mojo:1832). */
int strut_gpu_commit(StrutHandle* h);
/* committed -> trial (fiber2d.mojo:4222). */
int strut_gpu_revert(StrutHandle* h);

/* ---- known-answer drivers ---------------------------------------------------------- */
/* section_path: one FiberSection2d, a path of (eps0, kappa) pairs; after each point the
 * section is committed.  out: n_points x 5 = N, Mz, k11, k12, k22. */
int strut_gpu_section_path(const StrutUniMaterial* materials, int32_t num_materials,
                           const StrutFiber* fibers, int32_t num_fibers,
                           const double* eps0_kappa, int32_t n_points, double* out);
/* section_path for one FiberSection3d (section_path.mojo:463-556): a path of (eps0, kappa_y,
 * kappa_z) triples, committed after each point.  out: n_points x 9 = N, My, Mz, k11, k12, k13,
 * k22, k23, k33 (fiber3d.mojo:769-836). */
int strut_gpu_section3d_path(const StrutUniMaterial* materials, int32_t num_materials,
                             const StrutFiber* fibers, int32_t num_fibers, const double* path,
                             int32_t n_points, double* out);
/* material_path: one uniaxial material, a strain history, commit after each strain (the
 * scalar uniaxial path of materials/uniaxial/ops.mojo:117-174). out: n x 2 stress, tangent. */
int strut_gpu_material_path(const StrutUniMaterial* material, const double* strains,
                            int32_t n, double* out);
/* Batched section evaluation: n_inst instances of one FiberSection2d, each with its own
 * fiber history.  Evaluates every instance at its (eps0, kappa) from committed state and
 * writes N, Mz, k11, k12, k22 per instance; if commit != 0 the trial state becomes the
 * committed state.  Repeated calls continue the same histories (state lives in the handle). */
typedef struct StrutSectionBatch StrutSectionBatch;
int strut_gpu_section_batch_create(const StrutUniMaterial* materials, int32_t num_materials,
                                   const StrutFiber* fibers, int32_t num_fibers,
                                   int32_t n_inst, StrutSectionBatch** out);
int strut_gpu_section_batch_destroy(StrutSectionBatch* b);
/* eps0_kappa_dev / resp_dev are DEVICE pointers (n_inst x 2 and n_inst x 5). */
int strut_gpu_section_eval_batch(StrutSectionBatch* b, const double* eps0_kappa_dev,
                                 double* resp_dev, int32_t commit, void* stream);
/* Copies the committed fiber state of one instance to the host in the section's family
 * order (Steel02 fibers, then Concrete02, then Steel01), 16 doubles per fiber, unused slots 0:
 *   Steel02:    eps sig tan epsmin epsmax epspl epss0 sigs0 epsr sigr, slot 15 = kon
 *   Concrete02: eps sig tan ecmin dept
 *   Steel01:    eps sig tan epsp alpha
 * Pass out = NULL to query *n_fibers only. */
int strut_gpu_section_batch_state(StrutSectionBatch* b, int32_t instance, double* out,
                                  int32_t* n_fibers);

/* ---- learned Newton predictor: the per-node network ---------------------------------------
 * No counterpart in the reference (Strut has no learned predictor).  A per-node MLP with
 * n_in <= 48 features, two hidden layers of 128 GELU (tanh form) units and n_out <= 16
 * outputs, run on the tensor cores (tcgen05, bf16 operands, fp32 accumulation) with fp32
 * master parameters packed as W1 (n_in x 128, W[k][j] maps input k to output j), b1 (128),
 * W2 (128 x 128), b2 (128), W3 (128 x n_out), b3 (n_out). */
typedef struct StrutMlp StrutMlp;
int strut_gpu_mlp_create(int32_t n_in, int32_t n_out, StrutMlp** out);
int strut_gpu_mlp_destroy(StrutMlp* m);
int32_t strut_gpu_mlp_param_count(const StrutMlp* m);
int strut_gpu_mlp_set_params(StrutMlp* m, const float* params);
int strut_gpu_mlp_get_params(const StrutMlp* m, float* params);
/* y (n x n_out) = network(x (n x n_in)); host buffers. */
int strut_gpu_mlp_forward(StrutMlp* m, const float* x, int32_t n, float* y);
/* Mean squared error of the network on (x, t) and its gradient with respect to the packed
 * parameters (the tensor-core backward pass; one batch of all n rows). */
int strut_gpu_mlp_loss_grad(StrutMlp* m, const float* x, const float* t, int32_t n, float* loss,
                            float* grads);
/* Adam (beta 0.9 / 0.999, eps 1e-8) on minibatches of `batch` rows, `epochs` passes over the n
 * rows in a seeded random order; *loss_out = mean squared error over the last pass. */
int strut_gpu_mlp_train(StrutMlp* m, const float* x, const float* t, int32_t n, int32_t epochs,
                        int32_t batch, float lr, uint64_t seed, float* loss_out);

/* ---- learned Newton predictor on an analysis ----------------------------------------------
 * No counterpart in the reference.  Attaches a trained network (not owned; it must outlive the
 * attachment) to every instance of the handle: each step, per node with a free dof, the features
 * (converged increments of the node's dofs at the 4 previous steps, ground acceleration at this
 * and the 15 previous steps, node height over frame height; x_norm = (x - x_mean) * x_scale,
 * 4 ndf + 17 of them) give a correction to the step's Newmark predictor (network output *
 * y_scale per dof), the learned guess being predictor + correction (slave dofs of multi-point
 * constraints then follow their masters).  The step starts from that guess.  Its first Newton
 * iteration assembles the residual R(u_l) and effective tangent K_eff at the guess u_l and
 * compares |R(u_l)| with the Newmark predictor u_p's residual to first order,
 * |R(u_l) + K_eff (u_l - u_p)|: when the learned one is the larger the step goes back to u_p
 * (the plain predictor is the fallback) and that evaluation is not counted as an iteration.  The
 * iterations then run to the same convergence test.  Instances must use Newton and have their
 * band in shared memory.  m = NULL detaches (the plain method). */
int strut_gpu_set_predictor(StrutHandle* h, StrutMlp* m, const float* x_mean, const float* x_scale,
                            const float* y_scale);
/* Number of predicted nodes (all instances), i.e. rows of strut_gpu_predictor_features. */
int32_t strut_gpu_predictor_nodes(const StrutHandle* h);
/* First iterations offered a learned guess, and how many kept it. */
int strut_gpu_predictor_stats(const StrutHandle* h, int64_t* offered, int64_t* chosen);
/* The normalised features of the next step, nodes x (4 ndf + 17) (tests). */
int strut_gpu_predictor_features(StrutHandle* h, float* out);

/* ---- band factor-solve that allocates nothing -------------------------------------------
 * No counterpart in the reference.  For callers that cannot let a library allocate device
 * memory: a host that reserves the device's memory for itself up front, or one that must not
 * trigger the device-wide synchronisation a cudaMalloc / cudaFree can cause between Newton
 * iterations.  Factors and solves one BandGeneral (band_dev: n x (2*half_bw+1), slot
 * row*(2bw+1) + (col-row+bw)) or BandSPD (band_dev: n x (half_bw+1), slot row*(bw+1) +
 * (row-col)) system held in device memory, with the kernels of strut_gpu_factor_solve, on
 * `stream`; writes x_dev and *status_dev (0 ok, 2 singular or not positive definite).  The
 * BandGeneral dense partial-pivot fallback works in a static device buffer compiled into the
 * library (2 MiB, held by every GPU that loads the library until the process exits), so n is
 * limited to 512: a larger n returns STRUT_BAD_ARG, a band too wide for shared memory
 * STRUT_UNSUPPORTED.  Nothing in that buffer has to be cleared: each call writes what it reads.
 * Every call on a device shares the buffer, so calls whose kernels may overlap on the GPU
 * (unordered streams) race and must be serialised by the caller.  The first call on a device
 * looks up the buffer's address and sets the kernel's shared-memory limit; make it before any
 * stream capture.  Those addresses belong to the device's context as it was then: after a
 * cudaDeviceReset in the same process this entry point is not supported.  Both systems are
 * held in shared memory in the general n x (2*half_bw+1) layout (BandSPD's lower band expanded
 * into it), so one shared-memory limit, (n (2 half_bw + 1) + 4 n) doubles within the device's
 * opt-in limit, applies to both.  Returns after the launch (asynchronous). */
int strut_gpu_band_solve_noalloc(const double* band_dev, int32_t n, int32_t half_bw,
                                 int32_t system, const double* rhs_dev, double* x_dev,
                                 int32_t* status_dev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* STRUT_CUDA_H */

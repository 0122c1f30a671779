// Host side of libstrut_cuda.so: packs Strut model descriptions into the device layout
// described in kernels.cuh, drives the Newmark-Newton loop and implements the C ABI of
// include/strut_cuda.h.
//
// Step loop (src/mojo/solver/run_case/analysis/transient_nonlinear.mojo:1698-3110):
//   predictor_kernel            Newmark predictor + ground-motion load, activate instances
//   repeat (Newton):
//     element_state_kernel      every element of every still-active instance
//     instance_newton_kernel    assembly gather, residual, band factor/solve, update, test
//     (host reads the number of still-active instances)
//   commit_kernel               fiber commit, basic-deformation sync, element-force records
//   post_step_kernel            Newmark velocity / acceleration update
//   record_disp_kernel          displacement records
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "strut_cuda.h"
#include "element_kernels.cuh"
#include "kat_kernels.cuh"
#include "fiber_stream_kernels.cuh"
#include "solver_kernels.cuh"
#include "largeband_kernels.cuh"
#include "shell_kernels.cuh"
#include "predictor_kernels.cuh"
#include "section_record_kernels.cuh"

using namespace strut;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(STRUT_CUDA_ERROR, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

inline int round4(int x) { return (x + 3) & ~3; }

DevMat make_devmat(const StrutUniMaterial& m) {
    DevMat d;
    std::memset(&d, 0, sizeof(d));
    d.type = m.type;
    for (int i = 0; i < 11; ++i) d.p[i] = m.p[i];
    const double* p = m.p;
    if (m.type == STRUT_MAT_CONCRETE02) {
        const double fc = p[0], epsc0 = p[1], fcu = p[2], epscu = p[3], rat = p[4], ft = p[5],
                     Ets = p[6];
        const double Ec0 = (2.0 * fc) / epsc0;
        d.k[C2K_EC0] = Ec0;
        d.k[C2K_EPSR] = (fcu - rat * Ec0 * epscu) / (Ec0 * (1.0 - rat));
        d.k[C2K_SIGMR] = Ec0 * d.k[C2K_EPSR];
        d.k[C2K_EPS0T] = ft / Ec0;
        d.k[C2K_EPSUT] = ft * (1.0 / Ets + 1.0 / Ec0);
    } else if (m.type == STRUT_MAT_STEEL02) {
        const double Fy = p[0], E0 = p[1], b = p[2], a2 = p[7], a4 = p[9];
        const double Esh = b * E0, epsy = Fy / E0;
        d.k[S2K_ESH] = Esh;
        d.k[S2K_EPSY] = epsy;
        d.k[S2K_SIGINI_E0] = p[10] / E0;
        d.k[S2K_DPOS] = 2.0 * (a4 * epsy);
        d.k[S2K_DNEG] = 2.0 * (a2 * epsy);
        d.k[S2K_E0MESH] = E0 - Esh;
        d.k[S2K_ESHEPSY] = Esh * epsy;
    } else if (m.type == STRUT_MAT_CONCRETE01) {
        d.k[C1K_EC0] = (2.0 * p[0]) / p[1];
    } else if (m.type == STRUT_MAT_STEEL01) {
        const double E0 = p[1], b = p[2];
        const double H = (b * E0) / (1.0 - b);
        d.k[S1K_H] = H;
        d.k[S1K_EH] = (E0 * H) / (E0 + H);
        d.k[S1K_E0PH] = E0 + H;
    }
    return d;
}

double initial_tangent(const StrutUniMaterial& m) {
    switch (m.type) {
        case STRUT_MAT_ELASTIC: return m.p[0];
        case STRUT_MAT_STEEL01: return m.p[1];
        case STRUT_MAT_CONCRETE01: return (2.0 * m.p[0]) / m.p[1];
        case STRUT_MAT_STEEL02: return m.p[1];
        case STRUT_MAT_CONCRETE02: return (2.0 * m.p[0]) / m.p[1];
        default: return 0.0;
    }
}

// Host image of the fiber geometry and section definitions.
struct SectionPack {
    std::vector<DevSection> secs;
    std::vector<double> y, z, a;
    std::vector<int> m;
};

// Builds one FiberSection2d definition (fiber2d.mojo:3323-3455: area centroid, families,
// initial flexibility) or, with dim 3, one FiberSection3d (fiber3d.mojo:633-720: centroid
// (y_bar, z_bar) = (sum A y, sum A z) / sum A, coordinates relative to it).  Families are
// stored in the order Steel02 | Concrete02 | Steel01 | Concrete01 | Elastic.  mat_base offsets material
// indices into the global table.
int pack_section(const StrutUniMaterial* mats, int nmat, const StrutFiber* fibers, int off,
                 int count, int mat_base, int dim, SectionPack& sp) {
    if (count <= 0) return fail(STRUT_BAD_ARG, "section without fibers");
    double area_sum = 0.0, qz_sum = 0.0, qy_sum = 0.0;
    for (int i = 0; i < count; ++i) {
        const StrutFiber& f = fibers[off + i];
        if (f.material < 0 || f.material >= nmat) return fail(STRUT_BAD_ARG, "fiber material out of range");
        const int t = mats[f.material].type;
        if (t != STRUT_MAT_ELASTIC && t != STRUT_MAT_STEEL01 && t != STRUT_MAT_STEEL02 &&
            t != STRUT_MAT_CONCRETE02 && t != STRUT_MAT_CONCRETE01)
            return fail(STRUT_UNSUPPORTED, "fiber material type not implemented on this path");
        area_sum += f.area;
        qy_sum += f.area * f.z;
        qz_sum += f.area * f.y;
    }
    if (!(area_sum > 0.0)) return fail(STRUT_BAD_ARG, "section total area must be > 0");
    const double y_bar = qz_sum / area_sum;
    const double z_bar = dim == 3 ? qy_sum / area_sum : 0.0;
    DevSection sd;
    std::memset(&sd, 0, sizeof(sd));
    sd.geo_off = (int)sp.y.size();
    double ik11 = 0.0, ik12 = 0.0, ik22 = 0.0;
    for (int i = 0; i < count; ++i) {
        const StrutFiber& f = fibers[off + i];
        const double y_rel = f.y - y_bar;
        const double ks = initial_tangent(mats[f.material]) * f.area;
        ik11 += ks;
        ik12 += -ks * y_rel;
        ik22 += ks * y_rel * y_rel;
    }
    const int order[5] = {STRUT_MAT_STEEL02, STRUT_MAT_CONCRETE02, STRUT_MAT_STEEL01,
                          STRUT_MAT_CONCRETE01, STRUT_MAT_ELASTIC};
    int counts[5] = {0, 0, 0, 0, 0};
    for (int fam = 0; fam < 5; ++fam) {
        for (int i = 0; i < count; ++i) {
            const StrutFiber& f = fibers[off + i];
            if (mats[f.material].type != order[fam]) continue;
            sp.y.push_back(f.y - y_bar);
            sp.z.push_back(dim == 3 ? f.z - z_bar : 0.0);
            sp.a.push_back(f.area);
            sp.m.push_back(mat_base + f.material);
            counts[fam]++;
        }
    }
    sd.n_s2 = counts[0];
    sd.n_c2 = counts[1];
    sd.n_s1 = counts[2];
    sd.n_c1 = counts[3];
    sd.n_el = counts[4];
    sd.all_elastic = (sd.n_s2 + sd.n_c2 + sd.n_s1 + sd.n_c1) == 0;
    sd.el_uniform = 0;
    if (sd.n_el > 0) {
        sd.el_uniform = 1;
        double E0 = -1.0;
        for (int i = 0; i < count; ++i) {
            const StrutFiber& f = fibers[off + i];
            if (mats[f.material].type != STRUT_MAT_ELASTIC) continue;
            const double E = mats[f.material].p[0];
            if (E0 < 0.0) E0 = E;
            else if (E != E0) sd.el_uniform = 0;
        }
    }
    sd.dim = dim;
    const double det = ik11 * ik22 - ik12 * ik12;
    if (dim == 2 && std::fabs(det) > 1.0e-40) {
        const double inv_det = 1.0 / det;
        sd.init_valid = 1;
        sd.f00 = ik22 * inv_det;
        sd.f01 = -ik12 * inv_det;
        sd.f11 = ik11 * inv_det;
    }
    sp.secs.push_back(sd);
    return STRUT_OK;
}

// Local axes of a 3D beam-column (rows x, y, z) from its end coordinates and vecxz
// (elements/utils.mojo:59-140; force_beam_column3d.mojo:172-222).
bool rotation3d_host(const double* x1, const double* x2, int has_vecxz, const double* vxz,
                     double* R) {
    const double dx = x2[0] - x1[0], dy = x2[1] - x1[1], dz = x2[2] - x1[2];
    const double n = std::sqrt(dx * dx + dy * dy + dz * dz);
    if (n == 0.0) return false;
    const double lx = dx / n, ly = dy / n, lz = dz / n;
    double vx = 1.0, vy = 0.0, vz = 0.0;
    if (has_vecxz) {
        vx = vxz[0];
        vy = vxz[1];
        vz = vxz[2];
    } else if (std::fabs(lx) >= 0.9) {
        vx = 0.0;
        vy = 1.0;
        if (std::fabs(ly) >= 0.9) {
            vy = 0.0;
            vz = 1.0;
        }
    }
    double yx = vy * lz - vz * ly, yy = vz * lx - vx * lz, yz = vx * ly - vy * lx;
    const double yn = std::sqrt(yx * yx + yy * yy + yz * yz);
    if (yn == 0.0) return false;
    yx /= yn;
    yy /= yn;
    yz /= yn;
    R[0] = lx;
    R[1] = ly;
    R[2] = lz;
    R[3] = yx;
    R[4] = yy;
    R[5] = yz;
    R[6] = ly * yz - lz * yy;
    R[7] = lz * yx - lx * yz;
    R[8] = lx * yy - ly * yx;
    return true;
}

double path_eval(const StrutExcitation& x, double t) {
    // eval_time_series_input, Path with dt (src/mojo/solver/time_series.mojo:71-90)
    const int n = x.count;
    if (n == 0) return 0.0;
    if (t < x.start_time) return 0.0;
    const double incr = (t - x.start_time) / x.dt;
    const int incr1 = (int)std::floor(incr);
    const int incr2 = incr1 + 1;
    if (incr2 >= n) {
        if (x.use_last) return x.factor * x.values[n - 1];
        return 0.0;
    }
    const double v1 = x.values[incr1], v2 = x.values[incr2];
    return x.factor * (v1 + (v2 - v1) * (incr - (double)incr1));
}

template <typename T>
int upload(T** dptr, const std::vector<T>& h, std::vector<void*>& allocs) {
    const size_t n = std::max<size_t>(h.size(), 1);
    CK(cudaMalloc((void**)dptr, n * sizeof(T)));
    allocs.push_back(*dptr);
    if (!h.empty()) CK(cudaMemcpy(*dptr, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return STRUT_OK;
}

template <typename T>
int dzeros(T** dptr, size_t n, std::vector<void*>& allocs) {
    n = std::max<size_t>(n, 1);
    CK(cudaMalloc((void**)dptr, n * sizeof(T)));
    allocs.push_back(*dptr);
    CK(cudaMemset(*dptr, 0, n * sizeof(T)));
    return STRUT_OK;
}

#define TRY(x)                       \
    do {                             \
        int rc_ = (x);               \
        if (rc_ != STRUT_OK) return rc_; \
    } while (0)

}  // namespace

struct ExcHost {
    int num;
    StrutExcitation x[2];
    std::vector<double> vals[2];
};

struct StrutHandle {
    int n_inst = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<void*> allocs;
    std::vector<DevInst> insts;
    std::vector<ExcHost> exc;
    std::vector<int> rec_off, n_rec, rece_off, n_rece;
    std::vector<std::vector<int>> rece_map;  // record entry -> unique element record slot
    int n_rec_total = 0, n_rece_slots = 0;
    int ef_w = 6;                    // doubles per element record slot: 6, or 12 with 3D
    std::vector<int> inst_nd;        // element dofs (2 ndf) of each instance
    int ndf_all = 3;                 // ndf shared by every instance, -1 when mixed
    int* d_rec3 = nullptr;           // recorded 3D elements (record pass after commit)
    int n_rec3 = 0;
    // section recorders: one slot per (instance, record), instance-major
    SecRec* d_secrec = nullptr;
    int n_sec_slots = 0;
    std::vector<int> sec_off, sec_n;
    double* d_hist_sec = nullptr;
    long long ek_total = 0, ef_total = 0;
    std::vector<DevShell> shells_h;  // linear shells of all instances
    DevShell* d_shells = nullptr;
    int n_shells = 0;
    // instances whose band is factored in global memory
    int n_large = 0, large_rows = 0, max_large_n = 0, lfactor_grid = 1, max_factor_grid = 1;
    long long lband_total = 0;
    size_t lfactor_smem = 16;
    int max_large_bw = 0;
    std::vector<int> large_list_h;
    int* d_large_list = nullptr;
    int* d_large_rowbase = nullptr;
    GridBarrier* d_gb = nullptr;
    double* d_wbuf = nullptr;
    int lfactor_wide = 0;      // the 16-column / 640-thread factorisation (half bands beyond 352)
    double* d_lpan = nullptr;  // factored panel, CTA 0 -> the other CTAs
    int* d_lpiv = nullptr;     // its row permutation
    int n_slaves_total = 0;          // slave dofs of every instance (multi-point constraints)
    int n_free_total = 0, n_dofs_total = 0, n_elem = 0;
    long long band_total = 0;
    int any_modified = 0;  // an instance runs ModifiedNewton(Initial)
    int any_chain = 0;     // an instance's solver chain has more than one attempt
    bool pred_owns_base = false;  // A.u_base / estate_base belong to the attached predictor
    int max_nip = 1;
    size_t elem_smem = 0, inst_smem = 0;
    int max_iters_global = 1;
    std::vector<int> max_fibers_per_section;
    // device
    DevElem* d_elems = nullptr;
    DevInst* d_insts = nullptr;
    Geo geo;
    FiberState fs;
    double* d_estate = nullptr;
    double* d_ek = nullptr;
    double* d_ef = nullptr;
    InstArrays A;
    int* d_free_inst = nullptr;
    int* d_free_dir = nullptr;
    int* d_rec_dof = nullptr;
    int* d_rece_base = nullptr;
    int* d_elem_err = nullptr;
    int elem_grid = 1;  // resident element CTAs (persistent element kernel)
    unsigned long long* d_counters = nullptr;
    double* d_ag = nullptr;
    int ag_cap = 0;
    double* d_hist_disp = nullptr;
    double* d_hist_ef = nullptr;
    int* d_hist_iters = nullptr;
    int hist_cap = 0;
    int steps_done = 0;
    int* h_ctrl = nullptr;  // pinned: nactive
    bool state_determined = false;
    bool prof = false;
    StrutKernelProfile P;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    DevCtl* d_ctl = nullptr;
    int* d_fail_step = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    const void* graph_keys[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    double* d_rhs = nullptr;
    std::vector<long long> elem_fibers;  // fibers per element (all families)
    // node table of the learned predictor: nodes with a free dof, instance order then node order
    std::vector<int> pn_free;   // per node ndf global free indices (-1: not free)
    std::vector<int> pn_inst;
    std::vector<float> pn_h;    // height / instance height
    int pn_ndf = 3;
    struct PredState* pred = nullptr;
    double commit_bytes_total = 0.0;
    long long dense_total = 0;
    StrutTuning tune = {1, 0, 0, 0, {0, 0, 0, 0}};
    int default_factor_grid = 1;
    int tune_gen = 0;       // bumped by strut_gpu_set_tuning (the graph bakes launch shapes in)
    int graph_tune_gen = -1;
    ~StrutHandle();
    void release() {
        for (void* p : allocs) cudaFree(p);
        if (d_hist_disp) cudaFree(d_hist_disp);
        if (d_hist_ef) cudaFree(d_hist_ef);
        if (d_hist_iters) cudaFree(d_hist_iters);
        if (d_hist_sec) cudaFree(d_hist_sec);
        if (d_ag) cudaFree(d_ag);
        if (h_ctrl) cudaFreeHost(h_ctrl);
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

struct PredState;
static void pred_free(PredState* p);
StrutHandle::~StrutHandle() {
    if (pred) pred_free(pred);
    release();
}
// learned predictor steps of a Newton step (defined with the predictor's host code)
static int pred_launch(StrutHandle* h);
static int pred_add_nodes(StrutHandle* h, cudaGraph_t body, cudaGraphNode_t dep, cudaGraphNode_t* last);

static int prof_begin(StrutHandle* h) {
    if (h->prof) CK(cudaEventRecord(h->ev0, h->stream));
    return STRUT_OK;
}

static int prof_end(StrutHandle* h, int k) {
    if (!h->prof) return STRUT_OK;
    CK(cudaEventRecord(h->ev1, h->stream));
    CK(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    h->P.ms[k] += ms;
    h->P.launches[k] += 1;
    return STRUT_OK;
}

// Element state kernel: kTeamThreads threads per element CTA.  Commit kernel: one team of 128
// threads per integration point up to 5 points, else 64.
using CommitKernel = decltype(&commit_kernel<128>);
using ElemKernel = decltype(&element_state_kernel<2>);
// Element CTA sizes: 640 (one CTA per SM), 320, 224 and 160 threads (more CTAs per SM where
// shared memory allows: more elements in flight, each with fewer threads).  The 3D kernel's
// epilogue needs 172 threads, so 160 is 2D only.
static bool elem_threads_ok(const StrutHandle* h, int t) {
    return t == kTeamThreads || t == kTeamThreads / 2 || t == 224 || (t == 160 && h->ndf_all != 6);
}
static int elem_threads_of(const StrutHandle* h) {
    return h->tune.element_threads != 0 && elem_threads_ok(h, h->tune.element_threads) ? h->tune.element_threads
                                                                                        : kTeamThreads;
}
static ElemKernel elem_kernel_of(const StrutHandle* h) {
    return h->ndf_all == 6 ? element_state_kernel<3> : element_state_kernel<2>;
}
static dim3 elem_block(const StrutHandle* h) { return dim3(elem_threads_of(h)); }
// Resident CTAs of the element kernel the handle's tuning selects (its persistent grid).
static int elem_grid_of(StrutHandle* h) {
    int per_sm = 0, n_sm = 0;
    CK(cudaFuncSetAttribute(elem_kernel_of(h), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->elem_smem));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, elem_kernel_of(h), (int)elem_block(h).x, h->elem_smem));
    CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, h->device));
    if (per_sm < 1) return fail(STRUT_UNSUPPORTED, "element kernel does not fit on an SM");
    h->elem_grid = std::max(1, std::min(h->n_elem, per_sm * n_sm));
    return STRUT_OK;
}
static int commit_team_of(const StrutHandle* h) {
    // the commit kernel is launched with at most kTeamThreads threads: team x points
    if (h->tune.commit_team == 64 || (h->tune.commit_team == 128 && h->max_nip <= 5)) return h->tune.commit_team;
    return h->max_nip <= 5 ? 128 : 64;
}
static CommitKernel commit_kernel_of(const StrutHandle* h) {
    return commit_team_of(h) == 128 ? commit_kernel<128> : commit_kernel<64>;
}
static dim3 commit_block(const StrutHandle* h) { return dim3(commit_team_of(h) * h->max_nip); }

// all_elems: every element (set-up and single-iteration entries); otherwise the list of
// elements of the instances still iterating.
static RecPass rec_pass_of(const StrutHandle* h) {
    RecPass rp;
    rp.list = h->d_rec3;
    rp.n = h->n_rec3;
    rp.hist_ef = h->d_hist_ef;
    rp.rece_base = h->d_rece_base;
    rp.slots = std::max(h->n_rece_slots, 1);
    rp.ef_w = h->ef_w;
    return rp;
}

// Record pass of the recorded 3D beam-columns after a step's commit.
static int launch_record_pass(StrutHandle* h) {
    if (h->n_rec3 == 0) return STRUT_OK;
    elem_kernel_of(h)<<<std::min(h->n_rec3, h->elem_grid), elem_block(h), h->elem_smem, h->stream>>>(
        h->d_elems, h->geo, h->fs, h->A.u_full, h->d_estate, h->d_ek, h->d_ef, h->A.active,
        h->A.status, h->d_elem_err, h->d_counters, h->A.el, (const DevCtl*)h->d_ctl,
        (int)ELEM_MODE_RECORD, h->n_elem, rec_pass_of(h));
    CK(cudaGetLastError());
    return STRUT_OK;
}

static int launch_elements(StrutHandle* h, int all_elems = 0) {
    if (h->prof) CK(cudaMemsetAsync(h->d_counters + 5, 0, sizeof(unsigned long long), h->stream));
    TRY(prof_begin(h));
    elem_kernel_of(h)<<<all_elems ? h->n_elem : h->elem_grid, elem_block(h), h->elem_smem, h->stream>>>(
        h->d_elems, h->geo, h->fs, h->A.u_full, h->d_estate, h->d_ek, h->d_ef, h->A.active,
        h->A.status, h->d_elem_err, h->d_counters, h->A.el, (const DevCtl*)h->d_ctl,
        all_elems ? (int)ELEM_MODE_ALL : (int)ELEM_MODE_LIST, h->n_elem, rec_pass_of(h));
    CK(cudaGetLastError());
    if (h->n_shells > 0) {
        shell_force_kernel<<<(h->n_shells * 32 + 255) / 256, 256, 0, h->stream>>>(h->d_shells, h->n_shells, h->d_ek,
                                                                                h->d_ef, h->A.u_full);
        CK(cudaGetLastError());
    }
    TRY(prof_end(h, 0));
    if (h->prof) {
        unsigned long long mx = 0;
        CK(cudaMemcpy(&mx, h->d_counters + 5, sizeof(mx), cudaMemcpyDeviceToHost));
        h->P.launches[5] += 1;
        h->P.bytes[5] += (double)mx;
        h->P.ms[5] = h->P.ms[0];
    }
    return STRUT_OK;
}

// Instances with a global-memory band: assembly (or the exported band), cooperative blocked LU
// with partial pivoting, back substitution + update + test.  mode as the instance kernel; EXPORT stops after
// the assembly.
static int launch_large(StrutHandle* h, int mode, const DevInst* insts = nullptr, InstArrays* Aover = nullptr) {
    if (h->n_large == 0) return STRUT_OK;
    InstArrays A = Aover ? *Aover : h->A;
    if (!Aover) A.bytes_counter = h->d_counters + 4;
    if (!insts) insts = h->d_insts;
    if (mode == INST_MODE_SOLVE_EXPORTED) {
        large_load_exported_kernel<<<dim3(64, h->n_large), 256, 0, h->stream>>>(insts, A, h->d_large_list,
                                                                                h->n_large, h->d_gb, h->d_wbuf);
    } else {
        const int blocks = (h->large_rows * 32 + 255) / 256;
        large_assemble_kernel<<<blocks, 256, 0, h->stream>>>(insts, A, h->d_large_list, h->d_large_rowbase,
                                                            h->n_large, h->large_rows, mode, h->d_gb,
                                                            h->d_wbuf);
    }
    CK(cudaGetLastError());
    if (mode == INST_MODE_EXPORT) return STRUT_OK;
    if (mode == INST_MODE_NEWTON && A.dual && A.skip) {
        large_learned_check_kernel<<<h->n_large, 256, 0, h->stream>>>(insts, A, h->d_large_list, h->n_large);
        CK(cudaGetLastError());
    }
    {
        int n_large = h->n_large;
        GridBarrier* gb = h->d_gb;
        const int* ll = h->d_large_list;
        double* wb = h->d_wbuf;
        double* lpan = h->d_lpan;
        int* lpiv = h->d_lpiv;
        void* args[] = {(void*)&insts, (void*)&A,  (void*)&ll,   (void*)&n_large, (void*)&mode,
                        (void*)&gb,    (void*)&wb, (void*)&lpan, (void*)&lpiv};
        if (h->lfactor_wide)
            CK(cudaLaunchCooperativeKernel((const void*)large_factor_kernel<kPanelWide, kLargeThreadsWide>,
                                           dim3(h->lfactor_grid), dim3(kLargeThreadsWide), args, h->lfactor_smem,
                                           h->stream));
        else
            CK(cudaLaunchCooperativeKernel((const void*)large_factor_kernel<kPanel, kLargeThreads>,
                                           dim3(h->lfactor_grid), dim3(kLargeThreads), args, h->lfactor_smem,
                                           h->stream));
    }
    large_solve_kernel<<<h->n_large, kSolveThreads, large_solve_smem(h->max_large_n), h->stream>>>(insts, A, h->d_large_list, h->n_large, mode,
                                                                    h->d_wbuf, h->d_gb);
    CK(cudaGetLastError());
    return STRUT_OK;
}

static int launch_instances(StrutHandle* h, int mode, int step) {
    InstArrays A = h->A;
    A.hist_iters = (mode == INST_MODE_NEWTON && step >= 0) ? h->d_hist_iters : nullptr;
    A.bytes_counter = h->d_counters + 4;
    TRY(prof_begin(h));
    instance_newton_kernel<<<h->n_inst, 256, h->inst_smem, h->stream>>>(h->d_insts, A, mode, step);
    CK(cudaGetLastError());
    TRY(launch_large(h, mode, nullptr, &A));
    TRY(prof_end(h, 1));
    return STRUT_OK;
}

static int ensure_history(StrutHandle* h, int need) {
    if (need <= h->hist_cap) return STRUT_OK;
    int cap = std::max(need, std::max(64, 2 * h->hist_cap));
    double* nd = nullptr;
    double* ne = nullptr;
    int* ni = nullptr;
    double* ns = nullptr;
    const int sw = h->ndf_all == 6 ? 4 : 2;
    CK(cudaMalloc((void**)&ns, (size_t)cap * std::max(h->n_sec_slots, 1) * sw * sizeof(double)));
    CK(cudaMalloc((void**)&nd, (size_t)cap * std::max(h->n_rec_total, 1) * sizeof(double)));
    CK(cudaMalloc((void**)&ne, (size_t)cap * std::max(h->n_rece_slots, 1) * h->ef_w * sizeof(double)));
    CK(cudaMalloc((void**)&ni, (size_t)cap * h->n_inst * sizeof(int)));
    CK(cudaMemset(ni, 0, (size_t)cap * h->n_inst * sizeof(int)));
    if (h->hist_cap > 0 && h->steps_done > 0) {
        CK(cudaMemcpy(nd, h->d_hist_disp, (size_t)h->steps_done * std::max(h->n_rec_total, 1) * sizeof(double),
                      cudaMemcpyDeviceToDevice));
        CK(cudaMemcpy(ne, h->d_hist_ef, (size_t)h->steps_done * std::max(h->n_rece_slots, 1) * h->ef_w * sizeof(double),
                      cudaMemcpyDeviceToDevice));
        CK(cudaMemcpy(ni, h->d_hist_iters, (size_t)h->steps_done * h->n_inst * sizeof(int),
                      cudaMemcpyDeviceToDevice));
        CK(cudaMemcpy(ns, h->d_hist_sec, (size_t)h->steps_done * std::max(h->n_sec_slots, 1) * sw * sizeof(double),
                      cudaMemcpyDeviceToDevice));
    }
    if (h->d_hist_sec) cudaFree(h->d_hist_sec);
    h->d_hist_sec = ns;
    if (h->d_hist_disp) cudaFree(h->d_hist_disp);
    if (h->d_hist_ef) cudaFree(h->d_hist_ef);
    if (h->d_hist_iters) cudaFree(h->d_hist_iters);
    h->d_hist_disp = nd;
    h->d_hist_ef = ne;
    h->d_hist_iters = ni;
    h->hist_cap = cap;
    return STRUT_OK;
}

template <typename T, size_t... I>
static void fill_params(T& t, void** p, std::index_sequence<I...>) {
    ((p[I] = (void*)&std::get<I>(t)), ...);
}

// Adds a kernel node with the given launch configuration and arguments (copied at creation).
template <typename... P, typename... Q>
static int add_kernel_node(cudaGraphNode_t* node, cudaGraph_t g, const cudaGraphNode_t* deps,
                           size_t ndeps, void (*func)(P...), dim3 grid, dim3 block, size_t smem,
                           Q... args) {
    std::tuple<std::decay_t<P>...> vals(args...);
    void* params[sizeof...(P) > 0 ? sizeof...(P) : 1];
    fill_params(vals, params, std::index_sequence_for<P...>{});
    cudaKernelNodeParams kp;
    std::memset(&kp, 0, sizeof(kp));
    kp.func = (void*)func;
    kp.gridDim = grid;
    kp.blockDim = block;
    kp.sharedMemBytes = (unsigned)smem;
    kp.kernelParams = params;
    kp.extra = nullptr;
    CK(cudaGraphAddKernelNode(node, g, deps, ndeps, &kp));
    return STRUT_OK;
}

static int add_while_node(cudaGraphNode_t* node, cudaGraph_t g, const cudaGraphNode_t* deps,
                          size_t ndeps, cudaGraphConditionalHandle handle, cudaGraph_t* body) {
    alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
    std::memset(raw, 0, sizeof(raw));
    cudaGraphNodeParams* np = reinterpret_cast<cudaGraphNodeParams*>(raw);
    np->type = cudaGraphNodeTypeConditional;
    np->conditional.handle = handle;
    np->conditional.type = cudaGraphCondTypeWhile;
    np->conditional.size = 1;
    CK(cudaGraphAddNode(node, g, deps, ndeps, np));
    *body = np->conditional.phGraph_out[0];
    return STRUT_OK;
}

// The whole step loop as one CUDA graph: an outer WHILE over steps (condition set by
// step_end_kernel) around predictor -> inner WHILE over Newton iterations (element state
// determination, instance Newton kernel, newton_check_kernel sets the condition) -> commit ->
// Newmark update -> displacement records -> step_end.  The host synchronises once per run.
static int build_graph(StrutHandle* h) {
    if (h->gexec) {
        cudaGraphExecDestroy(h->gexec);
        h->gexec = nullptr;
    }
    if (h->graph) {
        cudaGraphDestroy(h->graph);
        h->graph = nullptr;
    }
    cudaGraph_t g;
    CK(cudaGraphCreate(&g, 0));
    h->graph = g;
    cudaGraphConditionalHandle outer, inner;
    CK(cudaGraphConditionalHandleCreate(&outer, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNode_t n_outer;
    cudaGraph_t body;
    TRY(add_while_node(&n_outer, g, nullptr, 0, outer, &body));
    CK(cudaGraphConditionalHandleCreate(&inner, body, 1, cudaGraphCondAssignDefault));
    const int nF = h->n_free_total;
    const int tb = 256;
    const int npred = std::max(nF, h->n_inst);
    InstArrays A = h->A;
    A.hist_iters = h->d_hist_iters;
    A.ctl = h->d_ctl;
    A.bytes_counter = h->d_counters + 4;
    cudaGraphNode_t n_pred, n_inner, n_commit, n_post, n_rec, n_end;
    TRY(add_kernel_node(&n_pred, body, nullptr, 0, predictor_kernel, dim3((npred + tb - 1) / tb), dim3(tb), 0,
                        (const DevInst*)h->d_insts, A, (const int*)h->d_free_inst, (const int*)h->d_free_dir,
                        (const double*)h->d_ag, nF, h->n_inst, h->d_ctl, inner, 1));
    cudaGraph_t ibody;
    cudaGraphNode_t n_before_inner = n_pred;
    if (h->any_chain || h->pred) {
        // the element state at the step's start, for a retry of the solver chain or the return
        // from the learned guess to the predictor
        cudaGraphNode_t n_snap;
        TRY(add_kernel_node(&n_snap, body, &n_pred, 1, copy_doubles_kernel, dim3(592), dim3(tb), 0,
                            (const double*)h->d_estate, h->A.estate_base, (long long)h->n_elem * kEStride));
        n_before_inner = n_snap;
    }
    if (h->n_slaves_total > 0) {
        cudaGraphNode_t n_sl;
        TRY(add_kernel_node(&n_sl, body, &n_before_inner, 1, slave_enforce_kernel, dim3((h->n_slaves_total + tb - 1) / tb),
                            dim3(tb), 0, A, h->n_slaves_total));
        n_before_inner = n_sl;
    }
    if (h->pred) TRY(pred_add_nodes(h, body, n_before_inner, &n_before_inner));
    TRY(add_while_node(&n_inner, body, &n_before_inner, 1, inner, &ibody));
    cudaGraphNode_t n_el, n_in, n_chk;
    TRY(add_kernel_node(&n_el, ibody, nullptr, 0, elem_kernel_of(h), dim3(h->elem_grid),
                        elem_block(h), h->elem_smem, (const DevElem*)h->d_elems, h->geo,
                        h->fs, (const double*)h->A.u_full, h->d_estate, h->d_ek, h->d_ef,
                        (const int*)h->A.active, h->A.status, h->d_elem_err, h->d_counters, h->A.el,
                        (const DevCtl*)h->d_ctl, (int)ELEM_MODE_LIST, h->n_elem, rec_pass_of(h)));
    cudaGraphNode_t n_after_el = n_el;
    if (h->n_shells > 0) {
        cudaGraphNode_t n_sh;
        TRY(add_kernel_node(&n_sh, ibody, &n_el, 1, shell_force_kernel, dim3((h->n_shells * 32 + 255) / 256),
                            dim3(256), 0, (const DevShell*)h->d_shells, h->n_shells, (const double*)h->d_ek, h->d_ef,
                            (const double*)h->A.u_full));
        n_after_el = n_sh;
    }
    TRY(add_kernel_node(&n_in, ibody, &n_after_el, 1, instance_newton_kernel, dim3(h->n_inst), dim3(256),
                        h->inst_smem, (const DevInst*)h->d_insts, A, (int)INST_MODE_NEWTON, 0));
    cudaGraphNode_t n_before_chk = n_in;
    TRY(add_kernel_node(&n_chk, ibody, &n_before_chk, 1, newton_check_kernel, dim3(1), dim3(32), 0, h->d_ctl,
                        (const int*)h->A.nactive, inner, 1));
    TRY(add_kernel_node(&n_commit, body, &n_inner, 1, commit_kernel_of(h), dim3(h->n_elem),
                        commit_block(h), 0, (const DevElem*)h->d_elems, h->geo, h->fs,
                        (const double*)h->A.u_full, h->d_estate, (const int*)h->A.status, h->d_hist_ef,
                        (const int*)h->d_rece_base, std::max(h->n_rece_slots, 1), h->ef_w, (const DevCtl*)h->d_ctl));
    cudaGraphNode_t n_after_commit = n_commit;
    if (h->n_rec3 > 0) {
        cudaGraphNode_t n_rp;
        TRY(add_kernel_node(&n_rp, body, &n_commit, 1, elem_kernel_of(h), dim3(std::min(h->n_rec3, h->elem_grid)),
                            elem_block(h), h->elem_smem, (const DevElem*)h->d_elems, h->geo, h->fs,
                            (const double*)h->A.u_full, h->d_estate, h->d_ek, h->d_ef, (const int*)h->A.active,
                            h->A.status, h->d_elem_err, h->d_counters, h->A.el, (const DevCtl*)h->d_ctl,
                            (int)ELEM_MODE_RECORD, h->n_elem, rec_pass_of(h)));
        n_after_commit = n_rp;
    }
    TRY(add_kernel_node(&n_post, body, &n_after_commit, 1, post_step_kernel, dim3((nF + tb - 1) / tb), dim3(tb), 0,
                        (const DevInst*)h->d_insts, A, (const int*)h->d_free_inst, nF));
    cudaGraphNode_t last = n_post;
    if (h->n_rec_total > 0) {
        TRY(add_kernel_node(&n_rec, body, &n_post, 1, record_disp_kernel, dim3((h->n_rec_total + tb - 1) / tb),
                            dim3(tb), 0, (const double*)h->A.u_full, (const int*)h->d_rec_dof, h->n_rec_total,
                            h->d_hist_disp, (const DevCtl*)h->d_ctl));
        last = n_rec;
    }
    if (h->n_sec_slots > 0) {
        cudaGraphNode_t n_sec;
        TRY(add_kernel_node(&n_sec, body, &last, 1, record_sections_kernel, dim3((h->n_sec_slots * 32 + 255) / 256),
                            dim3(256), 0, (const DevElem*)h->d_elems, h->geo, h->fs, (const double*)h->A.u_full,
                            (const double*)h->d_estate, (const SecRec*)h->d_secrec, h->n_sec_slots,
                            h->ndf_all == 6 ? 4 : 2, h->d_hist_sec, (const DevCtl*)h->d_ctl));
        last = n_sec;
    }
    TRY(add_kernel_node(&n_end, body, &last, 1, step_end_kernel, dim3(1), dim3(256), 0, h->d_ctl,
                        (const int*)h->A.status, h->d_fail_step, h->n_inst, h->A.nactive, h->A.el, outer, 1));
    CK(cudaGraphInstantiate(&h->gexec, g, 0));
    h->graph_keys[0] = h->d_hist_disp;
    h->graph_keys[1] = h->d_hist_ef;
    h->graph_keys[2] = h->d_hist_iters;
    h->graph_keys[3] = h->d_ag;
    h->graph_keys[5] = h->d_hist_sec;
    h->graph_keys[4] = h->pred;
    h->graph_tune_gen = h->tune_gen;
    return STRUT_OK;
}

static int ensure_graph(StrutHandle* h) {
    if (h->gexec && h->graph_tune_gen == h->tune_gen && h->graph_keys[0] == h->d_hist_disp && h->graph_keys[1] == h->d_hist_ef &&
        h->graph_keys[2] == h->d_hist_iters && h->graph_keys[3] == h->d_ag && h->graph_keys[4] == h->pred &&
        h->graph_keys[5] == h->d_hist_sec)
        return STRUT_OK;
    return build_graph(h);
}

extern "C" {

int strut_gpu_abi_version(void) { return STRUT_ABI_VERSION; }

const char* strut_gpu_last_error(void) { return g_last_error.c_str(); }

int strut_gpu_create(const StrutModelDesc* models, int32_t num_instances, int32_t device,
                     StrutHandle** out) {
    if (!models || num_instances <= 0 || !out) return fail(STRUT_BAD_ARG, "bad arguments");
    *out = nullptr;
    if (device >= 0) CK(cudaSetDevice(device));
    StrutHandle* h = new StrutHandle();
    int rc = STRUT_OK;
    auto bail = [&](int code) {
        delete h;
        return code;
    };
    CK(cudaGetDevice(&h->device));
    h->n_inst = num_instances;
    std::vector<DevMat> mats;
    SectionPack sp;
    std::vector<DevElem> elems;
    std::vector<double> Mff, Mrff, fconst;
    std::vector<int> free_dof, free_inst, free_dir, rec_dof, rece_base;
    std::vector<long long> slot_ptr(1, 0);
    std::vector<int> slot_contrib;
    std::vector<int> fint_ptr(1, 0), fint_contrib;
    std::vector<double> slot_coef, fint_coef;        // filled when some instance has constraints
    std::vector<int> sl_dof, sl_ptr(1, 0), sl_master;
    std::vector<double> sl_coef;
    bool any_mpc = false;
    for (int inst = 0; inst < num_instances; ++inst) any_mpc = any_mpc || models[inst].num_slaves > 0;
    long long c2_total = 0, s2_total = 0, s1_total = 0, c1_total = 0;
    std::vector<int> sec_base(num_instances);
    int u_off = 0, f_off = 0;
    long long band_off = 0;
    long long dense_off = 0;
    h->insts.resize(num_instances);
    h->exc.resize(num_instances);
    h->rec_off.resize(num_instances);
    h->n_rec.resize(num_instances);
    h->rece_off.resize(num_instances);
    h->n_rece.resize(num_instances);
    h->rece_map.resize(num_instances);
    for (int inst = 0; inst < num_instances; ++inst) {
        const StrutModelDesc& d = models[inst];
        const bool three_d = d.ndm == 3 && d.ndf == 6;
        if (!three_d && (d.ndm != 2 || d.ndf != 3))
            return bail(fail(STRUT_UNSUPPORTED, "frames with ndm 2, ndf 3 or ndm 3, ndf 6"));
        const int nd = 2 * d.ndf;
        h->inst_nd.push_back(nd);
        if (inst == 0) h->ndf_all = d.ndf;
        else if (h->ndf_all != d.ndf)
            return bail(fail(STRUT_UNSUPPORTED, "a batch holds either 2D (ndf 3) or 3D (ndf 6) frames"));
        if (three_d) h->ef_w = 12;
        if (d.num_free <= 0 || d.num_elements <= 0 || d.num_dofs != d.num_nodes * d.ndf)
            return bail(fail(STRUT_BAD_ARG, "inconsistent model sizes"));
        if (d.system != STRUT_SYSTEM_BAND_GENERAL && d.system != STRUT_SYSTEM_BAND_SPD)
            return bail(fail(STRUT_UNSUPPORTED, "only BandGeneral and BandSPD"));
        if (d.beta_k_comm != 0.0)
            return bail(fail(STRUT_UNSUPPORTED, "rayleigh betaKComm is not implemented on this path"));
        if (!(d.beta > 0.0) || !(d.dt > 0.0)) return bail(fail(STRUT_BAD_ARG, "Newmark beta and dt must be > 0"));
        if (d.max_iters <= 0) return bail(fail(STRUT_BAD_ARG, "max_iters must be > 0"));
        const int mat_base = (int)mats.size();
        for (int i = 0; i < d.num_materials; ++i) mats.push_back(make_devmat(d.materials[i]));
        sec_base[inst] = (int)sp.secs.size();
        for (int s = 0; s < d.num_sections; ++s) {
            rc = pack_section(d.materials, d.num_materials, d.fibers, d.sections[s].fiber_offset,
                              d.sections[s].fiber_count, mat_base, three_d ? 3 : 2, sp);
            if (rc != STRUT_OK) return bail(rc);
        }
        // free numbering / masses
        int nf = d.num_free;
        std::vector<int> free_of_dof(d.num_dofs);
        bool has_mass = false;
        std::vector<double> mff(nf, 0.0), mrff(nf, 0.0), fcf(nf, 0.0);
        std::vector<int> fdof(nf, -1);
        for (int dof = 0; dof < d.num_dofs; ++dof) {
            const int fi = d.free_index[dof];
            free_of_dof[dof] = fi;
            if (fi < 0) continue;
            if (fi >= nf) return bail(fail(STRUT_BAD_ARG, "free index out of range"));
            fdof[fi] = dof;
            if (d.mass[dof] != 0.0) {
                mff[fi] += d.mass[dof] * 1.0 * 1.0;
                has_mass = true;
            }
            if (d.mass_rayleigh && d.mass_rayleigh[dof] != 0.0) mrff[fi] += d.mass_rayleigh[dof] * 1.0 * 1.0;
            if (d.f_const) fcf[fi] = d.f_const[dof];
        }
        if (!has_mass) return bail(fail(STRUT_BAD_ARG, "transient_nonlinear requires masses on free dofs"));
        // collapse rows of every dof (loader.mojo:2239-2380): a free dof maps to itself, a
        // slave to its retained dofs, a fixed dof to nothing
        std::vector<int> slave_of(d.num_dofs, -1);
        const int sl0 = (int)sl_dof.size();
        if (d.num_slaves < 0 || (d.num_slaves > 0 && (!d.slave_dof || !d.slave_ptr || !d.slave_master || !d.slave_coef)))
            return bail(fail(STRUT_BAD_ARG, "slave arrays missing"));
        for (int k = 0; k < d.num_slaves; ++k) {
            const int sd = d.slave_dof[k];
            if (sd < 0 || sd >= d.num_dofs || d.free_index[sd] >= 0 || slave_of[sd] >= 0)
                return bail(fail(STRUT_BAD_ARG, "slave dof out of range, free, or repeated"));
            if (d.mass[sd] != 0.0 || (d.mass_rayleigh && d.mass_rayleigh[sd] != 0.0))
                return bail(fail(STRUT_UNSUPPORTED, "mass on a constrained (slave) dof"));
            slave_of[sd] = k;
            if (d.slave_ptr[k + 1] < d.slave_ptr[k]) return bail(fail(STRUT_BAD_ARG, "slave_ptr not increasing"));
            sl_dof.push_back(u_off + sd);
            for (int t = d.slave_ptr[k]; t < d.slave_ptr[k + 1]; ++t) {
                const int md = d.slave_master[t];
                if (md < 0 || md >= d.num_dofs) return bail(fail(STRUT_BAD_ARG, "retained dof out of range"));
                sl_master.push_back(u_off + md);
                sl_coef.push_back(d.slave_coef[t]);
            }
            sl_ptr.push_back((int)sl_master.size());
        }
        for (int k = 0; k < d.num_slaves; ++k)
            for (int t = d.slave_ptr[k]; t < d.slave_ptr[k + 1]; ++t)
                if (slave_of[d.slave_master[t]] >= 0)
                    return bail(fail(STRUT_BAD_ARG, "a retained dof cannot itself be constrained"));
        auto rows_of = [&](int dof, std::vector<std::pair<int, double>>& out) {
            out.clear();
            if (slave_of[dof] >= 0) {
                const int k = slave_of[dof];
                for (int t = d.slave_ptr[k]; t < d.slave_ptr[k + 1]; ++t)
                    out.emplace_back(d.free_index[d.slave_master[t]], d.slave_coef[t]);
            } else if (d.free_index[dof] >= 0) {
                out.emplace_back(d.free_index[dof], 1.0);
            }
        };
        if (d.num_slaves > 0 && d.f_const) {
            // F_const collapsed onto the retained dofs (loader.mojo:2344)
            std::vector<double> red(d.num_dofs, 0.0);
            for (int dof = 0; dof < d.num_dofs; ++dof) {
                if (slave_of[dof] >= 0) {
                    const int k = slave_of[dof];
                    for (int t = d.slave_ptr[k]; t < d.slave_ptr[k + 1]; ++t)
                        red[d.slave_master[t]] += d.slave_coef[t] * d.f_const[dof];
                } else if (d.free_index[dof] >= 0) {
                    red[dof] += 1.0 * d.f_const[dof];
                }
            }
            for (int dof = 0; dof < d.num_dofs; ++dof)
                if (d.free_index[dof] >= 0) fcf[d.free_index[dof]] = red[dof];
        }
        {
            double hmax = 0.0;
            for (int nd = 0; nd < d.num_nodes; ++nd) hmax = std::max(hmax, d.node_coords[d.ndm * nd + d.ndm - 1]);
            for (int nd = 0; nd < d.num_nodes; ++nd) {
                bool any = false;
                for (int k = 0; k < d.ndf; ++k) any = any || d.free_index[nd * d.ndf + k] >= 0;
                if (!any) continue;
                for (int k = 0; k < d.ndf; ++k) {
                    const int fi = d.free_index[nd * d.ndf + k];
                    h->pn_free.push_back(fi >= 0 ? f_off + fi : -1);
                }
                h->pn_inst.push_back(inst);
                const double y = d.node_coords[d.ndm * nd + d.ndm - 1];
                h->pn_h.push_back(hmax > 0.0 ? (float)(y / hmax) : 0.0f);
            }
            h->pn_ndf = d.ndf;
        }
        for (int fi = 0; fi < nf; ++fi) {
            if (fdof[fi] < 0) return bail(fail(STRUT_BAD_ARG, "free numbering has holes"));
            Mff.push_back(mff[fi]);
            Mrff.push_back(mrff[fi]);
            fconst.push_back(fcf[fi]);
            free_dof.push_back(u_off + fdof[fi]);
            free_inst.push_back(inst);
            free_dir.push_back((fdof[fi] % d.ndf) + 1);
        }
        // elements
        const int e0 = (int)elems.size();
        int bw = 0;
        std::vector<int> efree((size_t)nd * d.num_elements);
        std::vector<int> rec_slot(d.num_elements, -1);
        std::vector<int>& rmap = h->rece_map[inst];
        int nslots = 0;
        for (int j = 0; j < d.num_record_elements; ++j) {
            const int re = d.record_elements[j];
            if (re < 0 || re >= d.num_elements) return bail(fail(STRUT_BAD_ARG, "recorded element out of range"));
            if (rec_slot[re] < 0) rec_slot[re] = nslots++;
            rmap.push_back(rec_slot[re]);
        }
        for (int e = 0; e < d.num_elements; ++e) {
            const StrutFrameElement& ed = d.elements[e];
            const bool el3 = ed.type == STRUT_ELEM_FORCE_BEAM_COLUMN_3D || ed.type == STRUT_ELEM_DISP_BEAM_COLUMN_3D;
            const bool el2 = ed.type == STRUT_ELEM_FORCE_BEAM_COLUMN_2D || ed.type == STRUT_ELEM_DISP_BEAM_COLUMN_2D;
            if (three_d ? !el3 : !el2)
                return bail(fail(STRUT_UNSUPPORTED, "element type not implemented on this path"));
            if (ed.geom != STRUT_GEOM_LINEAR && ed.geom != STRUT_GEOM_PDELTA &&
                !(three_d && ed.geom == STRUT_GEOM_COROTATIONAL))
                return bail(fail(STRUT_UNSUPPORTED, three_d ? "geomTransf must be Linear, PDelta or Corotational"
                                                            : "geomTransf must be Linear or PDelta"));
            if (ed.section < 0 || ed.section >= d.num_sections || ed.integration < 0 ||
                ed.integration >= d.num_integrations)
                return bail(fail(STRUT_BAD_ARG, "element section / integration out of range"));
            const StrutBeamIntegration& r = d.integrations[ed.integration];
            if (r.num_int_pts < 1 || r.num_int_pts > kMaxIp)
                return bail(fail(STRUT_BAD_ARG, "num_int_pts out of range"));
            DevElem E;
            std::memset(&E, 0, sizeof(E));
            E.type = ed.type;
            E.geom = ed.geom;
            E.nip = r.num_int_pts;
            E.sec = sec_base[inst] + ed.section;
            E.inst = inst;
            E.rec = rec_slot[e];
            E.nd = nd;
            for (int a = 0; a < nd; ++a) {
                if (ed.dof[a] < 0 || ed.dof[a] >= d.num_dofs) return bail(fail(STRUT_BAD_ARG, "element dof out of range"));
                E.dof[a] = u_off + ed.dof[a];
                efree[(size_t)nd * e + a] = free_of_dof[ed.dof[a]];
            }
            if (ed.node_i < 0 || ed.node_i >= d.num_nodes || ed.node_j < 0 || ed.node_j >= d.num_nodes)
                return bail(fail(STRUT_BAD_ARG, "element node out of range"));
            if (three_d) {
                for (int c = 0; c < 3; ++c) {
                    E.X1[c] = d.node_coords[3 * ed.node_i + c];
                    E.X2[c] = d.node_coords[3 * ed.node_j + c];
                    E.vxz[c] = ed.vecxz[c];
                }
                E.has_vecxz = ed.has_vecxz ? 1 : 0;
                const double dx = E.X2[0] - E.X1[0], dy = E.X2[1] - E.X1[1], dz = E.X2[2] - E.X1[2];
                E.L = std::sqrt(dx * dx + dy * dy + dz * dz);
                if (E.L == 0.0) return bail(fail(STRUT_BAD_ARG, "zero-length element"));
                E.inv_L = 1.0 / E.L;
                if (!rotation3d_host(E.X1, E.X2, E.has_vecxz, E.vxz, E.R))
                    return bail(fail(STRUT_BAD_ARG, "invalid beam3d vecxz orientation"));
                E.G = d.sections[ed.section].G;
                E.J = d.sections[ed.section].J;
            } else {
                const double x1 = d.node_coords[2 * ed.node_i], y1 = d.node_coords[2 * ed.node_i + 1];
                const double x2 = d.node_coords[2 * ed.node_j], y2 = d.node_coords[2 * ed.node_j + 1];
                const double dx = x2 - x1, dy = y2 - y1;
                E.L = std::hypot(dx, dy);
                if (E.L == 0.0) return bail(fail(STRUT_BAD_ARG, "zero-length element"));
                E.inv_L = 1.0 / E.L;
                E.c = dx * E.inv_L;
                E.s = dy * E.inv_L;
                E.c_div = dx / E.L;
                E.s_div = dy / E.L;
                E.L_sync = std::sqrt(dx * dx + dy * dy);
                E.c_sync = dx / E.L_sync;
                E.s_sync = dy / E.L_sync;
            }
            E.ek_off = h->ek_total;
            E.ef_off = h->ef_total;
            h->ek_total += (long long)nd * nd;
            h->ef_total += nd;
            for (int ip = 0; ip < E.nip; ++ip) {
                E.xi[ip] = r.xi[ip];
                E.w[ip] = r.w[ip];
            }
            const DevSection& sd = sp.secs[E.sec];
            E.s2_off = (int)s2_total;
            E.s2_blk = round4(E.nip * sd.n_s2);
            s2_total += E.s2_blk;
            E.c2_off = (int)c2_total;
            E.c2_blk = round4(E.nip * sd.n_c2);
            c2_total += E.c2_blk;
            E.s1_off = (int)s1_total;
            E.s1_blk = round4(E.nip * sd.n_s1);
            s1_total += E.s1_blk;
            E.c1_off = (int)c1_total;
            E.c1_blk = round4(E.nip * sd.n_c1);
            c1_total += E.c1_blk;
            h->max_nip = std::max(h->max_nip, E.nip);
            // staged history (Concrete02 without dept) + derived constants (Concrete02 5, Steel02
            // 12 doubles per fiber) + the section's fiber y + per-fiber stress and tangent of
            // every point
            const int n_tot = sd.n_s2 + sd.n_c2 + sd.n_s1 + sd.n_c1 + sd.n_el;
            const size_t smem = 8 * (size_t)(4 * E.c2_blk + 10 * E.s2_blk + 5 * E.s1_blk + 6 * E.c1_blk) +
                                4 * (size_t)E.s2_blk +
                                8 * (size_t)(5 * E.c2_blk + 12 * E.s2_blk) +
                                8 * (size_t)((three_d ? 2 : 1) * ((n_tot + 1) & ~1) + 2 * E.nip * n_tot);
            h->elem_smem = std::max(h->elem_smem, smem);
            h->elem_fibers.push_back((long long)E.nip * (sd.n_s2 + sd.n_c2 + sd.n_s1 + sd.n_c1 + sd.n_el));
            {
                // committed history read once (Concrete02 / Steel01 5 doubles, Concrete01 6,
                // Steel02 10 doubles + kon), element state read + written, k and f written,
                // the element's dofs read, the element record itself
                const double fib = (double)E.nip * (40.0 * sd.n_c2 + 84.0 * sd.n_s2 + 40.0 * sd.n_s1 +
                                                    48.0 * sd.n_c1);
                const double est = three_d ? 8.0 * (5 + 3 * E.nip) : 8.0 * (6 + 2 * E.nip);
                E.io_bytes = fib + 2.0 * est + 8.0 * (nd * nd + nd) + 8.0 * nd + (double)sizeof(DevElem);
                E.commit_bytes = 2.0 * fib + est + 8.0 * nd + (double)sizeof(DevElem);
            }
            elems.push_back(E);
            for (int a = 0; a < nd; ++a) {
                const int ia = efree[(size_t)nd * e + a];
                if (ia < 0) continue;
                for (int b = a + 1; b < nd; ++b) {
                    const int ib = efree[(size_t)nd * e + b];
                    if (ib < 0) continue;
                    bw = std::max(bw, std::abs(ia - ib));
                }
            }
        }
        // linear shells (elements/shell4.mojo:10-363): constant 24 x 24 stiffness after the frame
        // elements' entries, their free-dof pairs in the band
        const int sh0 = (int)h->shells_h.size();
        std::vector<int> sfree((size_t)24 * d.num_shells);
        if (d.num_shells > 0 && (d.ndm != 3 || d.ndf != 6 || !d.shells))
            return bail(fail(STRUT_BAD_ARG, "shells need ndm 3, ndf 6 and a shell array"));
        for (int s = 0; s < d.num_shells; ++s) {
            const StrutShellElement& se = d.shells[s];
            DevShell S;
            std::memset(&S, 0, sizeof(S));
            for (int k = 0; k < 4; ++k) {
                if (se.nodes[k] < 0 || se.nodes[k] >= d.num_nodes) return bail(fail(STRUT_BAD_ARG, "shell node out of range"));
                S.x[k] = d.node_coords[3 * se.nodes[k]];
                S.y[k] = d.node_coords[3 * se.nodes[k] + 1];
                S.z[k] = d.node_coords[3 * se.nodes[k] + 2];
            }
            if (!(se.E > 0.0 && se.h > 0.0 && se.nu > -1.0 && se.nu < 0.5))
                return bail(fail(STRUT_BAD_ARG, "shell section needs E > 0, h > 0, -1 < nu < 0.5"));
            S.E = se.E;
            S.nu = se.nu;
            S.h = se.h;
            for (int a = 0; a < 24; ++a) {
                const int dof = se.dof[a];
                if (dof < 0 || dof >= d.num_dofs) return bail(fail(STRUT_BAD_ARG, "shell dof out of range"));
                S.dof[a] = u_off + dof;
                sfree[(size_t)24 * s + a] = d.free_index[dof];
            }
            S.ek_off = h->ek_total;
            S.ef_off = h->ef_total;
            h->ek_total += 576;
            h->ef_total += 24;
            h->shells_h.push_back(S);
            for (int a = 0; a < 24; ++a) {
                const int ia = sfree[(size_t)24 * s + a];
                if (ia < 0) continue;
                for (int b = a + 1; b < 24; ++b) {
                    const int ib = sfree[(size_t)24 * s + b];
                    if (ib >= 0) bw = std::max(bw, std::abs(ia - ib));
                }
            }
        }
        const int rw = 2 * bw + 1;
        // band slot contributions, element order (stiffness_internal_frame2d.mojo:594-619)
        std::vector<std::vector<int>> slots((size_t)nf * rw);
        std::vector<std::vector<int>> fcontr(nf);
        std::vector<std::vector<double>> slotc, fc;
        if (any_mpc) {
            slotc.resize((size_t)nf * rw);
            fc.resize(nf);
        }
        if (d.num_slaves == 0) {
            for (int e = 0; e < d.num_elements; ++e) {
                const DevElem& E = elems[e0 + e];
                for (int a = 0; a < nd; ++a) {
                    const int ia = efree[(size_t)nd * e + a];
                    if (ia < 0) continue;
                    for (int b = 0; b < nd; ++b) {
                        const int ib = efree[(size_t)nd * e + b];
                        if (ib < 0) continue;
                        const size_t sl = (size_t)ia * rw + (ib - ia + bw);
                        slots[sl].push_back((int)(E.ek_off + a * nd + b));
                        if (any_mpc) slotc[sl].push_back(1.0);
                    }
                    fcontr[ia].push_back((int)(E.ef_off + a));
                    if (any_mpc) fc[ia].push_back(1.0);
                }
            }
            for (int s = 0; s < d.num_shells; ++s) {
                const DevShell& S = h->shells_h[sh0 + s];
                for (int a = 0; a < 24; ++a) {
                    const int ia = sfree[(size_t)24 * s + a];
                    if (ia < 0) continue;
                    for (int b = 0; b < 24; ++b) {
                        const int ib = sfree[(size_t)24 * s + b];
                        if (ib < 0) continue;
                        const size_t sl = (size_t)ia * rw + (ib - ia + bw);
                        slots[sl].push_back((int)(S.ek_off + a * 24 + b));
                        if (any_mpc) slotc[sl].push_back(1.0);
                    }
                    fcontr[ia].push_back((int)(S.ef_off + a));
                    if (any_mpc) fc[ia].push_back(1.0);
                }
            }
        } else {
            // collapse c_i k c_j onto the retained free dofs; entries outside the half width
            // detected from the elements' free dofs are dropped, as Strut's band load drops
            // them (linear_solver_backend.mojo:413-427)
            std::vector<std::pair<int, double>> ra, rb;
            for (int e = 0; e < d.num_elements; ++e) {
                const DevElem& E = elems[e0 + e];
                for (int a = 0; a < nd; ++a) {
                    rows_of(d.elements[e].dof[a], ra);
                    for (int b = 0; b < nd; ++b) {
                        rows_of(d.elements[e].dof[b], rb);
                        for (auto& ta : ra)
                            for (auto& tb : rb) {
                                if (ta.first < 0 || tb.first < 0 || std::abs(ta.first - tb.first) > bw) continue;
                                if (ta.second == 0.0 || tb.second == 0.0) continue;
                                const size_t sl = (size_t)ta.first * rw + (tb.first - ta.first + bw);
                                slots[sl].push_back((int)(E.ek_off + a * nd + b));
                                slotc[sl].push_back(ta.second * tb.second);
                            }
                    }
                    for (auto& ta : ra) {
                        if (ta.first < 0 || ta.second == 0.0) continue;
                        fcontr[ta.first].push_back((int)(E.ef_off + a));
                        fc[ta.first].push_back(ta.second);
                    }
                }
            }
            for (int s = 0; s < d.num_shells; ++s) {
                const DevShell& S = h->shells_h[sh0 + s];
                for (int a = 0; a < 24; ++a) {
                    rows_of(d.shells[s].dof[a], ra);
                    for (int b = 0; b < 24; ++b) {
                        rows_of(d.shells[s].dof[b], rb);
                        for (auto& ta : ra)
                            for (auto& tb : rb) {
                                if (ta.first < 0 || tb.first < 0 || std::abs(ta.first - tb.first) > bw) continue;
                                if (ta.second == 0.0 || tb.second == 0.0) continue;
                                const size_t sl = (size_t)ta.first * rw + (tb.first - ta.first + bw);
                                slots[sl].push_back((int)(S.ek_off + a * 24 + b));
                                slotc[sl].push_back(ta.second * tb.second);
                            }
                    }
                    for (auto& ta : ra) {
                        if (ta.first < 0 || ta.second == 0.0) continue;
                        fcontr[ta.first].push_back((int)(S.ef_off + a));
                        fc[ta.first].push_back(ta.second);
                    }
                }
            }
        }
        for (size_t k = 0; k < slots.size(); ++k) {
            slot_contrib.insert(slot_contrib.end(), slots[k].begin(), slots[k].end());
            if (any_mpc) slot_coef.insert(slot_coef.end(), slotc[k].begin(), slotc[k].end());
            slot_ptr.push_back((long long)slot_contrib.size());
        }
        for (int k = 0; k < nf; ++k) {
            fint_contrib.insert(fint_contrib.end(), fcontr[k].begin(), fcontr[k].end());
            if (any_mpc) fint_coef.insert(fint_coef.end(), fc[k].begin(), fc[k].end());
            fint_ptr.push_back((int)fint_contrib.size());
        }
        DevInst I;
        std::memset(&I, 0, sizeof(I));
        I.sl_off = sl0;
        I.n_sl = d.num_slaves;
        I.n = nf;
        I.bw = bw;
        I.rw = rw;
        I.num_dofs = d.num_dofs;
        I.u_off = u_off;
        I.f_off = f_off;
        I.band_off = band_off;
        I.slot_ptr_off = band_off;
        I.dense_off = dense_off;
        if ((size_t)nf * rw * sizeof(double) + 6 * sizeof(double) * (size_t)nf <= 220 * 1024)
            dense_off += (long long)nf * nf;
        I.elem_off = e0;
        I.n_elem = d.num_elements;
        I.fint_ptr_off = f_off;
        I.max_iters = d.max_iters;
        I.test_type = d.test_type;
        if (d.algorithm < STRUT_ALGORITHM_NEWTON || d.algorithm > STRUT_ALGORITHM_MODIFIED_NEWTON_INITIAL)
            return bail(fail(STRUT_BAD_ARG, "unknown algorithm"));
        I.algorithm = d.algorithm;
        {
            // the solver chain: as given, or the primary settings followed by Newton when the
            // primary algorithm is not Newton (transient_nonlinear.mojo:758-830)
            if (d.num_attempts < 0 || d.num_attempts > STRUT_MAX_ATTEMPTS)
                return bail(fail(STRUT_BAD_ARG, "num_attempts must be 0.." + std::to_string(STRUT_MAX_ATTEMPTS)));
            StrutSolverAttempt ch[STRUT_MAX_ATTEMPTS];
            int na = d.num_attempts;
            if (na > 0) {
                for (int k = 0; k < na; ++k) ch[k] = d.attempts[k];
            } else {
                ch[0].algorithm = d.algorithm;
                ch[0].test_type = d.test_type;
                ch[0].max_iters = d.max_iters;
                ch[0].tol = d.tol;
                na = 1;
                if (d.algorithm != STRUT_ALGORITHM_NEWTON) {
                    ch[1] = ch[0];
                    ch[1].algorithm = STRUT_ALGORITHM_NEWTON;
                    na = 2;
                }
            }
            I.n_att = na;
            int total = 0;
            for (int k = 0; k < na; ++k) {
                if (ch[k].algorithm < STRUT_ALGORITHM_NEWTON || ch[k].algorithm > STRUT_ALGORITHM_MODIFIED_NEWTON_INITIAL ||
                    ch[k].test_type < STRUT_TEST_MAX_DISP_INCR || ch[k].test_type > STRUT_TEST_ENERGY_INCR ||
                    ch[k].max_iters < 1)
                    return bail(fail(STRUT_BAD_ARG, "solver attempt out of range"));
                I.att_alg[k] = ch[k].algorithm;
                I.att_test[k] = ch[k].test_type;
                I.att_maxit[k] = ch[k].max_iters;
                I.att_tol[k] = ch[k].tol;
                if (ch[k].algorithm != STRUT_ALGORITHM_NEWTON) h->any_modified = 1;
                total += ch[k].max_iters;
            }
            if (na > 1) h->any_chain = 1;
            h->max_iters_global = std::max(h->max_iters_global, total);
        }
        I.spd = d.system == STRUT_SYSTEM_BAND_SPD;
        I.has_damping = d.alpha_m != 0.0 || d.beta_k != 0.0 || d.beta_k_init != 0.0 || d.beta_k_comm != 0.0;
        I.dt = d.dt;
        I.gamma = d.gamma;
        I.beta = d.beta;
        I.a0 = 1.0 / (d.beta * d.dt * d.dt);
        I.a1 = d.gamma / (d.beta * d.dt);
        I.a2 = 1.0 / (d.beta * d.dt);
        I.a3 = 1.0 / (2.0 * d.beta) - 1.0;
        I.coeff = d.dt * d.dt * (0.5 - d.beta);
        I.tol = d.tol;
        I.alpha_m = d.alpha_m;
        I.beta_k = d.beta_k;
        I.beta_k_init = d.beta_k_init;
        I.beta_k_comm = d.beta_k_comm;
        {
            // gathered element k / f entries, the band written to shared memory is not HBM;
            // K_init band, the gather lists, and the free-dof vectors
            long long ncontrib = 0, nfc = 0;
            for (auto& v : slots) ncontrib += (long long)v.size();
            for (auto& v : fcontr) nfc += (long long)v.size();
            I.io_bytes = 12.0 * ncontrib + 12.0 * nfc + 8.0 * (double)nf * rw * (d.beta_k_init != 0.0) +
                         8.0 * ((double)nf * rw + 1) + 8.0 * 14.0 * nf;
        }
        I.rec_off = h->n_rec_total;
        I.n_rec = d.num_record_dofs;
        I.rece_off = h->n_rece_slots;
        I.n_rece = nslots;
        h->rec_off[inst] = h->n_rec_total;
        h->n_rec[inst] = d.num_record_dofs;
        h->rece_off[inst] = h->n_rece_slots;
        h->n_rece[inst] = nslots;
        rece_base.push_back(h->n_rece_slots);
        for (int j = 0; j < d.num_record_dofs; ++j) {
            if (d.record_dofs[j] < 0 || d.record_dofs[j] >= d.num_dofs) return bail(fail(STRUT_BAD_ARG, "record dof out of range"));
            rec_dof.push_back(u_off + d.record_dofs[j]);
        }
        h->n_rec_total += d.num_record_dofs;
        h->n_rece_slots += nslots;
        const size_t ismem = ((size_t)nf * rw + 6 * (size_t)nf) * sizeof(double);
        if (ismem > 220 * 1024) {
            // band too large for shared memory: blocked factorisation in global memory
            if (I.spd)
                return bail(fail(STRUT_UNSUPPORTED, "BandSPD bands beyond shared memory are not implemented"));
            for (int k = 0; k < I.n_att; ++k)
                if (I.att_alg[k] != STRUT_ALGORITHM_NEWTON)
                    return bail(fail(STRUT_UNSUPPORTED, "ModifiedNewton on bands beyond shared memory is not implemented"));
            const size_t fsm = bw > kLargeMaxBw ? large_factor_smem(kPanelWide, kLargeThreadsWide)
                                                : large_factor_smem(kPanel, kLargeThreads);
            if (fsm > 220 * 1024 || bw > kLargeMaxBwWide)
                return bail(fail(STRUT_UNSUPPORTED, "band width too large for the blocked factorisation"));
            if (large_solve_smem(nf) > 220 * 1024)
                return bail(fail(STRUT_UNSUPPORTED, "system too large for the band substitution"));
            I.large = 1;
            I.large_idx = h->n_large++;
            I.lrw = 3 * bw + 1;  // columns i - bw .. i + 2 bw: room for the pivot rows' fill
            I.lband_off = h->lband_total;
            h->lband_total += (long long)nf * I.lrw;
            h->large_list_h.push_back(inst);
            h->max_large_n = std::max(h->max_large_n, nf);
            h->max_large_bw = std::max(h->max_large_bw, bw);
            h->lfactor_smem = std::max(h->lfactor_smem, fsm);
        } else {
            h->inst_smem = std::max(h->inst_smem, ismem);
        }
        h->insts[inst] = I;
        // excitations
        ExcHost& ex = h->exc[inst];
        ex.num = d.num_excitations;
        if (ex.num < 0 || ex.num > 2) return bail(fail(STRUT_BAD_ARG, "num_excitations must be 0..2"));
        for (int x = 0; x < ex.num; ++x) {
            ex.x[x] = d.excitation[x];
            if (ex.x[x].direction < 1 || ex.x[x].direction > 2) return bail(fail(STRUT_BAD_ARG, "excitation direction must be 1 or 2"));
            if (ex.x[x].count > 0 && !(ex.x[x].dt > 0.0)) return bail(fail(STRUT_BAD_ARG, "Path time series dt must be > 0"));
            ex.vals[x].assign(ex.x[x].values, ex.x[x].values + ex.x[x].count);
            ex.x[x].values = ex.vals[x].data();
        }
        if (ex.num == 2 && ex.x[0].direction == ex.x[1].direction)
            return bail(fail(STRUT_BAD_ARG, "two excitations must act in different directions"));
        u_off += d.num_dofs;
        f_off += nf;
        band_off += (long long)nf * rw;
    }
    for (const DevElem& E : elems) h->commit_bytes_total += E.commit_bytes;
    h->n_free_total = f_off;
    h->n_dofs_total = u_off;
    h->n_elem = (int)elems.size();
    h->band_total = band_off;
    h->dense_total = dense_off;
    if (h->elem_smem > 200 * 1024) return bail(fail(STRUT_UNSUPPORTED, "element fiber history exceeds shared memory"));
    h->elem_smem = std::max<size_t>(h->elem_smem, 16);
    CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    if ((rc = elem_grid_of(h)) != STRUT_OK) return bail(rc);
    CK(cudaFuncSetAttribute(instance_newton_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)std::max<size_t>(h->inst_smem, 16)));
    auto& al = h->allocs;
    // geometry and definitions
    DevMat* d_mats;
    DevSection* d_secs;
    double *d_y, *d_z, *d_a;
    int* d_m;
    if ((rc = upload(&d_mats, mats, al)) || (rc = upload(&d_secs, sp.secs, al)) ||
        (rc = upload(&d_y, sp.y, al)) || (rc = upload(&d_z, sp.z, al)) || (rc = upload(&d_a, sp.a, al)) ||
        (rc = upload(&d_m, sp.m, al)) || (rc = upload(&h->d_elems, elems, al)) ||
        (rc = upload(&h->d_insts, h->insts, al)))
        return bail(rc);
    {
        // recorded 3D beam-columns: their recorded force comes from a state determination after
        // the step's commit
        std::vector<int> rec3;
        for (int e = 0; e < (int)elems.size(); ++e)
            if (elems[e].nd == 12 && elems[e].rec >= 0) rec3.push_back(e);
        h->n_rec3 = (int)rec3.size();
        if ((rc = upload(&h->d_rec3, rec3, al))) return bail(rc);
    }
    {
        // section recorders
        std::vector<SecRec> secs;
        h->sec_off.assign(num_instances, 0);
        h->sec_n.assign(num_instances, 0);
        for (int i = 0; i < num_instances; ++i) {
            const StrutModelDesc& d = models[i];
            h->sec_off[i] = (int)secs.size();
            h->sec_n[i] = std::max(d.num_record_sections, 0);
            if (d.num_record_sections > 0 && !d.record_sections)
                return bail(fail(STRUT_BAD_ARG, "record_sections is NULL"));
            for (int k = 0; k < d.num_record_sections; ++k) {
                const StrutSectionRecord& sr = d.record_sections[k];
                if (sr.element < 0 || sr.element >= d.num_elements)
                    return bail(fail(STRUT_BAD_ARG, "section recorder element out of range"));
                const int ge = h->insts[i].elem_off + sr.element;
                if (sr.section < 0 || sr.section >= elems[ge].nip)
                    return bail(fail(STRUT_BAD_ARG, "section recorder section index out of range"));
                if (sr.kind != STRUT_SECTION_FORCE && sr.kind != STRUT_SECTION_DEFORMATION)
                    return bail(fail(STRUT_BAD_ARG, "section recorder kind must be force or deformation"));
                if (elems[ge].type == STRUT_ELEM_FORCE_BEAM_COLUMN_3D && elems[ge].rec < 0)
                    return bail(fail(STRUT_BAD_ARG, "a forceBeamColumn3d section recorder needs its element "
                                                    "recorded too (Strut's recorder re-runs its state determination)"));
                secs.push_back(SecRec{ge, sr.section, sr.kind, i});
            }
        }
        h->n_sec_slots = (int)secs.size();
        if (h->n_sec_slots > 0 && (rc = upload(&h->d_secrec, secs, al))) return bail(rc);
    }
    h->geo.y = d_y;
    h->geo.z = d_z;
    h->geo.a = d_a;
    h->geo.m = d_m;
    h->geo.mats = d_mats;
    h->geo.secs = d_secs;
    // fiber history: committed state initialised from each material (core.mojo:203-263)
    {
        const long long c2n = round4((int)std::max<long long>(c2_total, 4));
        const long long s2n = round4((int)std::max<long long>(s2_total, 4));
        const long long s1n = round4((int)std::max<long long>(s1_total, 4));
        const long long c1n = round4((int)std::max<long long>(c1_total, 4));
        std::vector<double> c2(5 * c2n, 0.0), s2(10 * s2n, 0.0), s1(5 * s1n, 0.0), c1(6 * c1n, 0.0);
        std::vector<int> kon(s2n, 0);
        for (const DevElem& E : elems) {
            const DevSection& sd = sp.secs[E.sec];
            for (int ip = 0; ip < E.nip; ++ip) {
                int base = sd.geo_off;
                for (int j = 0; j < sd.n_s2; ++j) {
                    const DevMat& m = mats[sp.m[base + j]];
                    const long long idx = E.s2_off + ip * sd.n_s2 + j;
                    s2[2 * s2n + idx] = m.p[1];
                    s2[4 * s2n + idx] = m.k[S2K_EPSY];
                    s2[3 * s2n + idx] = -m.k[S2K_EPSY];
                    if (m.p[10] != 0.0) {
                        s2[0 * s2n + idx] = m.k[S2K_SIGINI_E0];
                        s2[1 * s2n + idx] = m.p[10];
                    }
                }
                base += sd.n_s2;
                for (int j = 0; j < sd.n_c2; ++j) {
                    const DevMat& m = mats[sp.m[base + j]];
                    c2[2 * c2n + E.c2_off + ip * sd.n_c2 + j] = m.k[C2K_EC0];
                }
                base += sd.n_c2;
                for (int j = 0; j < sd.n_s1; ++j) {
                    const DevMat& m = mats[sp.m[base + j]];
                    s1[2 * s1n + E.s1_off + ip * sd.n_s1 + j] = m.p[1];
                }
                base += sd.n_s1;
                for (int j = 0; j < sd.n_c1; ++j) {
                    const DevMat& m = mats[sp.m[base + j]];
                    c1[2 * c1n + E.c1_off + ip * sd.n_c1 + j] = m.k[C1K_EC0];
                    c1[5 * c1n + E.c1_off + ip * sd.n_c1 + j] = m.k[C1K_EC0];
                }
            }
        }
        if ((rc = upload(&h->fs.c2, c2, al)) || (rc = upload(&h->fs.s2, s2, al)) ||
            (rc = upload(&h->fs.s2_kon, kon, al)) || (rc = upload(&h->fs.s1, s1, al)) ||
            (rc = upload(&h->fs.c1, c1, al)))
            return bail(rc);
        h->fs.c2_n = c2n;
        h->fs.s2_n = s2n;
        h->fs.s1_n = s1n;
        h->fs.c1_n = c1n;
    }
    InstArrays& A = h->A;
    std::memset(&A, 0, sizeof(A));
    const size_t nF = h->n_free_total;
    if ((rc = dzeros(&h->d_estate, (size_t)h->n_elem * kEStride, al)) ||
        (rc = dzeros(&h->d_ek, (size_t)h->ek_total, al)) ||
        (rc = dzeros(&h->d_ef, (size_t)h->ef_total, al)) || (rc = dzeros(&A.u_f, nF, al)) ||
        (rc = dzeros(&A.v_f, nF, al)) || (rc = dzeros(&A.a_f, nF, al)) ||
        (rc = dzeros(&A.u_n, nF, al)) || (rc = dzeros(&A.v_n, nF, al)) ||
        (rc = dzeros(&A.a_n, nF, al)) || (rc = dzeros(&A.P_f, nF, al)) ||
        (rc = dzeros(&A.du, nF, al)) || (rc = dzeros(&A.R, nF, al)) ||
        (rc = dzeros(&A.u_full, (size_t)h->n_dofs_total, al)) ||
        (rc = dzeros(&A.active, (size_t)h->n_inst, al)) ||
        (rc = dzeros(&A.status, (size_t)h->n_inst, al)) ||
        (rc = dzeros(&A.iters, (size_t)h->n_inst, al)) || (rc = dzeros(&A.nactive, 4, al)) ||
        (rc = dzeros(&A.export_band, (size_t)h->band_total, al)) ||
        (rc = dzeros(&A.export_f, nF, al)) || (rc = dzeros(&h->d_rhs, nF, al)) ||
        (rc = dzeros(&h->d_elem_err, (size_t)h->n_elem, al)) ||
        (rc = dzeros(&h->d_counters, 8, al)) || (rc = dzeros(&A.dense, (size_t)h->dense_total, al)) ||
        (rc = dzeros(&A.piv, nF, al)) || (rc = dzeros(&A.fallbacks, (size_t)h->n_inst, al)) ||
        (rc = dzeros(&A.el.list[0], (size_t)h->n_elem, al)) || (rc = dzeros(&A.el.list[1], (size_t)h->n_elem, al)) ||
        (rc = dzeros(&A.el.count, 2, al)) || (rc = dzeros(&A.el.next, 2, al)) ||
        (rc = dzeros(&A.el.hard[0], (size_t)kFanCap, al)) || (rc = dzeros(&A.el.hard[1], (size_t)kFanCap, al)) ||
        (rc = dzeros(&A.el.hard_count, 2, al)) || (rc = dzeros(&A.el.fan_done, (size_t)2 * kFanCap, al)) ||
        (rc = dzeros(&A.el.fan_first, (size_t)2 * kFanCap, al)))
        return bail(rc);
    {
        // attempt fan-out of forceBeamColumn2d elements (none in a 3D handle)
        bool any_fbc2d = false;
        for (int i = 0; i < num_instances && !any_fbc2d; ++i)
            for (int k = 0; k < models[i].num_elements; ++k)
                if (models[i].elements[k].type == STRUT_ELEM_FORCE_BEAM_COLUMN_2D) {
                    any_fbc2d = true;
                    break;
                }
        if (any_fbc2d &&
            ((rc = dzeros(&A.el.hard_flag, (size_t)h->n_elem, al)) ||
             (rc = dzeros(&A.el.fan_rec, (size_t)2 * kFanCap * kFanAttempts * kFanRec, al)) ||
             (rc = dzeros(&A.el.fan_round, (size_t)2 * kFanCap * kFanRound, al)) ||
             (rc = dzeros(&A.el.rq, (size_t)2 * kRoundQ, al)) || (rc = dzeros(&A.el.rq_tail, 2, al)) ||
             (rc = dzeros(&A.el.fan_finished, 2, al)) || (rc = dzeros(&A.el.q_err, 1, al))))
            return bail(rc);
    }
    if (h->any_modified &&
        ((rc = dzeros(&A.kfrz, (size_t)h->band_total, al)) || (rc = dzeros(&A.lufrz, (size_t)h->band_total, al)) ||
         (rc = dzeros(&A.lu_dense, (size_t)h->n_inst, al))))
        return bail(rc);
    if (h->any_chain &&
        ((rc = dzeros(&A.attempt, (size_t)h->n_inst, al)) || (rc = dzeros(&A.iters_prev, (size_t)h->n_inst, al)) ||
         (rc = dzeros(&A.u_base, nF, al)) || (rc = dzeros(&A.estate_base, (size_t)h->n_elem * kEStride, al))))
        return bail(rc);
    double* d_Mff;
    double* d_Mrff;
    double* d_fconst;
    int* d_free_dof;
    long long* d_slot_ptr;
    int* d_slot_contrib;
    int* d_fint_ptr;
    int* d_fint_contrib;
    double* d_Kinit;
    if ((rc = upload(&d_Mff, Mff, al)) || (rc = upload(&d_Mrff, Mrff, al)) ||
        (rc = upload(&d_fconst, fconst, al)) || (rc = upload(&d_free_dof, free_dof, al)) ||
        (rc = upload(&h->d_free_inst, free_inst, al)) || (rc = upload(&h->d_free_dir, free_dir, al)) ||
        (rc = upload(&d_slot_ptr, slot_ptr, al)) || (rc = upload(&d_slot_contrib, slot_contrib, al)) ||
        (rc = upload(&d_fint_ptr, fint_ptr, al)) || (rc = upload(&d_fint_contrib, fint_contrib, al)) ||
        (rc = upload(&h->d_rec_dof, rec_dof, al)) || (rc = upload(&h->d_rece_base, rece_base, al)) ||
        (rc = dzeros(&d_Kinit, (size_t)h->band_total, al)))
        return bail(rc);
    A.Mff = d_Mff;
    A.Mrff = d_Mrff;
    A.fconst = d_fconst;
    A.free_dof = d_free_dof;
    A.slot_ptr = d_slot_ptr;
    A.slot_contrib = d_slot_contrib;
    A.fint_ptr = d_fint_ptr;
    A.fint_contrib = d_fint_contrib;
    A.ek = h->d_ek;
    A.ef = h->d_ef;
    A.Kinit = d_Kinit;
    if (any_mpc) {
        double *d_sc, *d_fc, *d_slc;
        int *d_sld, *d_slp, *d_slm;
        if ((rc = upload(&d_sc, slot_coef, al)) || (rc = upload(&d_fc, fint_coef, al)) ||
            (rc = upload(&d_sld, sl_dof, al)) || (rc = upload(&d_slp, sl_ptr, al)) ||
            (rc = upload(&d_slm, sl_master, al)) || (rc = upload(&d_slc, sl_coef, al)))
            return bail(rc);
        A.slot_coef = d_sc;
        A.fint_coef = d_fc;
        A.sl_dof = d_sld;
        A.sl_ptr = d_slp;
        A.sl_master = d_slm;
        A.sl_coef = d_slc;
        h->n_slaves_total = (int)sl_dof.size();
    }
    if ((rc = dzeros(&h->d_ctl, 1, al))) return bail(rc);
    {
        std::vector<int> neg(h->n_inst, -1);
        if ((rc = upload(&h->d_fail_step, neg, al))) return bail(rc);
    }
    A.ctl = h->d_ctl;
    A.estate = h->d_estate;
    A.n_free_total = h->n_free_total;
    A.n_inst = h->n_inst;
    A.dual = 0;
    if (h->n_large > 0) {
        std::vector<int> rowbase(h->n_large + 1, 0);
        for (int li = 0; li < h->n_large; ++li) rowbase[li + 1] = rowbase[li] + h->insts[h->large_list_h[li]].n;
        h->large_rows = rowbase[h->n_large];
        std::vector<int> lstat(h->n_large, -1);
        if ((rc = upload(&h->d_large_list, h->large_list_h, al)) || (rc = upload(&h->d_large_rowbase, rowbase, al)) ||
            (rc = dzeros(&A.lband, (size_t)h->lband_total, al)) || (rc = upload(&A.lstatus, lstat, al)) ||
            (rc = dzeros(&h->d_gb, 1, al)) || (rc = dzeros(&h->d_wbuf, nF, al)) ||
            (rc = dzeros(&h->d_lpan, (size_t)std::max(kPanel * kLargeThreads, kPanelWide * kLargeThreadsWide), al)) ||
            (rc = dzeros(&h->d_lpiv, (size_t)std::max(kLargeThreads, kLargeThreadsWide), al)))
            return bail(rc);
        {
            const int polls = kBarrierPolls;
            CK(cudaMemcpy((char*)h->d_gb + offsetof(GridBarrier, limit), &polls, sizeof(int), cudaMemcpyHostToDevice));
        }
        h->lfactor_wide = h->max_large_bw > kLargeMaxBw ? 1 : 0;
        const void* fk = h->lfactor_wide ? (const void*)large_factor_kernel<kPanelWide, kLargeThreadsWide>
                                         : (const void*)large_factor_kernel<kPanel, kLargeThreads>;
        CK(cudaFuncSetAttribute(fk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->lfactor_smem));
        int per_sm = 0, n_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fk, h->lfactor_wide ? kLargeThreadsWide : kLargeThreads,
                                                         h->lfactor_smem));
        CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, h->device));
        if (per_sm < 1) return bail(fail(STRUT_UNSUPPORTED, "band factorisation kernel does not fit on an SM"));
        // one CTA per SM at most, all co-resident (cooperative launch), and no more than one
        // panel's trailing tiles can use
        h->lfactor_grid = std::max(1, std::min(n_sm, large_factor_tiles(h->max_large_bw)));
        h->default_factor_grid = h->lfactor_grid;
        h->max_factor_grid = n_sm * per_sm;
        CK(cudaFuncSetAttribute(large_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)large_solve_smem(h->max_large_n)));
    }
    CK(cudaMallocHost((void**)&h->h_ctrl, 4 * sizeof(int)));
    CK(cudaEventCreate(&h->ev0));
    CK(cudaEventCreate(&h->ev1));
    std::memset(&h->P, 0, sizeof(h->P));
    // initial assembly at the initial displacements (transient_nonlinear.mojo:1207-1453): K_init
    // for betaKInit; the trial fiber state it produces is discarded (revert) by construction.
    {
        std::vector<int> ones(h->n_inst, 1);
        CK(cudaMemcpy(A.active, ones.data(), sizeof(int) * h->n_inst, cudaMemcpyHostToDevice));
        if (!h->shells_h.empty()) {
            h->n_shells = (int)h->shells_h.size();
            int* d_err = nullptr;
            if ((rc = upload(&h->d_shells, h->shells_h, al)) || (rc = dzeros(&d_err, 1, al))) return bail(rc);
            shell_stiffness_kernel<<<(h->n_shells + 63) / 64, 64, 0, h->stream>>>(h->d_shells, h->n_shells, h->d_ek,
                                                                                d_err);
            CK(cudaGetLastError());
            int herr = 0;
            CK(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            if (herr) return bail(fail(STRUT_BAD_ARG, "shell with a singular Jacobian"));
        }
        if ((rc = launch_elements(h, 1)) != STRUT_OK) return bail(rc);
        // Kinit = K gathered in element order; the export path of the instance kernel with
        // a0 = a1 = 0 and no damping would equal K, but a dedicated gather keeps it exact.
        std::vector<DevInst> tmp = h->insts;
        for (auto& I : tmp) {
            I.a0 = 0.0;
            I.a1 = 0.0;
            I.has_damping = 0;
            I.spd = 0;
        }
        DevInst* d_tmp;
        if ((rc = upload(&d_tmp, tmp, al))) return bail(rc);
        InstArrays B = A;
        B.export_band = d_Kinit;
        instance_newton_kernel<<<h->n_inst, 256, h->inst_smem, h->stream>>>(d_tmp, B, INST_MODE_EXPORT, -1);
        CK(cudaGetLastError());
        if ((rc = launch_large(h, INST_MODE_EXPORT, d_tmp, &B)) != STRUT_OK) return bail(rc);
        CK(cudaStreamSynchronize(h->stream));
        std::vector<int> st(h->n_inst);
        CK(cudaMemcpy(st.data(), A.status, sizeof(int) * h->n_inst, cudaMemcpyDeviceToHost));
        for (int i = 0; i < h->n_inst; ++i)
            if (st[i] != 0) return bail(fail(st[i], "initial assembly failed for instance " + std::to_string(i)));
    }
    *out = h;
    return STRUT_OK;
}

int strut_gpu_destroy(StrutHandle* h) {
    if (!h) return STRUT_BAD_ARG;
    cudaStreamSynchronize(h->stream);
    delete h;
    return STRUT_OK;
}

int strut_gpu_num_instances(const StrutHandle* h) { return h ? h->n_inst : 0; }

int strut_gpu_run_steps(StrutHandle* h, int32_t n_steps, StrutStepStats* stats) {
    if (!h || n_steps < 0) return fail(STRUT_BAD_ARG, "bad arguments");
    StrutStepStats st;
    std::memset(&st, 0, sizeof(st));
    st.failed_instance = -1;
    st.failed_step = -1;
    TRY(ensure_history(h, h->steps_done + n_steps));
    // ground accelerations of every step of this call: per instance 2 values + 2 flags
    if (h->ag_cap < n_steps) {
        if (h->d_ag) cudaFree(h->d_ag);
        h->d_ag = nullptr;
        CK(cudaMalloc((void**)&h->d_ag, (size_t)n_steps * 4 * h->n_inst * sizeof(double)));
        h->ag_cap = n_steps;
    }
    {
        std::vector<double> ag((size_t)n_steps * 4 * h->n_inst, 0.0);
        for (int s = 0; s < n_steps; ++s) {
            const int step = h->steps_done + s;
            for (int i = 0; i < h->n_inst; ++i) {
                const double t = (double)(step + 1) * h->insts[i].dt;
                double* row = &ag[((size_t)s * h->n_inst + i) * 4];
                for (int x = 0; x < h->exc[i].num; ++x) {
                    const int dir = h->exc[i].x[x].direction;
                    row[dir - 1] = path_eval(h->exc[i].x[x], t);
                    row[2 + dir - 1] = 1.0;
                }
            }
        }
        if (n_steps > 0)
            CK(cudaMemcpyAsync(h->d_ag, ag.data(), ag.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    CK(cudaMemsetAsync(h->d_counters, 0, 8 * sizeof(unsigned long long), h->stream));
    const int nF = h->n_free_total;
    const int tb = 256;
    int rc = STRUT_OK;
    const int step0 = h->steps_done;
    {
        DevCtl c;
        std::memset(&c, 0, sizeof(c));
        c.step = step0;
        c.step0 = step0;
        c.n_end = step0 + n_steps;
        c.max_iters = h->max_iters_global;
        c.single = h->n_inst == 1;
        c.fan = h->tune.fan_out ? 1 : 0;
        if (!c.fan && h->A.el.hard_flag)
            CK(cudaMemsetAsync(h->A.el.hard_flag, 0, sizeof(int) * (size_t)h->n_elem, h->stream));
        CK(cudaMemcpyAsync(h->d_ctl, &c, sizeof(c), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemsetAsync(h->A.nactive, 0, 4 * sizeof(int), h->stream));
        CK(cudaMemsetAsync(h->A.el.count, 0, 2 * sizeof(int), h->stream));
        CK(cudaMemsetAsync(h->A.el.next, 0, 2 * sizeof(int), h->stream));
        CK(cudaMemsetAsync(h->A.el.hard_count, 0, 2 * sizeof(int), h->stream));
        if (h->A.el.rq) {
            // the attempt queue starts empty (-1 entries) for every run
            CK(cudaMemsetAsync(h->A.el.rq, 0xFF, sizeof(long long) * 2 * kRoundQ, h->stream));
            CK(cudaMemsetAsync(h->A.el.rq_tail, 0, 2 * sizeof(int), h->stream));
            CK(cudaMemsetAsync(h->A.el.fan_finished, 0, 2 * sizeof(int), h->stream));
        }
        CK(cudaStreamSynchronize(h->stream));
    }
    if (n_steps > 0 && !h->prof && h->n_large == 0) {
        // (instances with a global-memory band run the host-driven loop: their cooperative
        // factorisation is launched with cudaLaunchCooperativeKernel)
        TRY(ensure_graph(h));
        CK(cudaGraphLaunch(h->gexec, h->stream));
    } else {
        // host-driven loop (profiling: per-launch event timing on the launching stream)
        cudaGraphConditionalHandle none = 0;
        for (int s = 0; s < n_steps; ++s) {
            const int step = step0 + s;
            const int npred = std::max(nF, h->n_inst);
            TRY(prof_begin(h));
            predictor_kernel<<<(npred + tb - 1) / tb, tb, 0, h->stream>>>(
                h->d_insts, h->A, h->d_free_inst, h->d_free_dir, h->d_ag, nF, h->n_inst, h->d_ctl, none, 0);
            CK(cudaGetLastError());
            if (h->any_chain || h->pred) {
                copy_doubles_kernel<<<592, tb, 0, h->stream>>>(h->d_estate, h->A.estate_base,
                                                               (long long)h->n_elem * kEStride);
                CK(cudaGetLastError());
            }
            if (h->n_slaves_total > 0) {
                slave_enforce_kernel<<<(h->n_slaves_total + tb - 1) / tb, tb, 0, h->stream>>>(h->A, h->n_slaves_total);
                CK(cudaGetLastError());
            }
            TRY(prof_end(h, 3));
            if (h->pred) {
                TRY(prof_begin(h));
                TRY(pred_launch(h));
                TRY(prof_end(h, 6));
            }
            for (int it = 0; it < h->max_iters_global; ++it) {
                TRY(launch_elements(h));
                TRY(launch_instances(h, INST_MODE_NEWTON, step));
                newton_check_kernel<<<1, 32, 0, h->stream>>>(h->d_ctl, h->A.nactive, none, 0);
                CK(cudaGetLastError());
                CK(cudaMemcpyAsync(h->h_ctrl, h->A.nactive, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
                CK(cudaStreamSynchronize(h->stream));
                if (h->h_ctrl[0] <= 0) break;
            }
            TRY(prof_begin(h));
            commit_kernel_of(h)<<<h->n_elem, commit_block(h), 0, h->stream>>>(
                h->d_elems, h->geo, h->fs, h->A.u_full, h->d_estate, h->A.status, h->d_hist_ef, h->d_rece_base,
                std::max(h->n_rece_slots, 1), h->ef_w, h->d_ctl);
            CK(cudaGetLastError());
            TRY(launch_record_pass(h));
            TRY(prof_end(h, 2));
            TRY(prof_begin(h));
            post_step_kernel<<<(nF + tb - 1) / tb, tb, 0, h->stream>>>(h->d_insts, h->A, h->d_free_inst, nF);
            CK(cudaGetLastError());
            TRY(prof_end(h, 4));
            if (h->prof) h->P.bytes[2] += h->commit_bytes_total;
            if (h->n_rec_total > 0) {
                record_disp_kernel<<<(h->n_rec_total + tb - 1) / tb, tb, 0, h->stream>>>(
                    h->A.u_full, h->d_rec_dof, h->n_rec_total, h->d_hist_disp, h->d_ctl);
                CK(cudaGetLastError());
            }
            if (h->n_sec_slots > 0) {
                record_sections_kernel<<<(h->n_sec_slots * 32 + 255) / 256, 256, 0, h->stream>>>(
                    h->d_elems, h->geo, h->fs, h->A.u_full, h->d_estate, h->d_secrec, h->n_sec_slots,
                    h->ndf_all == 6 ? 4 : 2, h->d_hist_sec, h->d_ctl);
                CK(cudaGetLastError());
            }
            step_end_kernel<<<1, 256, 0, h->stream>>>(h->d_ctl, h->A.status, h->d_fail_step, h->n_inst,
                                                      h->A.nactive, h->A.el, none, 0);
            CK(cudaGetLastError());
            if (h->n_inst == 1) {
                int s0 = 0;
                CK(cudaMemcpyAsync(&s0, h->A.status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
                CK(cudaStreamSynchronize(h->stream));
                if (s0 != 0) break;
            }
        }
    }
    CK(cudaStreamSynchronize(h->stream));
    {
        DevCtl c;
        CK(cudaMemcpy(&c, h->d_ctl, sizeof(c), cudaMemcpyDeviceToHost));
        st.steps_done = c.step - step0;
        h->steps_done = c.step;
        std::vector<int> status(h->n_inst), fstep(h->n_inst);
        CK(cudaMemcpy(status.data(), h->A.status, sizeof(int) * h->n_inst, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(fstep.data(), h->d_fail_step, sizeof(int) * h->n_inst, cudaMemcpyDeviceToHost));
        // the first failure of this run: earliest step, then lowest instance
        for (int i = 0; i < h->n_inst; ++i) {
            if (status[i] == 0 || fstep[i] < step0) continue;
            if (st.failed_instance < 0 || fstep[i] < st.failed_step) {
                st.failed_instance = i;
                st.failed_step = fstep[i];
                rc = status[i];
            }
        }
    }
    CK(cudaStreamSynchronize(h->stream));
    unsigned long long cnt[8];
    CK(cudaMemcpy(cnt, h->d_counters, sizeof(cnt), cudaMemcpyDeviceToHost));
    if (h->prof) {
        // element kernel: the fiber-state update bytes of its section evaluations
        h->P.bytes[0] += (double)cnt[7];
        h->P.bytes[1] += (double)cnt[4];
        h->P.bytes[3] += (double)st.steps_done * 8.0 * 12.0 * h->n_free_total;
        h->P.bytes[4] += (double)st.steps_done * 8.0 * 8.0 * h->n_free_total;
    }
    st.local_element_iterations = (int64_t)cnt[0];
    st.fanned_out = (int64_t)cnt[6];
    st.section_evaluations = (int64_t)cnt[1];
    {
        const int first = h->steps_done - st.steps_done;
        if (st.steps_done > 0) {
            std::vector<int> it((size_t)st.steps_done * h->n_inst);
            CK(cudaMemcpy(it.data(), h->d_hist_iters + (size_t)first * h->n_inst, it.size() * sizeof(int),
                          cudaMemcpyDeviceToHost));
            long long tot = 0, fac = 0;
            for (size_t k = 0; k < it.size(); ++k) {
                tot += it[k];
                // ModifiedNewton factors once per step
                fac += h->insts[k % h->n_inst].algorithm == STRUT_ALGORITHM_NEWTON ? it[k] : (it[k] > 0 ? 1 : 0);
            }
            st.global_newton_iterations = tot;
            st.factorizations = fac;
        }
    }
    // fiber updates: per section evaluation, the section's fiber count
    st.fiber_updates = (int64_t)cnt[2];
    if (h->A.el.q_err) {
        int qe = 0;
        CK(cudaMemcpy(&qe, h->A.el.q_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (qe) {
            rc = fail(STRUT_CUDA_ERROR, "a wait on the element attempt queue ran out");
            CK(cudaMemset(h->A.el.q_err, 0, sizeof(int)));
        }
    }
    st.status = rc;
    if (rc != STRUT_OK) {
        std::vector<int> ee(h->n_elem);
        CK(cudaMemcpy(ee.data(), h->d_elem_err, sizeof(int) * h->n_elem, cudaMemcpyDeviceToHost));
        g_last_error = "instance " + std::to_string(st.failed_instance) + " failed at step " +
                       std::to_string(st.failed_step) + " with status " + std::to_string(rc);
    }
    if (stats) *stats = st;
    return rc;
}

int strut_gpu_get_history(StrutHandle* h, int32_t instance, double* disp, double* eforce,
                          int32_t* iters) {
    if (!h || instance < 0 || instance >= h->n_inst) return fail(STRUT_BAD_ARG, "bad arguments");
    const int S = h->steps_done;
    if (S == 0) return STRUT_OK;
    if (disp && h->n_rec[instance] > 0) {
        std::vector<double> all((size_t)S * h->n_rec_total);
        CK(cudaMemcpy(all.data(), h->d_hist_disp, all.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int s = 0; s < S; ++s)
            for (int j = 0; j < h->n_rec[instance]; ++j)
                disp[(size_t)s * h->n_rec[instance] + j] = all[(size_t)s * h->n_rec_total + h->rec_off[instance] + j];
    }
    if (eforce && !h->rece_map[instance].empty()) {
        const int slots = std::max(h->n_rece_slots, 1), W = h->ef_w, nd = h->inst_nd[instance];
        std::vector<double> all((size_t)S * slots * W);
        CK(cudaMemcpy(all.data(), h->d_hist_ef, all.size() * sizeof(double), cudaMemcpyDeviceToHost));
        const auto& mp = h->rece_map[instance];
        for (int s = 0; s < S; ++s)
            for (size_t j = 0; j < mp.size(); ++j)
                for (int c = 0; c < nd; ++c)
                    eforce[((size_t)s * mp.size() + j) * nd + c] =
                        all[((size_t)s * slots + h->rece_off[instance] + mp[j]) * W + c];
    }
    if (iters) {
        std::vector<int> all((size_t)S * h->n_inst);
        CK(cudaMemcpy(all.data(), h->d_hist_iters, all.size() * sizeof(int), cudaMemcpyDeviceToHost));
        for (int s = 0; s < S; ++s) iters[s] = all[(size_t)s * h->n_inst + instance];
    }
    return STRUT_OK;
}

int strut_gpu_get_history_all(StrutHandle* h, double* disp, double* eforce, int32_t* iters) {
    if (!h) return fail(STRUT_BAD_ARG, "bad arguments");
    const int S = h->steps_done;
    if (S == 0) return STRUT_OK;
    if (disp && h->n_rec_total > 0) {
        std::vector<double> all((size_t)S * h->n_rec_total);
        CK(cudaMemcpy(all.data(), h->d_hist_disp, all.size() * sizeof(double), cudaMemcpyDeviceToHost));
        size_t o = 0;
        for (int i = 0; i < h->n_inst; ++i)
            for (int s = 0; s < S; ++s)
                for (int j = 0; j < h->n_rec[i]; ++j) disp[o++] = all[(size_t)s * h->n_rec_total + h->rec_off[i] + j];
    }
    if (eforce) {
        const int slots = std::max(h->n_rece_slots, 1), W = h->ef_w;
        std::vector<double> all((size_t)S * slots * W);
        CK(cudaMemcpy(all.data(), h->d_hist_ef, all.size() * sizeof(double), cudaMemcpyDeviceToHost));
        size_t o = 0;
        for (int i = 0; i < h->n_inst; ++i) {
            const auto& mp = h->rece_map[i];
            const int nd = h->inst_nd[i];
            for (int s = 0; s < S; ++s)
                for (size_t j = 0; j < mp.size(); ++j)
                    for (int c = 0; c < nd; ++c)
                        eforce[o++] = all[((size_t)s * slots + h->rece_off[i] + mp[j]) * W + c];
        }
    }
    if (iters) {
        std::vector<int> all((size_t)S * h->n_inst);
        CK(cudaMemcpy(all.data(), h->d_hist_iters, all.size() * sizeof(int), cudaMemcpyDeviceToHost));
        size_t o = 0;
        for (int i = 0; i < h->n_inst; ++i)
            for (int s = 0; s < S; ++s) iters[o++] = all[(size_t)s * h->n_inst + i];
    }
    return STRUT_OK;
}

int strut_gpu_get_section_history(StrutHandle* h, int32_t instance, double* out) {
    if (!h || instance < 0 || instance >= h->n_inst) return fail(STRUT_BAD_ARG, "bad arguments");
    const int S = h->steps_done, n = h->sec_n[instance];
    if (S == 0 || n == 0) return STRUT_OK;
    if (!out) return fail(STRUT_BAD_ARG, "bad arguments");
    const int W = h->ndf_all == 6 ? 4 : 2;
    std::vector<double> all((size_t)S * h->n_sec_slots * W);
    CK(cudaMemcpy(all.data(), h->d_hist_sec, all.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (int s = 0; s < S; ++s)
        for (int k = 0; k < n; ++k)
            for (int c = 0; c < W; ++c)
                out[((size_t)s * n + k) * W + c] = all[((size_t)s * h->n_sec_slots + h->sec_off[instance] + k) * W + c];
    return STRUT_OK;
}

int strut_gpu_instance_status(const StrutHandle* h, int32_t* status) {
    if (!h || !status) return fail(STRUT_BAD_ARG, "bad arguments");
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(status, h->A.status, sizeof(int) * h->n_inst, cudaMemcpyDeviceToHost));
    return STRUT_OK;
}

int strut_gpu_get_state(StrutHandle* h, int32_t instance, double* u_free, double* v_free,
                        double* a_free) {
    if (!h || instance < 0 || instance >= h->n_inst) return fail(STRUT_BAD_ARG, "bad arguments");
    const DevInst& I = h->insts[instance];
    CK(cudaStreamSynchronize(h->stream));
    if (u_free) CK(cudaMemcpy(u_free, h->A.u_f + I.f_off, I.n * sizeof(double), cudaMemcpyDeviceToHost));
    if (v_free) CK(cudaMemcpy(v_free, h->A.v_f + I.f_off, I.n * sizeof(double), cudaMemcpyDeviceToHost));
    if (a_free) CK(cudaMemcpy(a_free, h->A.a_f + I.f_off, I.n * sizeof(double), cudaMemcpyDeviceToHost));
    return STRUT_OK;
}

int strut_gpu_set_profiling(StrutHandle* h, int32_t enabled) {
    if (!h) return fail(STRUT_BAD_ARG, "bad arguments");
    h->prof = enabled != 0;
    if (h->prof) std::memset(&h->P, 0, sizeof(h->P));
    return STRUT_OK;
}

int strut_gpu_set_tuning(StrutHandle* h, const StrutTuning* t) {
    if (!h) return fail(STRUT_BAD_ARG, "bad arguments");
    StrutTuning d = {1, 0, 0, 0, {0, 0, 0, 0}};
    if (t) {
        if ((t->fan_out != 0 && t->fan_out != 1) || (t->commit_team != 0 && t->commit_team != 64 && t->commit_team != 128) ||
            (t->commit_team == 128 && h->max_nip > 5) || t->factor_ctas < 0 ||
            (t->element_threads != 0 && !elem_threads_ok(h, t->element_threads)))
            return fail(STRUT_BAD_ARG, "tuning value out of range");
        d = *t;
    }
    const StrutTuning old = h->tune;
    h->tune = d;
    if (elem_grid_of(h) != STRUT_OK) {
        h->tune = old;
        elem_grid_of(h);
        return fail(STRUT_UNSUPPORTED, "the element kernel with that many threads does not fit on an SM");
    }
    h->lfactor_grid = d.factor_ctas > 0 ? std::min(d.factor_ctas, h->max_factor_grid) : h->default_factor_grid;
    h->tune_gen += 1;
    return STRUT_OK;
}

int strut_gpu_set_wait_limit(StrutHandle* h, int32_t polls) {
    if (!h || polls < 0) return fail(STRUT_BAD_ARG, "bad arguments");
    if (!h->d_gb) return STRUT_OK;  // no cooperative factorisation in this handle
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy((char*)h->d_gb + offsetof(GridBarrier, limit), &polls, sizeof(int), cudaMemcpyHostToDevice));
    return STRUT_OK;
}

int strut_gpu_get_tuning(const StrutHandle* h, StrutTuning* out) {
    if (!h || !out) return fail(STRUT_BAD_ARG, "bad arguments");
    *out = h->tune;
    out->commit_team = commit_team_of(h);
    out->element_threads = elem_threads_of(h);
    out->factor_ctas = h->n_large ? h->lfactor_grid : 0;
    return STRUT_OK;
}

int strut_gpu_get_profile(const StrutHandle* h, StrutKernelProfile* out) {
    if (!h || !out) return fail(STRUT_BAD_ARG, "bad arguments");
    *out = h->P;
    return STRUT_OK;
}

void* strut_gpu_stream(const StrutHandle* h) { return h ? (void*)h->stream : nullptr; }

int strut_gpu_band_info(const StrutHandle* h, int32_t instance, int32_t* half_bw, int32_t* row_width) {
    if (!h || instance < 0 || instance >= h->n_inst) return fail(STRUT_BAD_ARG, "bad arguments");
    const DevInst& I = h->insts[instance];
    if (half_bw) *half_bw = I.bw;
    if (row_width) *row_width = I.spd ? I.bw + 1 : I.rw;
    return STRUT_OK;
}

int strut_gpu_state_determination(StrutHandle* h, const double* u_free, double* f_int_free,
                                  double* band_out) {
    if (!h || !u_free) return fail(STRUT_BAD_ARG, "bad arguments");
    const int nF = h->n_free_total;
    CK(cudaMemcpyAsync(h->A.u_f, u_free, nF * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    scatter_free_kernel<<<(nF + 255) / 256, 256, 0, h->stream>>>(h->A.u_f, h->A.free_dof, h->A.u_full, nF);
    CK(cudaGetLastError());
    if (h->n_slaves_total > 0) {
        slave_enforce_kernel<<<(h->n_slaves_total + 255) / 256, 256, 0, h->stream>>>(h->A, h->n_slaves_total);
        CK(cudaGetLastError());
    }
    std::vector<int> ones(h->n_inst, 1), zeros(h->n_inst, 0);
    CK(cudaMemcpyAsync(h->A.active, ones.data(), sizeof(int) * h->n_inst, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->A.status, zeros.data(), sizeof(int) * h->n_inst, cudaMemcpyHostToDevice, h->stream));
    TRY(launch_elements(h, 1));
    TRY(launch_instances(h, INST_MODE_EXPORT, -1));
    CK(cudaStreamSynchronize(h->stream));
    std::vector<int> st(h->n_inst);
    CK(cudaMemcpy(st.data(), h->A.status, sizeof(int) * h->n_inst, cudaMemcpyDeviceToHost));
    for (int i = 0; i < h->n_inst; ++i)
        if (st[i] != 0) return fail(st[i], "state determination failed for instance " + std::to_string(i));
    if (f_int_free) CK(cudaMemcpy(f_int_free, h->A.export_f, nF * sizeof(double), cudaMemcpyDeviceToHost));
    if (band_out) {
        std::vector<double> band((size_t)h->band_total);
        CK(cudaMemcpy(band.data(), h->A.export_band, band.size() * sizeof(double), cudaMemcpyDeviceToHost));
        size_t o = 0;
        for (int i = 0; i < h->n_inst; ++i) {
            const DevInst& I = h->insts[i];
            for (int r = 0; r < I.n; ++r) {
                if (I.spd) {
                    for (int k = 0; k <= I.bw; ++k) {  // slot row*(bw+1) + (row - col)
                        const int col = r - k;
                        band_out[o++] = col >= 0 ? band[I.band_off + (size_t)r * I.rw + (col - r + I.bw)] : 0.0;
                    }
                } else {
                    for (int k = 0; k < I.rw; ++k) band_out[o++] = band[I.band_off + (size_t)r * I.rw + k];
                }
            }
        }
    }
    h->state_determined = true;
    return STRUT_OK;
}

int strut_gpu_factor_solve(StrutHandle* h, const double* rhs, double* du) {
    if (!h || !rhs || !du) return fail(STRUT_BAD_ARG, "bad arguments");
    if (!h->state_determined) return fail(STRUT_BAD_ARG, "call strut_gpu_state_determination first");
    const int nF = h->n_free_total;
    CK(cudaMemcpyAsync(h->d_rhs, rhs, nF * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    InstArrays A = h->A;
    A.rhs_in = h->d_rhs;
    std::vector<int> zeros(h->n_inst, 0);
    CK(cudaMemcpyAsync(h->A.status, zeros.data(), sizeof(int) * h->n_inst, cudaMemcpyHostToDevice, h->stream));
    instance_newton_kernel<<<h->n_inst, 256, h->inst_smem, h->stream>>>(h->d_insts, A, INST_MODE_SOLVE_EXPORTED, -1);
    CK(cudaGetLastError());
    TRY(launch_large(h, INST_MODE_SOLVE_EXPORTED, nullptr, &A));
    CK(cudaStreamSynchronize(h->stream));
    std::vector<int> st(h->n_inst);
    CK(cudaMemcpy(st.data(), h->A.status, sizeof(int) * h->n_inst, cudaMemcpyDeviceToHost));
    for (int i = 0; i < h->n_inst; ++i)
        if (st[i] != 0) return fail(st[i], "factorization failed for instance " + std::to_string(i));
    CK(cudaMemcpy(du, h->A.du, nF * sizeof(double), cudaMemcpyDeviceToHost));
    return STRUT_OK;
}

int strut_gpu_commit(StrutHandle* h) {
    if (!h) return fail(STRUT_BAD_ARG, "bad arguments");
    commit_kernel_of(h)<<<h->n_elem, commit_block(h), 0, h->stream>>>(
        h->d_elems, h->geo, h->fs, h->A.u_full, h->d_estate, h->A.status, nullptr, h->d_rece_base, 1,
        h->ef_w, h->d_ctl);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    return STRUT_OK;
}

int strut_gpu_revert(StrutHandle* h) {
    // Trial fiber state is never stored (it is recomputed from committed state on demand), so
    // committed -> trial has nothing to copy.
    if (!h) return fail(STRUT_BAD_ARG, "bad arguments");
    return STRUT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// known-answer drivers and batched section evaluation
// ---------------------------------------------------------------------------------------
struct StrutSectionBatch {
    int n_inst = 0;
    std::vector<void*> allocs;
    Geo geo;
    DevSection sd;
    BatchState bs;  // bs.n_inst: allocated instances (a whole number of tiles), the field stride
    // streaming kernel: stage geometry, tiles, persistent grid (0: the stages do not fit, one warp
    // per instance instead)
    FsLayout L{};
    int n_mats = 0;
    long long n_tiles = 0;
    int grid = 0;
    size_t smem = 0;
    int* d_err = nullptr;
    ~StrutSectionBatch() {
        for (void* p : allocs) cudaFree(p);
    }
};

extern "C" {

int strut_gpu_material_path(const StrutUniMaterial* material, const double* strains, int32_t n,
                            double* out) {
    if (!material || (n > 0 && (!strains || !out)) || n < 0) return fail(STRUT_BAD_ARG, "bad arguments");
    if (n == 0) return STRUT_OK;
    DevMat m = make_devmat(*material);
    double *d_s = nullptr, *d_o = nullptr;
    CK(cudaMalloc((void**)&d_s, n * sizeof(double)));
    CK(cudaMalloc((void**)&d_o, 2 * n * sizeof(double)));
    CK(cudaMemcpy(d_s, strains, n * sizeof(double), cudaMemcpyHostToDevice));
    material_path_kernel<<<1, 32>>>(m, d_s, n, d_o);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(out, d_o, 2 * n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d_s);
    cudaFree(d_o);
    if (e != cudaSuccess) return fail(STRUT_CUDA_ERROR, cudaGetErrorString(e));
    return STRUT_OK;
}

}  // extern "C"

// Initial committed state (UniMaterialState(mat_def), core.mojo:203-263) of n_inst copies of
// the section sp.secs[0], laid out as section_batch_kernel reads it.
static void batch_initial_state(const SectionPack& sp, const std::vector<DevMat>& mats, long long n_inst,
                                std::vector<double>& s2, std::vector<double>& c2, std::vector<double>& s1,
                                std::vector<double>& c1, std::vector<int>& kon) {
    const DevSection& sd = sp.secs[0];
    const int P2 = fs_pad4(sd.n_s2), P3 = fs_pad4(sd.n_c2), P1 = fs_pad4(sd.n_s1), P4 = fs_pad4(sd.n_c1);
    const long long n2 = n_inst * P2, n3 = n_inst * P3, n1 = n_inst * P1, n4 = n_inst * P4;
    s2.assign(10 * std::max<long long>(n2, 1), 0.0);
    c2.assign(5 * std::max<long long>(n3, 1), 0.0);
    s1.assign(5 * std::max<long long>(n1, 1), 0.0);
    c1.assign(6 * std::max<long long>(n4, 1), 0.0);
    kon.assign(std::max<long long>(n2, 1), 0);
    for (long long i = 0; i < n_inst; ++i) {
        int base = sd.geo_off;
        for (int j = 0; j < sd.n_s2; ++j) {
            const DevMat& m = mats[sp.m[base + j]];
            const long long idx = i * P2 + j;
            s2[2 * n2 + idx] = m.p[1];
            s2[4 * n2 + idx] = m.k[S2K_EPSY];
            s2[3 * n2 + idx] = -m.k[S2K_EPSY];
            if (m.p[10] != 0.0) {
                s2[idx] = m.k[S2K_SIGINI_E0];
                s2[n2 + idx] = m.p[10];
            }
        }
        base += sd.n_s2;
        for (int j = 0; j < sd.n_c2; ++j) c2[2 * n3 + i * P3 + j] = mats[sp.m[base + j]].k[C2K_EC0];
        base += sd.n_c2;
        for (int j = 0; j < sd.n_s1; ++j) s1[2 * n1 + i * P1 + j] = mats[sp.m[base + j]].p[1];
        base += sd.n_s1;
        for (int j = 0; j < sd.n_c1; ++j) {
            c1[2 * n4 + i * P4 + j] = mats[sp.m[base + j]].k[C1K_EC0];
            c1[5 * n4 + i * P4 + j] = mats[sp.m[base + j]].k[C1K_EC0];
        }
    }
}

// Persistent grid of the streaming kernel: as many CTAs per SM as the occupancy calculator
// allows with this section's two stages; 0 when they do not fit at all.
static int fs_configure(StrutSectionBatch* b) {
    int dev = 0, optin = 0, n_sm = 1;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
    b->L = fs_layout(b->sd);
    b->L.n_mats = b->n_mats;
    b->smem = fs_smem_bytes(b->L);
    b->n_tiles = (b->n_inst + kFsTile - 1) / kFsTile;
    b->grid = 0;
    if (b->smem + 1024 > (size_t)optin) return STRUT_OK;
    CK(cudaFuncSetAttribute(fiber_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem));
    int resident = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, fiber_stream_kernel, fs_threads(b->L), b->smem));
    if (resident < 1) return STRUT_OK;
    b->grid = (int)std::min<long long>(b->n_tiles, (long long)n_sm * resident);
    return STRUT_OK;
}

extern "C" {

int strut_gpu_section_batch_create(const StrutUniMaterial* materials, int32_t num_materials,
                                   const StrutFiber* fibers, int32_t num_fibers, int32_t n_inst,
                                   StrutSectionBatch** out) {
    if (!materials || !fibers || num_fibers <= 0 || n_inst <= 0 || !out) return fail(STRUT_BAD_ARG, "bad arguments");
    *out = nullptr;
    SectionPack sp;
    int rc = pack_section(materials, num_materials, fibers, 0, num_fibers, 0, 2, sp);
    if (rc != STRUT_OK) return rc;
    std::vector<DevMat> mats;
    for (int i = 0; i < num_materials; ++i) mats.push_back(make_devmat(materials[i]));
    StrutSectionBatch* b = new StrutSectionBatch();
    b->n_inst = n_inst;
    b->n_mats = num_materials;
    b->sd = sp.secs[0];
    DevMat* d_mats;
    DevSection* d_secs;
    double *d_y, *d_a;
    int* d_m;
    auto& al = b->allocs;
    if ((rc = upload(&d_mats, mats, al)) || (rc = upload(&d_secs, sp.secs, al)) || (rc = upload(&d_y, sp.y, al)) ||
        (rc = upload(&d_a, sp.a, al)) || (rc = upload(&d_m, sp.m, al))) {
        delete b;
        return rc;
    }
    b->geo.y = d_y;
    b->geo.a = d_a;
    b->geo.m = d_m;
    b->geo.mats = d_mats;
    b->geo.secs = d_secs;
    std::vector<double> s2, c2, s1, c1;
    std::vector<int> kon;
    if ((rc = fs_configure(b)) != STRUT_OK) {
        delete b;
        return rc;
    }
    const long long n_alloc = b->n_tiles * kFsTile;  // whole tiles: a tile's copies stay in bounds
    batch_initial_state(sp, mats, n_alloc, s2, c2, s1, c1, kon);
    if ((rc = upload(&b->bs.s2, s2, al)) || (rc = upload(&b->bs.c2, c2, al)) || (rc = upload(&b->bs.s1, s1, al)) ||
        (rc = upload(&b->bs.c1, c1, al)) || (rc = upload(&b->bs.kon, kon, al))) {
        delete b;
        return rc;
    }
    b->bs.n_inst = n_alloc;
    b->bs.p_s2 = b->L.p_s2;
    b->bs.p_c2 = b->L.p_c2;
    b->bs.p_s1 = b->L.p_s1;
    b->bs.p_c1 = b->L.p_c1;
    if ((rc = dzeros(&b->d_err, 1, al))) {
        delete b;
        return rc;
    }
    *out = b;
    return STRUT_OK;
}

int strut_gpu_section_batch_destroy(StrutSectionBatch* b) {
    if (!b) return STRUT_BAD_ARG;
    cudaDeviceSynchronize();
    delete b;
    return STRUT_OK;
}

int strut_gpu_section_eval_batch(StrutSectionBatch* b, const double* eps0_kappa_dev, double* resp_dev,
                                 int32_t commit, void* stream) {
    if (!b || !eps0_kappa_dev || !resp_dev) return fail(STRUT_BAD_ARG, "bad arguments");
    if (b->grid > 0) {
        fiber_stream_kernel<<<b->grid, fs_threads(b->L), b->smem, (cudaStream_t)stream>>>(
            b->geo, b->sd, b->bs, b->L, (long long)b->n_inst, b->n_tiles, eps0_kappa_dev, resp_dev, commit ? 1 : 0,
            b->d_err);
    } else {
        // a section whose stages do not fit in shared memory: one warp per instance
        const long long threads = (long long)b->n_inst * 32;
        const int tb = 256;
        section_batch_kernel<<<(unsigned)((threads + tb - 1) / tb), tb, 0, (cudaStream_t)stream>>>(
            b->geo, b->sd, b->bs, (long long)b->n_inst, eps0_kappa_dev, resp_dev, commit ? 1 : 0);
    }
    CK(cudaGetLastError());
    return STRUT_OK;
}

int strut_gpu_section_batch_state(StrutSectionBatch* b, int32_t instance, double* out, int32_t* n_fibers) {
    if (!b || instance < 0 || instance >= b->n_inst) return fail(STRUT_BAD_ARG, "bad arguments");
    const DevSection& sd = b->sd;
    const int nf = sd.n_s2 + sd.n_c2 + sd.n_s1 + sd.n_c1;
    if (n_fibers) *n_fibers = nf;
    if (!out) return STRUT_OK;
    CK(cudaDeviceSynchronize());
    {
        int err = 0;
        CK(cudaMemcpy(&err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (err) return fail(STRUT_CUDA_ERROR, "a bulk copy of the streaming fiber kernel did not complete");
    }
    // 16 doubles per fiber: the family's committed fields in declaration order, kon in slot 15
    std::vector<double> o((size_t)nf * 16, 0.0);
    const int P2 = b->bs.p_s2, P3 = b->bs.p_c2, P1 = b->bs.p_s1, P4 = b->bs.p_c1;
    const long long n2 = b->bs.n_inst * P2, n3 = b->bs.n_inst * P3, n1 = b->bs.n_inst * P1, n4 = b->bs.n_inst * P4;
    for (int j = 0; j < sd.n_s2; ++j) {
        for (int f = 0; f < 10; ++f)
            CK(cudaMemcpy(&o[(size_t)j * 16 + f], b->bs.s2 + f * n2 + (long long)instance * P2 + j, sizeof(double),
                          cudaMemcpyDeviceToHost));
        int kon = 0;
        CK(cudaMemcpy(&kon, b->bs.kon + (long long)instance * P2 + j, sizeof(int), cudaMemcpyDeviceToHost));
        o[(size_t)j * 16 + 15] = kon;
    }
    for (int j = 0; j < sd.n_c2; ++j)
        for (int f = 0; f < 5; ++f)
            CK(cudaMemcpy(&o[(size_t)(sd.n_s2 + j) * 16 + f], b->bs.c2 + f * n3 + (long long)instance * P3 + j,
                          sizeof(double), cudaMemcpyDeviceToHost));
    for (int j = 0; j < sd.n_s1; ++j)
        for (int f = 0; f < 5; ++f)
            CK(cudaMemcpy(&o[(size_t)(sd.n_s2 + sd.n_c2 + j) * 16 + f],
                          b->bs.s1 + f * n1 + (long long)instance * P1 + j, sizeof(double), cudaMemcpyDeviceToHost));
    for (int j = 0; j < sd.n_c1; ++j)
        for (int f = 0; f < 6; ++f)
            CK(cudaMemcpy(&o[(size_t)(sd.n_s2 + sd.n_c2 + sd.n_s1 + j) * 16 + f],
                          b->bs.c1 + f * n4 + (long long)instance * P4 + j, sizeof(double), cudaMemcpyDeviceToHost));
    std::memcpy(out, o.data(), o.size() * sizeof(double));
    return STRUT_OK;
}

int strut_gpu_section_path(const StrutUniMaterial* materials, int32_t num_materials, const StrutFiber* fibers,
                           int32_t num_fibers, const double* eps0_kappa, int32_t n_points, double* out) {
    if (n_points < 0 || (n_points > 0 && (!eps0_kappa || !out))) return fail(STRUT_BAD_ARG, "bad arguments");
    StrutSectionBatch* b = nullptr;
    int rc = strut_gpu_section_batch_create(materials, num_materials, fibers, num_fibers, 1, &b);
    if (rc != STRUT_OK) return rc;
    double *d_ek = nullptr, *d_r = nullptr;
    cudaError_t e = cudaMalloc((void**)&d_ek, 2 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc((void**)&d_r, 5 * sizeof(double));
    for (int p = 0; p < n_points && e == cudaSuccess && rc == STRUT_OK; ++p) {
        e = cudaMemcpy(d_ek, eps0_kappa + 2 * p, 2 * sizeof(double), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) break;
        rc = strut_gpu_section_eval_batch(b, d_ek, d_r, 1, nullptr);
        if (rc != STRUT_OK) break;
        e = cudaMemcpy(out + 5 * p, d_r, 5 * sizeof(double), cudaMemcpyDeviceToHost);
    }
    if (d_ek) cudaFree(d_ek);
    if (d_r) cudaFree(d_r);
    strut_gpu_section_batch_destroy(b);
    if (e != cudaSuccess) return fail(STRUT_CUDA_ERROR, cudaGetErrorString(e));
    return rc;
}

int strut_gpu_section3d_path(const StrutUniMaterial* materials, int32_t num_materials,
                             const StrutFiber* fibers, int32_t num_fibers, const double* path,
                             int32_t n_points, double* out) {
    if (!materials || !fibers || num_fibers <= 0 || n_points < 0 || (n_points > 0 && (!path || !out)))
        return fail(STRUT_BAD_ARG, "bad arguments");
    SectionPack sp;
    int rc = pack_section(materials, num_materials, fibers, 0, num_fibers, 0, 3, sp);
    if (rc != STRUT_OK) return rc;
    if (n_points == 0) return STRUT_OK;
    std::vector<DevMat> mats;
    for (int i = 0; i < num_materials; ++i) mats.push_back(make_devmat(materials[i]));
    std::vector<double> s2, c2, s1, c1;
    std::vector<int> kon;
    batch_initial_state(sp, mats, 1, s2, c2, s1, c1, kon);
    std::vector<void*> al;
    auto cleanup = [&]() {
        for (void* p : al) cudaFree(p);
    };
    DevMat* d_mats = nullptr;
    double *d_y = nullptr, *d_z = nullptr, *d_a = nullptr, *d_path = nullptr, *d_out = nullptr;
    int* d_m = nullptr;
    BatchState bs;
    std::memset(&bs, 0, sizeof(bs));
    std::vector<double> pv(path, path + 3 * (size_t)n_points);
    if ((rc = upload(&d_mats, mats, al)) || (rc = upload(&d_y, sp.y, al)) || (rc = upload(&d_z, sp.z, al)) ||
        (rc = upload(&d_a, sp.a, al)) || (rc = upload(&d_m, sp.m, al)) || (rc = upload(&bs.s2, s2, al)) ||
        (rc = upload(&bs.c2, c2, al)) || (rc = upload(&bs.s1, s1, al)) || (rc = upload(&bs.c1, c1, al)) ||
        (rc = upload(&bs.kon, kon, al)) ||
        (rc = upload(&d_path, pv, al)) || (rc = dzeros(&d_out, 9 * (size_t)n_points, al))) {
        cleanup();
        return rc;
    }
    bs.n_inst = 1;
    bs.p_s2 = fs_pad4(sp.secs[0].n_s2);
    bs.p_c2 = fs_pad4(sp.secs[0].n_c2);
    bs.p_s1 = fs_pad4(sp.secs[0].n_s1);
    bs.p_c1 = fs_pad4(sp.secs[0].n_c1);
    Geo g;
    std::memset(&g, 0, sizeof(g));
    g.y = d_y;
    g.z = d_z;
    g.a = d_a;
    g.m = d_m;
    g.mats = d_mats;
    section3d_path_kernel<<<1, 32>>>(g, sp.secs[0], bs, d_path, n_points, d_out);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(out, d_out, 9 * (size_t)n_points * sizeof(double), cudaMemcpyDeviceToHost);
    cleanup();
    if (e != cudaSuccess) return fail(STRUT_CUDA_ERROR, cudaGetErrorString(e));
    return STRUT_OK;
}

}  // extern "C"
#include "mlp_host.cuh"
#include "predictor_host.cuh"
#include "noalloc.cuh"

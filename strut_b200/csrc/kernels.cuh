// Device data layout and kernels of the batched transient hot path (sm_100a, FP64).
//
// HBM layout (all instances concatenated, instance-major):
//   fiber geometry   per section definition, families contiguous: Steel02 | Concrete02 |
//                    Steel01 | Concrete01 | Elastic; y (and z) relative to the area centroid,
//                    area, material index
//   fiber history    structure-of-arrays per family, committed state only.  Element e owns
//                    one block per family: [ip0 fibers | ip1 fibers | ...] padded to 4 entries,
//                    so every field block is a 32-byte aligned contiguous run that one
//                    cp.async.bulk moves into shared memory.
//   element state    128 doubles per element.  2D: q0..q2 | eps0[10] | kappa[10] | v0..v2 (the
//                    forceBeamColumn2d "force_basic_q" block of loader.mojo:1757-1771; for
//                    dispBeamColumn2d the section deformations of the last state
//                    determination), then the cached section responses at those
//                    deformations.  3D: q0..q4 | eps0[10] | kappa_y[10] | kappa_z[10]
//                    (forceBeamColumn3d's block, loader.mojo:1836-1840), then the cached
//                    responses (N, My, Mz and the six flexibility terms per point)
//   element output   k (nd x nd global) and f (nd) per element, nd = 6 (2D) or 12 (3D), at
//                    the element's own offsets
//   instance arrays  free-dof vectors, band Kinit, gather lists for band slots and F_int
//
// Trial fiber state is never written to HBM: a fiber's trial state is a pure function of its
// committed state and strain, so the commit kernel recomputes it from the section deformations
// stored in the element state and writes it over the committed state.
#pragma once

#include <cstdint>

#include "fiber_device.cuh"

namespace strut {

constexpr int kMaxIp = 10;
// Threads of an element CTA (element state determination; the commit kernel uses one team of
// 128 (up to 5 integration points) or 64 (up to 10) threads per integration point).
constexpr int kTeamThreads = 640;
constexpr int kEStride = 128;  // doubles of element state
constexpr int kEq = 0, kEe = 3, kEk = 13, kEv = 23;
// Section responses at the stored deformations (N, Mz and the 2x2 flexibility), valid flag.
// A forceBeamColumn state determination starts by re-evaluating every section at the stored
// deformations (force_beam_column2d.mojo:877-925); when nothing changed since the evaluation
// that produced them, those responses are these, bit for bit.
constexpr int kEcv = 26, kEcN = 27, kEcM = 37, kEc00 = 47, kEc01 = 57, kEc11 = 67;
// 3D element state: basic forces, section deformations, cache flag, cached resultants
// (N, My, Mz) and flexibilities (f11, f12, f13, f22, f23, f33) per point.
constexpr int kE3q = 0, kE3e = 5, kE3y = 15, kE3z = 25, kE3cv = 35, kE3cs = 36, kE3cf = 66;
static_assert(kE3cf + 6 * kMaxIp <= kEStride, "3D element state fits the stride");

struct DevSection {
    int n_s2, n_c2, n_s1, n_el;
    int geo_off;
    int el_uniform;
    int init_valid;
    int all_elastic;
    int dim, n_c1;
    double f00, f01, f11;
};

struct DevElem {
    int type, geom, nip, sec;
    int inst, rec;              // rec: recorder slot of this element in its instance or -1
    int nd, has_vecxz;          // element dofs (6 or 12); vecxz given (3D)
    int dof[12];                // absolute indices into the concatenated full u vector
    int s2_off, c2_off, s1_off; // block offsets into family arrays
    int s2_blk, c2_blk, s1_blk; // block lengths (multiples of 4)
    int c1_off, c1_blk;         // Concrete01 block
    long long ek_off, ef_off;   // offsets of this element's k (nd x nd) and f (nd)
    double L, inv_L, c, s, c_div, s_div, L_sync, c_sync, s_sync;
    double xi[kMaxIp], w[kMaxIp];
    // 3D: local axes (rows x, y, z) of the undeformed element, end coordinates and vecxz for
    // the Corotational axes, torsional G and J of the section
    double R[9], X1[3], X2[3], vxz[3], G, J;
    double io_bytes;            // algorithmic HBM bytes of one state determination
    double commit_bytes;        // algorithmic HBM bytes of one commit
};

// Algorithmic HBM bytes of one evaluation of a section's fibers: per fiber-state update its
// committed history read and its trial history written (Concrete02 5 + 5 doubles, Steel02 10 + 10
// doubles and kon, Steel01 eps_p and alpha read, five doubles written, Concrete01 6 + 6 doubles;
// elastic fibers have no history).
__host__ __device__ __forceinline__ unsigned long long section_update_bytes(const DevSection& sd) {
    return 80ull * sd.n_c2 + 168ull * sd.n_s2 + 56ull * sd.n_s1 + 96ull * sd.n_c1;
}

struct DevInst {
    int n, bw, rw, num_dofs;
    int u_off, f_off;
    long long band_off;
    long long slot_ptr_off;  // slot_ptr has n*rw + 1 entries per instance
    int fint_ptr_off;        // fint_ptr has n + 1 entries per instance
    int max_iters, test_type, spd, has_damping;
    int rec_off, n_rec, rece_off, n_rece;
    double a0, a1, a2, a3, dt, gamma, beta, coeff, tol;
    double alpha_m, beta_k, beta_k_init, beta_k_comm;
    double io_bytes;  // algorithmic HBM bytes of one Newton iteration of this instance
    long long dense_off;  // offset of this instance's n x n fallback scratch
    int elem_off, n_elem; // this instance's elements (contiguous)
    int large, large_idx; // band in global memory (too large for shared memory), its index
    long long lband_off;  // offset of its band in the global band buffer
    int lrw, pad_l;       // slots per row of that band (3 bw + 1)
    int algorithm, pad_al; // STRUT_ALGORITHM_* (Newton, ModifiedNewton, ModifiedNewtonInitial)
    int sl_off, n_sl;     // this instance's slave dofs (multi-point constraints)
    // solver chain (transient_nonlinear.mojo:758-830, 1925-1942): attempt k's algorithm, test,
    // iteration limit and tolerance; attempt 0 is (algorithm, test_type, max_iters, tol)
    int n_att, pad_att;
    int att_alg[4], att_test[4], att_maxit[4];
    double att_tol[4];
};

// The solver settings of an instance's current attempt.
struct Attempt {
    int alg, test, max_iters;
    double tol;
};

// Elements of the instances still iterating, rebuilt every Newton iteration and double
// buffered on the parity of DevCtl::iter: the predictor lists every element of the live
// instances into buffer 0, the instance kernel of iteration i lists the elements of an
// instance that has not converged into buffer (i + 1) & 1, and the element kernel of
// iteration i reads buffer i & 1 and clears the other one's count.  The order inside a list
// does not matter: elements are independent.
//
// Attempt fan-out.  forceBeamColumn2d tries an increment with three schemes at up to four
// subdivision levels, each attempt starting again from the element's accepted state
// (force_beam_column2d.mojo:1669-1763), so the twelve attempts of one pass are independent.  An
// element whose previous state determination needed more than the first level (hard_flag) is
// listed once more in `hard`, and the element kernel runs its twelve attempts on twelve CTAs at
// once: each writes its outcome to fan_rec, the last to finish takes the first success in the
// reference's order (level by level, scheme 0, 1, 2) and carries on from there as the sequential
// algorithm would, so the result is the sequential one bit for bit.  Its plain list entry carries
// kFanBit and is skipped.  At most kFanCap elements are fanned out per list.
//
// Later passes fan out too.  When the chosen attempt leaves part of the increment (an accepted
// subdivision), the sequential algorithm starts a new pass over the remainder from level 1; the
// resolving CTA saves the element's accepted state in the slot's round record, posts the next
// pass's twelve attempts to a queue that the persistent CTAs of the same launch take work from,
// and leaves the element; the pass's last attempt resolves it in turn.  CTAs whose next ticket lies
// beyond the posted items wait for one while any fanned element is unresolved.  A pass is fanned
// out only while the sequential loop's guard leaves room for all four levels; otherwise the
// resolving CTA goes on sequentially, so the result is the sequential one bit for bit.
constexpr int kFanAttempts = 12;  // 4 subdivision levels x 3 schemes
constexpr int kFanCap = 512;
constexpr int kFanRec = 88;       // doubles per attempt record
constexpr int kFanBit = 0x40000000;
constexpr int kFanRound = 96;     // doubles per round record (the state a pass starts from)
constexpr int kRoundQ = 8192;     // queue entries per list buffer (a ring)
constexpr int kQueuePolls = 1 << 26;  // bound on a queue wait (polls with a short sleep)
// round record fields
enum {
    kFRound = 0, kFGuard = 1, kFLocal = 2, kFEvals = 3, kFHard = 4, kFCValid = 5, kFBestOk = 6,
    kFAccV = 7, kFAccQ = 10, kFRem = 13, kFBest = 16, kFSvsE = 26, kFSvsK = 36, kFCN = 46, kFCM = 56,
    kFC00 = 66, kFC01 = 76, kFC11 = 86
};

struct ElemList {
    int* list[2];
    int* count;  // 2 entries
    int* next;   // 2 entries: work counter of the persistent element kernel
    int* hard[2];       // elements fanned out in this list (kFanCap entries each)
    int* hard_count;    // 2 entries (may exceed kFanCap; only the first kFanCap are fanned out)
    int* hard_flag;     // per element: its last state determination needed a subdivision
    int* fan_done;      // 2 x kFanCap: attempts finished per slot, zeroed when the slot is
                        // handed out; every launch over the list adds kFanAttempts, so the
                        // last attempt of a launch is the one that finds count % 12 == 11
    double* fan_rec;    // 2 x kFanCap x kFanAttempts x kFanRec attempt records
    int* fan_first;     // 2 x kFanCap: the earliest attempt that has succeeded (kFanAttempts:
                        // none yet); a later attempt stops as soon as it sees an earlier success
    double* fan_round;  // 2 x kFanCap x kFanRound: the state each slot's current pass starts from
    long long* rq;      // 2 x kRoundQ: posted attempts, (ticket << 16) | (slot x 12 + attempt);
                        // -1 when free (the taker frees it)
    int* rq_tail;       // 2 entries: queue tickets handed to posted attempts
    int* fan_finished;  // 2 entries: fanned elements of the list that are resolved
    int* q_err;         // a queue wait that ran out
};

// List entry of element e in list buffer `buf`: a flagged element also gets a fan slot.
__device__ __forceinline__ int list_entry(const ElemList& el, int buf, int e) {
    if (el.hard_flag && el.hard_flag[e]) {
        const int slot = atomicAdd(&el.hard_count[buf], 1);
        if (slot < kFanCap) {
            el.hard[buf][slot] = e;
            el.fan_done[buf * kFanCap + slot] = 0;
            el.fan_first[buf * kFanCap + slot] = kFanAttempts;
            if (el.fan_round) el.fan_round[(size_t)(buf * kFanCap + slot) * kFanRound + kFRound] = 1.0;
            return e | kFanBit;
        }
    }
    return e;
}

// Step / iteration control on the device (read by the kernels, advanced by step_end_kernel).
struct DevCtl {
    int step;       // absolute index of the step being computed
    int step0;      // first step of the current run (ground-motion table row 0)
    int n_end;      // run stops before this step
    int iter;       // Newton iteration of the current step
    int max_iters;  // max over instances
    int single;     // single-instance handle: stop at the failing step
    int fan;        // attempt fan-out enabled (StrutTuning.fan_out)
    int pad1;
};

struct FiberState {
    // family arrays: field f of family X lives at X + f * X_n
    double* c2;
    long long c2_n;
    double* s2;
    int* s2_kon;
    long long s2_n;
    double* s1;
    long long s1_n;
    double* c1;  // Concrete01: eps, sig, tan, min strain, end strain, unloading slope
    long long c1_n;
};

struct Geo {
    const double* y;
    const double* z;  // 3D sections (0 for 2D sections)
    const double* a;
    const int* m;
    const DevMat* mats;
    const DevSection* secs;
};

}  // namespace strut

// Fused element state determination for forceBeamColumn2d / dispBeamColumn2d on sm_100a.
//
// One CTA per element (a persistent grid claiming elements from a list).  The element's
// committed fiber history (all of its sections, all families) is staged into shared memory with
// cp.async.bulk (the TMA unit's bulk copy) completing on an mbarrier, and the constants each
// fiber's trial rule derives from its committed state are computed once per launch.  Every
// section evaluation of the element-level flexibility iteration then reads shared memory only,
// in two phases: the trial stress and tangent of every fiber of every integration point (one
// fiber per thread, Steel02 fibers on one warp per SM sub-partition), then the section sums in a
// fixed chunked order.  Warp 0 runs the element algebra with one lane per integration point
// (section flexibilities, 3x3 inverse, work-norm test); thread 0 runs the subdivision and scheme
// fallbacks.  The per-iteration latency of one element is what bounds a batch whose slowest
// record keeps failing its local iteration, so the work between barriers is kept short.
//
// Algorithm (paths relative to the Strut project root):
//   src/mojo/elements/force_beam_column2d.mojo:223-272 (3x3 inverse), 608-801 (exact elastic,
//   initial basic tangent), 804-1189 (_force_beam_column2d_try_increment), 1418-1920 (entry:
//   schemes x subdivisions, basic -> local -> global); src/mojo/sections/fiber2d.mojo:3042-3086
//   (section flexibility); src/mojo/elements/disp_beam_column2d.mojo:114-254.
#pragma once

#include "kernels.cuh"

namespace strut {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// cp.async.bulk global -> shared, completing transaction bytes on the mbarrier.
// dst/src 16-byte aligned, bytes a multiple of 16.  No multicast.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, "
        "1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// Bounded wait: gives up after a fixed number of polls (each try_wait itself suspends for a
// hardware time slice), reports it, and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase) {
    for (int i = 0; i < (1 << 20); ++i)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

enum { ELEM_ERR_NONE = 0, ELEM_ERR_TMA_TIMEOUT = 1, ELEM_ERR_FAILED = 2 };

// Section teams: each integration point of an element is evaluated by a team of TEAM threads
// (64 or 128).  The team's section sums follow one canonical order whatever TEAM is: fiber j of a
// family (family-local index) is accumulated by virtual lane j % 128 in increasing j, each block of
// 32 virtual lanes is summed by a shuffle butterfly, and the four block sums are added in block
// order.  A record's result therefore never depends on the launch shape of the batch it is in.
constexpr int kVLanes = 128;
constexpr int kVBlocks = kVLanes / 32;

// element-level scratch in shared memory
struct ElemScratch {
    double q[3], acc_q[3], acc_v[3], v[3], rem[3], att[3], tv[3], zero3[3];
    double svs_e[kMaxIp], svs_k[kMaxIp];  // accepted section deformations
    double vs_e[kMaxIp], vs_k[kMaxIp];    // element state section deformations
    double pt_e[kMaxIp], pt_k[kMaxIp];    // points to evaluate
    double resp[kMaxIp][5];
    double raw[kMaxIp][6];                // section sums of the last evaluation
    double scr[kMaxIp][12];               // per-point terms of the element algebra (lanes < nip of warp 0)
    double sub_e[kMaxIp], sub_k[kMaxIp], ssr_n[kMaxIp], ssr_m[kMaxIp];
    double fs00[kMaxIp], fs01[kMaxIp], fs11[kMaxIp];
    double best[10];
    double c_n[kMaxIp], c_m[kMaxIp], c_f00[kMaxIp], c_f01[kMaxIp], c_f11[kMaxIp];
    double ul[6];
    double k[36];
    double f[6];
    int best_ok;
    int c_valid;
    int flag;
    int sing;  // some section of the last evaluation had a singular tangent
    int loop_ctrl;
    int local_iters;
    int section_evals;
    int hard;  // this determination needed a subdivided increment (fan out next time)
};

// Family views of the element's committed history (shared memory, or global memory with the
// family length as field stride).
struct StageView {
    const double* c2;   // staged: 4 fields x c2_blk (eps sig tan ecmin; dept only enters the
                        // derived constants, which read it from a separate buffer)
    const double* s2;   // 10 fields x s2_blk
    const int* kon;     // s2_blk
    const double* s1;   // 5 fields x s1_blk
    const double* c1;   // 6 fields x c1_blk
    const double* c2d;  // C2Derived, 5 fields x c2_blk (shared-memory views only)
    const double* s2d;  // S2Derived, 12 fields x s2_blk (shared-memory views only)
    int c2_blk, s2_blk, s1_blk, c1_blk;
};

__device__ __forceinline__ void load_c1(const StageView& sv, int idx, C1State& c) {
    const int B = sv.c1_blk;
    c.eps = sv.c1[0 * B + idx];
    c.sig = sv.c1[1 * B + idx];
    c.tan = sv.c1[2 * B + idx];
    c.emin = sv.c1[3 * B + idx];
    c.eend = sv.c1[4 * B + idx];
    c.slope = sv.c1[5 * B + idx];
}

// The staged Concrete02 fields; dept is not staged (set to 0 here: the stress and tangent given
// the derived constants do not use it).
__device__ __forceinline__ void load_c2(const StageView& sv, int idx, C2State& c) {
    const int B = sv.c2_blk;
    c.eps = sv.c2[0 * B + idx];
    c.sig = sv.c2[1 * B + idx];
    c.tan = sv.c2[2 * B + idx];
    c.ecmin = sv.c2[3 * B + idx];
    c.dept = 0.0;
}

__device__ __forceinline__ void load_s2(const StageView& sv, int idx, S2State& c) {
    const int B = sv.s2_blk;
    c.eps = sv.s2[0 * B + idx];
    c.sig = sv.s2[1 * B + idx];
    c.tan = sv.s2[2 * B + idx];
    c.epsmin = sv.s2[3 * B + idx];
    c.epsmax = sv.s2[4 * B + idx];
    c.epspl = sv.s2[5 * B + idx];
    c.epss0 = sv.s2[6 * B + idx];
    c.sigs0 = sv.s2[7 * B + idx];
    c.epsr = sv.s2[8 * B + idx];
    c.sigr = sv.s2[9 * B + idx];
    c.kon = sv.kon[idx];
}

// Derived constants of every Concrete02 / Steel02 fiber of the staged element, computed once
// per launch by the whole CTA (the committed state does not change inside a launch).  A
// Concrete02 fiber's dept comes from c2_dept: the element's dept field, in global memory or
// copied into shared memory beside the staged history.  The two
// branch curves of a Steel02 fiber (each with its own pow) are two work items, given to the last
// threads of the CTA, so they run beside the Concrete02 items instead of after them.
__device__ __forceinline__ void derive_c2(const Geo& g, const DevSection& sd, const StageView& sv,
                                          const double* __restrict__ c2_dept, double* c2d, int idx) {
    C2State c;
    load_c2(sv, idx, c);
    c.dept = c2_dept[idx];
    const int j = idx % sd.n_c2;
    C2Derived d;
    concrete02_derive(g.mats[__ldg(g.m + sd.geo_off + sd.n_s2 + j)], c, d);
    const int B = sv.c2_blk;
    c2d[0 * B + idx] = d.sigmm;
    c2d[1 * B + idx] = d.er;
    c2d[2 * B + idx] = d.ept;
    c2d[3 * B + idx] = d.epn;
    c2d[4 * B + idx] = d.etn;
}

// Branch curve k (0: strain increasing, 1: decreasing) of Steel02 fiber idx (steel02_derive).
__device__ __forceinline__ void derive_s2(const Geo& g, const DevSection& sd, const StageView& sv, double* s2d,
                                          int idx, int k) {
    S2State c;
    load_s2(sv, idx, c);
    const int j = idx % sd.n_s2;
    const DevMat& m = g.mats[__ldg(g.m + sd.geo_off + j)];
    S2State t;
    steel02_branch(m, c, k == 0, t);
    S2Curve cv;
    steel02_curve_of(m, t, cv);
    const int B = sv.s2_blk;
    s2d[(6 * k + 0) * B + idx] = cv.epsr;
    s2d[(6 * k + 1) * B + idx] = cv.sigr;
    s2d[(6 * k + 2) * B + idx] = cv.denom;
    s2d[(6 * k + 3) * B + idx] = cv.dsig;
    s2d[(6 * k + 4) * B + idx] = cv.R;
    s2d[(6 * k + 5) * B + idx] = cv.invR;
}

__device__ __forceinline__ void derive_element(const Geo& g, const DevSection& sd, const DevElem& E,
                                               const StageView& sv, const double* __restrict__ c2_dept,
                                               double* c2d, double* s2d) {
    const int nc = E.nip * sd.n_c2, ns2 = 2 * E.nip * sd.n_s2;
    const int nt = blockDim.x, tid = threadIdx.x;
    if (ns2 > 0 && ns2 <= nt / 2) {
        // Concrete02 on the first nt - ns2 threads, one Steel02 branch on each of the others
        const int split = nt - ns2;
        if (tid < split) {
            for (int idx = tid; idx < nc; idx += split) derive_c2(g, sd, sv, c2_dept, c2d, idx);
        } else {
            const int q = tid - split;
            derive_s2(g, sd, sv, s2d, q >> 1, q & 1);
        }
        return;
    }
    for (int idx = tid; idx < nc; idx += nt) derive_c2(g, sd, sv, c2_dept, c2d, idx);
    for (int q = tid; q < ns2; q += nt) derive_s2(g, sd, sv, s2d, q >> 1, q & 1);
}

__device__ __forceinline__ void acc_fiber(double* a, double fs, double ks, double y) {
    a[0] += fs;
    a[1] += -fs * y;
    a[2] += ks;
    a[3] += -ks * y;
    a[4] += ks * y * y;
}

// Team evaluation of section `ip` of an element at (eps0, kappa); r is the thread's rank in
// the team.  Writes the team's per-block partial sums (N, Mz, k11, k12, k22, elastic k12) to
// part[kVBlocks][6]; the caller adds them in block order after a barrier.
template <int TEAM>
__device__ __forceinline__ void section_eval_team(const Geo& g, const DevSection& sd,
                                                  const StageView& sv, int ip, double eps0,
                                                  double kappa, int r, double (*part)[6]) {
    constexpr int NS = kVLanes / TEAM;  // virtual lanes per thread
    double acc[NS][6];
#pragma unroll
    for (int s = 0; s < NS; ++s)
#pragma unroll
        for (int c = 0; c < 6; ++c) acc[s][c] = 0.0;
    int base = sd.geo_off;
    for (int j0 = 0; j0 < sd.n_s2; j0 += kVLanes) {
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const int j = j0 + s * TEAM + r;
            if (j >= sd.n_s2) continue;
            const int idx = ip * sd.n_s2 + j;
            const int B = sv.s2_blk;
            S2State c;
            c.eps = sv.s2[0 * B + idx];
            c.sig = sv.s2[1 * B + idx];
            c.tan = sv.s2[2 * B + idx];
            c.epsmin = sv.s2[3 * B + idx];
            c.epsmax = sv.s2[4 * B + idx];
            c.epspl = sv.s2[5 * B + idx];
            c.epss0 = sv.s2[6 * B + idx];
            c.sigs0 = sv.s2[7 * B + idx];
            c.epsr = sv.s2[8 * B + idx];
            c.sigr = sv.s2[9 * B + idx];
            c.kon = sv.kon[idx];
            const double y = __ldg(g.y + base + j), A = __ldg(g.a + base + j);
            S2State t;
            steel02_trial(g.mats[__ldg(g.m + base + j)], c, eps0 - y * kappa, t);
            acc_fiber(acc[s], t.sig * A, t.tan * A, y);
        }
    }
    base += sd.n_s2;
    for (int j0 = 0; j0 < sd.n_c2; j0 += kVLanes) {
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const int j = j0 + s * TEAM + r;
            if (j >= sd.n_c2) continue;
            const int idx = ip * sd.n_c2 + j;
            const int B = sv.c2_blk;
            C2State c;
            c.eps = sv.c2[0 * B + idx];
            c.sig = sv.c2[1 * B + idx];
            c.tan = sv.c2[2 * B + idx];
            c.ecmin = sv.c2[3 * B + idx];
            c.dept = sv.c2[4 * B + idx];
            const double y = __ldg(g.y + base + j), A = __ldg(g.a + base + j);
            C2State t;
            concrete02_trial(g.mats[__ldg(g.m + base + j)], c, eps0 - y * kappa, t);
            acc_fiber(acc[s], t.sig * A, t.tan * A, y);
        }
    }
    base += sd.n_c2;
    for (int j0 = 0; j0 < sd.n_s1; j0 += kVLanes) {
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const int j = j0 + s * TEAM + r;
            if (j >= sd.n_s1) continue;
            const int idx = ip * sd.n_s1 + j;
            const int B = sv.s1_blk;
            S1State c;
            c.eps = sv.s1[0 * B + idx];
            c.sig = sv.s1[1 * B + idx];
            c.tan = sv.s1[2 * B + idx];
            c.epsp = sv.s1[3 * B + idx];
            c.alpha = sv.s1[4 * B + idx];
            const double y = __ldg(g.y + base + j), A = __ldg(g.a + base + j);
            S1State t;
            steel01_trial(g.mats[__ldg(g.m + base + j)], c, eps0 - y * kappa, t);
            acc_fiber(acc[s], t.sig * A, t.tan * A, y);
        }
    }
    base += sd.n_s1;
    for (int j0 = 0; j0 < sd.n_c1; j0 += kVLanes) {
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const int j = j0 + s * TEAM + r;
            if (j >= sd.n_c1) continue;
            C1State c, t;
            load_c1(sv, ip * sd.n_c1 + j, c);
            const double y = __ldg(g.y + base + j), A = __ldg(g.a + base + j);
            concrete01_trial(g.mats[__ldg(g.m + base + j)], c, eps0 - y * kappa, t);
            acc_fiber(acc[s], t.sig * A, t.tan * A, y);
        }
    }
    base += sd.n_c1;
    for (int j0 = 0; j0 < sd.n_el; j0 += kVLanes) {
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const int j = j0 + s * TEAM + r;
            if (j >= sd.n_el) continue;
            const double y = __ldg(g.y + base + j), A = __ldg(g.a + base + j);
            const double E = g.mats[__ldg(g.m + base + j)].p[0];
            const double ks = E * A;
            const double fs = ks * (eps0 - y * kappa);
            acc[s][0] += fs;
            acc[s][1] += -fs * y;
            acc[s][2] += ks;
            acc[s][5] += -ks * y;
            acc[s][4] += ks * y * y;
        }
    }
    const int lane = r & 31, w = r >> 5;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        double v[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) v[c] = warp_sum(acc[s][c]);
        if (lane == 0) {
#pragma unroll
            for (int c = 0; c < 6; ++c) part[s * (TEAM / 32) + w][c] = v[c];
        }
    }
}

// Section resultants and tangent from the block partial sums, in block order.
// fiber2d.mojo:3491-3499: a section whose elastic fibers share one modulus reports no
// elastic k12 contribution.
__device__ __forceinline__ void section_finish(const DevSection& sd, const double (*part)[6],
                                               double* out) {
    double v[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        double t = part[0][c];
#pragma unroll
        for (int b = 1; b < kVBlocks; ++b) t += part[b][c];
        v[c] = t;
    }
    out[0] = v[0];
    out[1] = v[1];
    out[2] = v[2];
    out[3] = v[3] + (sd.el_uniform ? 0.0 : v[5]);
    out[4] = v[4];
}

__device__ __forceinline__ bool invert3(const double* F, double* k) {
    const double a = F[0], b = F[1], c = F[2], d = F[3], e = F[4], f = F[5], g = F[6],
                 h = F[7], i = F[8];
    const double co00 = e * i - f * h;
    const double co01 = -(d * i - f * g);
    const double co02 = d * h - e * g;
    const double co10 = -(b * i - c * h);
    const double co11 = a * i - c * g;
    const double co12 = -(a * h - b * g);
    const double co20 = b * f - c * e;
    const double co21 = -(a * f - c * d);
    const double co22 = a * e - b * d;
    const double det = a * co00 + b * co01 + c * co02;
    if (fabs(det) <= 1.0e-40) return false;
    const double inv_det = 1.0 / det;
    k[0] = co00 * inv_det;
    k[1] = co10 * inv_det;
    k[2] = co20 * inv_det;
    k[3] = co01 * inv_det;
    k[4] = co11 * inv_det;
    k[5] = co21 * inv_det;
    k[6] = co02 * inv_det;
    k[7] = co12 * inv_det;
    k[8] = co22 * inv_det;
    return true;
}

__device__ __forceinline__ void flex_accum(double* F, double wL, double bmi, double bmj,
                                           double f00, double f01, double f11) {
    const double f10 = f01;
    F[0] += wL * f00;
    F[1] += wL * f01 * bmi;
    F[2] += wL * f01 * bmj;
    F[3] += wL * bmi * f10;
    F[4] += wL * bmi * f11 * bmi;
    F[5] += wL * bmi * f11 * bmj;
    F[6] += wL * bmj * f10;
    F[7] += wL * bmj * f11 * bmi;
    F[8] += wL * bmj * f11 * bmj;
}

// ---- two-phase evaluation of all integration points of an element ----------------------
//
// Phase 1 computes the trial stress and tangent (times area) of every fiber of every point at
// S.pt into fo[(ip * n_tot + g) * 2 + {0, 1}] (g: the fiber's index in the section, families in
// order Steel02 | Concrete02 | Steel01 | Elastic).  Steel02 fibers (two pow calls each) go to
// the first warps (32 consecutive fibers per warp), the other families to the remaining warps,
// again 32 consecutive fibers per warp so that the staged arrays are read without bank
// conflicts and no warp mixes the two code paths.
//
// Phase 2 forms the section sums in a fixed order: every value of point ip is summed over eight
// contiguous chunks of the section's fibers, each chunk sequentially by one thread (which
// carries all six sums of its chunk), and the eight chunk sums are added by a fixed pairwise tree.  The order does not depend on the launch shape, so a
// record's result never depends on the batch it runs in.  Raw sums: N, Mz, k11, k12 of the
// non-elastic fibers, k22, k12 of the elastic fibers (fiber2d.mojo:1338-1351, 3459-3501).

__device__ __forceinline__ int steel_warps(int n_items, int n_warps) {
    if (n_items <= 0) return 0;
    int ws = (n_items + 31) / 32;
    if (ws > n_warps / 2) ws = n_warps / 2;
    return ws < 1 ? 1 : ws;
}

__device__ __forceinline__ void fiber_phase(const Geo& g, const DevSection& sd,
                                            const StageView& sv, const DevElem& E,
                                            const double* pe, const double* pk, double* fo) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int nip = E.nip;
    const int n_tot = sd.n_s2 + sd.n_c2 + sd.n_s1 + sd.n_c1 + sd.n_el;
    const int n_s = nip * sd.n_s2;
    const int ws = steel_warps(n_s, nw);
    if (w < ws) {
        for (int i = w * 32 + lane; i < n_s; i += ws * 32) {
            const int ip = i / sd.n_s2, j = i - ip * sd.n_s2;
            const int idx = ip * sd.n_s2 + j;
            S2State c;
            load_s2(sv, idx, c);
            const double y = __ldg(g.y + sd.geo_off + j), A = __ldg(g.a + sd.geo_off + j);
            const DevMat& mat = g.mats[__ldg(g.m + sd.geo_off + j)];
            const double eps = steel02_strain(mat, pe[ip] - y * pk[ip]);
            const double deps = eps - c.eps;
            double sig, tan;
            if (steel02_no_change(c, deps)) {
                tan = mat.p[1];
                sig = mat.p[10];
            } else {
                const int B = sv.s2_blk, k = steel02_up(c, deps) ? 0 : 6;
                S2Curve cv;
                cv.epsr = sv.s2d[(k + 0) * B + idx];
                cv.sigr = sv.s2d[(k + 1) * B + idx];
                cv.denom = sv.s2d[(k + 2) * B + idx];
                cv.dsig = sv.s2d[(k + 3) * B + idx];
                cv.R = sv.s2d[(k + 4) * B + idx];
                cv.invR = sv.s2d[(k + 5) * B + idx];
                steel02_curve_eval(mat, cv, eps, sig, tan);
            }
            double* o = fo + 2 * (ip * n_tot + j);
            o[0] = sig * A;
            o[1] = tan * A;
        }
        return;
    }
    const int n_o_sec = sd.n_c2 + sd.n_s1 + sd.n_c1 + sd.n_el;
    const int n_o = nip * n_o_sec;
    const int nwo = nw - ws;
    for (int k = (w - ws) * 32 + lane; k < n_o; k += nwo * 32) {
        const int ip = k / n_o_sec, jj = k - ip * n_o_sec;
        const double e0 = pe[ip], ka = pk[ip];
        const int gi = sd.n_s2 + jj;  // index in the section
        const double y = __ldg(g.y + sd.geo_off + gi), A = __ldg(g.a + sd.geo_off + gi);
        const DevMat& mat = g.mats[__ldg(g.m + sd.geo_off + gi)];
        double* o = fo + 2 * (ip * n_tot + gi);
        if (jj < sd.n_c2) {
            const int idx = ip * sd.n_c2 + jj;
            C2State c;
            load_c2(sv, idx, c);
            const int B = sv.c2_blk;
            C2Derived d;
            d.sigmm = sv.c2d[0 * B + idx];
            d.er = sv.c2d[1 * B + idx];
            d.ept = sv.c2d[2 * B + idx];
            d.epn = sv.c2d[3 * B + idx];
            d.etn = sv.c2d[4 * B + idx];
            double sig, tan;
            concrete02_sig_tan(mat, c, d, e0 - y * ka, sig, tan);
            o[0] = sig * A;
            o[1] = tan * A;
        } else if (jj < sd.n_c2 + sd.n_s1) {
            const int idx = ip * sd.n_s1 + (jj - sd.n_c2);
            const int B = sv.s1_blk;
            S1State c;
            c.eps = sv.s1[0 * B + idx];
            c.sig = sv.s1[1 * B + idx];
            c.tan = sv.s1[2 * B + idx];
            c.epsp = sv.s1[3 * B + idx];
            c.alpha = sv.s1[4 * B + idx];
            S1State t;
            steel01_trial(mat, c, e0 - y * ka, t);
            o[0] = t.sig * A;
            o[1] = t.tan * A;
        } else if (jj < sd.n_c2 + sd.n_s1 + sd.n_c1) {
            C1State c, t;
            load_c1(sv, ip * sd.n_c1 + (jj - sd.n_c2 - sd.n_s1), c);
            concrete01_trial(mat, c, e0 - y * ka, t);
            o[0] = t.sig * A;
            o[1] = t.tan * A;
        } else {
            // elastic: ks = E A, fs = ks (eps0 - y kappa)
            const double ks = mat.p[0] * A;
            o[0] = ks * (e0 - y * ka);
            o[1] = ks;
        }
    }
}

// Phase 2: thread t < nip * 8 sums chunk t % 8 of point t / 8 (the elastic fibers, last in the
// section, in a loop of their own); the eight chunk threads of a point are consecutive lanes and
// combine their sums by a fixed pairwise tree ((c0 + c1) + (c2 + c3)) + ((c4 + c5) + (c6 + c7)).
__device__ __forceinline__ void sum_phase(const DevSection& sd, int nip, const double* ys,
                                          const double* fo, double (*raw)[6]) {
    const int t = threadIdx.x;
    const int n_sum = nip * 8;
    if ((t & ~31) >= n_sum) return;  // whole warp outside
    const int n_tot = sd.n_s2 + sd.n_c2 + sd.n_s1 + sd.n_c1 + sd.n_el;
    const int n_nl = n_tot - sd.n_el;
    const bool act = t < n_sum;
    const int ip = t >> 3, b = t & 7;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, a4 = 0.0, a5 = 0.0;
    if (act) {
        const int cs = (n_tot + 7) >> 3;
        const int g0 = b * cs, g1 = min(g0 + cs, n_tot);
        const double* f = fo + 2 * ip * n_tot;
        const int gm = min(g1, n_nl);
#pragma unroll 4
        for (int gg = g0; gg < gm; ++gg) {
            const double fs = f[2 * gg], ks = f[2 * gg + 1], y = ys[gg];
            a0 += fs;
            a1 += -fs * y;
            a2 += ks;
            a3 += -ks * y;
            a4 += ks * y * y;
        }
        for (int gg = max(g0, n_nl); gg < g1; ++gg) {
            const double fs = f[2 * gg], ks = f[2 * gg + 1], y = ys[gg];
            a0 += fs;
            a1 += -fs * y;
            a2 += ks;
            a5 += -ks * y;
            a4 += ks * y * y;
        }
    }
    double a[6] = {a0, a1, a2, a3, a4, a5};
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        double p = a[c];
        p += __shfl_down_sync(0xffffffffu, p, 1);  // (c0+c1), (c2+c3), ...
        p += __shfl_down_sync(0xffffffffu, p, 2);  // ((c0+c1)+(c2+c3)), ...
        p += __shfl_down_sync(0xffffffffu, p, 4);
        if (act && b == 0) raw[ip][c] = p;
    }
}

// Both phases for every point of the element at S.pt; S.raw holds the sums afterwards.
__device__ __forceinline__ void eval_sections(const Geo& g, const DevSection& sd, const StageView& sv,
                                              const DevElem& E, ElemScratch& S, const double* ys,
                                              double* fo) {
    fiber_phase(g, sd, sv, E, S.pt_e, S.pt_k, fo);
    __syncthreads();
    sum_phase(sd, E.nip, ys, fo, S.raw);
    if (threadIdx.x == 0) S.section_evals += E.nip;
    __syncthreads();
}

// Resultants and tangent of a point from its raw sums (uniform-modulus elastic k12 quirk of
// fiber2d.mojo:3491-3499).
__device__ __forceinline__ void raw_resp(const DevSection& sd, const double* raw, double& N,
                                         double& M, double& k11, double& k12, double& k22) {
    N = raw[0];
    M = raw[1];
    k11 = raw[2];
    k12 = raw[3] + (sd.el_uniform ? 0.0 : raw[5]);
    k22 = raw[4];
}

// Section flexibility (fiber_section2d_batch_eval_same_def): false if |det| <= 1e-40.
__device__ __forceinline__ bool sec_flex(double k11, double k12, double k22, double& f00,
                                         double& f01, double& f11) {
    const double det = k11 * k22 - k12 * k12;
    if (fabs(det) <= 1.0e-40) return false;
    const double inv_det = 1.0 / det;
    f00 = k22 * inv_det;
    f01 = -k12 * inv_det;
    f11 = k11 * inv_det;
    return true;
}

// Sums, over the lanes 0..nip-1 of warp 0 in lane order, the NV values each lane put in
// scr[lane][0..NV-1]; every lane gets the same sums.  Warp 0 only.
template <int NV>
__device__ __forceinline__ void lane_ordered_sums(double (*scr)[12], int nip, double* out) {
    __syncwarp();
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v] = 0.0;
    for (int ip = 0; ip < nip; ++ip) {
#pragma unroll
        for (int v = 0; v < NV; ++v) out[v] += scr[ip][v];
    }
    __syncwarp();
}

// Flexibility integration terms of one point (flex_accum's nine products); lane = point.
__device__ __forceinline__ void flex_terms(double* o, double wL, double bmi, double bmj, double f00,
                                           double f01, double f11) {
    const double f10 = f01;
    o[0] = wL * f00;
    o[1] = wL * f01 * bmi;
    o[2] = wL * f01 * bmj;
    o[3] = wL * bmi * f10;
    o[4] = wL * bmi * f11 * bmi;
    o[5] = wL * bmi * f11 * bmj;
    o[6] = wL * bmj * f10;
    o[7] = wL * bmj * f11 * bmi;
    o[8] = wL * bmj * f11 * bmj;
}

// _force_beam_column2d_try_increment (force_beam_column2d.mojo:804-1189), executed
// collectively: every thread evaluates fibers, warp 0 runs the element algebra with one lane per
// integration point.  Starting state: S.q, S.vs_*; on success S.q / S.vs_* hold the converged
// state, S.best the result, and the section-response cache is refreshed.  Compiled once (not
// inlined): an attempt run by the sequential loop and the same attempt run by a fanned-out CTA
// execute the same instructions, so their floating-point results are the same bit for bit.
// stop / my: a fanned-out attempt (my = its index) gives up as soon as *stop, the earliest
// successful attempt of its element, is below it; null in the sequential order.
__device__ __noinline__ bool fbc_try_increment(const Geo& g, const DevSection& sd, const StageView& sv,
                                  const DevElem& E, ElemScratch& S, const double* base,
                                  const double* dv, int scheme, const double* ys, double* fo,
                                  const int* stop, int my) {
    const int tid = threadIdx.x, lane = tid & 31;
    const bool w0 = tid < 32;
    const int nip = E.nip;
    const bool act = w0 && lane < nip;
    if (!sd.init_valid) return false;
    const double xi = act ? E.xi[lane] : 0.0, wL = act ? E.w[lane] * E.L : 0.0;
    const double bmi = xi - 1.0, bmj = xi;
    // per-point state, held by lane ip of warp 0
    double sub_e = 0.0, sub_k = 0.0, ssr_n = 0.0, ssr_m = 0.0, f00 = 0.0, f01 = 0.0, f11 = 0.0;
    double pe = 0.0, pk = 0.0;
    double q0 = 0.0, q1 = 0.0, q2 = 0.0;
    const int num_iters = scheme == 1 ? 100 : 10;
    const bool cached = S.c_valid != 0;
    if (w0) {
        q0 = S.q[0];
        q1 = S.q[1];
        q2 = S.q[2];
        if (act) {
            sub_e = S.vs_e[lane];
            sub_k = S.vs_k[lane];
            if (!cached) {
                S.pt_e[lane] = sub_e;
                S.pt_k[lane] = sub_k;
            }
        }
    }
    if (!cached) {
        __syncthreads();
        eval_sections(g, sd, sv, E, S, ys, fo);
    }
    // the next points: s(q) - s_r through the section flexibility (initial flexibility for
    // scheme 1 and for the first iteration of scheme 2)
    auto next_points = [&](bool use_init) {
        const double ss0 = q0 + 0.0;
        const double ss1 = bmi * q1 + bmj * q2 + 0.0;
        const double dss0 = ss0 - ssr_n;
        const double dss1 = ss1 - ssr_m;
        const double a00 = use_init ? sd.f00 : f00;
        const double a01 = use_init ? sd.f01 : f01;
        const double a11 = use_init ? sd.f11 : f11;
        pe = sub_e + (a00 * dss0 + a01 * dss1);
        pk = sub_k + (a01 * dss0 + a11 * dss1);
        if (act) {
            S.pt_e[lane] = pe;
            S.pt_k[lane] = pk;
        }
    };
    if (w0) {
        int ok = 1;
        if (cached) {
            if (act) {
                ssr_n = S.c_n[lane];
                ssr_m = S.c_m[lane];
                f00 = S.c_f00[lane];
                f01 = S.c_f01[lane];
                f11 = S.c_f11[lane];
            }
        } else {
            bool good = true;
            if (act) {
                double k11, k12, k22;
                raw_resp(sd, S.raw[lane], ssr_n, ssr_m, k11, k12, k22);
                good = sec_flex(k11, k12, k22, f00, f01, f11);
            }
            ok = __all_sync(0xffffffffu, good) ? 1 : 0;
        }
        if (ok) {
            if (act) flex_terms(S.scr[lane], wL, bmi, bmj, f00, f01, f11);
            double P[9], pk9[9];
            lane_ordered_sums<9>(S.scr, nip, P);
            if (invert3(P, pk9)) {
                q0 += (pk9[0] * dv[0] + pk9[1] * dv[1] + pk9[2] * dv[2]);
                q1 += (pk9[3] * dv[0] + pk9[4] * dv[1] + pk9[5] * dv[2]);
                q2 += (pk9[6] * dv[0] + pk9[7] * dv[1] + pk9[8] * dv[2]);
            }
            next_points(scheme == 1 || scheme == 2);
        }
        if (lane == 0) S.flag = ok;
    }
    __syncthreads();
    if (!S.flag) return false;
    const double t0 = base[0] + dv[0], t1 = base[1] + dv[1], t2 = base[2] + dv[2];
    for (int it = 0; it < num_iters; ++it) {
        eval_sections(g, sd, sv, E, S, ys, fo);
        if (w0) {
            bool good = true;
            double N = 0.0, M = 0.0, n00 = 0.0, n01 = 0.0, n11 = 0.0;
            if (act) {
                double k11, k12, k22;
                raw_resp(sd, S.raw[lane], N, M, k11, k12, k22);
                good = sec_flex(k11, k12, k22, n00, n01, n11);
            }
            int res = 0;
            if (__all_sync(0xffffffffu, good)) {
                const double ss0 = q0 + 0.0;
                const double ss1 = bmi * q1 + bmj * q2 + 0.0;
                sub_e = pe;
                sub_k = pk;
                ssr_n = N;
                ssr_m = M;
                f00 = n00;
                f01 = n01;
                f11 = n11;
                const double dr0 = ss0 - ssr_n;
                const double dr1 = ss1 - ssr_m;
                const double dvr0 = n00 * dr0 + n01 * dr1;
                const double dvr1 = n01 * dr0 + n11 * dr1;
                if (act) {
                    flex_terms(S.scr[lane], wL, bmi, bmj, n00, n01, n11);
                    S.scr[lane][9] = wL * (pe + dvr0);
                    S.scr[lane][10] = wL * bmi * (pk + dvr1);
                    S.scr[lane][11] = wL * bmj * (pk + dvr1);
                }
                double F[12], k[9];
                lane_ordered_sums<12>(S.scr, nip, F);
                if (invert3(F, k)) {
                    const double r0 = t0 - F[9];
                    const double r1 = t1 - F[10];
                    const double r2 = t2 - F[11];
                    const double dq0 = k[0] * r0 + k[1] * r1 + k[2] * r2;
                    const double dq1 = k[3] * r0 + k[4] * r1 + k[5] * r2;
                    const double dq2 = k[6] * r0 + k[7] * r1 + k[8] * r2;
                    const double work = fabs(r0 * dq0 + r1 * dq1 + r2 * dq2);
                    q0 += dq0;
                    q1 += dq1;
                    q2 += dq2;
                    res = 1;
                    if (work < 1.0e-12) {
                        res = 2;
                        if (act) {
                            S.vs_e[lane] = sub_e;
                            S.vs_k[lane] = sub_k;
                            S.c_n[lane] = ssr_n;
                            S.c_m[lane] = ssr_m;
                            S.c_f00[lane] = f00;
                            S.c_f01[lane] = f01;
                            S.c_f11[lane] = f11;
                        }
                        if (lane == 0) {
                            S.c_valid = 1;
                            S.best[0] = q0;
                            S.best[1] = q1;
                            S.best[2] = q2;
                            S.best[3] = k[0];
                            S.best[4] = k[1];
                            S.best[5] = k[2];
                            S.best[6] = k[3];
                            S.best[7] = k[4];
                            S.best[8] = k[5];
                            S.best[9] = k[8];
                        }
                    } else if (it + 1 < num_iters) {
                        next_points(scheme == 1);
                    }
                }
            }
            if (lane == 0) {
                S.local_iters++;
                // an earlier attempt of a fanned-out element has succeeded: this one is moot
                if (stop && *(volatile const int*)stop < my) res = 0;
                S.flag = res;
                if (res) {
                    S.q[0] = q0;
                    S.q[1] = q1;
                    S.q[2] = q2;
                }
            }
        }
        __syncthreads();
        const int f = S.flag;
        if (f == 0) return false;
        if (f == 2) return true;
    }
    return false;
}

__device__ __forceinline__ double max_abs3(const double* v) {
    double m = fabs(v[0]);
    if (fabs(v[1]) > m) m = fabs(v[1]);
    if (fabs(v[2]) > m) m = fabs(v[2]);
    return m;
}

__device__ __forceinline__ void u_to_local(double c, double s, const double* ug, double* ul) {
    ul[0] = c * ug[0] + s * ug[1];
    ul[1] = -s * ug[0] + c * ug[1];
    ul[2] = ug[2];
    ul[3] = c * ug[3] + s * ug[4];
    ul[4] = -s * ug[3] + c * ug[4];
    ul[5] = ug[5];
}

__device__ __forceinline__ void k_to_global(double* k, double c, double s) {
    for (int i = 0; i < 6; ++i) {
        const double k0 = k[i * 6 + 0], k1 = k[i * 6 + 1], k3 = k[i * 6 + 3], k4 = k[i * 6 + 4];
        k[i * 6 + 0] = c * k0 - s * k1;
        k[i * 6 + 1] = s * k0 + c * k1;
        k[i * 6 + 3] = c * k3 - s * k4;
        k[i * 6 + 4] = s * k3 + c * k4;
    }
    for (int r0 = 0; r0 <= 3; r0 += 3) {
        const int r1 = r0 + 1;
        for (int j = 0; j < 6; ++j) {
            const double a = k[r0 * 6 + j], b = k[r1 * 6 + j];
            k[r0 * 6 + j] = c * a - s * b;
            k[r1 * 6 + j] = s * a + c * b;
        }
    }
}

__device__ __forceinline__ void f_to_global(double* f, double c, double s) {
    const double f0 = f[0], f1 = f[1], f3 = f[3], f4 = f[4];
    f[0] = c * f0 - s * f1;
    f[1] = s * f0 + c * f1;
    f[3] = c * f3 - s * f4;
    f[4] = s * f3 + c * f4;
}

__device__ __forceinline__ void basic_map(int col, double inv_L, double* a) {
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

__device__ __forceinline__ double curv_shape(int idx, double inv_L, double inv_L_sq, double xi) {
    switch (idx) {
        case 1: return (-6.0 + 12.0 * xi) * inv_L_sq;
        case 2: return (-4.0 + 6.0 * xi) * inv_L;
        case 4: return (6.0 - 12.0 * xi) * inv_L_sq;
        case 5: return (-2.0 + 6.0 * xi) * inv_L;
        default: return 0.0;
    }
}

__device__ __forceinline__ double axial_shape(int idx, double inv_L) {
    if (idx == 0) return -inv_L;
    if (idx == 3) return inv_L;
    return 0.0;
}

// One attempt of an element's fan-out (level fa / 3, scheme fa % 3 of the first subdivision
// pass, force_beam_column2d.mojo:1669-1763) from the accepted state in S, its outcome recorded in
// the fan slot; the last attempt to finish resolves the pass.  Returns -2 for an attempt that is
// not the last (the caller stops), else the first successful attempt in the reference's order
// (-1: none), with S as the sequential algorithm leaves it after that acceptance: q, the section
// deformations and the response cache of the chosen attempt, the accepted basic state advanced,
// S.loop_ctrl 1 when nothing remains, else 0 with S.att the remainder; S.local_iters and
// S.section_evals count the attempts the sequential algorithm would have run.  Not inlined: it
// runs at most once per element determination and keeps the sequential path's registers free.
__device__ __noinline__ int fan_attempt(const Geo& g, const DevSection& sd, const StageView& sv,
                                        const DevElem& E, ElemScratch& S, const ElemList& el, int cur,
                                        int fslot, int fa, const double* ys, double* fo) {
    const int tid = threadIdx.x, nip = E.nip;
    const int level = fa / 3, scheme = fa - 3 * (fa / 3);
    if (tid == 0) {
        for (int l = 0; l < level; ++l)
            for (int i = 0; i < 3; ++i) S.att[i] /= 10.0;
        for (int i = 0; i < 3; ++i) {
            S.tv[i] = S.acc_v[i] + S.att[i];
            S.q[i] = S.acc_q[i];
        }
        for (int ip = 0; ip < nip; ++ip) {
            S.vs_e[ip] = S.svs_e[ip];
            S.vs_k[ip] = S.svs_k[ip];
        }
    }
    __syncthreads();
    int* first = el.fan_first + cur * kFanCap + fslot;
    const bool ok = fbc_try_increment(g, sd, sv, E, S, S.acc_v, S.att, scheme, ys, fo, first, fa);
    if (ok && threadIdx.x == 0) atomicMin(first, fa);
    double* const slot_rec = el.fan_rec + (size_t)(cur * kFanCap + fslot) * kFanAttempts * kFanRec;
    double* rec = slot_rec + (size_t)fa * kFanRec;
    if (tid == 0) {
        rec[0] = ok ? 1.0 : 0.0;
        rec[1] = (double)S.local_iters;
        rec[2] = (double)S.section_evals;
        for (int i = 0; i < 3; ++i) rec[3 + i] = S.q[i];
        for (int i = 0; i < 10; ++i) rec[6 + i] = S.best[i];
        rec[86] = (double)S.c_valid;
    } else if (tid <= nip) {
        const int ip = tid - 1;
        rec[16 + ip] = S.vs_e[ip];
        rec[26 + ip] = S.vs_k[ip];
        rec[36 + ip] = S.c_n[ip];
        rec[46 + ip] = S.c_m[ip];
        rec[56 + ip] = S.c_f00[ip];
        rec[66 + ip] = S.c_f01[ip];
        rec[76 + ip] = S.c_f11[ip];
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) {
        const int old = atomicAdd(&el.fan_done[cur * kFanCap + fslot], 1);
        S.flag = (old % kFanAttempts) == kFanAttempts - 1;
    }
    __syncthreads();
    if (!S.flag) return -2;
    __threadfence();
    if (tid == 0) {
        int best_a = -1;
        long long li = 0, se = 0;
        for (int a = 0; a < kFanAttempts; ++a) {
            const double* r = slot_rec + (size_t)a * kFanRec;
            li += (long long)__ldcg(r + 1);
            se += (long long)__ldcg(r + 2);
            if (__ldcg(r) != 0.0) {
                best_a = a;
                break;
            }
        }
        S.local_iters = (int)li;
        S.section_evals = (int)se;
        S.loop_ctrl = best_a;
        if (best_a < 0 || best_a >= 3) S.hard = 1;
    }
    __syncthreads();
    const int best_a = S.loop_ctrl;
    if (best_a < 0) return -1;
    const double* r = slot_rec + (size_t)best_a * kFanRec;
    if (tid == 0) {
        for (int i = 0; i < 3; ++i) S.q[i] = __ldcg(r + 3 + i);
        for (int i = 0; i < 10; ++i) S.best[i] = __ldcg(r + 6 + i);
        S.c_valid = (int)__ldcg(r + 86);
        // S.att holds this CTA's own level: recompute the chosen one's
        for (int i = 0; i < 3; ++i) S.att[i] = S.rem[i];
        for (int l = 0; l < best_a / 3; ++l)
            for (int i = 0; i < 3; ++i) S.att[i] /= 10.0;
        for (int i = 0; i < 3; ++i) S.tv[i] = S.acc_v[i] + S.att[i];
    } else if (tid <= nip) {
        const int ip = tid - 1;
        S.vs_e[ip] = __ldcg(r + 16 + ip);
        S.vs_k[ip] = __ldcg(r + 26 + ip);
        S.c_n[ip] = __ldcg(r + 36 + ip);
        S.c_m[ip] = __ldcg(r + 46 + ip);
        S.c_f00[ip] = __ldcg(r + 56 + ip);
        S.c_f01[ip] = __ldcg(r + 66 + ip);
        S.c_f11[ip] = __ldcg(r + 76 + ip);
    }
    __syncthreads();
    // the acceptance of the sequential loop
    if (tid == 0) {
        for (int i = 0; i < 3; ++i) {
            S.acc_v[i] = S.tv[i];
            S.acc_q[i] = S.best[i];
        }
        for (int ip = 0; ip < nip; ++ip) {
            S.svs_e[ip] = S.vs_e[ip];
            S.svs_k[ip] = S.vs_k[ip];
        }
        S.best_ok = 1;
        for (int i = 0; i < 3; ++i) S.rem[i] = S.v[i] - S.acc_v[i];
        if (max_abs3(S.rem) <= 1.0e-12) {
            S.loop_ctrl = 1;
        } else {
            for (int i = 0; i < 3; ++i) S.att[i] = S.rem[i];
            S.loop_ctrl = 0;
        }
    }
    __syncthreads();
    return best_a;
}

// Copies a POD struct from global to shared memory with 4-byte words.
template <typename T>
__device__ __forceinline__ void copy_struct(T* dst, const T* src) {
    static_assert(sizeof(T) % 4 == 0, "4-byte multiple");
    const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
    uint32_t* d = reinterpret_cast<uint32_t*>(dst);
    for (int i = threadIdx.x; i < (int)(sizeof(T) / 4); i += blockDim.x) d[i] = s[i];
}

// Stages the element's committed fiber history into shared memory: stage_issue (the views, and
// thread 0's bulk copies) then stage_wait; stage_element does both.  bar was initialised once for
// the CTA; phase is the parity of its next completion (every thread tracks the same value).
// stage_wait returns false (and sets *err) if the bulk copy did not complete within the bounded
// wait.
__device__ __forceinline__ void stage_layout(const DevElem& E, double* sm, StageView& sv) {
    double* c2 = sm;
    double* s2 = c2 + 4 * E.c2_blk;
    double* s1 = s2 + 10 * E.s2_blk;
    double* c1 = s1 + 5 * E.s1_blk;
    int* kon = reinterpret_cast<int*>(c1 + 6 * E.c1_blk);
    sv.c2 = c2;
    sv.s2 = s2;
    sv.s1 = s1;
    sv.c1 = c1;
    sv.kon = kon;
    // derived constants follow the staged history (kon occupies s2_blk ints, s2_blk % 4 == 0)
    sv.c2d = reinterpret_cast<const double*>(kon + E.s2_blk);
    sv.s2d = sv.c2d + 5 * E.c2_blk;
    sv.c2_blk = E.c2_blk;
    sv.s2_blk = E.s2_blk;
    sv.s1_blk = E.s1_blk;
    sv.c1_blk = E.c1_blk;
}

// dept (optional): shared-memory destination of the Concrete02 dept field (E.c2_blk doubles,
// 16-byte aligned), copied with the history.
__device__ __forceinline__ uint32_t stage_issue(const DevElem& E, const FiberState& fs, double* sm,
                                                uint64_t* bar, StageView& sv, double* dept = nullptr) {
    stage_layout(E, sm, sv);
    double* c2 = const_cast<double*>(sv.c2);
    double* s2 = const_cast<double*>(sv.s2);
    double* s1 = const_cast<double*>(sv.s1);
    double* c1 = const_cast<double*>(sv.c1);
    int* kon = const_cast<int*>(sv.kon);
    if (!E.c2_blk) dept = nullptr;
    const uint32_t bytes = (uint32_t)(8 * (4 * E.c2_blk + 10 * E.s2_blk + 5 * E.s1_blk + 6 * E.c1_blk) +
                                      4 * E.s2_blk + (dept ? 8 * E.c2_blk : 0));
    if (bytes == 0) return 0u;
    if (threadIdx.x == 0) {
        // the previous element's reads of this buffer (generic proxy) come before the copies
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive_expect_tx(bar, bytes);
        for (int f = 0; f < 4 && E.c2_blk; ++f)
            bulk_g2s(c2 + f * E.c2_blk, fs.c2 + f * fs.c2_n + E.c2_off, 8u * E.c2_blk, bar);
        if (dept) bulk_g2s(dept, fs.c2 + 4 * fs.c2_n + E.c2_off, 8u * E.c2_blk, bar);
        for (int f = 0; f < 10 && E.s2_blk; ++f)
            bulk_g2s(s2 + f * E.s2_blk, fs.s2 + f * fs.s2_n + E.s2_off, 8u * E.s2_blk, bar);
        if (E.s2_blk) bulk_g2s(kon, fs.s2_kon + E.s2_off, 4u * E.s2_blk, bar);
        for (int f = 0; f < 5 && E.s1_blk; ++f)
            bulk_g2s(s1 + f * E.s1_blk, fs.s1 + f * fs.s1_n + E.s1_off, 8u * E.s1_blk, bar);
        for (int f = 0; f < 6 && E.c1_blk; ++f)
            bulk_g2s(c1 + f * E.c1_blk, fs.c1 + f * fs.c1_n + E.c1_off, 8u * E.c1_blk, bar);
    }
    return bytes;
}

__device__ __forceinline__ bool stage_wait(uint32_t bytes, uint64_t* bar, uint32_t& phase, int* err) {
    if (bytes == 0) return true;
    const uint32_t ph = phase;
    phase ^= 1u;
    const bool ok = mbar_wait_bounded(bar, ph);
    // every thread takes the same branch
    if (__syncthreads_or(ok ? 0 : 1)) {
        if (threadIdx.x == 0) *err = ELEM_ERR_TMA_TIMEOUT;
        // let the copies land before the CTA stops (second bounded wait)
        mbar_wait_bounded(bar, ph);
        return false;
    }
    return true;
}

__device__ __forceinline__ bool stage_element(const DevElem& E, const FiberState& fs,
                                              double* sm, uint64_t* bar, uint32_t& phase,
                                              StageView& sv, int* err) {
    return stage_wait(stage_issue(E, fs, sm, bar, sv), bar, phase, err);
}

}  // namespace strut

#include "element3d_kernels.cuh"

namespace strut {

// Elements processed by one launch of the element kernel.
enum { ELEM_MODE_LIST = 0, ELEM_MODE_ALL = 1, ELEM_MODE_RECORD = 2 };

// Record pass after a step's commit: the recorded 3D beam-columns of the live instances, whose
// recorded force is a full state determination at the converged displacements
// (helpers.mojo:544-775; for forceBeamColumn3d this also moves its trial basic forces and section
// deformations, as in Strut).
struct RecPass {
    const int* list;      // element indices
    int n;
    double* hist_ef;      // step-major: [step][slot][ef_w]
    const int* rece_base; // first record slot of each instance
    int slots, ef_w;
};

// State determination of every element of the active instances: k (nd x nd global), f (nd)
// and the element state.  One CTA of kTeamThreads threads (or half as many, two CTAs per SM) per
// element at a time; one compiled kernel serves both block sizes, so the arithmetic is the same.
//
// Persistent: the grid is sized to the resident CTAs of the device and each CTA claims elements
// from the list of the instances still iterating (all elements when all_elems is set), so a
// Newton iteration of a few slow records launches no idle CTAs and a slow element does not hold
// up elements queued behind it on the same CTA.
//
// Saves the accepted state a fanned element's next pass starts from in its round record and posts
// the pass's twelve attempts to the list's queue (thread 0 of the resolving CTA).
__device__ __noinline__ void post_next_pass(const ElemList& el, int cur, int fslot, double* R, int round, int guard,
                                            const ElemScratch& S, int nip) {
    R[kFRound] = (double)(round + 1);
    R[kFGuard] = (double)guard;
    R[kFLocal] = (double)S.local_iters;
    R[kFEvals] = (double)S.section_evals;
    R[kFHard] = (double)S.hard;
    R[kFCValid] = (double)S.c_valid;
    R[kFBestOk] = (double)S.best_ok;
    for (int i = 0; i < 3; ++i) {
        R[kFAccV + i] = S.acc_v[i];
        R[kFAccQ + i] = S.acc_q[i];
        R[kFRem + i] = S.att[i];
    }
    for (int i = 0; i < 10; ++i) R[kFBest + i] = S.best[i];
    for (int ip = 0; ip < nip; ++ip) {
        R[kFSvsE + ip] = S.svs_e[ip];
        R[kFSvsK + ip] = S.svs_k[ip];
        R[kFCN + ip] = S.c_n[ip];
        R[kFCM + ip] = S.c_m[ip];
        R[kFC00 + ip] = S.c_f00[ip];
        R[kFC01 + ip] = S.c_f01[ip];
        R[kFC11 + ip] = S.c_f11[ip];
    }
    el.fan_first[cur * kFanCap + fslot] = kFanAttempts;
    __threadfence();
    const int d0 = atomicAdd(&el.rq_tail[cur], kFanAttempts);
    long long* q = el.rq + (size_t)cur * kRoundQ;
    for (int a = 0; a < kFanAttempts; ++a) {
        const int d = d0 + a;
        const long long v = ((long long)d << 16) | (long long)(fslot * kFanAttempts + a);
        // an entry is free once its previous attempt was taken (bounded wait)
        int n = 0;
        while (atomicCAS(reinterpret_cast<unsigned long long*>(q + d % kRoundQ), ~0ull, (unsigned long long)v) !=
               ~0ull) {
            if (++n > kQueuePolls) {
                atomicExch(el.q_err, 1);
                break;
            }
            __nanosleep(128);
        }
    }
}

// Takes the posted attempt with queue ticket d: returns slot x 12 + attempt, or -1 once every
// fanned element of the list is resolved and no attempt has ticket d (thread 0).
__device__ __noinline__ int take_posted(const ElemList& el, int cur, int d, int n_slots) {
    volatile long long* q = el.rq + (size_t)cur * kRoundQ + d % kRoundQ;
    for (int n = 0; n < kQueuePolls; ++n) {
        const long long v = *q;
        if (v >= 0 && (v >> 16) == (long long)d) {
            __threadfence();
            *q = -1;  // free the entry
            return (int)(v & 0xFFFF);
        }
        if (*(volatile int*)(el.fan_finished + cur) >= n_slots && *(volatile int*)(el.rq_tail + cur) <= d)
            return -1;
        __nanosleep(n < 256 ? 64 : 512);
    }
    atomicExch(el.q_err, 1);
    return -1;
}

// Element-level scratch of the element kernel: the 3D scratch exists only in the 3D instance (a
// smaller static footprint lets more 2D element CTAs share an SM).
template <int DIM>
union ElemScratchOf {
    ElemScratch s2;
    ElemScratch3 s3;
};
template <>
union ElemScratchOf<2> {
    ElemScratch s2;
};

// DIM 2 instantiates the 2D elements' code only, DIM 3 the 3D elements' (a batch holds one kind).
template <int DIM>
__global__ void __launch_bounds__(kTeamThreads) element_state_kernel(
    const DevElem* __restrict__ elems, Geo g, FiberState fs, const double* __restrict__ u_full,
    double* __restrict__ estate, double* __restrict__ ek, double* __restrict__ ef,
    const int* __restrict__ active, int* __restrict__ status, int* __restrict__ elem_err,
    unsigned long long* __restrict__ counters, ElemList el, const DevCtl* __restrict__ ctl,
    int mode, int n_elem, RecPass rp) {
    extern __shared__ __align__(128) double smem_fib[];
    __shared__ DevElem E;
    __shared__ DevSection sd;
    __shared__ ElemScratchOf<DIM> SU;
    ElemScratch& S = SU.s2;
    const int all_elems = mode != ELEM_MODE_LIST;
    __shared__ __align__(8) uint64_t bar;
    const int tid = threadIdx.x;
    if (tid == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __shared__ int s_next;
    __shared__ int s_fan;    // a fan attempt has already counted itself in (fan_done)
    __shared__ int s_round;  // pass of the fanned element this CTA works on (1: the first)
    __shared__ int s_item;   // posted attempt taken from the queue (-1: none)
    const int cur = all_elems ? 0 : (ctl->iter & 1);
    // fanned-out elements of this list (their attempts come first in the work order)
    const int n_fan = all_elems ? 0 : min(el.hard_count[cur], (int)kFanCap) * kFanAttempts;
    if (!all_elems && blockIdx.x == 0 && tid == 0) {
        el.count[cur ^ 1] = 0;
        el.next[cur ^ 1] = 0;
        el.hard_count[cur ^ 1] = 0;
        if (el.rq) {
            el.rq_tail[cur ^ 1] = 0;
            el.fan_finished[cur ^ 1] = 0;
        }
    }
    const int total = mode == ELEM_MODE_ALL ? n_elem
                    : mode == ELEM_MODE_RECORD ? rp.n : n_fan + el.count[cur];
    __syncthreads();
    uint32_t phase = 0;
    bool stop = false;
    // fslot >= 0: attempt fa of the fan-out of element e in slot fslot of this list
    auto process = [&](const int e, const int fslot, const int fa) -> void {
    copy_struct(&E, elems + e);
    __syncthreads();
    // the instance's flag and the section record are read together (the section of an element
    // that is not run is read but not used)
    const bool skip = mode == ELEM_MODE_RECORD ? status[E.inst] != 0 : !active[E.inst];
    copy_struct(&sd, g.secs + E.sec);
    if (skip) {
        // a fanned element that is not run still counts as resolved (its first attempt's CTA)
        if (fslot >= 0 && fa == 0 && tid == 0 && el.rq) atomicAdd(&el.fan_finished[cur], 1);
        return;
    }
    if constexpr (DIM == 3) {
        __syncthreads();
        double* rec_out = nullptr;
        if (mode == ELEM_MODE_RECORD)
            rec_out = rp.hist_ef + ((size_t)ctl->step * rp.slots + rp.rece_base[E.inst] + E.rec) * rp.ef_w;
        element3d_process(g, sd, E, e, fs, u_full, estate, ek, ef, status, elem_err, counters, SU.s3,
                          smem_fib, &bar, phase, stop, rec_out);
        return;
    }
    __syncthreads();
    // the bulk copies of the fiber history go out first, with the Concrete02 dept field into the
    // buffer of the per-fiber results (free until the first evaluation); the element state and
    // the section's fiber y are read while they are in flight
    StageView sv;
    stage_layout(E, smem_fib, sv);
    const int n_tot = sd.n_s2 + sd.n_c2 + sd.n_s1 + sd.n_c1 + sd.n_el;
    double* ys = const_cast<double*>(sv.s2d) + 12 * E.s2_blk;
    double* fo = ys + ((n_tot + 1) & ~1);
    int err = ELEM_ERR_NONE;
    const uint32_t stage_bytes = stage_issue(E, fs, smem_fib, &bar, sv, fo);
    {
        const double* es = estate + (size_t)e * kEStride;
        if (tid < E.nip) {
            const int ip = tid;
            const double ve = es[kEe + ip], vk = es[kEk + ip];
            S.vs_e[ip] = ve;
            S.vs_k[ip] = vk;
            if (E.type == 2) {  // the accepted section deformations start as the element's
                S.svs_e[ip] = ve;
                S.svs_k[ip] = vk;
            }
            S.c_n[ip] = es[kEcN + ip];
            S.c_m[ip] = es[kEcM + ip];
            S.c_f00[ip] = es[kEc00 + ip];
            S.c_f01[ip] = es[kEc01 + ip];
            S.c_f11[ip] = es[kEc11 + ip];
        } else if (tid == 32) {
            // the displacements in the element's frame and (forceBeamColumn2d) the basic
            // deformations, the accepted state and the increment still to apply
            double ug[6], ul[6], q[3], av[3];
            for (int a = 0; a < 6; ++a) ug[a] = u_full[E.dof[a]];
            for (int i = 0; i < 3; ++i) {
                q[i] = es[kEq + i];
                av[i] = es[kEv + i];
            }
            const bool cv = es[kEcv] != 0.0;
            if (E.type == 2)
                u_to_local(E.c, E.s, ug, ul);
            else
                u_to_local(E.c_div, E.s_div, ug, ul);
            for (int a = 0; a < 6; ++a) S.ul[a] = ul[a];
            S.local_iters = 0;
            S.section_evals = 0;
            S.hard = 0;
            for (int i = 0; i < 3; ++i) {
                S.q[i] = q[i];
                S.acc_v[i] = av[i];
                S.zero3[i] = 0.0;
            }
            S.c_valid = E.type == 2 && cv;
            if (E.type == 2) {
                const double chord = (ul[4] - ul[1]) / E.L;
                const double v[3] = {ul[3] - ul[0], ul[2] - chord, ul[5] - chord};
                for (int i = 0; i < 3; ++i) {
                    S.v[i] = v[i];
                    S.acc_q[i] = q[i];
                    const double r = v[i] - av[i];
                    S.rem[i] = r;
                    S.att[i] = r;
                }
                S.best_ok = 0;
                S.loop_ctrl = 0;
            }
        }
    }
    for (int gg = tid; gg < n_tot; gg += blockDim.x) ys[gg] = __ldg(g.y + sd.geo_off + gg);
    const bool staged = stage_wait(stage_bytes, &bar, phase, &err);  // a CTA barrier when copies ran
    if (!stage_bytes) __syncthreads();
    if (!staged) {
        if (tid == 0) {
            elem_err[e] = err;
            status[E.inst] = 5;
        }
        stop = true;
        return;
    }
    derive_element(g, sd, E, sv, fo, const_cast<double*>(sv.c2d), const_cast<double*>(sv.s2d));
    __syncthreads();
    const int nip = E.nip;
    if (E.type == 3) {
        // ---------------- dispBeamColumn2d ----------------
        const double L = E.L, inv_L = 1.0 / L, inv_L_sq = inv_L * inv_L;
        if (tid < nip) {
            const double xi = E.xi[tid];
            const double b1 = curv_shape(1, inv_L, inv_L_sq, xi);
            const double b2 = curv_shape(2, inv_L, inv_L_sq, xi);
            const double b4 = curv_shape(4, inv_L, inv_L_sq, xi);
            const double b5 = curv_shape(5, inv_L, inv_L_sq, xi);
            const double eps0 = (-inv_L) * S.ul[0] + inv_L * S.ul[3];
            const double kappa = b1 * S.ul[1] + b2 * S.ul[2] + b4 * S.ul[4] + b5 * S.ul[5];
            S.pt_e[tid] = eps0;
            S.pt_k[tid] = kappa;
            S.vs_e[tid] = eps0;
            S.vs_k[tid] = kappa;
        }
        __syncthreads();
        eval_sections(g, sd, sv, E, S, ys, fo);
        if (tid < nip) {
            double* r = S.resp[tid];
            raw_resp(sd, S.raw[tid], r[0], r[1], r[2], r[3], r[4]);
        }
        __syncthreads();
        if (tid < 36) {
            const int a = tid / 6, b = tid % 6;
            double kab = 0.0;
            for (int ip = 0; ip < nip; ++ip) {
                const double xi = E.xi[ip], wL = E.w[ip] * L;
                const double ban = axial_shape(a, inv_L), bam = curv_shape(a, inv_L, inv_L_sq, xi);
                const double bbn = axial_shape(b, inv_L), bbm = curv_shape(b, inv_L, inv_L_sq, xi);
                const double dN = S.resp[ip][2] * bbn + S.resp[ip][3] * bbm;
                const double dM = S.resp[ip][3] * bbn + S.resp[ip][4] * bbm;
                kab += wL * (ban * dN + bam * dM);
            }
            S.k[tid] = kab;
        } else if (tid < 42) {
            const int a = tid - 36;
            double fa = 0.0;
            for (int ip = 0; ip < nip; ++ip) {
                const double xi = E.xi[ip], wL = E.w[ip] * L;
                const double ban = axial_shape(a, inv_L), bam = curv_shape(a, inv_L, inv_L_sq, xi);
                fa += wL * (ban * S.resp[ip][0] + bam * S.resp[ip][1]);
            }
            S.f[a] = fa;
        }
        __syncthreads();
        if (tid == 0) {
            if (E.geom == 1) {
                double avg = 0.0;
                for (int ip = 0; ip < nip; ++ip) avg += E.w[ip] * S.resp[ip][0];
                const double al = avg / L;
                S.k[1 * 6 + 1] += al;
                S.k[4 * 6 + 4] += al;
                S.k[1 * 6 + 4] -= al;
                S.k[4 * 6 + 1] -= al;
                const double ps = (S.ul[1] - S.ul[4]) * al;
                S.f[1] += ps;
                S.f[4] -= ps;
            }
            k_to_global(S.k, E.c_div, E.s_div);
            f_to_global(S.f, E.c_div, E.s_div);
            for (int ip = 0; ip < nip; ++ip) {
                estate[(size_t)e * kEStride + kEe + ip] = S.vs_e[ip];
                estate[(size_t)e * kEStride + kEk + ip] = S.vs_k[ip];
            }
        }
        __syncthreads();
        if (tid < 36) ek[E.ek_off + tid] = S.k[tid];
        else if (tid < 42) ef[E.ef_off + tid - 36] = S.f[tid - 36];
        if (tid == 0) {
            atomicAdd(&counters[3], (unsigned long long)E.io_bytes);
            atomicAdd(&counters[1], (unsigned long long)nip);
            atomicAdd(&counters[2], (unsigned long long)nip *
                                        (sd.n_s2 + sd.n_c2 + sd.n_s1 + sd.n_c1 + sd.n_el));
            atomicAdd(&counters[7], (unsigned long long)nip * section_update_bytes(sd));
        }
        return;
    }
    // ---------------- forceBeamColumn2d ----------------
    // (basic deformations, accepted state and increment were set up while the history was staged)
    const double L = E.L;
    const double inv_L = E.inv_L;
    // a later pass of a fanned-out element starts from the state its previous pass accepted
    if (fslot >= 0 && tid == 0) {
        const double* R = el.fan_round + (size_t)(cur * kFanCap + fslot) * kFanRound;
        s_round = (int)__ldcg(R + kFRound);
        if (s_round > 1) {
            for (int i = 0; i < 3; ++i) {
                S.acc_v[i] = __ldcg(R + kFAccV + i);
                S.acc_q[i] = __ldcg(R + kFAccQ + i);
                S.rem[i] = __ldcg(R + kFRem + i);
                S.att[i] = S.rem[i];
            }
            for (int i = 0; i < 10; ++i) S.best[i] = __ldcg(R + kFBest + i);
            S.best_ok = (int)__ldcg(R + kFBestOk);
            S.c_valid = (int)__ldcg(R + kFCValid);
            for (int ip = 0; ip < nip; ++ip) {
                S.svs_e[ip] = __ldcg(R + kFSvsE + ip);
                S.svs_k[ip] = __ldcg(R + kFSvsK + ip);
                S.c_n[ip] = __ldcg(R + kFCN + ip);
                S.c_m[ip] = __ldcg(R + kFCM + ip);
                S.c_f00[ip] = __ldcg(R + kFC00 + ip);
                S.c_f01[ip] = __ldcg(R + kFC01 + ip);
                S.c_f11[ip] = __ldcg(R + kFC11 + ip);
            }
        }
    }
    if (fslot >= 0) __syncthreads();
    int converged = 0;
    if (sd.all_elastic) {
        // _force_beam_column2d_exact_elastic_state (section evaluations there only set trial
        // fiber state, which this design does not store)
        if (tid == 0) {
            int ok = 0;
            if (sd.init_valid) {
                double F[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                double vl0 = 0.0, vl1 = 0.0, vl2 = 0.0;
                for (int ip = 0; ip < nip; ++ip) {
                    const double xi = E.xi[ip], wL = E.w[ip] * L;
                    const double bmi = xi - 1.0, bmj = xi;
                    flex_accum(F, wL, bmi, bmj, sd.f00, sd.f01, sd.f11);
                    vl0 += wL * (sd.f00 * 0.0 + sd.f01 * 0.0);
                    vl1 += wL * bmi * (sd.f01 * 0.0 + sd.f11 * 0.0);
                    vl2 += wL * bmj * (sd.f01 * 0.0 + sd.f11 * 0.0);
                }
                double k[9];
                if (invert3(F, k)) {
                    const double r0 = S.v[0] - vl0, r1 = S.v[1] - vl1, r2 = S.v[2] - vl2;
                    const double q0 = k[0] * r0 + k[1] * r1 + k[2] * r2;
                    const double q1 = k[3] * r0 + k[4] * r1 + k[5] * r2;
                    const double q2 = k[6] * r0 + k[7] * r1 + k[8] * r2;
                    for (int ip = 0; ip < nip; ++ip) {
                        const double xi = E.xi[ip];
                        const double axial = q0 + 0.0;
                        const double moment = (xi - 1.0) * q1 + xi * q2 + 0.0;
                        S.vs_e[ip] = sd.f00 * axial + sd.f01 * moment;
                        S.vs_k[ip] = sd.f01 * axial + sd.f11 * moment;
                        S.svs_e[ip] = S.vs_e[ip];
                        S.svs_k[ip] = S.vs_k[ip];
                    }
                    S.q[0] = q0;
                    S.q[1] = q1;
                    S.q[2] = q2;
                    for (int i = 0; i < 3; ++i) {
                        S.acc_v[i] = S.v[i];
                        S.acc_q[i] = S.q[i];
                        S.rem[i] = 0.0;
                    }
                    S.best[0] = q0;
                    S.best[1] = q1;
                    S.best[2] = q2;
                    for (int i = 0; i < 6; ++i) S.best[3 + i] = k[i];
                    S.best[9] = k[8];
                    S.best_ok = 1;
                    S.c_valid = 0;
                    ok = 1;
                }
            }
            S.flag = ok;
        }
        __syncthreads();
        converged = S.flag;
    }
    // a fanned-out element with nothing to subdivide runs on its first attempt's CTA alone
    if (fslot >= 0 && fa != 0 && (converged || max_abs3(S.rem) <= 1.0e-16)) return;
    if (!converged) {
        if (max_abs3(S.rem) <= 1.0e-16) {
            for (int scheme = 0; scheme < 3; ++scheme) {
                if (tid == 0) {
                    for (int i = 0; i < 3; ++i) S.q[i] = S.acc_q[i];
                    for (int ip = 0; ip < nip; ++ip) {
                        S.vs_e[ip] = S.svs_e[ip];
                        S.vs_k[ip] = S.svs_k[ip];
                    }
                }
                __syncthreads();
                if (!fbc_try_increment(g, sd, sv, E, S, S.acc_v, S.zero3, scheme, ys, fo, nullptr, 0)) continue;
                if (tid == 0) S.best_ok = 1;
                converged = 1;
                break;
            }
        } else {
            int num_subdivide = 1;
            int guard = 0;
            bool run_loop = true;
            if (fslot >= 0) {
                const int best_a = fan_attempt(g, sd, sv, E, S, el, cur, fslot, fa, ys, fo);
                if (best_a == -2) {
                    s_fan = 1;
                    return;  // not the last attempt: the last one finishes the element
                }
                double* R = el.fan_round + (size_t)(cur * kFanCap + fslot) * kFanRound;
                const int round = s_round;
                const int guard_before = round > 1 ? (int)__ldcg(R + kFGuard) : 0;
                if (tid == 0) {
                    s_fan = 1;
                    if (round > 1) {  // the passes before this one
                        S.local_iters += (int)__ldcg(R + kFLocal);
                        S.section_evals += (int)__ldcg(R + kFEvals);
                        if (__ldcg(R + kFHard) != 0.0) S.hard = 1;
                    }
                }
                if (best_a < 0) {
                    run_loop = false;  // every attempt failed: the initial-tangent fallback
                    guard = guard_before + 4;
                } else {
                    if (S.loop_ctrl == 1) {
                        converged = 1;
                        run_loop = false;
                    }
                    guard = guard_before + best_a / 3 + 1;
                    // the next pass over the remainder, fanned out while the guard leaves room
                    // for all four of its levels
                    if (run_loop && guard + 4 <= 10000) {
                        __syncthreads();
                        if (tid == 0) post_next_pass(el, cur, fslot, R, round, guard, S, nip);
                        __syncthreads();
                        return;
                    }
                }
            }
            while (run_loop && num_subdivide <= 4 && guard < 10000) {
                ++guard;
                int scheme_success = 0;
                for (int scheme = 0; scheme < 3; ++scheme) {
                    // warp 0 restores the accepted state (and first forms the trial deformation)
                    if (tid < 32) {
                        if (tid < 3) {
                            if (scheme == 0) S.tv[tid] = S.acc_v[tid] + S.att[tid];
                            S.q[tid] = S.acc_q[tid];
                        }
                        if (tid < nip) {
                            S.vs_e[tid] = S.svs_e[tid];
                            S.vs_k[tid] = S.svs_k[tid];
                        }
                    }
                    __syncthreads();
                    if (!fbc_try_increment(g, sd, sv, E, S, S.acc_v, S.att, scheme, ys, fo, nullptr, 0)) continue;
                    if (tid < 32) {
                        // accept the partial step; every lane forms the remainder and its test
                        double rm[3];
                        for (int i = 0; i < 3; ++i) rm[i] = S.v[i] - S.tv[i];
                        const bool done = max_abs3(rm) <= 1.0e-12;
                        if (tid < 3) {
                            const double r = tid == 0 ? rm[0] : tid == 1 ? rm[1] : rm[2];
                            S.acc_v[tid] = S.tv[tid];
                            S.acc_q[tid] = S.best[tid];
                            S.rem[tid] = r;
                            if (!done) S.att[tid] = r;
                        }
                        if (tid < nip) {
                            S.svs_e[tid] = S.vs_e[tid];
                            S.svs_k[tid] = S.vs_k[tid];
                        }
                        if (tid == 0) {
                            S.best_ok = 1;
                            S.loop_ctrl = done ? 1 : 0;
                        }
                    }
                    __syncthreads();
                    scheme_success = 1;
                    if (S.loop_ctrl == 1) converged = 1;
                    else num_subdivide = 1;
                    break;
                }
                if (converged) break;
                if (scheme_success) continue;
                if (tid == 0) {
                    for (int i = 0; i < 3; ++i) S.att[i] /= 10.0;
                    S.hard = 1;
                }
                __syncthreads();
                num_subdivide += 1;
            }
        }
    }
    if (tid == 0) {
        int fail = 0;
        if (!converged) {
            for (int i = 0; i < 3; ++i) S.q[i] = S.acc_q[i];
            for (int ip = 0; ip < nip; ++ip) {
                S.vs_e[ip] = S.svs_e[ip];
                S.vs_k[ip] = S.svs_k[ip];
            }
        }
        if (!S.best_ok) {
            // _force_beam_column2d_initial_basic_tangent fallback
            double F[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int ip = 0; ip < nip; ++ip) {
                const double xi = E.xi[ip], wL = E.w[ip] * L;
                flex_accum(F, wL, xi - 1.0, xi, sd.f00, sd.f01, sd.f11);
            }
            double k[9];
            if (sd.init_valid && invert3(F, k)) {
                S.best[0] = S.q[0];
                S.best[1] = S.q[1];
                S.best[2] = S.q[2];
                for (int i = 0; i < 6; ++i) S.best[3 + i] = k[i];
                S.best[9] = k[8];
            } else {
                fail = 1;
            }
        }
        S.flag = fail;
        // element state: q, section deformations, accepted basic deformation
        for (int i = 0; i < 3; ++i) {
            estate[(size_t)e * kEStride + kEq + i] = S.q[i];
            estate[(size_t)e * kEStride + kEv + i] = S.acc_v[i];
        }
        double* es = estate + (size_t)e * kEStride;
        for (int ip = 0; ip < nip; ++ip) {
            es[kEe + ip] = S.vs_e[ip];
            es[kEk + ip] = S.vs_k[ip];
            es[kEcN + ip] = S.c_n[ip];
            es[kEcM + ip] = S.c_m[ip];
            es[kEc00 + ip] = S.c_f00[ip];
            es[kEc01 + ip] = S.c_f01[ip];
            es[kEc11 + ip] = S.c_f11[ip];
        }
        es[kEcv] = S.c_valid ? 1.0 : 0.0;
        if (el.hard_flag && mode == ELEM_MODE_LIST) el.hard_flag[e] = ctl->fan ? S.hard : 0;
        if (fslot >= 0) {
            atomicAdd(&counters[6], 1ull);
            atomicAdd(&el.fan_finished[cur], 1);  // the fanned element is resolved
        }
    }
    __syncthreads();
    if (S.flag) {
        if (tid == 0) {
            elem_err[e] = ELEM_ERR_FAILED;
            status[E.inst] = 7;
        }
        return;
    }
    if (tid < 36) {
        const int a = tid / 6, b = tid % 6;
        const double* B = S.best;
        const double kb[9] = {B[3], B[4], B[5], B[6], B[7], B[8], B[5], B[8], B[9]};
        double av[3], bv[3];
        basic_map(a, inv_L, av);
        basic_map(b, inv_L, bv);
        S.k[tid] = av[0] * (kb[0] * bv[0] + kb[1] * bv[1] + kb[2] * bv[2]) +
                   av[1] * (kb[3] * bv[0] + kb[4] * bv[1] + kb[5] * bv[2]) +
                   av[2] * (kb[6] * bv[0] + kb[7] * bv[1] + kb[8] * bv[2]);
    }
    __syncthreads();
    if (tid == 0) {
        const double q0 = S.best[0], q1 = S.best[1], q2 = S.best[2];
        if (E.geom == 1) {
            const double ql = q0 * inv_L;
            S.k[1 * 6 + 1] += ql;
            S.k[4 * 6 + 4] += ql;
            S.k[1 * 6 + 4] -= ql;
            S.k[4 * 6 + 1] -= ql;
        }
        S.f[0] = -q0 + 0.0;
        S.f[1] = (q1 + q2) * inv_L + 0.0;
        S.f[2] = q1;
        S.f[3] = q0;
        S.f[4] = -(q1 + q2) * inv_L + 0.0;
        S.f[5] = q2;
        if (E.geom == 1) {
            const double ps = (S.ul[1] - S.ul[4]) * q0 * inv_L;
            S.f[1] += ps;
            S.f[4] -= ps;
        }
        k_to_global(S.k, E.c, E.s);
        f_to_global(S.f, E.c, E.s);
        atomicAdd(&counters[3], (unsigned long long)E.io_bytes);
        atomicAdd(&counters[0], (unsigned long long)S.local_iters);
        atomicMax(&counters[5], (unsigned long long)S.local_iters);
        atomicAdd(&counters[1], (unsigned long long)S.section_evals);
        atomicAdd(&counters[2], (unsigned long long)S.section_evals *
                                    (sd.n_s2 + sd.n_c2 + sd.n_s1 + sd.n_c1 + sd.n_el));
        atomicAdd(&counters[7], (unsigned long long)S.section_evals * section_update_bytes(sd));
    }
    __syncthreads();
    if (tid < 36) ek[E.ek_off + tid] = S.k[tid];
    else if (tid < 42) ef[E.ef_off + tid - 36] = S.f[tid - 36];
    };
    // first element by block index, then dynamically: thread 0 claims the next list entry while
    // the CTA works on the current one (the claim's latency hides behind the element)
    // Tickets beyond the list are attempts of later passes of fanned elements, posted while the
    // launch runs (el.rq); a CTA holding such a ticket waits for its attempt while any fanned
    // element is unresolved.
    int li = blockIdx.x;
    const bool queue = mode == ELEM_MODE_LIST && n_fan > 0 && el.rq != nullptr;
    while (!stop && (li < total || queue)) {
        int item = -1;  // slot x 12 + attempt of a fan-out attempt
        if (li >= total) {
            if (tid == 0) s_item = take_posted(el, cur, li - total, n_fan / kFanAttempts);
            __syncthreads();
            item = s_item;
            __syncthreads();
            if (item < 0) break;
        } else if (mode == ELEM_MODE_LIST && li < n_fan) {
            item = li;
        }
        int claimed = li + gridDim.x;
        if (!all_elems && tid == 0) claimed = atomicAdd(&el.next[cur], 1) + gridDim.x;
        int pe = -1;
        const bool fan_item = item >= 0;
        if (mode == ELEM_MODE_ALL) {
            pe = li;
        } else if (mode == ELEM_MODE_RECORD) {
            pe = rp.list[li];
        } else if (fan_item) {
            pe = el.hard[cur][item / kFanAttempts];
        } else {
            const int ent = el.list[cur][li - n_fan];
            if (!(ent & kFanBit)) pe = ent;
        }
        if (tid == 0) s_fan = 0;
        if (pe >= 0) process(pe, fan_item ? item / kFanAttempts : -1, fan_item ? item % kFanAttempts : 0);
        if (fan_item) {
            __syncthreads();
            // every attempt counts itself in exactly once, whatever path it took
            if (tid == 0 && !s_fan) {
                __threadfence();
                atomicAdd(&el.fan_done[cur * kFanCap + item / kFanAttempts], 1);
            }
        }
        if (tid == 0) s_next = claimed;
        __syncthreads();
        li = s_next;
        __syncthreads();
    }
}

// Commit: recompute each fiber's trial state at the section deformation stored in the element
// state and write it over the committed state (fiber2d.mojo:4191-4221); then the
// forceBeamColumn2d basic-deformation sync from the converged displacements
// (helpers.mojo:1832-1883) and, for recorded elements, the global end forces
// (helpers.mojo:1500-1600 for forceBeamColumn2d; a section evaluation at the converged
// displacements from the new committed state for dispBeamColumn2d).
template <int TEAM>
__global__ void __launch_bounds__(kTeamThreads) commit_kernel(
    const DevElem* __restrict__ elems, Geo g, FiberState fs, const double* __restrict__ u_full,
    double* __restrict__ estate, const int* __restrict__ status, double* __restrict__ rec_base,
    const int* __restrict__ rece_base, int rec_slots, int ef_w, const DevCtl* __restrict__ ctl) {
    __shared__ DevElem E;
    __shared__ DevSection sd;
    __shared__ double resp[kMaxIp][5];
    __shared__ double part[kMaxIp][kVBlocks][6];
    __shared__ double ul[6];
    const int e = blockIdx.x;
    const int tid = threadIdx.x, team = tid / TEAM, r = tid % TEAM;
    double* rec_out = rec_base ? rec_base + (size_t)ctl->step * rec_slots * ef_w : nullptr;
    copy_struct(&E, elems + e);
    __syncthreads();
    if (status[E.inst] != 0) return;
    copy_struct(&sd, g.secs + E.sec);
    __syncthreads();
    const int nip = E.nip;
    const bool three_d = E.nd == 12;
    if (team < nip) {
        // strain of a fiber: eps0 - y kappa (2D); eps0 + z kappa_y - y kappa_z (3D)
        const double* es = estate + (size_t)e * kEStride;
        const double eps0 = three_d ? es[kE3e + team] : es[kEe + team];
        const double kappa = three_d ? es[kE3z + team] : es[kEk + team];
        const double kappa_y = three_d ? es[kE3y + team] : 0.0;
        const double* gz = three_d ? g.z : nullptr;
        auto strain = [&](int gi) {
            const double y = __ldg(g.y + gi);
            return three_d ? eps0 + __ldg(gz + gi) * kappa_y - y * kappa : eps0 - y * kappa;
        };
        int base = sd.geo_off;
        for (int j = r; j < sd.n_s2; j += TEAM) {
            const long long idx = E.s2_off + team * sd.n_s2 + j;
            double* F = fs.s2 + idx;
            const long long N = fs.s2_n;
            S2State c, t;
            c.eps = F[0 * N]; c.sig = F[1 * N]; c.tan = F[2 * N]; c.epsmin = F[3 * N];
            c.epsmax = F[4 * N]; c.epspl = F[5 * N]; c.epss0 = F[6 * N]; c.sigs0 = F[7 * N];
            c.epsr = F[8 * N]; c.sigr = F[9 * N]; c.kon = fs.s2_kon[idx];
            steel02_trial(g.mats[__ldg(g.m + base + j)], c, strain(base + j), t);
            F[0 * N] = t.eps; F[1 * N] = t.sig; F[2 * N] = t.tan; F[3 * N] = t.epsmin;
            F[4 * N] = t.epsmax; F[5 * N] = t.epspl; F[6 * N] = t.epss0; F[7 * N] = t.sigs0;
            F[8 * N] = t.epsr; F[9 * N] = t.sigr; fs.s2_kon[idx] = t.kon;
        }
        base += sd.n_s2;
        for (int j = r; j < sd.n_c2; j += TEAM) {
            const long long idx = E.c2_off + team * sd.n_c2 + j;
            double* F = fs.c2 + idx;
            const long long N = fs.c2_n;
            C2State c, t;
            c.eps = F[0]; c.sig = F[N]; c.tan = F[2 * N]; c.ecmin = F[3 * N]; c.dept = F[4 * N];
            concrete02_trial(g.mats[__ldg(g.m + base + j)], c, strain(base + j), t);
            F[0] = t.eps; F[N] = t.sig; F[2 * N] = t.tan; F[3 * N] = t.ecmin; F[4 * N] = t.dept;
        }
        base += sd.n_c2;
        for (int j = r; j < sd.n_s1; j += TEAM) {
            const long long idx = E.s1_off + team * sd.n_s1 + j;
            double* F = fs.s1 + idx;
            const long long N = fs.s1_n;
            S1State c, t;
            c.eps = F[0]; c.sig = F[N]; c.tan = F[2 * N]; c.epsp = F[3 * N]; c.alpha = F[4 * N];
            steel01_trial(g.mats[__ldg(g.m + base + j)], c, strain(base + j), t);
            F[0] = t.eps; F[N] = t.sig; F[2 * N] = t.tan; F[3 * N] = t.epsp; F[4 * N] = t.alpha;
        }
        base += sd.n_s1;
        for (int j = r; j < sd.n_c1; j += TEAM) {
            const long long idx = E.c1_off + team * sd.n_c1 + j;
            double* F = fs.c1 + idx;
            const long long N = fs.c1_n;
            C1State c, t;
            c.eps = F[0]; c.sig = F[N]; c.tan = F[2 * N]; c.emin = F[3 * N]; c.eend = F[4 * N];
            c.slope = F[5 * N];
            concrete01_trial(g.mats[__ldg(g.m + base + j)], c, strain(base + j), t);
            F[0] = t.eps; F[N] = t.sig; F[2 * N] = t.tan; F[3 * N] = t.emin; F[4 * N] = t.eend;
            F[5 * N] = t.slope;
        }
    }
    if (three_d) {
        // 3D recorders run as a separate pass (element state determination after commit)
        if (tid == 0 && sd.n_s1 > 0) estate[(size_t)e * kEStride + kE3cv] = 0.0;
        return;
    }
    if (tid == 0) {
        double ug[6];
        for (int a = 0; a < 6; ++a) ug[a] = u_full[E.dof[a]];
        // After commit the stored deformations evaluated from the new committed state give the
        // same Concrete02 / Steel02 / Elastic responses bit for bit (zero strain increment);
        // Steel01's return map may move by rounding, so its sections drop the cache.
        if (sd.n_s1 > 0) estate[(size_t)e * kEStride + kEcv] = 0.0;
        if (E.type == 2) {
            u_to_local(E.c_sync, E.s_sync, ug, ul);
            const double chord = (ul[4] - ul[1]) / E.L_sync;
            estate[(size_t)e * kEStride + kEv + 0] = ul[3] - ul[0];
            estate[(size_t)e * kEStride + kEv + 1] = ul[2] - chord;
            estate[(size_t)e * kEStride + kEv + 2] = ul[5] - chord;
            if (E.rec >= 0 && rec_out) {
                const double inv_L = 1.0 / E.L_sync;
                const double q0 = estate[(size_t)e * kEStride + 0];
                const double q1 = estate[(size_t)e * kEStride + 1];
                const double q2 = estate[(size_t)e * kEStride + 2];
                const double shear = (q1 + q2) * inv_L;
                double f[6] = {-q0 + 0.0, shear + 0.0, q1, q0, -shear + 0.0, q2};
                if (E.geom == 1) {
                    const double ps = (ul[1] - ul[4]) * q0 * inv_L;
                    f[1] += ps;
                    f[4] -= ps;
                }
                f_to_global(f, E.c_sync, E.s_sync);
                double* out = rec_out + ((size_t)rece_base[E.inst] + E.rec) * ef_w;
                for (int i = 0; i < 6; ++i) out[i] = f[i];
            }
        } else {
            u_to_local(E.c_div, E.s_div, ug, ul);
        }
    }
    if (E.type != 3 || E.rec < 0 || !rec_out) return;
    __syncthreads();
    // dispBeamColumn2d recorder: section evaluation at the converged displacements from the
    // just-committed state (each thread reads back exactly the fibers it wrote)
    const double L = E.L, inv_L = 1.0 / L, inv_L_sq = inv_L * inv_L;
    if (team < nip) {
        const double xi = E.xi[team];
        const double eps0 = (-inv_L) * ul[0] + inv_L * ul[3];
        const double kappa = curv_shape(1, inv_L, inv_L_sq, xi) * ul[1] +
                             curv_shape(2, inv_L, inv_L_sq, xi) * ul[2] +
                             curv_shape(4, inv_L, inv_L_sq, xi) * ul[4] +
                             curv_shape(5, inv_L, inv_L_sq, xi) * ul[5];
        // StageView over global memory: field stride = family length
        StageView gv;
        gv.c2 = fs.c2 + E.c2_off;
        gv.s2 = fs.s2 + E.s2_off;
        gv.kon = fs.s2_kon + E.s2_off;
        gv.s1 = fs.s1 + E.s1_off;
        gv.c1 = fs.c1 + E.c1_off;
        gv.c2_blk = (int)fs.c2_n;
        gv.s2_blk = (int)fs.s2_n;
        gv.s1_blk = (int)fs.s1_n;
        gv.c1_blk = (int)fs.c1_n;
        section_eval_team<TEAM>(g, sd, gv, team, eps0, kappa, r, part[team]);
    }
    __syncthreads();
    if (team < nip && r == 0) section_finish(sd, part[team], resp[team]);
    __syncthreads();
    if (tid == 0) {
        double f[6] = {0, 0, 0, 0, 0, 0};
        double avg = 0.0;
        for (int ip = 0; ip < nip; ++ip) {
            const double xi = E.xi[ip], wL = E.w[ip] * L;
            avg += E.w[ip] * resp[ip][0];
            for (int a = 0; a < 6; ++a)
                f[a] += wL * (axial_shape(a, inv_L) * resp[ip][0] +
                              curv_shape(a, inv_L, inv_L_sq, xi) * resp[ip][1]);
        }
        if (E.geom == 1) {
            const double ps = (ul[1] - ul[4]) * (avg / L);
            f[1] += ps;
            f[4] -= ps;
        }
        f_to_global(f, E.c_div, E.s_div);
        double* out = rec_out + ((size_t)rece_base[E.inst] + E.rec) * ef_w;
        for (int i = 0; i < 6; ++i) out[i] = f[i];
    }
}

}  // namespace strut

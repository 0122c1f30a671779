// Streaming fiber-state update of many FiberSection2d instances (sm_100a, FP64).
//
// The throughput form of fiber_section2d_set_trial_from_offset
// (src/mojo/sections/fiber2d.mojo:3982-4024, families 1785-1972 and 2301-2516, accumulation
// 1338-1351, elastic fibers 3459-3501) over a batch of instances of one section, each with its
// own committed history: every call reads each fiber's committed state once, computes its trial
// state at eps0 - y kappa, writes it back as the new committed state (commit != 0) and forms each
// instance's resultants and tangent.  Bound: HBM (80 B per Concrete02 fiber, 168 B per Steel02
// fiber, 56 B per Steel01 fiber, 96 B per Concrete01 fiber, read + write).
//
// Layout (BatchState): field f of fiber j of instance i of a family at f * N + i * P + j, with P
// the family's length padded to a multiple of 4 and N = bs.n_inst * P (bs.n_inst: allocated
// instances), so every field of one instance is a contiguous, 16-byte aligned run.
//
// One warp per CTA, as many CTAs per SM as shared memory allows (14 for a 148-fiber section),
// each walking its own instances with a private two-stage pipeline: while the warp updates
// instance k from shared memory, the TMA unit (cp.async.bulk, mbarrier completion, no multicast)
// brings instance k + 1's committed history into the other stage.  No CTA-wide barrier: the
// warps of an SM never wait for one another, so a warp that meets the slow Steel02 branch holds
// up nobody else.  Each lane writes its fibers' new state straight back to HBM (consecutive lanes
// write consecutive fibers, so the stores coalesce), and the per-fiber stress and tangent (times
// area) go to shared memory, from which eight lanes form the instance's sums in the element
// kernel's fixed order (eight chunks of the section's fibers, each summed sequentially, then a
// pairwise tree), so results do not depend on the launch shape.
#pragma once

#include "element_kernels.cuh"
#include "kat_kernels.cuh"

namespace strut {

constexpr int kFsMinCtasPerSm = 16;  // register budget: 128 per thread

__host__ __device__ inline int fs_pad4(int n) { return (n + 3) & ~3; }

// Stage geometry of one instance (identical for every instance of the batch).
struct FsLayout {
    int n_s2, n_c2, n_s1, n_c1, n_el, n_tot;
    int p_s2, p_c2, p_s1, p_c1;                    // padded family lengths
    int off_s2, off_c2, off_s1, off_c1, off_kon;  // offsets in a stage, in doubles
    int stage_doubles;                            // one stage, kon included, a multiple of 2
    uint32_t bytes_s2, bytes_c2, bytes_s1, bytes_c1, bytes_kon, bytes_total;  // per field / stage
};

__host__ __device__ inline FsLayout fs_layout(const DevSection& sd) {
    FsLayout L;
    L.n_s2 = sd.n_s2;
    L.n_c2 = sd.n_c2;
    L.n_s1 = sd.n_s1;
    L.n_c1 = sd.n_c1;
    L.n_el = sd.n_el;
    L.n_tot = sd.n_s2 + sd.n_c2 + sd.n_s1 + sd.n_c1 + sd.n_el;
    L.p_s2 = fs_pad4(sd.n_s2);
    L.p_c2 = fs_pad4(sd.n_c2);
    L.p_s1 = fs_pad4(sd.n_s1);
    L.p_c1 = fs_pad4(sd.n_c1);
    L.off_s2 = 0;
    L.off_c2 = L.off_s2 + 10 * L.p_s2;
    L.off_s1 = L.off_c2 + 5 * L.p_c2;
    L.off_c1 = L.off_s1 + 5 * L.p_s1;
    L.off_kon = L.off_c1 + 6 * L.p_c1;
    L.stage_doubles = L.off_kon + L.p_s2 / 2;
    L.bytes_s2 = 8u * L.p_s2;
    L.bytes_c2 = 8u * L.p_c2;
    L.bytes_s1 = 8u * L.p_s1;
    L.bytes_c1 = 8u * L.p_c1;
    L.bytes_kon = 4u * L.p_s2;
    L.bytes_total = 10u * L.bytes_s2 + 5u * L.bytes_c2 + 5u * L.bytes_s1 + 6u * L.bytes_c1 + L.bytes_kon;
    return L;
}

// Dynamic shared memory of one CTA: two stages and the per-fiber (sig A, tan A) of an instance.
__host__ __device__ inline size_t fs_smem_bytes(const FsLayout& L) {
    return 8u * (2u * (size_t)L.stage_doubles + 2u * (size_t)L.n_tot);
}

// Issues the bulk copies of instance i's committed history into a stage (one lane).
__device__ __forceinline__ void fs_load(const FsLayout& L, const BatchState& bs, long long N2, long long N3,
                                        long long N1, long long N4, long long i, double* st, uint64_t* bar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_arrive_expect_tx(bar, L.bytes_total);
    if (L.bytes_s2) {
        for (int f = 0; f < 10; ++f)
            bulk_g2s(st + L.off_s2 + f * L.p_s2, bs.s2 + f * N2 + i * L.p_s2, L.bytes_s2, bar);
        bulk_g2s(st + L.off_kon, bs.kon + i * L.p_s2, L.bytes_kon, bar);
    }
    if (L.bytes_c2)
        for (int f = 0; f < 5; ++f)
            bulk_g2s(st + L.off_c2 + f * L.p_c2, bs.c2 + f * N3 + i * L.p_c2, L.bytes_c2, bar);
    if (L.bytes_s1)
        for (int f = 0; f < 5; ++f)
            bulk_g2s(st + L.off_s1 + f * L.p_s1, bs.s1 + f * N1 + i * L.p_s1, L.bytes_s1, bar);
    if (L.bytes_c1)
        for (int f = 0; f < 6; ++f)
            bulk_g2s(st + L.off_c1 + f * L.p_c1, bs.c1 + f * N4 + i * L.p_c1, L.bytes_c1, bar);
}

// n_inst instances; ek: n_inst x 2 (eps0, kappa); resp: n_inst x 5 (N, Mz, k11, k12, k22).  CTA c
// takes instances c, c + gridDim.x, ...  *err is set when a bulk copy does not complete within
// the bounded wait.
__global__ void __launch_bounds__(32, kFsMinCtasPerSm) fiber_stream_kernel(Geo g, DevSection sd, BatchState bs,
                                                                           FsLayout L, long long n_inst,
                                                                           const double* __restrict__ ek,
                                                                           double* __restrict__ resp, int commit,
                                                                           int* __restrict__ err) {
    extern __shared__ __align__(128) double fs_smem[];
    __shared__ __align__(8) uint64_t bar[2];
    const int lane = threadIdx.x;
    constexpr unsigned full = 0xffffffffu;
    double* fk = fs_smem + 2 * L.stage_doubles;  // n_tot x {sig A, tan A}
    const long long N2 = bs.n_inst * L.p_s2, N3 = bs.n_inst * L.p_c2, N1 = bs.n_inst * L.p_s1,
                    N4 = bs.n_inst * L.p_c1;
    if (lane == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    __syncwarp();
    long long i = blockIdx.x;
    if (i >= n_inst) return;
    if (lane == 0) fs_load(L, bs, N2, N3, N1, N4, i, fs_smem, &bar[0]);
    // strains of the current instance in lanes 0 (eps0) and 1 (kappa), loaded one instance ahead
    double ek_next = lane < 2 ? __ldg(ek + 2 * i + lane) : 0.0;
    uint32_t phases = 0u;  // bit s: parity of stage s's next completion
    const int geo_c2 = sd.geo_off + L.n_s2, geo_s1 = geo_c2 + L.n_c2, geo_c1 = geo_s1 + L.n_s1,
              geo_el = geo_c1 + L.n_c1;
    const int b_c2 = L.n_s2, b_s1 = b_c2 + L.n_c2, b_c1 = b_s1 + L.n_s1, b_el = b_c1 + L.n_c1;
    for (int k = 0; i < n_inst; ++k, i += gridDim.x) {
        const int s = k & 1;
        const double* st = fs_smem + s * L.stage_doubles;
        const long long nx = i + gridDim.x;
        if (nx < n_inst && lane == 0)
            fs_load(L, bs, N2, N3, N1, N4, nx, fs_smem + (s ^ 1) * L.stage_doubles, &bar[s ^ 1]);
        const double e0 = __shfl_sync(full, ek_next, 0), ka = __shfl_sync(full, ek_next, 1);
        if (nx < n_inst && lane < 2) ek_next = __ldg(ek + 2 * nx + lane);
        const uint32_t ph = (phases >> s) & 1u;
        const bool ok = mbar_wait_bounded(&bar[s], ph);
        phases ^= 1u << s;
        if (__any_sync(full, !ok)) {
            if (lane == 0) {
                *err = 1;
                // let the copies in flight land before the CTA stops
                mbar_wait_bounded(&bar[s], ph);
                if (nx < n_inst) mbar_wait_bounded(&bar[s ^ 1], (phases >> (s ^ 1)) & 1u);
            }
            return;
        }
        // phase 1: every fiber of the instance in section order (Steel02, Concrete02, Steel01,
        // Concrete01, elastic); the new committed state goes back to the same places in HBM
        for (int j = lane; j < L.n_tot; j += 32) {
            double sA, tA;
            if (j < b_c2) {
                const double* F = st + L.off_s2 + j;
                const int gi = sd.geo_off + j;
                const double y = __ldg(g.y + gi), A = __ldg(g.a + gi);
                S2State c, t;
                c.eps = F[0]; c.sig = F[L.p_s2]; c.tan = F[2 * L.p_s2]; c.epsmin = F[3 * L.p_s2];
                c.epsmax = F[4 * L.p_s2]; c.epspl = F[5 * L.p_s2]; c.epss0 = F[6 * L.p_s2];
                c.sigs0 = F[7 * L.p_s2]; c.epsr = F[8 * L.p_s2]; c.sigr = F[9 * L.p_s2];
                c.kon = reinterpret_cast<const int*>(st + L.off_kon)[j];
                steel02_trial(g.mats[__ldg(g.m + gi)], c, e0 - y * ka, t);
                if (commit) {
                    double* G = bs.s2 + i * L.p_s2 + j;
                    G[0] = t.eps; G[N2] = t.sig; G[2 * N2] = t.tan; G[3 * N2] = t.epsmin; G[4 * N2] = t.epsmax;
                    G[5 * N2] = t.epspl; G[6 * N2] = t.epss0; G[7 * N2] = t.sigs0; G[8 * N2] = t.epsr;
                    G[9 * N2] = t.sigr;
                    bs.kon[i * L.p_s2 + j] = t.kon;
                }
                sA = t.sig * A;
                tA = t.tan * A;
            } else if (j < b_s1) {
                const int jj = j - b_c2;
                const double* F = st + L.off_c2 + jj;
                const int gi = geo_c2 + jj;
                const double y = __ldg(g.y + gi), A = __ldg(g.a + gi);
                C2State c, t;
                c.eps = F[0]; c.sig = F[L.p_c2]; c.tan = F[2 * L.p_c2]; c.ecmin = F[3 * L.p_c2];
                c.dept = F[4 * L.p_c2];
                concrete02_trial(g.mats[__ldg(g.m + gi)], c, e0 - y * ka, t);
                if (commit) {
                    double* G = bs.c2 + i * L.p_c2 + jj;
                    G[0] = t.eps; G[N3] = t.sig; G[2 * N3] = t.tan; G[3 * N3] = t.ecmin; G[4 * N3] = t.dept;
                }
                sA = t.sig * A;
                tA = t.tan * A;
            } else if (j < b_c1) {
                const int jj = j - b_s1;
                const double* F = st + L.off_s1 + jj;
                const int gi = geo_s1 + jj;
                const double y = __ldg(g.y + gi), A = __ldg(g.a + gi);
                S1State c, t;
                c.eps = F[0]; c.sig = F[L.p_s1]; c.tan = F[2 * L.p_s1]; c.epsp = F[3 * L.p_s1];
                c.alpha = F[4 * L.p_s1];
                steel01_trial(g.mats[__ldg(g.m + gi)], c, e0 - y * ka, t);
                if (commit) {
                    double* G = bs.s1 + i * L.p_s1 + jj;
                    G[0] = t.eps; G[N1] = t.sig; G[2 * N1] = t.tan; G[3 * N1] = t.epsp; G[4 * N1] = t.alpha;
                }
                sA = t.sig * A;
                tA = t.tan * A;
            } else if (j < b_el) {
                const int jj = j - b_c1;
                const double* F = st + L.off_c1 + jj;
                const int gi = geo_c1 + jj;
                const double y = __ldg(g.y + gi), A = __ldg(g.a + gi);
                C1State c, t;
                c.eps = F[0]; c.sig = F[L.p_c1]; c.tan = F[2 * L.p_c1]; c.emin = F[3 * L.p_c1];
                c.eend = F[4 * L.p_c1]; c.slope = F[5 * L.p_c1];
                concrete01_trial(g.mats[__ldg(g.m + gi)], c, e0 - y * ka, t);
                if (commit) {
                    double* G = bs.c1 + i * L.p_c1 + jj;
                    G[0] = t.eps; G[N4] = t.sig; G[2 * N4] = t.tan; G[3 * N4] = t.emin; G[4 * N4] = t.eend;
                    G[5 * N4] = t.slope;
                }
                sA = t.sig * A;
                tA = t.tan * A;
            } else {
                const int gi = geo_el + (j - b_el);
                const double y = __ldg(g.y + gi), A = __ldg(g.a + gi);
                const double ks = g.mats[__ldg(g.m + gi)].p[0] * A;
                sA = ks * (e0 - y * ka);
                tA = ks;
            }
            fk[2 * j] = sA;
            fk[2 * j + 1] = tA;
        }
        __syncwarp();
        // phase 2: lane b < 8 sums chunk b (the element kernel's order: running sums over a
        // chunk, the elastic fibers' k12 apart, then a pairwise tree over the eight chunks)
        {
            const int n_nl = L.n_tot - L.n_el;
            double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, a4 = 0.0, a5 = 0.0;
            if (lane < 8) {
                const int cs = (L.n_tot + 7) >> 3;
                const int g0 = lane * cs, g1 = min(g0 + cs, L.n_tot);
                const int gm = min(g1, n_nl);
                for (int gg = g0; gg < gm; ++gg) {
                    const double fs = fk[2 * gg], ks = fk[2 * gg + 1], y = __ldg(g.y + sd.geo_off + gg);
                    a0 += fs;
                    a1 += -fs * y;
                    a2 += ks;
                    a3 += -ks * y;
                    a4 += ks * y * y;
                }
                for (int gg = max(g0, n_nl); gg < g1; ++gg) {
                    const double fs = fk[2 * gg], ks = fk[2 * gg + 1], y = __ldg(g.y + sd.geo_off + gg);
                    a0 += fs;
                    a1 += -fs * y;
                    a2 += ks;
                    a5 += -ks * y;
                    a4 += ks * y * y;
                }
            }
            a0 += __shfl_down_sync(full, a0, 1); a1 += __shfl_down_sync(full, a1, 1);
            a2 += __shfl_down_sync(full, a2, 1); a3 += __shfl_down_sync(full, a3, 1);
            a4 += __shfl_down_sync(full, a4, 1); a5 += __shfl_down_sync(full, a5, 1);
            a0 += __shfl_down_sync(full, a0, 2); a1 += __shfl_down_sync(full, a1, 2);
            a2 += __shfl_down_sync(full, a2, 2); a3 += __shfl_down_sync(full, a3, 2);
            a4 += __shfl_down_sync(full, a4, 2); a5 += __shfl_down_sync(full, a5, 2);
            a0 += __shfl_down_sync(full, a0, 4); a1 += __shfl_down_sync(full, a1, 4);
            a2 += __shfl_down_sync(full, a2, 4); a3 += __shfl_down_sync(full, a3, 4);
            a4 += __shfl_down_sync(full, a4, 4); a5 += __shfl_down_sync(full, a5, 4);
            if (lane == 0) {
                double* o = resp + 5 * i;
                o[0] = a0;
                o[1] = a1;
                o[2] = a2;
                o[3] = a3 + (sd.el_uniform ? 0.0 : a5);
                o[4] = a4;
            }
        }
        __syncwarp();  // fk and this stage are rewritten for later instances
    }
}

}  // namespace strut

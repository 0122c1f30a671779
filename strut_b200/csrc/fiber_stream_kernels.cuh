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
// instances, a multiple of the tile), so every field of a tile of kFsTile consecutive instances
// is one contiguous, 16-byte aligned run: one bulk copy per field and tile.
//
// Warp-specialised CTAs, several per SM: kFsTile instance warps, each owning one instance of the
// tile (its Concrete02, Steel01, Concrete01 and elastic fibers, then its sums), and W_s steel
// warps that take the Steel02 fibers of all the tile's instances together, so the expensive
// Menegotto-Pinto branch runs on full warps instead of a few lanes of every instance warp.  Two
// stages: the TMA unit (cp.async.bulk, mbarrier completion, no multicast) brings tile k + 2 into a
// stage as soon as every warp has read tile k from it.  The warps hand work to one another through
// mbarriers only (stage full / stage read / steel results written / sums done), never a CTA-wide
// barrier, so a warp that finishes its part of a tile goes on to the next one.  Each lane writes
// its fibers' new state straight back to HBM (consecutive lanes, consecutive fibers), and the
// per-fiber stress and tangent (times area) go to shared memory, from which eight lanes of the
// instance warp form the sums in the element kernel's fixed order (eight chunks of the section's
// fibers, each summed sequentially, then a pairwise tree), so results do not depend on the launch
// shape.
#pragma once

#include "element_kernels.cuh"
#include "kat_kernels.cuh"

namespace strut {

constexpr int kFsTile = 4;        // instances per tile = instance warps per CTA
constexpr int kFsMaxSteelWarps = 4;

__host__ __device__ inline int fs_pad4(int n) { return (n + 3) & ~3; }

// Stage geometry of one tile (identical for every tile of the batch).
struct FsLayout {
    int n_s2, n_c2, n_s1, n_c1, n_el, n_tot;
    int p_s2, p_c2, p_s1, p_c1;                    // padded family lengths (per instance)
    int off_s2, off_c2, off_s1, off_c1, off_kon;  // offsets in a stage, in doubles
    int stage_doubles;                            // one stage, kon included, a multiple of 2
    int steel_warps;                              // W_s (0 without Steel02 fibers)
    float inv_s2;                                 // 1 / n_s2
    uint32_t bytes_s2, bytes_c2, bytes_s1, bytes_c1, bytes_kon, bytes_total;  // per field / tile
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
    constexpr int T = kFsTile;
    L.off_s2 = 0;
    L.off_c2 = L.off_s2 + 10 * T * L.p_s2;
    L.off_s1 = L.off_c2 + 5 * T * L.p_c2;
    L.off_c1 = L.off_s1 + 5 * T * L.p_s1;
    L.off_kon = L.off_c1 + 6 * T * L.p_c1;
    L.stage_doubles = L.off_kon + T * L.p_s2 / 2;
    const int ws = (T * sd.n_s2 + 31) / 32;
    L.steel_warps = ws < kFsMaxSteelWarps ? ws : kFsMaxSteelWarps;
    L.inv_s2 = sd.n_s2 ? 1.0f / sd.n_s2 : 0.0f;
    L.bytes_s2 = 8u * T * L.p_s2;
    L.bytes_c2 = 8u * T * L.p_c2;
    L.bytes_s1 = 8u * T * L.p_s1;
    L.bytes_c1 = 8u * T * L.p_c1;
    L.bytes_kon = 4u * T * L.p_s2;
    L.bytes_total = 10u * L.bytes_s2 + 5u * L.bytes_c2 + 5u * L.bytes_s1 + 6u * L.bytes_c1 + L.bytes_kon;
    return L;
}

// Threads of a CTA: the instance warps and the steel warps.
__host__ __device__ inline int fs_threads(const FsLayout& L) { return 32 * (kFsTile + L.steel_warps); }

// Dynamic shared memory of one CTA: two stages and, per stage, the per-fiber (sig A, tan A) of
// the tile's instances.
__host__ __device__ inline size_t fs_smem_bytes(const FsLayout& L) {
    return 8u * (2u * (size_t)L.stage_doubles + 2u * (size_t)kFsTile * 2u * (size_t)L.n_tot);
}

// q = r / n for 0 <= r < 2^22 and n >= 1, from a float estimate corrected to the exact quotient.
__device__ __forceinline__ int fs_div(int r, int n, float inv) {
    int q = __float2int_rz(__int2float_rz(r) * inv);
    if (q * n > r) --q;
    else if ((q + 1) * n <= r) ++q;
    return q;
}

__device__ __forceinline__ void fs_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Issues the bulk copies of tile t's committed history into a stage (one lane).
__device__ __forceinline__ void fs_load(const FsLayout& L, const BatchState& bs, long long N2, long long N3,
                                        long long N1, long long N4, long long t, double* st, uint64_t* bar) {
    constexpr int T = kFsTile;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_arrive_expect_tx(bar, L.bytes_total);
    if (L.bytes_s2) {
        for (int f = 0; f < 10; ++f)
            bulk_g2s(st + L.off_s2 + f * T * L.p_s2, bs.s2 + f * N2 + t * T * L.p_s2, L.bytes_s2, bar);
        bulk_g2s(st + L.off_kon, bs.kon + t * T * L.p_s2, L.bytes_kon, bar);
    }
    if (L.bytes_c2)
        for (int f = 0; f < 5; ++f)
            bulk_g2s(st + L.off_c2 + f * T * L.p_c2, bs.c2 + f * N3 + t * T * L.p_c2, L.bytes_c2, bar);
    if (L.bytes_s1)
        for (int f = 0; f < 5; ++f)
            bulk_g2s(st + L.off_s1 + f * T * L.p_s1, bs.s1 + f * N1 + t * T * L.p_s1, L.bytes_s1, bar);
    if (L.bytes_c1)
        for (int f = 0; f < 6; ++f)
            bulk_g2s(st + L.off_c1 + f * T * L.p_c1, bs.c1 + f * N4 + t * T * L.p_c1, L.bytes_c1, bar);
}

// One fiber of a non-Steel02 family of instance i (section index j >= n_s2): trial state from the
// stage at strain e, new committed state to HBM when commit, (sig A, tan A) returned.
__device__ __forceinline__ void fs_other_fiber(const Geo& g, const DevSection& sd, const BatchState& bs,
                                               const FsLayout& L, const double* st, int w, long long i, int j,
                                               double e0, double ka, long long N3, long long N1, long long N4,
                                               int commit, double& sA, double& tA) {
    constexpr int T = kFsTile;
    const int gi = sd.geo_off + j;
    const double y = __ldg(g.y + gi), A = __ldg(g.a + gi);
    const DevMat& mat = g.mats[__ldg(g.m + gi)];
    const double e = e0 - y * ka;
    int jj = j - L.n_s2;
    if (jj < L.n_c2) {
        const int S = T * L.p_c2;
        const double* F = st + L.off_c2 + w * L.p_c2 + jj;
        C2State c, t;
        c.eps = F[0]; c.sig = F[S]; c.tan = F[2 * S]; c.ecmin = F[3 * S]; c.dept = F[4 * S];
        concrete02_trial(mat, c, e, t);
        if (commit) {
            double* G = bs.c2 + i * L.p_c2 + jj;
            G[0] = t.eps; G[N3] = t.sig; G[2 * N3] = t.tan; G[3 * N3] = t.ecmin; G[4 * N3] = t.dept;
        }
        sA = t.sig * A;
        tA = t.tan * A;
        return;
    }
    jj -= L.n_c2;
    if (jj < L.n_s1) {
        const int S = T * L.p_s1;
        const double* F = st + L.off_s1 + w * L.p_s1 + jj;
        S1State c, t;
        c.eps = F[0]; c.sig = F[S]; c.tan = F[2 * S]; c.epsp = F[3 * S]; c.alpha = F[4 * S];
        steel01_trial(mat, c, e, t);
        if (commit) {
            double* G = bs.s1 + i * L.p_s1 + jj;
            G[0] = t.eps; G[N1] = t.sig; G[2 * N1] = t.tan; G[3 * N1] = t.epsp; G[4 * N1] = t.alpha;
        }
        sA = t.sig * A;
        tA = t.tan * A;
        return;
    }
    jj -= L.n_s1;
    if (jj < L.n_c1) {
        const int S = T * L.p_c1;
        const double* F = st + L.off_c1 + w * L.p_c1 + jj;
        C1State c, t;
        c.eps = F[0]; c.sig = F[S]; c.tan = F[2 * S]; c.emin = F[3 * S]; c.eend = F[4 * S]; c.slope = F[5 * S];
        concrete01_trial(mat, c, e, t);
        if (commit) {
            double* G = bs.c1 + i * L.p_c1 + jj;
            G[0] = t.eps; G[N4] = t.sig; G[2 * N4] = t.tan; G[3 * N4] = t.emin; G[4 * N4] = t.eend;
            G[5 * N4] = t.slope;
        }
        sA = t.sig * A;
        tA = t.tan * A;
        return;
    }
    const double ks = mat.p[0] * A;  // elastic
    sA = ks * e;
    tA = ks;
}

// Sums of one instance from its per-fiber (sig A, tan A): lane b < 8 sums chunk b (running sums
// over a chunk, the elastic fibers' k12 apart), then a pairwise tree over the eight chunks; lane 0
// writes N, Mz, k11, k12, k22.  Whole warp.
__device__ __forceinline__ void fs_sums(const Geo& g, const DevSection& sd, const FsLayout& L, const double* fk,
                                        int lane, double* out) {
    constexpr unsigned full = 0xffffffffu;
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
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
        a0 += __shfl_down_sync(full, a0, o);
        a1 += __shfl_down_sync(full, a1, o);
        a2 += __shfl_down_sync(full, a2, o);
        a3 += __shfl_down_sync(full, a3, o);
        a4 += __shfl_down_sync(full, a4, o);
        a5 += __shfl_down_sync(full, a5, o);
    }
    if (lane == 0) {
        out[0] = a0;
        out[1] = a1;
        out[2] = a2;
        out[3] = a3 + (sd.el_uniform ? 0.0 : a5);
        out[4] = a4;
    }
}

// n_inst instances in n_tiles tiles (state allocated for n_tiles * kFsTile instances); ek:
// n_inst x 2 (eps0, kappa); resp: n_inst x 5 (N, Mz, k11, k12, k22).  fs_threads(L) threads; CTA c
// takes tiles c, c + gridDim.x, ...  *err is set when a wait does not complete within its bound
// (the warps then stop; the loading lane first lets its copies in flight land).
__global__ void __launch_bounds__(32 * (kFsTile + kFsMaxSteelWarps), 2)
    fiber_stream_kernel(Geo g, DevSection sd, BatchState bs, FsLayout L, long long n_inst, long long n_tiles,
                        const double* __restrict__ ek, double* __restrict__ resp, int commit,
                        int* __restrict__ err) {
    constexpr int T = kFsTile;
    constexpr unsigned all = 0xffffffffu;
    extern __shared__ __align__(128) double fs_smem[];
    // per stage: full (bulk copies landed), read (every warp has read the stage), steel (the
    // Steel02 results of the tile are in fk), summed (every instance warp has read fk)
    __shared__ __align__(8) uint64_t bar_full[2], bar_read[2], bar_steel[2], bar_summed[2];
    __shared__ double s_ek[kFsMaxSteelWarps][2 * T];  // strains of the tile, per steel warp
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int W = T + L.steel_warps;
    double* const fkb = fs_smem + 2 * L.stage_doubles;  // [stage][instance] x n_tot x {sig A, tan A}
    const long long N2 = bs.n_inst * L.p_s2, N3 = bs.n_inst * L.p_c2, N1 = bs.n_inst * L.p_s1,
                    N4 = bs.n_inst * L.p_c1;
    if (threadIdx.x == 0) {
        for (int s = 0; s < 2; ++s) {
            mbar_init(&bar_full[s], 1);
            mbar_init(&bar_read[s], W);
            mbar_init(&bar_steel[s], L.steel_warps > 0 ? L.steel_warps : 1);
            mbar_init(&bar_summed[s], T);
        }
        mbar_fence_init();
    }
    __syncthreads();  // barrier initialisation: the kernel's only CTA-wide barrier
    const long long t0 = blockIdx.x;
    if (t0 >= n_tiles) return;
    const long long G = gridDim.x;
    // the loading lane (lane 0 of warp 0) tracks the copies it issued and nobody has waited for
    uint32_t pend = 0u, pend_par = 0u;  // bit s: stage s has a copy in flight / its phase parity
    if (threadIdx.x == 0) {
        fs_load(L, bs, N2, N3, N1, N4, t0, fs_smem, &bar_full[0]);
        pend |= 1u;
        if (t0 + G < n_tiles) {
            fs_load(L, bs, N2, N3, N1, N4, t0 + G, fs_smem + L.stage_doubles, &bar_full[1]);
            pend |= 2u;
        }
    }
    bool ok = true;
    if (warp < T) {
        // ---- instance warp w: its instance's non-Steel02 fibers, then its sums
        const int w = warp;
        auto strain = [&](long long t) -> double {
            const long long i = t * T + w;
            return (lane < 2 && t < n_tiles && i < n_inst) ? __ldg(ek + 2 * i + lane) : 0.0;
        };
        double ek_cur = strain(t0);
        for (int k = 0;; ++k) {
            const long long t = t0 + k * G;
            if (t >= n_tiles) break;
            const int s = k & 1;
            const uint32_t par = (uint32_t)(k >> 1) & 1u;
            const double* st = fs_smem + s * L.stage_doubles;
            double* fk = fkb + (size_t)(s * T + w) * 2 * L.n_tot;
            const long long i = t * T + w;
            const bool valid = i < n_inst;
            const double e0 = __shfl_sync(all, ek_cur, 0), ka = __shfl_sync(all, ek_cur, 1);
            ek_cur = strain(t + G);
            ok = __all_sync(all, mbar_wait_bounded(&bar_full[s], par));
            if (!ok) break;
            if (threadIdx.x == 0) pend &= ~(1u << s);
            if (valid)
                for (int j = L.n_s2 + lane; j < L.n_tot; j += 32) {
                    double sA, tA;
                    fs_other_fiber(g, sd, bs, L, st, w, i, j, e0, ka, N3, N1, N4, commit, sA, tA);
                    fk[2 * j] = sA;
                    fk[2 * j + 1] = tA;
                }
            __syncwarp();
            if (lane == 0) fs_arrive(&bar_read[s]);
            if (L.steel_warps) {
                ok = __all_sync(all, mbar_wait_bounded(&bar_steel[s], par));
                if (!ok) break;
            }
            if (valid) fs_sums(g, sd, L, fk, lane, resp + 5 * i);
            __syncwarp();
            if (lane == 0) fs_arrive(&bar_summed[s]);
            // the loading lane refills stage s with tile t + 2G once every warp has read tile t
            if (threadIdx.x == 0 && t + 2 * G < n_tiles) {
                if (mbar_wait_bounded(&bar_read[s], par)) {
                    fs_load(L, bs, N2, N3, N1, N4, t + 2 * G, fs_smem + s * L.stage_doubles, &bar_full[s]);
                    pend |= 1u << s;
                    pend_par = (pend_par & ~(1u << s)) | ((par ^ 1u) << s);
                } else {
                    ok = false;
                }
            }
            ok = __shfl_sync(all, ok ? 1 : 0, 0) != 0;
            if (!ok) break;
        }
    } else {
        // ---- steel warp v: the Steel02 fibers of every instance of the tile
        const int v = warp - T;
        const int n_items = T * L.n_s2;
        auto strains = [&](long long t) -> double {
            const long long q = 2 * t * T + lane;
            return (lane < 2 * T && t < n_tiles && q < 2 * n_inst) ? __ldg(ek + q) : 0.0;
        };
        double ek_cur = strains(t0);
        for (int k = 0;; ++k) {
            const long long t = t0 + k * G;
            if (t >= n_tiles) break;
            const int s = k & 1;
            const uint32_t par = (uint32_t)(k >> 1) & 1u;
            const double* st = fs_smem + s * L.stage_doubles;
            if (lane < 2 * T) s_ek[v][lane] = ek_cur;
            __syncwarp();
            ek_cur = strains(t + G);
            ok = __all_sync(all, mbar_wait_bounded(&bar_full[s], par));
            // fk of this stage is free once the instance warps have summed tile t - 2G
            if (ok && k >= 2) ok = __all_sync(all, mbar_wait_bounded(&bar_summed[s], par ^ 1u));
            if (!ok) break;
            for (int q = v * 32 + lane; q < n_items; q += 32 * L.steel_warps) {
                const int inst = fs_div(q, L.n_s2, L.inv_s2), j = q - inst * L.n_s2;
                const long long i = t * T + inst;
                if (i >= n_inst) continue;
                const int S = T * L.p_s2, x = inst * L.p_s2 + j;
                const double* F = st + L.off_s2 + x;
                const int gi = sd.geo_off + j;
                const double y = __ldg(g.y + gi), A = __ldg(g.a + gi);
                S2State c, tr;
                c.eps = F[0]; c.sig = F[S]; c.tan = F[2 * S]; c.epsmin = F[3 * S]; c.epsmax = F[4 * S];
                c.epspl = F[5 * S]; c.epss0 = F[6 * S]; c.sigs0 = F[7 * S]; c.epsr = F[8 * S]; c.sigr = F[9 * S];
                c.kon = reinterpret_cast<const int*>(st + L.off_kon)[x];
                steel02_trial(g.mats[__ldg(g.m + gi)], c, s_ek[v][2 * inst] - y * s_ek[v][2 * inst + 1], tr);
                if (commit) {
                    double* Gp = bs.s2 + i * L.p_s2 + j;
                    Gp[0] = tr.eps; Gp[N2] = tr.sig; Gp[2 * N2] = tr.tan; Gp[3 * N2] = tr.epsmin;
                    Gp[4 * N2] = tr.epsmax; Gp[5 * N2] = tr.epspl; Gp[6 * N2] = tr.epss0; Gp[7 * N2] = tr.sigs0;
                    Gp[8 * N2] = tr.epsr; Gp[9 * N2] = tr.sigr;
                    bs.kon[i * L.p_s2 + j] = tr.kon;
                }
                double* fk = fkb + (size_t)(s * T + inst) * 2 * L.n_tot;
                fk[2 * j] = tr.sig * A;
                fk[2 * j + 1] = tr.tan * A;
            }
            __syncwarp();
            if (lane == 0) {
                fs_arrive(&bar_read[s]);
                fs_arrive(&bar_steel[s]);
            }
        }
    }
    if (!ok) {
        if (lane == 0) *err = 1;
        // let the copies in flight land before the CTA's shared memory can be released
        if (threadIdx.x == 0)
            for (int s = 0; s < 2; ++s)
                if (pend & (1u << s)) mbar_wait_bounded(&bar_full[s], (pend_par >> s) & 1u);
    }
}

}  // namespace strut

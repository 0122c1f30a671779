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
// Warp-specialised CTAs, several per SM: kFsTile instance warps share the tile's Concrete02,
// Steel01, Concrete01 and elastic fibers (flattened over the tile's instances, so the warps' last
// round is nearly full), and W_s steel warps take the Steel02 fibers of all the tile's instances
// together, so the expensive Menegotto-Pinto branch runs on full warps instead of a few lanes of
// every warp.  Two stages: the TMA unit (cp.async.bulk, mbarrier completion, no multicast) brings
// tile k + 2 into a stage as soon as every warp has read tile k from it.  The warps hand work to
// one another through mbarriers only (stage full / stage read / steel and instance results
// written / sums done), never a CTA-wide barrier: one instance warp per tile forms the four
// instances' sums with all 32 lanes once every result is in, while the others go on to the next
// tile.  Each lane writes its fibers' new state straight back to HBM (consecutive lanes,
// consecutive fibers), and the per-fiber stress and tangent (times area) go to shared memory, from
// which the sums are formed in the element kernel's fixed order (eight chunks of the section's
// fibers, each summed sequentially, then a pairwise tree), so results do not depend on the launch
// shape.  The section's fiber geometry and materials are copied to shared memory once per CTA.
#pragma once

#include "element_kernels.cuh"
#include "kat_kernels.cuh"

namespace strut {

constexpr int kFsTile = 4;        // instances per tile = instance warps per CTA
constexpr int kFsMaxSteelWarps = 4;
constexpr int kFsMaxMats = 16;    // materials copied to shared memory (more: read from global)

__host__ __device__ inline int fs_pad4(int n) { return (n + 3) & ~3; }

// Stage geometry of one tile (identical for every tile of the batch).
struct FsLayout {
    int n_s2, n_c2, n_s1, n_c1, n_el, n_tot;
    int p_s2, p_c2, p_s1, p_c1;                    // padded family lengths (per instance)
    int off_s2, off_c2, off_s1, off_c1, off_kon;  // offsets in a stage, in doubles
    int stage_doubles;                            // one stage, kon included, a multiple of 2
    int steel_warps;                              // W_s (0 without Steel02 fibers)
    int n_mats;                                   // materials of the batch
    int n_oth;                                    // non-Steel02 fibers of a section
    float inv_s2, inv_oth;                        // 1 / n_s2, 1 / n_oth
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
    L.n_mats = 0;
    L.n_oth = L.n_tot - sd.n_s2;
    L.inv_s2 = sd.n_s2 ? 1.0f / sd.n_s2 : 0.0f;
    L.inv_oth = L.n_oth ? 1.0f / L.n_oth : 0.0f;
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

// Dynamic shared memory of one CTA: two stages; per stage, the per-fiber (sig A, tan A) of the
// tile's instances; the section's fiber y and area; the materials (when at most kFsMaxMats); the
// fibers' material indices.
__host__ __device__ inline size_t fs_fk_doubles(const FsLayout& L) { return 2u * kFsTile * 2u * (size_t)L.n_tot; }
__host__ __device__ inline size_t fs_geo_doubles(const FsLayout& L) {
    return 2u * (size_t)L.n_tot + (L.n_mats <= kFsMaxMats ? (sizeof(DevMat) / 8) * (size_t)L.n_mats : 0u);
}
__host__ __device__ inline size_t fs_smem_bytes(const FsLayout& L) {
    return 8u * (2u * (size_t)L.stage_doubles + fs_fk_doubles(L) + fs_geo_doubles(L)) + 4u * (size_t)L.n_tot;
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


// The section's fiber geometry as the kernel reads it (shared memory).
struct FsGeo {
    const double* y;
    const double* a;
    const int* m;
    const DevMat* mats;
};

// One fiber of a non-Steel02 family of tile instance w (global instance i, section index
// j >= n_s2): trial state from the stage at strain e0 - y ka, new committed state to HBM when
// commit, (sig A, tan A) returned.
__device__ __forceinline__ void fs_other_fiber(const FsGeo& G, const BatchState& bs, const FsLayout& L,
                                               const double* st, int w, long long i, int j, double e0, double ka,
                                               long long N3, long long N1, long long N4, int commit, double& sA,
                                               double& tA) {
    constexpr int T = kFsTile;
    const double y = G.y[j], A = G.a[j];
    const DevMat& mat = G.mats[G.m[j]];
    const double e = e0 - y * ka;
    int jj = j - L.n_s2;
    if (jj < L.n_c2) {
        const int S = T * L.p_c2;
        const double* F = st + L.off_c2 + w * L.p_c2 + jj;
        C2State c, t;
        c.eps = F[0]; c.sig = F[S]; c.tan = F[2 * S]; c.ecmin = F[3 * S]; c.dept = F[4 * S];
        concrete02_trial(mat, c, e, t);
        if (commit) {
            double* Gp = bs.c2 + i * L.p_c2 + jj;
            Gp[0] = t.eps; Gp[N3] = t.sig; Gp[2 * N3] = t.tan; Gp[3 * N3] = t.ecmin; Gp[4 * N3] = t.dept;
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
            double* Gp = bs.s1 + i * L.p_s1 + jj;
            Gp[0] = t.eps; Gp[N1] = t.sig; Gp[2 * N1] = t.tan; Gp[3 * N1] = t.epsp; Gp[4 * N1] = t.alpha;
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
            double* Gp = bs.c1 + i * L.p_c1 + jj;
            Gp[0] = t.eps; Gp[N4] = t.sig; Gp[2 * N4] = t.tan; Gp[3 * N4] = t.emin; Gp[4 * N4] = t.eend;
            Gp[5 * N4] = t.slope;
        }
        sA = t.sig * A;
        tA = t.tan * A;
        return;
    }
    const double ks = mat.p[0] * A;  // elastic
    sA = ks * e;
    tA = ks;
}

// Sums of the tile's instances with one warp: lane 8 w + b sums chunk b of instance w (running
// sums over a chunk, the elastic fibers' k12 apart), then each instance's eight chunks are added
// by a pairwise tree; lane 8 w writes N, Mz, k11, k12, k22 of instance w (when valid).
__device__ __forceinline__ void fs_sums(const FsGeo& G, const DevSection& sd, const FsLayout& L, const double* fk,
                                        int lane, int n_valid, double* out) {
    constexpr unsigned full = 0xffffffffu;
    const int w = lane >> 3, b = lane & 7;
    const int n_nl = L.n_tot - L.n_el;
    const double* f = fk + (size_t)w * 2 * L.n_tot;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, a4 = 0.0, a5 = 0.0;
    if (w < n_valid) {
        const int cs = (L.n_tot + 7) >> 3;
        const int g0 = b * cs, g1 = min(g0 + cs, L.n_tot);
        const int gm = min(g1, n_nl);
        for (int gg = g0; gg < gm; ++gg) {
            const double fs = f[2 * gg], ks = f[2 * gg + 1], y = G.y[gg];
            a0 += fs;
            a1 += -fs * y;
            a2 += ks;
            a3 += -ks * y;
            a4 += ks * y * y;
        }
        for (int gg = max(g0, n_nl); gg < g1; ++gg) {
            const double fs = f[2 * gg], ks = f[2 * gg + 1], y = G.y[gg];
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
    if (b == 0 && w < n_valid) {
        double* o = out + 5 * w;
        o[0] = a0;
        o[1] = a1;
        o[2] = a2;
        o[3] = a3 + (sd.el_uniform ? 0.0 : a5);
        o[4] = a4;
    }
}

// n_inst instances in n_tiles tiles (state allocated for n_tiles * kFsTile instances); ek:
// n_inst x 2 (eps0, kappa); resp: n_inst x 5 (N, Mz, k11, k12, k22).  fs_threads(L) threads; CTA c
// takes tiles c, c + gridDim.x, ...  *err is set when a wait does not complete within its bound
// (the warps then stop together; the loading lane first lets its copies in flight land).
__global__ void __launch_bounds__(32 * (kFsTile + kFsMaxSteelWarps), 2)
    fiber_stream_kernel(Geo g, DevSection sd, BatchState bs, FsLayout L, long long n_inst, long long n_tiles,
                        const double* __restrict__ ek, double* __restrict__ resp, int commit,
                        int* __restrict__ err) {
    constexpr int T = kFsTile;
    constexpr unsigned all = 0xffffffffu;
    extern __shared__ __align__(128) double fs_smem[];
    // per stage: full (bulk copies landed), read (every warp has read the stage), steel / inst
    // (the steel / instance warps' results of the tile are in fk), summed (the tile's sums have
    // read fk)
    __shared__ __align__(8) uint64_t bar_full[2], bar_read[2], bar_steel[2], bar_inst[2], bar_summed[2];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int W = T + L.steel_warps;
    double* const fkb = fs_smem + 2 * L.stage_doubles;  // [stage][instance] x n_tot x {sig A, tan A}
    double* const gy = fkb + fs_fk_doubles(L);
    double* const ga = gy + L.n_tot;
    DevMat* const gm = reinterpret_cast<DevMat*>(ga + L.n_tot);
    int* const gmi = reinterpret_cast<int*>(gy + fs_geo_doubles(L));
    FsGeo G;
    G.y = gy;
    G.a = ga;
    G.m = gmi;
    G.mats = L.n_mats <= kFsMaxMats ? gm : g.mats;
    const long long N2 = bs.n_inst * L.p_s2, N3 = bs.n_inst * L.p_c2, N1 = bs.n_inst * L.p_s1,
                    N4 = bs.n_inst * L.p_c1;
    for (int j = threadIdx.x; j < L.n_tot; j += blockDim.x) {
        gy[j] = __ldg(g.y + sd.geo_off + j);
        ga[j] = __ldg(g.a + sd.geo_off + j);
        gmi[j] = __ldg(g.m + sd.geo_off + j);
    }
    if (L.n_mats <= kFsMaxMats)
        for (int q = threadIdx.x; q < L.n_mats * (int)(sizeof(DevMat) / 4); q += blockDim.x)
            reinterpret_cast<uint32_t*>(gm)[q] = __ldg(reinterpret_cast<const uint32_t*>(g.mats) + q);
    if (threadIdx.x == 0) {
        for (int s = 0; s < 2; ++s) {
            mbar_init(&bar_full[s], 1);
            mbar_init(&bar_read[s], W);
            mbar_init(&bar_steel[s], L.steel_warps > 0 ? L.steel_warps : 1);
            mbar_init(&bar_inst[s], T);
            mbar_init(&bar_summed[s], 1);
        }
        mbar_fence_init();
    }
    __syncthreads();  // geometry and barrier initialisation: the kernel's only CTA-wide barrier
    const long long t0 = blockIdx.x;
    if (t0 >= n_tiles) return;
    const long long G_ = gridDim.x;
    // the loading lane (lane 0 of warp 0) tracks the copies it issued and nobody has waited for
    uint32_t pend = 0u, pend_par = 0u;  // bit s: stage s has a copy in flight / its phase parity
    if (threadIdx.x == 0) {
        fs_load(L, bs, N2, N3, N1, N4, t0, fs_smem, &bar_full[0]);
        pend |= 1u;
        if (t0 + G_ < n_tiles) {
            fs_load(L, bs, N2, N3, N1, N4, t0 + G_, fs_smem + L.stage_doubles, &bar_full[1]);
            pend |= 2u;
        }
    }
    // strains of tile t: thread q < 2T of a warp loads value q (instance q / 2 of the tile)
    auto strains = [&](long long t) -> double {
        const long long q = 2 * t * T + lane;
        return (lane < 2 * T && t < n_tiles && q < 2 * n_inst) ? __ldg(ek + q) : 0.0;
    };
    bool ok = true;
    if (warp < T) {
        // ---- instance warps: the tile's non-Steel02 fibers, then (one warp per tile) the sums
        const int w = warp;
        const int n_items = T * L.n_oth;
        double ek_cur = strains(t0);
        for (int k = 0;; ++k) {
            const long long t = t0 + k * G_;
            if (t >= n_tiles) break;
            const int s = k & 1;
            const uint32_t par = (uint32_t)(k >> 1) & 1u;
            const double* st = fs_smem + s * L.stage_doubles;
            double* fk = fkb + (size_t)s * T * 2 * L.n_tot;
            const int n_valid = (int)min((long long)T, n_inst - t * T);
            const double ek_here = ek_cur;  // lanes 2q, 2q + 1: eps0, kappa of tile instance q
            ek_cur = strains(t + G_);
            ok = __all_sync(all, mbar_wait_bounded(&bar_full[s], par));
            // fk of this stage is free once the sums of tile t - 2G have read it
            if (ok && k >= 2) ok = __all_sync(all, mbar_wait_bounded(&bar_summed[s], par ^ 1u));
            if (!ok) break;
            if (threadIdx.x == 0) pend &= ~(1u << s);
            for (int base = w * 32; base < n_items; base += 32 * T) {
                const int q = base + lane;
                const int inst = q < n_items ? fs_div(q, L.n_oth, L.inv_oth) : 0;
                const double e0 = __shfl_sync(all, ek_here, 2 * inst), ka = __shfl_sync(all, ek_here, 2 * inst + 1);
                if (q >= n_items || inst >= n_valid) continue;
                const int j = L.n_s2 + (q - inst * L.n_oth);
                double sA, tA;
                fs_other_fiber(G, bs, L, st, inst, t * T + inst, j, e0, ka, N3, N1, N4, commit, sA, tA);
                double* f = fk + (size_t)inst * 2 * L.n_tot;
                f[2 * j] = sA;
                f[2 * j + 1] = tA;
            }
            __syncwarp();
            if (lane == 0) {
                fs_arrive(&bar_read[s]);
                fs_arrive(&bar_inst[s]);
            }
            // one warp per tile forms the sums once every warp's results are in fk; the others go
            // on to the next tile
            if (w == (k & (T - 1))) {
                ok = __all_sync(all, mbar_wait_bounded(&bar_inst[s], par));
                if (ok && L.steel_warps) ok = __all_sync(all, mbar_wait_bounded(&bar_steel[s], par));
                if (!ok) break;
                fs_sums(G, sd, L, fk, lane, n_valid, resp + 5 * t * T);
                __syncwarp();
                if (lane == 0) fs_arrive(&bar_summed[s]);
            }
            // the loading lane refills stage s with tile t + 2G once every warp has read tile t
            if (threadIdx.x == 0 && t + 2 * G_ < n_tiles) {
                if (mbar_wait_bounded(&bar_read[s], par)) {
                    fs_load(L, bs, N2, N3, N1, N4, t + 2 * G_, fs_smem + s * L.stage_doubles, &bar_full[s]);
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
        double ek_cur = strains(t0);
        for (int k = 0;; ++k) {
            const long long t = t0 + k * G_;
            if (t >= n_tiles) break;
            const int s = k & 1;
            const uint32_t par = (uint32_t)(k >> 1) & 1u;
            const double* st = fs_smem + s * L.stage_doubles;
            double* fk = fkb + (size_t)s * T * 2 * L.n_tot;
            // the tile's strains, one instance per lane pair; lanes read them by shuffle below
            const double ek_here = ek_cur;
            ek_cur = strains(t + G_);
            ok = __all_sync(all, mbar_wait_bounded(&bar_full[s], par));
            // fk of this stage is free once the sums of tile t - 2G have read it
            if (ok && k >= 2) ok = __all_sync(all, mbar_wait_bounded(&bar_summed[s], par ^ 1u));
            if (!ok) break;
            for (int base = v * 32; base < n_items; base += 32 * L.steel_warps) {
                const int q = base + lane;
                const int inst = q < n_items ? fs_div(q, L.n_s2, L.inv_s2) : 0;
                const double e0 = __shfl_sync(all, ek_here, 2 * inst), ka = __shfl_sync(all, ek_here, 2 * inst + 1);
                if (q >= n_items) continue;
                const int j = q - inst * L.n_s2;
                const long long i = t * T + inst;
                if (i >= n_inst) continue;
                const int S = T * L.p_s2, x = inst * L.p_s2 + j;
                const double* F = st + L.off_s2 + x;
                const double y = G.y[j], A = G.a[j];
                S2State c, tr;
                c.eps = F[0]; c.sig = F[S]; c.tan = F[2 * S]; c.epsmin = F[3 * S]; c.epsmax = F[4 * S];
                c.epspl = F[5 * S]; c.epss0 = F[6 * S]; c.sigs0 = F[7 * S]; c.epsr = F[8 * S]; c.sigr = F[9 * S];
                c.kon = reinterpret_cast<const int*>(st + L.off_kon)[x];
                steel02_trial(G.mats[G.m[j]], c, e0 - y * ka, tr);
                if (commit) {
                    double* Gp = bs.s2 + i * L.p_s2 + j;
                    Gp[0] = tr.eps; Gp[N2] = tr.sig; Gp[2 * N2] = tr.tan; Gp[3 * N2] = tr.epsmin;
                    Gp[4 * N2] = tr.epsmax; Gp[5 * N2] = tr.epspl; Gp[6 * N2] = tr.epss0; Gp[7 * N2] = tr.sigs0;
                    Gp[8 * N2] = tr.epsr; Gp[9 * N2] = tr.sigr;
                    bs.kon[i * L.p_s2 + j] = tr.kon;
                }
                double* f = fk + (size_t)inst * 2 * L.n_tot;
                f[2 * j] = tr.sig * A;
                f[2 * j + 1] = tr.tan * A;
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

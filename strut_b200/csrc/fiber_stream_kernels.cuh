// Streaming fiber-state update of many FiberSection2d instances (sm_100a, FP64).
//
// The throughput form of fiber_section2d_set_trial_from_offset
// (src/mojo/sections/fiber2d.mojo:3982-4024, families 1785-1972 and 2301-2516, accumulation
// 1338-1351, elastic fibers 3459-3501) over a batch of instances of one section, each with its
// own committed history: every call reads each fiber's committed state once, computes its trial
// state at eps0 - y kappa, writes it back as the new committed state (commit != 0) and forms each
// instance's resultants and tangent.  Bound: HBM (80 B per Concrete02 fiber, 168 B per Steel02
// fiber, read + write).
//
// Layout (BatchState): family field f of fiber j of instance i at f * N + i * n_fam + j with
// N = n_alloc * n_fam, n_alloc a multiple of the tile, so the fibers of a tile of consecutive
// instances are one contiguous 16-byte aligned run per field.
//
// Persistent CTAs (one of 512 threads or two of 256 per SM) walk the instance tiles with a
// two-stage pipeline: while the threads update tile k in shared memory, the TMA unit
// (cp.async.bulk, mbarrier completion, no multicast) brings tile k + 1 in; each thread writes its
// fibers' new state straight back to HBM (a warp's stores are consecutive, so they coalesce), so a
// stage is free again as soon as it has been read.  With two CTAs per SM one CTA's section sums
// and barriers overlap the other's fiber updates.  Inside a tile every thread takes fibers of the flattened (family, instance, fiber)
// order, so a warp's shared-memory accesses are consecutive; the per-fiber stress and tangent (times area) go
// to shared memory and each instance's sums are formed in the element kernel's fixed order (eight
// chunks of the section's fibers, each summed sequentially, then a pairwise tree), so results do
// not depend on the launch shape.
#pragma once

#include "element_kernels.cuh"
#include "kat_kernels.cuh"

namespace strut {

constexpr int kFsThreads = 512;      // one CTA per SM
constexpr int kFsThreadsPair = 256;  // two CTAs per SM
constexpr int kFsTileQuantum = 48;   // instances are allocated in multiples of every tile size (4..16)

// Per-tile geometry of the stage buffers, identical for every tile.
struct FsLayout {
    int T;                       // instances per tile (a multiple of 4)
    int n_s2, n_c2, n_s1, n_c1, n_el, n_tot;
    int off_c2, off_s2, off_s1, off_c1, off_kon;  // offsets in a stage, in doubles
    int stage_doubles;           // one stage, kon included, rounded to 16 bytes
    uint32_t bytes_c2, bytes_s2, bytes_s1, bytes_c1, bytes_kon;  // per field per tile
    float inv_s2, inv_c2, inv_s1, inv_c1, inv_el;  // 1 / family length (0 for an empty family)
};

// q = r / n for 0 <= r < 2^22 and n >= 1, from a float estimate corrected to the exact quotient.
__device__ __forceinline__ int fs_div(int r, int n, float inv) {
    int q = __float2int_rz(__int2float_rz(r) * inv);
    if (q * n > r) --q;
    else if ((q + 1) * n <= r) ++q;
    return q;
}

__host__ __device__ inline FsLayout fs_layout(const DevSection& sd, int T) {
    FsLayout L;
    L.T = T;
    L.n_s2 = sd.n_s2;
    L.n_c2 = sd.n_c2;
    L.n_s1 = sd.n_s1;
    L.n_c1 = sd.n_c1;
    L.n_el = sd.n_el;
    L.n_tot = sd.n_s2 + sd.n_c2 + sd.n_s1 + sd.n_c1 + sd.n_el;
    L.off_c2 = 0;
    L.off_s2 = L.off_c2 + 5 * T * sd.n_c2;
    L.off_s1 = L.off_s2 + 10 * T * sd.n_s2;
    L.off_c1 = L.off_s1 + 5 * T * sd.n_s1;
    L.off_kon = L.off_c1 + 6 * T * sd.n_c1;
    const int kon_doubles = (T * sd.n_s2 + 1) / 2;
    L.stage_doubles = (L.off_kon + kon_doubles + 1) & ~1;
    L.bytes_c2 = 8u * T * sd.n_c2;
    L.bytes_s2 = 8u * T * sd.n_s2;
    L.bytes_s1 = 8u * T * sd.n_s1;
    L.bytes_c1 = 8u * T * sd.n_c1;
    L.bytes_kon = 4u * T * sd.n_s2;
    L.inv_s2 = sd.n_s2 ? 1.0f / sd.n_s2 : 0.0f;
    L.inv_c2 = sd.n_c2 ? 1.0f / sd.n_c2 : 0.0f;
    L.inv_s1 = sd.n_s1 ? 1.0f / sd.n_s1 : 0.0f;
    L.inv_c1 = sd.n_c1 ? 1.0f / sd.n_c1 : 0.0f;
    L.inv_el = sd.n_el ? 1.0f / sd.n_el : 0.0f;
    return L;
}

// Dynamic shared memory: two stages, the per-fiber (sig A, tan A) of a tile, the strains.
__host__ __device__ inline size_t fs_smem_bytes(const FsLayout& L) {
    return 8u * (2u * L.stage_doubles + 2u * L.T * L.n_tot + 2u * L.T);
}

// Issues the bulk copies of tile `tile` of every family field into a stage (thread 0).
__device__ __forceinline__ void fs_load_tile(const FsLayout& L, const BatchState& bs, long long N2, long long N3,
                                             long long N1, long long N4, long long tile, double* st,
                                             uint64_t* bar) {
    const uint32_t total = 5 * L.bytes_c2 + 10 * L.bytes_s2 + 5 * L.bytes_s1 + 6 * L.bytes_c1 + L.bytes_kon;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_arrive_expect_tx(bar, total);
    const long long T = L.T;
    for (int f = 0; f < 5 && L.bytes_c2; ++f)
        bulk_g2s(st + L.off_c2 + f * T * L.n_c2, bs.c2 + f * N3 + tile * T * L.n_c2, L.bytes_c2, bar);
    for (int f = 0; f < 10 && L.bytes_s2; ++f)
        bulk_g2s(st + L.off_s2 + f * T * L.n_s2, bs.s2 + f * N2 + tile * T * L.n_s2, L.bytes_s2, bar);
    if (L.bytes_kon) bulk_g2s(st + L.off_kon, bs.kon + tile * T * L.n_s2, L.bytes_kon, bar);
    for (int f = 0; f < 5 && L.bytes_s1; ++f)
        bulk_g2s(st + L.off_s1 + f * T * L.n_s1, bs.s1 + f * N1 + tile * T * L.n_s1, L.bytes_s1, bar);
    for (int f = 0; f < 6 && L.bytes_c1; ++f)
        bulk_g2s(st + L.off_c1 + f * T * L.n_c1, bs.c1 + f * N4 + tile * T * L.n_c1, L.bytes_c1, bar);
}

// n_inst instances (state allocated for bs.n_inst >= n_tiles * T); ek: n_inst x 2 (eps0,
// kappa); resp: n_inst x 5 (N, Mz, k11, k12, k22).  *err is set when a bulk copy does not complete
// within the bounded wait.  THREADS x MINB = 512 threads per SM: both shapes have the same
// register budget (128 per thread).
template <int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) fiber_stream_kernel(Geo g, DevSection sd, BatchState bs, FsLayout L,
                                                                  long long n_inst, long long n_tiles,
                                                                  const double* __restrict__ ek,
                                                                  double* __restrict__ resp, int commit,
                                                                  int* __restrict__ err) {
    extern __shared__ __align__(128) double fs_smem[];
    __shared__ __align__(8) uint64_t bar[2];
    const int tid = threadIdx.x;
    constexpr int nt = THREADS;
    const int T = L.T;
    double* fk = fs_smem + 2 * L.stage_doubles;  // T x n_tot x {sig A, tan A}
    double* strain = fk + 2 * T * L.n_tot;       // T x {eps0, kappa}
    const long long n_alloc = bs.n_inst;  // allocated instances: the field stride
    const long long N2 = n_alloc * L.n_s2, N3 = n_alloc * L.n_c2, N1 = n_alloc * L.n_s1, N4 = n_alloc * L.n_c1;
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    long long tile = blockIdx.x;
    if (tile >= n_tiles) return;
    if (tid == 0) fs_load_tile(L, bs, N2, N3, N1, N4, tile, fs_smem, &bar[0]);
    uint32_t phases = 0u;  // bit s: parity of stage s's next completion
    const int geo_s2 = sd.geo_off, geo_c2 = geo_s2 + L.n_s2, geo_s1 = geo_c2 + L.n_c2, geo_c1 = geo_s1 + L.n_s1,
              geo_el = geo_c1 + L.n_c1;
    for (int k = 0; tile < n_tiles; ++k, tile += gridDim.x) {
        const int s = k & 1;
        double* st = fs_smem + s * L.stage_doubles;
        const long long next = tile + gridDim.x;
        if (next < n_tiles && tid == 0)
            fs_load_tile(L, bs, N2, N3, N1, N4, next, fs_smem + (s ^ 1) * L.stage_doubles, &bar[s ^ 1]);
        const long long i0 = tile * T;
        const int nvalid = (int)min((long long)T, n_inst - i0);
        for (int t = tid; t < 2 * T; t += nt) strain[t] = t < 2 * nvalid ? ek[2 * i0 + t] : 0.0;
        const uint32_t ph = (phases >> s) & 1u;
        const bool ok = mbar_wait_bounded(&bar[s], ph);
        phases ^= 1u << s;
        if (__syncthreads_or(ok ? 0 : 1)) {
            if (tid == 0) {
                *err = 1;
                // let the copies in flight land before the CTA stops
                mbar_wait_bounded(&bar[s], ph);
                if (next < n_tiles) mbar_wait_bounded(&bar[s ^ 1], (phases >> (s ^ 1)) & 1u);
            }
            return;
        }
        // phase 1: every fiber of the tile, flattened family by family; the new committed state
        // goes to the same places in HBM (Xg: this tile's fibers of family X, field stride NX)
        const int n_s2t = T * L.n_s2, n_c2t = T * L.n_c2, n_s1t = T * L.n_s1, n_c1t = T * L.n_c1, n_elt = T * L.n_el;
        double* const S2g = bs.s2 + tile * n_s2t;
        int* const Kg = bs.kon + tile * n_s2t;
        double* const C2g = bs.c2 + tile * n_c2t;
        double* const S1g = bs.s1 + tile * n_s1t;
        double* const C1g = bs.c1 + tile * n_c1t;
        const int n_items = n_s2t + n_c2t + n_s1t + n_c1t + n_elt;
        for (int it = tid; it < n_items; it += nt) {
            int r = it;
            if (r < n_s2t) {
                const int si = fs_div(r, L.n_s2, L.inv_s2), j = r - si * L.n_s2;
                if (si < nvalid) {
                    const double* F = st + L.off_s2 + r;
                    const int* K = reinterpret_cast<const int*>(st + L.off_kon) + r;
                    const int gi = geo_s2 + j;
                    const double y = __ldg(g.y + gi), A = __ldg(g.a + gi);
                    S2State c, t;
                    c.eps = F[0 * n_s2t]; c.sig = F[1 * n_s2t]; c.tan = F[2 * n_s2t]; c.epsmin = F[3 * n_s2t];
                    c.epsmax = F[4 * n_s2t]; c.epspl = F[5 * n_s2t]; c.epss0 = F[6 * n_s2t];
                    c.sigs0 = F[7 * n_s2t]; c.epsr = F[8 * n_s2t]; c.sigr = F[9 * n_s2t]; c.kon = *K;
                    steel02_trial(g.mats[__ldg(g.m + gi)], c, strain[2 * si] - y * strain[2 * si + 1], t);
                    if (commit) {
                        double* G = S2g + r;
                        G[0 * N2] = t.eps; G[1 * N2] = t.sig; G[2 * N2] = t.tan; G[3 * N2] = t.epsmin;
                        G[4 * N2] = t.epsmax; G[5 * N2] = t.epspl; G[6 * N2] = t.epss0;
                        G[7 * N2] = t.sigs0; G[8 * N2] = t.epsr; G[9 * N2] = t.sigr; Kg[r] = t.kon;
                    }
                    double* o = fk + 2 * (si * L.n_tot + j);
                    o[0] = t.sig * A;
                    o[1] = t.tan * A;
                }
                continue;
            }
            r -= n_s2t;
            if (r < n_c2t) {
                const int si = fs_div(r, L.n_c2, L.inv_c2), j = r - si * L.n_c2;
                if (si < nvalid) {
                    const double* F = st + L.off_c2 + r;
                    const int gi = geo_c2 + j;
                    const double y = __ldg(g.y + gi), A = __ldg(g.a + gi);
                    C2State c, t;
                    c.eps = F[0]; c.sig = F[n_c2t]; c.tan = F[2 * n_c2t]; c.ecmin = F[3 * n_c2t]; c.dept = F[4 * n_c2t];
                    concrete02_trial(g.mats[__ldg(g.m + gi)], c, strain[2 * si] - y * strain[2 * si + 1], t);
                    if (commit) {
                        double* G = C2g + r;
                        G[0] = t.eps; G[N3] = t.sig; G[2 * N3] = t.tan; G[3 * N3] = t.ecmin; G[4 * N3] = t.dept;
                    }
                    double* o = fk + 2 * (si * L.n_tot + L.n_s2 + j);
                    o[0] = t.sig * A;
                    o[1] = t.tan * A;
                }
                continue;
            }
            r -= n_c2t;
            if (r < n_s1t) {
                const int si = fs_div(r, L.n_s1, L.inv_s1), j = r - si * L.n_s1;
                if (si < nvalid) {
                    const double* F = st + L.off_s1 + r;
                    const int gi = geo_s1 + j;
                    const double y = __ldg(g.y + gi), A = __ldg(g.a + gi);
                    S1State c, t;
                    c.eps = F[0]; c.sig = F[n_s1t]; c.tan = F[2 * n_s1t]; c.epsp = F[3 * n_s1t]; c.alpha = F[4 * n_s1t];
                    steel01_trial(g.mats[__ldg(g.m + gi)], c, strain[2 * si] - y * strain[2 * si + 1], t);
                    if (commit) {
                        double* G = S1g + r;
                        G[0] = t.eps; G[N1] = t.sig; G[2 * N1] = t.tan; G[3 * N1] = t.epsp; G[4 * N1] = t.alpha;
                    }
                    double* o = fk + 2 * (si * L.n_tot + L.n_s2 + L.n_c2 + j);
                    o[0] = t.sig * A;
                    o[1] = t.tan * A;
                }
                continue;
            }
            r -= n_s1t;
            if (r < n_c1t) {
                const int si = fs_div(r, L.n_c1, L.inv_c1), j = r - si * L.n_c1;
                if (si < nvalid) {
                    const double* F = st + L.off_c1 + r;
                    const int gi = geo_c1 + j;
                    const double y = __ldg(g.y + gi), A = __ldg(g.a + gi);
                    C1State c, t;
                    c.eps = F[0]; c.sig = F[n_c1t]; c.tan = F[2 * n_c1t]; c.emin = F[3 * n_c1t];
                    c.eend = F[4 * n_c1t]; c.slope = F[5 * n_c1t];
                    concrete01_trial(g.mats[__ldg(g.m + gi)], c, strain[2 * si] - y * strain[2 * si + 1], t);
                    if (commit) {
                        double* G = C1g + r;
                        G[0] = t.eps; G[N4] = t.sig; G[2 * N4] = t.tan; G[3 * N4] = t.emin; G[4 * N4] = t.eend;
                        G[5 * N4] = t.slope;
                    }
                    double* o = fk + 2 * (si * L.n_tot + L.n_s2 + L.n_c2 + L.n_s1 + j);
                    o[0] = t.sig * A;
                    o[1] = t.tan * A;
                }
                continue;
            }
            r -= n_c1t;
            {
                const int si = fs_div(r, L.n_el, L.inv_el), j = r - si * L.n_el;
                if (si >= nvalid) continue;
                const int gi = geo_el + j;
                const double y = __ldg(g.y + gi), A = __ldg(g.a + gi);
                const double ks = g.mats[__ldg(g.m + gi)].p[0] * A;
                double* o = fk + 2 * (si * L.n_tot + L.n_tot - L.n_el + j);
                o[0] = ks * (strain[2 * si] - y * strain[2 * si + 1]);
                o[1] = ks;
            }
        }
        __syncthreads();
        // phase 2: thread t < 8 T sums chunk t % 8 of instance t / 8 (the element kernel's order:
        // running sums over a chunk, the elastic fibers' k12 apart, then a pairwise tree)
        {
            const int n_sum = 8 * T;
            const int n_nl = L.n_tot - L.n_el;
            for (int base = 0; base < n_sum; base += nt) {
                const int t = base + tid;
                if ((t & ~31) >= n_sum) break;  // whole warp outside
                const bool act = t < n_sum;
                const int si = t >> 3, b = t & 7;
                double a[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                if (act && si < nvalid) {
                    const int cs = (L.n_tot + 7) >> 3;
                    const int g0 = b * cs, g1 = min(g0 + cs, L.n_tot);
                    const double* f = fk + 2 * si * L.n_tot;
                    const int gm = min(g1, n_nl);
                    for (int gg = g0; gg < gm; ++gg) {
                        const double fs = f[2 * gg], ks = f[2 * gg + 1], y = __ldg(g.y + sd.geo_off + gg);
                        a[0] += fs;
                        a[1] += -fs * y;
                        a[2] += ks;
                        a[3] += -ks * y;
                        a[4] += ks * y * y;
                    }
                    for (int gg = max(g0, n_nl); gg < g1; ++gg) {
                        const double fs = f[2 * gg], ks = f[2 * gg + 1], y = __ldg(g.y + sd.geo_off + gg);
                        a[0] += fs;
                        a[1] += -fs * y;
                        a[2] += ks;
                        a[5] += -ks * y;
                        a[4] += ks * y * y;
                    }
                }
#pragma unroll
                for (int c = 0; c < 6; ++c) {
                    double p = a[c];
                    p += __shfl_down_sync(0xffffffffu, p, 1);
                    p += __shfl_down_sync(0xffffffffu, p, 2);
                    p += __shfl_down_sync(0xffffffffu, p, 4);
                    a[c] = p;
                }
                if (act && b == 0 && si < nvalid) {
                    double* o = resp + 5 * (i0 + si);
                    o[0] = a[0];
                    o[1] = a[1];
                    o[2] = a[2];
                    o[3] = a[3] + (sd.el_uniform ? 0.0 : a[5]);
                    o[4] = a[4];
                }
            }
        }
        __syncthreads();  // fk, strain and this stage are rewritten for later tiles
    }
}

}  // namespace strut

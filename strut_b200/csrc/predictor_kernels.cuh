// Learned Newton predictor: per-node features and the network's increments back to a displacement
// guess.
//
// Features of node p at step s (the step being computed, t = (s + 1) dt), n_in = 4 ndf + 17:
//   the converged increments of its ndf dofs at steps s-1, s-2, s-3, s-4 (0 for a constrained dof
//   or a step before the first), ground acceleration at steps s, s-1, ..., s-15 (one excitation)
//   or of each of the two components at steps s .. s-7 (0 before the record), the node height
//   over the instance's height; each normalised (x - mean) * scale.
// The network predicts, per dof and in units of y_scale, the correction the converged increment
// of step s needs over the Newmark predictor's (the plain predictor stays the reference point).  Strut has no
// learned predictor; the feature set is the one of the north-star configuration (2D: one ground
// component; 41 features for a 3D node).
#pragma once

#include "kernels.cuh"

namespace strut {

struct PredDev {
    int n_nodes, ndf, n_in, n_free, n_inst, ag_len;
    const int* node_free;   // n_nodes x ndf: global free index or -1
    const int* node_inst;
    const float* node_h;
    const float* x_mean;    // n_in
    const float* x_scale;   // n_in
    const float* y_scale;   // ndf
    const double* hist_du;  // 4 x n_free (slot = step % 4)
    const double* ag_full;  // 2 x n_inst x ag_len: ground acceleration of step s, per component
    const int* inst_comp;   // n_inst: excitation components of the instance (1 or 2)
};

__global__ void pred_features_kernel(PredDev P, const DevCtl* __restrict__ ctl, float* __restrict__ x) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P.n_nodes) return;
    const int s = ctl->step;
    const int inst = P.node_inst[p];
    float* xr = x + (size_t)p * P.n_in;
    int k = 0;
    for (int j = 0; j < 4; ++j) {
        const int sj = s - 1 - j;
        for (int d = 0; d < P.ndf; ++d, ++k) {
            const int fi = P.node_free[p * P.ndf + d];
            double v = 0.0;
            if (fi >= 0 && sj >= 0) v = P.hist_du[(size_t)(sj & 3) * P.n_free + fi];
            xr[k] = ((float)v - P.x_mean[k]) * P.x_scale[k];
        }
    }
    // one component: its 16 latest samples; two: the 8 latest of each
    const int two = P.inst_comp[inst] == 2;
    for (int j = 0; j < 16; ++j, ++k) {
        const int c = two ? j / 8 : 0, sj = s - (two ? j % 8 : j);
        const double v = (sj >= 0 && sj < P.ag_len) ? P.ag_full[((size_t)c * P.n_inst + inst) * P.ag_len + sj] : 0.0;
        xr[k] = ((float)v - P.x_mean[k]) * P.x_scale[k];
    }
    xr[k] = (P.node_h[p] - P.x_mean[k]) * P.x_scale[k];
}

// The learned guess: u += y * y_scale on the free dofs of every predicted node, u holding the
// Newmark predictor the step starts from (the network predicts the correction to it).  Each free
// dof belongs to one node, so every entry is updated by one thread.
__global__ void pred_scatter_kernel(PredDev P, const float* __restrict__ y, double* __restrict__ u_f,
                                    const int* __restrict__ free_dof, double* __restrict__ u_full) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= P.n_nodes * P.ndf) return;
    const int p = q / P.ndf, d = q % P.ndf;
    const int fi = P.node_free[p * P.ndf + d];
    if (fi < 0) return;
    const double u = u_f[fi] + (double)y[(size_t)p * P.ndf + d] * (double)P.y_scale[d];
    u_f[fi] = u;
    u_full[free_dof[fi]] = u;
}

__global__ void copy_doubles_kernel(const double* __restrict__ src, double* __restrict__ dst, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

}  // namespace strut

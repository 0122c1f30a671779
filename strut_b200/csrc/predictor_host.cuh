// Host side of the learned Newton predictor on an analysis handle (included once, by
// strut_cuda.cu, after the network's host code).
#pragma once

struct PredState {
    StrutMlp* mlp = nullptr;  // not owned
    strut::PredDev P{};
    int n_tiles = 0;
    std::vector<void*> allocs;
    float* d_x = nullptr;
    __nv_bfloat16* d_xt = nullptr;
    float* d_y = nullptr;
    long long* d_stats = nullptr;
    int* d_rejected = nullptr;
    int* d_skip = nullptr;
    bool owns_base = false;  // u_base / estate_base were allocated for the predictor
    ~PredState() {
        for (void* p : allocs) cudaFree(p);
    }
};

static void pred_free(PredState* p) { delete p; }

namespace {

template <typename T>
int pred_alloc(PredState* ps, T** p, size_t n) {
    CK(cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T)));
    CK(cudaMemset(*p, 0, std::max<size_t>(n, 1) * sizeof(T)));
    ps->allocs.push_back(*p);
    return STRUT_OK;
}


}  // namespace

// Feature and network launches after the Newmark predictor kernel of a step: the learned guess
// replaces the predictor's displacements (which u_base keeps) on every predicted free dof.
static int pred_launch(StrutHandle* h) {
    PredState* ps = h->pred;
    const int tb = 256;
    pred_features_kernel<<<(ps->P.n_nodes + tb - 1) / tb, tb, 0, h->stream>>>(ps->P, h->d_ctl, ps->d_x);
    const long long tot = (long long)ps->n_tiles * kMlpTile * kMlpKin;
    mlp_pack_x_kernel<<<(unsigned)((tot + tb - 1) / tb), tb, 0, h->stream>>>(ps->d_x, ps->P.n_nodes, ps->P.n_in,
                                                                            ps->d_xt, ps->n_tiles);
    mlp_forward_kernel<<<ps->n_tiles, 128, kMlpFwdSmem, h->stream>>>(ps->mlp->dev(), ps->d_xt, ps->P.n_nodes,
                                                                      ps->d_y, ps->P.ndf, ps->mlp->d_err);
    const int nq = ps->P.n_nodes * ps->P.ndf;
    pred_scatter_kernel<<<(nq + tb - 1) / tb, tb, 0, h->stream>>>(ps->P, ps->d_y, h->A.u_f, h->A.free_dof,
                                                                 h->A.u_full);
    CK(cudaGetLastError());
    if (h->n_slaves_total > 0) {
        // a learned value of a slave dof is overwritten by its constraint (helpers.mojo:3380-3400)
        slave_enforce_kernel<<<(h->n_slaves_total + tb - 1) / tb, tb, 0, h->stream>>>(h->A, h->n_slaves_total);
        CK(cudaGetLastError());
    }
    return STRUT_OK;
}

static int pred_add_nodes(StrutHandle* h, cudaGraph_t body, cudaGraphNode_t dep, cudaGraphNode_t* last) {
    PredState* ps = h->pred;
    const int tb = 256;
    cudaGraphNode_t c, d, e, f;
    TRY(add_kernel_node(&c, body, &dep, 1, pred_features_kernel, dim3((ps->P.n_nodes + tb - 1) / tb), dim3(tb), 0,
                        ps->P, (const DevCtl*)h->d_ctl, ps->d_x));
    const long long tot = (long long)ps->n_tiles * kMlpTile * kMlpKin;
    TRY(add_kernel_node(&d, body, &c, 1, mlp_pack_x_kernel, dim3((unsigned)((tot + tb - 1) / tb)), dim3(tb), 0,
                        (const float*)ps->d_x, ps->P.n_nodes, ps->P.n_in, ps->d_xt, ps->n_tiles));
    TRY(add_kernel_node(&e, body, &d, 1, mlp_forward_kernel, dim3(ps->n_tiles), dim3(128), (size_t)kMlpFwdSmem,
                        ps->mlp->dev(), (const __nv_bfloat16*)ps->d_xt, ps->P.n_nodes, ps->d_y, ps->P.ndf,
                        ps->mlp->d_err));
    const int nq = ps->P.n_nodes * ps->P.ndf;
    TRY(add_kernel_node(&f, body, &e, 1, pred_scatter_kernel, dim3((nq + tb - 1) / tb), dim3(tb), 0, ps->P,
                        (const float*)ps->d_y, h->A.u_f, (const int*)h->A.free_dof, h->A.u_full));
    *last = f;
    if (h->n_slaves_total > 0) {
        cudaGraphNode_t g;
        TRY(add_kernel_node(&g, body, &f, 1, slave_enforce_kernel, dim3((h->n_slaves_total + tb - 1) / tb), dim3(tb),
                            0, h->A, h->n_slaves_total));
        *last = g;
    }
    return STRUT_OK;
}

extern "C" {

int strut_gpu_set_predictor(StrutHandle* h, StrutMlp* m, const float* x_mean, const float* x_scale,
                            const float* y_scale) {
    if (!h) return fail(STRUT_BAD_ARG, "bad arguments");
    if (h->pred) {
        pred_free(h->pred);
        h->pred = nullptr;
    }
    h->A.dual = 0;
    h->A.hist_du = nullptr;
    h->A.pred_stats = nullptr;
    h->A.rejected = nullptr;
    h->A.skip = nullptr;
    if (h->pred_owns_base) {
        h->A.u_base = nullptr;
        h->A.estate_base = nullptr;
        h->pred_owns_base = false;
    }
    if (!m) return STRUT_OK;  // detached: the plain method
    if (h->ndf_all < 0) return fail(STRUT_UNSUPPORTED, "the learned predictor needs instances of one ndf");
    for (const DevInst& I : h->insts)
        for (int k = 0; k < I.n_att; ++k)
            if (I.att_alg[k] != STRUT_ALGORITHM_NEWTON)
                return fail(STRUT_UNSUPPORTED, "the learned predictor runs with the Newton algorithm");
    const int ndf = h->pn_ndf, n_in = 4 * ndf + 17;
    if (m->n_in != n_in || m->n_out != ndf)
        return fail(STRUT_BAD_ARG, "network must take " + std::to_string(n_in) + " features and give " +
                                       std::to_string(ndf) + " outputs");
    if (!x_mean || !x_scale || !y_scale) return fail(STRUT_BAD_ARG, "normalisation arrays required");
    PredState* ps = new PredState();
    ps->mlp = m;
    const int nn = (int)h->pn_inst.size();
    ps->n_tiles = (nn + kMlpTile - 1) / kMlpTile;
    // ground acceleration of every step of every instance, per excitation component, as the
    // step loop evaluates it: t = (s + 1) dt
    int ag_len = 1;
    for (int i = 0; i < h->n_inst; ++i)
        for (int c = 0; c < h->exc[i].num; ++c) {
            const StrutExcitation& x = h->exc[i].x[c];
            ag_len = std::max(ag_len, (int)std::ceil(x.count * x.dt / h->insts[i].dt) + 2);
        }
    std::vector<double> ag((size_t)2 * h->n_inst * ag_len, 0.0);
    std::vector<int> comp(h->n_inst, 1);
    for (int i = 0; i < h->n_inst; ++i) {
        comp[i] = h->exc[i].num == 2 ? 2 : 1;
        for (int c = 0; c < h->exc[i].num; ++c)
            for (int s = 0; s < ag_len; ++s)
                ag[((size_t)c * h->n_inst + i) * ag_len + s] = path_eval(h->exc[i].x[c], (s + 1) * h->insts[i].dt);
    }
    int rc = STRUT_OK;
    auto bail = [&](int code) {
        delete ps;
        return code;
    };
    int *d_nf, *d_ni, *d_comp;
    float *d_nh, *d_xm, *d_xs, *d_ys;
    double *d_hist, *d_ag;
    if ((rc = pred_alloc(ps, &d_nf, h->pn_free.size())) || (rc = pred_alloc(ps, &d_ni, (size_t)nn)) ||
        (rc = pred_alloc(ps, &d_nh, (size_t)nn)) || (rc = pred_alloc(ps, &d_xm, (size_t)n_in)) ||
        (rc = pred_alloc(ps, &d_xs, (size_t)n_in)) || (rc = pred_alloc(ps, &d_ys, (size_t)ndf)) ||
        (rc = pred_alloc(ps, &d_hist, (size_t)4 * h->n_free_total)) || (rc = pred_alloc(ps, &d_ag, ag.size())) ||
        (rc = pred_alloc(ps, &d_comp, comp.size())) ||
        (rc = pred_alloc(ps, &ps->d_x, (size_t)nn * n_in)) ||
        (rc = pred_alloc(ps, &ps->d_xt, (size_t)ps->n_tiles * kMlpBytesX / 2)) ||
        (rc = pred_alloc(ps, &ps->d_y, (size_t)nn * ndf)) ||
        (rc = pred_alloc(ps, &ps->d_stats, (size_t)2 * h->n_inst)) ||
        (rc = pred_alloc(ps, &ps->d_rejected, (size_t)h->n_inst)) || (rc = pred_alloc(ps, &ps->d_skip, (size_t)h->n_inst)))
        return bail(rc);
    double* d_u_base = h->A.u_base;
    double* d_estate_base = h->A.estate_base;
    if (!d_u_base) {
        // the predictor's displacements and the element state at the step's start, for the
        // return to the plain predictor
        if ((rc = pred_alloc(ps, &d_u_base, (size_t)h->n_free_total)) ||
            (rc = pred_alloc(ps, &d_estate_base, (size_t)h->n_elem * kEStride)))
            return bail(rc);
        ps->owns_base = true;
    }
    auto up = [&](void* dst, const void* src, size_t bytes) -> int {
        CK(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
        return STRUT_OK;
    };
    if ((rc = up(d_nf, h->pn_free.data(), h->pn_free.size() * 4)) || (rc = up(d_ni, h->pn_inst.data(), (size_t)nn * 4)) ||
        (rc = up(d_nh, h->pn_h.data(), (size_t)nn * 4)) || (rc = up(d_xm, x_mean, (size_t)n_in * 4)) ||
        (rc = up(d_xs, x_scale, (size_t)n_in * 4)) || (rc = up(d_ys, y_scale, (size_t)ndf * 4)) ||
        (rc = up(d_ag, ag.data(), ag.size() * 8)) || (rc = up(d_comp, comp.data(), comp.size() * 4)))
        return bail(rc);
    ps->P = PredDev{nn, ndf, n_in, h->n_free_total, h->n_inst, ag_len, d_nf, d_ni, d_nh, d_xm, d_xs, d_ys,
                    d_hist, d_ag, d_comp};
    h->pred = ps;
    h->A.dual = 1;
    h->A.rejected = ps->d_rejected;
    h->A.skip = ps->d_skip;
    h->A.u_base = d_u_base;
    h->A.estate_base = d_estate_base;
    h->pred_owns_base = ps->owns_base;
    h->A.pred_stats = ps->d_stats;
    h->A.hist_du = d_hist;
    return STRUT_OK;
}

int32_t strut_gpu_predictor_nodes(const StrutHandle* h) { return h ? (int32_t)h->pn_inst.size() : -1; }

int strut_gpu_predictor_stats(const StrutHandle* h, int64_t* offered, int64_t* chosen) {
    if (!h || !offered || !chosen) return fail(STRUT_BAD_ARG, "bad arguments");
    *offered = 0;
    *chosen = 0;
    if (!h->pred) return STRUT_OK;
    std::vector<long long> st((size_t)2 * h->n_inst);
    CK(cudaMemcpy(st.data(), h->pred->d_stats, st.size() * 8, cudaMemcpyDeviceToHost));
    for (int i = 0; i < h->n_inst; ++i) {
        *offered += st[2 * i];
        *chosen += st[2 * i + 1];
    }
    return STRUT_OK;
}

int strut_gpu_predictor_features(StrutHandle* h, float* out) {
    if (!h || !out || !h->pred) return fail(STRUT_BAD_ARG, "no predictor attached");
    PredState* ps = h->pred;
    DevCtl c;
    CK(cudaMemcpy(&c, h->d_ctl, sizeof(c), cudaMemcpyDeviceToHost));
    c.step = h->steps_done;  // features of the next step
    CK(cudaMemcpy(h->d_ctl, &c, sizeof(c), cudaMemcpyHostToDevice));
    pred_features_kernel<<<(ps->P.n_nodes + 255) / 256, 256, 0, h->stream>>>(ps->P, h->d_ctl, ps->d_x);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(out, ps->d_x, (size_t)ps->P.n_nodes * ps->P.n_in * 4, cudaMemcpyDeviceToHost));
    return STRUT_OK;
}

}  // extern "C"

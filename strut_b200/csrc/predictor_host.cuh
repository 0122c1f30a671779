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
    double* d_u_alt_f = nullptr;
    double* d_u_alt_full = nullptr;
    double* d_estate_alt = nullptr;
    double* d_ek_alt = nullptr;
    double* d_ef_alt = nullptr;
    long long* d_stats = nullptr;
    int* d_next_alt = nullptr;
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

ElemList alt_list(const StrutHandle* h) {
    ElemList el = h->A.el;
    el.next = h->pred->d_next_alt;
    return el;
}

}  // namespace

// Feature and network launches plus the element evaluation of the learned guess, after the
// Newmark predictor kernel of a step.
static int pred_launch(StrutHandle* h) {
    PredState* ps = h->pred;
    const int tb = 256;
    const long long ne = (long long)h->n_elem * kEStride;
    copy_doubles_kernel<<<592, tb, 0, h->stream>>>(h->d_estate, ps->d_estate_alt, ne);
    copy_doubles_kernel<<<148, tb, 0, h->stream>>>(h->A.u_full, ps->d_u_alt_full, h->n_dofs_total);
    pred_features_kernel<<<(ps->P.n_nodes + tb - 1) / tb, tb, 0, h->stream>>>(ps->P, h->d_ctl, h->A.status,
                                                                             ps->d_x, ps->d_next_alt);
    const long long tot = (long long)ps->n_tiles * kMlpTile * kMlpKin;
    mlp_pack_x_kernel<<<(unsigned)((tot + tb - 1) / tb), tb, 0, h->stream>>>(ps->d_x, ps->P.n_nodes, ps->P.n_in,
                                                                            ps->d_xt, ps->n_tiles);
    mlp_forward_kernel<<<ps->n_tiles, 128, kMlpFwdSmem, h->stream>>>(ps->mlp->dev(), ps->d_xt, ps->P.n_nodes,
                                                                      ps->d_y, ps->P.ndf, ps->mlp->d_err);
    const int nq = ps->P.n_nodes * ps->P.ndf;
    pred_scatter_kernel<<<(nq + tb - 1) / tb, tb, 0, h->stream>>>(ps->P, ps->d_y, h->A.u_f, h->A.free_dof,
                                                                 ps->d_u_alt_f, ps->d_u_alt_full);
    elem_kernel_of(h)<<<h->elem_grid, elem_block(h), h->elem_smem, h->stream>>>(
        h->d_elems, h->geo, h->fs, ps->d_u_alt_full, ps->d_estate_alt, ps->d_ek_alt, ps->d_ef_alt, h->A.active,
        h->A.status, h->d_elem_err, h->d_counters, alt_list(h), (const DevCtl*)h->d_ctl,
        (int)ELEM_MODE_LIST, h->n_elem, rec_pass_of(h));
    CK(cudaGetLastError());
    return STRUT_OK;
}

static int pred_add_nodes(StrutHandle* h, cudaGraph_t body, cudaGraphNode_t dep, cudaGraphNode_t* last) {
    PredState* ps = h->pred;
    const int tb = 256;
    const long long ne = (long long)h->n_elem * kEStride;
    cudaGraphNode_t a, b, c, d, e, f, g;
    TRY(add_kernel_node(&a, body, &dep, 1, copy_doubles_kernel, dim3(592), dim3(tb), 0, (const double*)h->d_estate,
                        ps->d_estate_alt, ne));
    TRY(add_kernel_node(&b, body, &a, 1, copy_doubles_kernel, dim3(148), dim3(tb), 0, (const double*)h->A.u_full,
                        ps->d_u_alt_full, (long long)h->n_dofs_total));
    TRY(add_kernel_node(&c, body, &b, 1, pred_features_kernel, dim3((ps->P.n_nodes + tb - 1) / tb), dim3(tb), 0,
                        ps->P, (const DevCtl*)h->d_ctl, (const int*)h->A.status, ps->d_x, ps->d_next_alt));
    const long long tot = (long long)ps->n_tiles * kMlpTile * kMlpKin;
    TRY(add_kernel_node(&d, body, &c, 1, mlp_pack_x_kernel, dim3((unsigned)((tot + tb - 1) / tb)), dim3(tb), 0,
                        (const float*)ps->d_x, ps->P.n_nodes, ps->P.n_in, ps->d_xt, ps->n_tiles));
    TRY(add_kernel_node(&e, body, &d, 1, mlp_forward_kernel, dim3(ps->n_tiles), dim3(128), (size_t)kMlpFwdSmem,
                        ps->mlp->dev(), (const __nv_bfloat16*)ps->d_xt, ps->P.n_nodes, ps->d_y, ps->P.ndf,
                        ps->mlp->d_err));
    const int nq = ps->P.n_nodes * ps->P.ndf;
    TRY(add_kernel_node(&f, body, &e, 1, pred_scatter_kernel, dim3((nq + tb - 1) / tb), dim3(tb), 0, ps->P,
                        (const float*)ps->d_y, (const double*)h->A.u_f, (const int*)h->A.free_dof, ps->d_u_alt_f,
                        ps->d_u_alt_full));
    TRY(add_kernel_node(&g, body, &f, 1, elem_kernel_of(h), dim3(h->elem_grid), elem_block(h), h->elem_smem,
                        (const DevElem*)h->d_elems, h->geo, h->fs, (const double*)ps->d_u_alt_full, ps->d_estate_alt,
                        ps->d_ek_alt, ps->d_ef_alt, (const int*)h->A.active, h->A.status, h->d_elem_err,
                        h->d_counters, alt_list(h), (const DevCtl*)h->d_ctl, (int)ELEM_MODE_LIST, h->n_elem,
                        rec_pass_of(h)));
    *last = g;
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
    if (!m) return STRUT_OK;  // detached: the plain method
    if (h->ndf_all < 0) return fail(STRUT_UNSUPPORTED, "the learned predictor needs instances of one ndf");
    if (h->n_large > 0)
        return fail(STRUT_UNSUPPORTED, "the learned predictor runs on instances whose band fits in shared memory");
    if (h->n_slaves_total > 0)
        return fail(STRUT_UNSUPPORTED, "the learned predictor does not run with multi-point constraints");
    if (h->n_shells > 0) return fail(STRUT_UNSUPPORTED, "the learned predictor does not run with shells");
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
    // ground acceleration of every step of every instance (first excitation), as the step loop
    // evaluates it: t = (s + 1) dt
    int ag_len = 1;
    for (int i = 0; i < h->n_inst; ++i)
        if (h->exc[i].num > 0) {
            const StrutExcitation& x = h->exc[i].x[0];
            ag_len = std::max(ag_len, (int)std::ceil(x.count * x.dt / h->insts[i].dt) + 2);
        }
    std::vector<double> ag((size_t)h->n_inst * ag_len, 0.0);
    for (int i = 0; i < h->n_inst; ++i)
        if (h->exc[i].num > 0)
            for (int s = 0; s < ag_len; ++s) ag[(size_t)i * ag_len + s] = path_eval(h->exc[i].x[0], (s + 1) * h->insts[i].dt);
    int rc = STRUT_OK;
    auto bail = [&](int code) {
        delete ps;
        return code;
    };
    int *d_nf, *d_ni;
    float *d_nh, *d_xm, *d_xs, *d_ys;
    double *d_hist, *d_ag;
    if ((rc = pred_alloc(ps, &d_nf, h->pn_free.size())) || (rc = pred_alloc(ps, &d_ni, (size_t)nn)) ||
        (rc = pred_alloc(ps, &d_nh, (size_t)nn)) || (rc = pred_alloc(ps, &d_xm, (size_t)n_in)) ||
        (rc = pred_alloc(ps, &d_xs, (size_t)n_in)) || (rc = pred_alloc(ps, &d_ys, (size_t)ndf)) ||
        (rc = pred_alloc(ps, &d_hist, (size_t)4 * h->n_free_total)) || (rc = pred_alloc(ps, &d_ag, ag.size())) ||
        (rc = pred_alloc(ps, &ps->d_x, (size_t)nn * n_in)) ||
        (rc = pred_alloc(ps, &ps->d_xt, (size_t)ps->n_tiles * kMlpBytesX / 2)) ||
        (rc = pred_alloc(ps, &ps->d_y, (size_t)nn * ndf)) || (rc = pred_alloc(ps, &ps->d_u_alt_f, (size_t)h->n_free_total)) ||
        (rc = pred_alloc(ps, &ps->d_u_alt_full, (size_t)h->n_dofs_total)) ||
        (rc = pred_alloc(ps, &ps->d_estate_alt, (size_t)h->n_elem * kEStride)) ||
        (rc = pred_alloc(ps, &ps->d_ek_alt, (size_t)h->ek_total)) ||
        (rc = pred_alloc(ps, &ps->d_ef_alt, (size_t)h->ef_total)) ||
        (rc = pred_alloc(ps, &ps->d_stats, (size_t)2 * h->n_inst)) || (rc = pred_alloc(ps, &ps->d_next_alt, 2)))
        return bail(rc);
    auto up = [&](void* dst, const void* src, size_t bytes) -> int {
        CK(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
        return STRUT_OK;
    };
    if ((rc = up(d_nf, h->pn_free.data(), h->pn_free.size() * 4)) || (rc = up(d_ni, h->pn_inst.data(), (size_t)nn * 4)) ||
        (rc = up(d_nh, h->pn_h.data(), (size_t)nn * 4)) || (rc = up(d_xm, x_mean, (size_t)n_in * 4)) ||
        (rc = up(d_xs, x_scale, (size_t)n_in * 4)) || (rc = up(d_ys, y_scale, (size_t)ndf * 4)) ||
        (rc = up(d_ag, ag.data(), ag.size() * 8)))
        return bail(rc);
    ps->P = PredDev{nn, ndf, n_in, h->n_free_total, h->n_inst, ag_len, d_nf, d_ni, d_nh, d_xm, d_xs, d_ys,
                    d_hist, d_ag};
    h->pred = ps;
    h->A.dual = 1;
    h->A.u_alt_f = ps->d_u_alt_f;
    h->A.ek_alt = ps->d_ek_alt;
    h->A.ef_alt = ps->d_ef_alt;
    h->A.estate_alt = ps->d_estate_alt;
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
    pred_features_kernel<<<(ps->P.n_nodes + 255) / 256, 256, 0, h->stream>>>(ps->P, h->d_ctl, h->A.status, ps->d_x,
                                                                             ps->d_next_alt);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(out, ps->d_x, (size_t)ps->P.n_nodes * ps->P.n_in * 4, cudaMemcpyDeviceToHost));
    return STRUT_OK;
}

}  // extern "C"

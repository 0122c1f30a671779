"""Learned Newton predictor: training data from the plain method's converged histories, feature
normalisation, and attaching a trained network to an analysis.

The predictor proposes each step's displacement increment node by node and the step starts from
that guess; its first Newton iteration compares the guess's residual with the plain Newmark
predictor's, estimated to first order from the tangent assembled at the guess, and goes back to
the plain predictor when the learned residual is the larger.  Newton converges to the same
NormDispIncr tolerance either way and the plain predictor is the fallback.  Strut has no learned predictor (this follows the north-star
configuration's network and features); the analysis path it plugs into is Strut's
transient_nonlinear Newton loop (src/mojo/solver/run_case/analysis/transient_nonlinear.mojo).

Features of a node at step s (n_in = 4 ndf + 17), matching the device's pred_features_kernel:
the converged increments of its ndf dofs at steps s-1 .. s-4, the ground acceleration at steps
s .. s-15 (t = (k + 1) dt), and the node height over the frame height.  Target: the correction the
node's converged increment at step s needs over the Newmark predictor's increment
dt v_{s-1} + dt^2 (1/2 - beta) a_{s-1} (transient_nonlinear.mojo:553-590), whose accuracy is
already third order; learning the correction keeps the network's bf16 precision from limiting the
guess.
"""
from __future__ import annotations

import ctypes as C
import copy

import numpy as np

from . import runtime

N_HIST = 4
N_AG = 16


def n_features(ndf: int) -> int:
    return N_HIST * ndf + N_AG + 1


def node_table(model):
    """Nodes with at least one free dof, in node order: (free index per dof or -1, height ratio)."""
    ndf, ndm = model.ndf, model.ndm
    heights = model.coords[ndm - 1::ndm]
    hmax = float(heights.max()) if heights.size else 0.0
    frees, hs = [], []
    for nd in range(model.num_nodes):
        fi = model.free_index[nd * ndf:(nd + 1) * ndf]
        if (fi >= 0).any():
            frees.append(fi.astype(np.int64))
            hs.append(np.float32(heights[nd] / hmax) if hmax > 0 else np.float32(0.0))
    return np.asarray(frees, dtype=np.int64).reshape(-1, ndf), np.asarray(hs, dtype=np.float32)


def path_eval(ex: dict, t: float) -> float:
    """Path time series with dt, linear interpolation (time_series.mojo:71-90)."""
    vals = ex["values"]
    n = len(vals)
    if n == 0 or t < ex["start_time"]:
        return 0.0
    incr = (t - ex["start_time"]) / ex["dt"]
    i1 = int(np.floor(incr))
    i2 = i1 + 1
    if i2 >= n:
        return ex["factor"] * vals[n - 1] if ex["use_last"] else 0.0
    v1, v2 = vals[i1], vals[i2]
    return ex["factor"] * (v1 + (v2 - v1) * (incr - i1))


def ground_series(model, steps: int, component: int = 0) -> np.ndarray:
    """Ground acceleration of steps 0..steps-1 of one excitation component, as the step loop
    evaluates it."""
    if len(model.excitations) <= component:
        return np.zeros(steps)
    ex = model.excitations[component]
    return np.array([path_eval(ex, (s + 1) * model.dt) for s in range(steps)])


def raw_features(model, u_free_hist: np.ndarray):
    """Unnormalised features and targets of every step and node of one converged history.

    u_free_hist: (steps, num_free) converged free displacements.  Returns X (steps * nodes, n_in)
    and T (steps * nodes, ndf), float32, step-major."""
    frees, hs = node_table(model)
    steps = u_free_hist.shape[0]
    ndf = model.ndf
    u = np.vstack([np.zeros((1, u_free_hist.shape[1])), u_free_hist])
    du = np.diff(u, axis=0)                           # du[s] = u_s - u_{s-1}
    du_pad = np.hstack([du, np.zeros((steps, 1))])    # column -1 -> 0 for constrained dofs
    col = np.where(frees >= 0, frees, du.shape[1])    # (nodes, ndf)
    node_du = du_pad[:, col]                          # (steps, nodes, ndf)
    nn = frees.shape[0]
    X = np.zeros((steps, nn, n_features(ndf)), dtype=np.float32)
    for j in range(N_HIST):
        sl = slice(j * ndf, (j + 1) * ndf)
        X[1 + j:, :, sl] = node_du[:steps - 1 - j].astype(np.float32)
    # one excitation: its 16 latest samples; two: the 8 latest of each component
    two = len(model.excitations) == 2
    for j in range(N_AG):
        c, lag = (j // 8, j % 8) if two else (0, j)
        ag = ground_series(model, steps, c)
        agp = np.concatenate([np.zeros(N_AG - 1), ag]).astype(np.float32)  # agp[k + 15] = ag[k]
        X[:, :, N_HIST * ndf + j] = agp[N_AG - 1 - lag:N_AG - 1 - lag + steps][:, None]
    X[:, :, -1] = hs[None, :]
    # Newmark velocity / acceleration of the converged history (transient_nonlinear.mojo:594-647)
    dt, gam, bet = model.dt, model.gamma, model.beta
    a0, a2, a3 = 1.0 / (bet * dt * dt), 1.0 / (bet * dt), 1.0 / (2.0 * bet) - 1.0
    nfree = u_free_hist.shape[1]
    v = np.zeros(nfree)
    a = np.zeros(nfree)
    pred = np.zeros((steps, nfree))
    for s in range(steps):
        pred[s] = dt * v + (dt * dt * (0.5 - bet)) * a
        an = a0 * du[s] - a2 * v - a3 * a
        v = v + dt * ((1.0 - gam) * a + gam * an)
        a = an
    corr = np.hstack([du - pred, np.zeros((steps, 1))])[:, col]
    T = corr.astype(np.float32)
    return X.reshape(-1, X.shape[-1]), T.reshape(-1, ndf)


def fit_normalisation(X: np.ndarray, T: np.ndarray):
    mean = X.mean(0).astype(np.float32)
    std = X.std(0).astype(np.float32)
    scale = np.where(std > 0, 1.0 / np.maximum(std, 1e-30), 1.0).astype(np.float32)
    y_scale = T.std(0).astype(np.float32)
    y_scale = np.where(y_scale > 0, y_scale, 1.0).astype(np.float32)
    return mean, scale, y_scale


def free_history(analysis, instance: int):
    """Converged free displacements (steps, num_free) of an analysis whose model records every
    dof (see record_all_dofs)."""
    m = analysis.models[instance]
    disp, _ef, _it = analysis.history(instance)
    fdof = np.full(m.num_free, -1)
    for dof, fi in enumerate(m.free_index):
        if fi >= 0:
            fdof[fi] = dof
    pos = {int(d): k for k, d in enumerate(m.record_dofs)}
    return disp[:, [pos[int(d)] for d in fdof]]


def record_all_dofs(model):
    """A copy of the model that records the displacement of every dof."""
    m = copy.copy(model)
    m.record_dofs = np.arange(model.num_dofs, dtype=np.int32)
    return m


class LearnedPredictor:
    """A trained per-node network with its normalisation, ready to attach to analyses."""

    def __init__(self, ndf: int, seed: int = 0):
        self.ndf = ndf
        self.n_in = n_features(ndf)
        self.net = runtime.Mlp(self.n_in, ndf)
        rng = np.random.default_rng(seed)
        H = runtime.Mlp.H
        self.net.set_params({
            "W1": (rng.standard_normal((self.n_in, H)) * np.sqrt(2.0 / self.n_in)).astype(np.float32),
            "b1": np.zeros(H, np.float32),
            "W2": (rng.standard_normal((H, H)) * np.sqrt(2.0 / H)).astype(np.float32),
            "b2": np.zeros(H, np.float32),
            "W3": (rng.standard_normal((H, ndf)) * np.sqrt(1.0 / H)).astype(np.float32),
            "b3": np.zeros(ndf, np.float32),
        })
        self.x_mean = np.zeros(self.n_in, np.float32)
        self.x_scale = np.ones(self.n_in, np.float32)
        self.y_scale = np.ones(ndf, np.float32)

    def fit(self, X: np.ndarray, T: np.ndarray, epochs: int = 20, batch: int = 8192, lr: float = 1e-3,
            seed: int = 0) -> float:
        """Normalises, then trains on the GPU (tensor-core forward and backward, Adam)."""
        self.x_mean, self.x_scale, self.y_scale = fit_normalisation(X, T)
        Xn = ((X - self.x_mean) * self.x_scale).astype(np.float32)
        Tn = (T / self.y_scale).astype(np.float32)
        return self.net.train(Xn, Tn, epochs=epochs, batch=batch, lr=lr, seed=seed)

    def predict(self, X: np.ndarray) -> np.ndarray:
        """Predicted correction to the Newmark predictor's increment, per node and dof."""
        Xn = ((X - self.x_mean) * self.x_scale).astype(np.float32)
        return self.net.forward(Xn) * self.y_scale

    def attach(self, analysis):
        f = C.POINTER(C.c_float)
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (self.x_mean, self.x_scale, self.y_scale)]
        runtime._check(runtime.lib().strut_gpu_set_predictor(analysis.h, self.net.m, *[a.ctypes.data_as(f) for a in arrs]),
                       "strut_gpu_set_predictor")
        analysis._predictor = self  # keeps the network alive while attached


def detach(analysis):
    runtime._check(runtime.lib().strut_gpu_set_predictor(analysis.h, None, None, None, None),
                   "strut_gpu_set_predictor")
    analysis._predictor = None


def stats(analysis):
    """(first iterations offered the learned guess, learned guess kept)."""
    o, c = C.c_int64(), C.c_int64()
    runtime._check(runtime.lib().strut_gpu_predictor_stats(analysis.h, C.byref(o), C.byref(c)),
                   "strut_gpu_predictor_stats")
    return o.value, c.value


def device_features(analysis) -> np.ndarray:
    """The device's (normalised) features of the next step, for tests."""
    n = int(runtime.lib().strut_gpu_predictor_nodes(analysis.h))
    p = analysis._predictor
    out = np.zeros((n, p.n_in), dtype=np.float32)
    runtime._check(runtime.lib().strut_gpu_predictor_features(analysis.h, out.ctypes.data_as(C.POINTER(C.c_float))),
                   "strut_gpu_predictor_features")
    return out

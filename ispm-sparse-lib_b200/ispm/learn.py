"""Learned per-row drop tolerances for the approximate inverse.

The reference tunes one global drop tolerance for fastainv_sym with a
golden-section search that costs a full build and solve per probe
(fastainv/droptol-tuning.h:4-103; DroptolTuner here).  This module replaces
that search with a prediction: per-row features of the matrix
(ispm_row_features) feed a 32 -> 64 -> 64 -> 2 MLP (ispm_mlp_*: BF16 weights,
FP32 accumulation, trained and run by the library's own GPU kernels) whose
two outputs are, per row j of the factor,

    out0 = log2(droptol_j / 0.01)      out1 = log(rescale_j)

fed to fastainv_sym_ex.  Training pairs come from the plain build and solve
themselves: every training system is built with fastainv_sym at a ladder of
global drop tolerances and solved with the mixed-precision PCG; the
tolerance with the least modelled solve cost (iterations x bytes moved per
iteration, vectors included) is the target of every row of that system.  The rescale head is
trained toward 1: measured row rescales (the modified-AINV row-sum
compensation at exponents 0.1 .. 1) raised iteration counts on this family.

Plain fastainv_sym stays the fallback and the yardstick: `gate` accepts the
learned factor only if PCG iterations drop (and the solve is not slower).

  python -m ispm.learn train  [--systems N] [--out PATH]
  python -m ispm.learn evaluate [--grid 128] [--contrast 1e4]
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
import time

import numpy as np

from . import (F32, F64, PCGSolver, _check, _lib, _ptr, _stream, csr_matrix, fastainv_sym,
               fastainv_sym_ex)

N_IN, N_H, N_OUT = 32, 64, 2
BASE_DROPTOL = 0.01
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                               "learned_droptol.npz")
TAUS = (0.08, 0.04, 0.02, 0.01, 0.005, 0.0025)

_DECLARED = False


def _declare():
    global _DECLARED
    if _DECLARED:
        return
    L = _lib()
    vp, i, ll, f = C.c_void_p, C.c_int, C.c_longlong, C.c_float
    L.ispm_mlp_n_params.argtypes = []
    L.ispm_mlp_n_params.restype = i
    L.ispm_mlp_create.argtypes = [vp, C.POINTER(vp)]
    L.ispm_mlp_create.restype = i
    L.ispm_mlp_get_params.argtypes = [vp, vp]
    L.ispm_mlp_get_params.restype = i
    L.ispm_mlp_set_params.argtypes = [vp, vp]
    L.ispm_mlp_set_params.restype = i
    L.ispm_mlp_forward.argtypes = [vp, ll, vp, vp, vp]
    L.ispm_mlp_forward.restype = i
    L.ispm_mlp_loss_grad.argtypes = [vp, ll, vp, vp, vp, vp, C.POINTER(C.c_double), vp]
    L.ispm_mlp_loss_grad.restype = i
    L.ispm_mlp_adam_step.argtypes = [vp, f, f, f, f, f, vp]
    L.ispm_mlp_adam_step.restype = i
    L.ispm_mlp_free.argtypes = [vp]
    L.ispm_mlp_free.restype = None
    L.ispm_row_features.argtypes = [i, vp, vp, vp, i, i, vp, vp]
    L.ispm_row_features.restype = i
    _DECLARED = True


def n_params() -> int:
    _declare()
    return int(_lib().ispm_mlp_n_params())


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform hidden layers, small output layer, zero biases."""
    rng = np.random.default_rng(seed)
    w1 = rng.uniform(-1, 1, (N_H, N_IN)) * math.sqrt(6.0 / N_IN)
    w2 = rng.uniform(-1, 1, (N_H, N_H)) * math.sqrt(6.0 / N_H)
    w3 = rng.uniform(-1, 1, (N_OUT, N_H)) * math.sqrt(1.0 / N_H)
    p = np.concatenate([w1.ravel(), np.zeros(N_H), w2.ravel(), np.zeros(N_H), w3.ravel(),
                        np.zeros(N_OUT)]).astype(np.float32)
    assert p.size == n_params()
    return p


class MLP:
    """The 32 -> 64 -> 64 -> 2 network on the current GPU (ispm_mlp)."""

    def __init__(self, params: np.ndarray | None = None, seed: int = 0):
        _declare()
        p = init_params(seed) if params is None else np.ascontiguousarray(params, np.float32)
        if p.size != n_params():
            raise ValueError(f"expected {n_params()} parameters, got {p.size}")
        h = C.c_void_p()
        _check(_lib().ispm_mlp_create(_ptr(p), C.byref(h)))
        self._h = h
        self._free = _lib().ispm_mlp_free

    def __del__(self):
        if getattr(self, "_h", None):
            self._free(self._h)
            self._h = None

    def params(self) -> np.ndarray:
        out = np.zeros(n_params(), np.float32)
        _check(_lib().ispm_mlp_get_params(self._h, _ptr(out)))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        _check(_lib().ispm_mlp_set_params(self._h, _ptr(p)))

    def forward(self, feat, stream=None):
        """feat: torch bfloat16 [n, 32] on the GPU -> torch float32 [n, 2]."""
        import torch
        out = torch.empty((feat.shape[0], N_OUT), dtype=torch.float32, device=feat.device)
        _check(_lib().ispm_mlp_forward(self._h, feat.shape[0], _ptr(feat), _ptr(out),
                                       _stream(stream)))
        return out

    def loss_grad(self, feat, target, weight=None, stream=None, want_grad=True):
        loss = C.c_double()
        g = np.zeros(n_params(), np.float32) if want_grad else None
        _check(_lib().ispm_mlp_loss_grad(self._h, feat.shape[0], _ptr(feat), _ptr(target),
                                         _ptr(weight), _ptr(g), C.byref(loss),
                                         _stream(stream)))
        return loss.value, g

    def adam_step(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0,
                  stream=None):
        _check(_lib().ispm_mlp_adam_step(self._h, lr, beta1, beta2, eps, weight_decay,
                                         _stream(stream)))

    def fit(self, feat, target, weight=None, epochs: int = 20, batch: int = 65536,
            lr: float = 2e-3, seed: int = 0, log=None):
        """Minibatch Adam over shuffled rows; returns the loss after each epoch
        (over the whole set)."""
        import torch
        gen = torch.Generator(device="cpu").manual_seed(seed)
        n = feat.shape[0]
        hist = []
        for ep in range(epochs):
            perm = torch.randperm(n, generator=gen).to(feat.device)
            fs, ts = feat[perm].contiguous(), target[perm].contiguous()
            ws = None if weight is None else weight[perm].contiguous()
            step_lr = lr * 0.5 * (1 + math.cos(math.pi * ep / max(epochs, 1)))
            for b0 in range(0, n, batch):
                b1 = min(n, b0 + batch)
                self.loss_grad(fs[b0:b1], ts[b0:b1], None if ws is None else ws[b0:b1],
                               want_grad=False)
                self.adam_step(step_lr)
            loss, _ = self.loss_grad(feat, target, weight, want_grad=False)
            hist.append(loss)
            if log:
                log(f"[learn] epoch {ep + 1}/{epochs} loss {loss:.5f}")
        return hist

    def save(self, path, meta=None):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez(path, params=self.params(), meta=json.dumps(meta or {}))

    @classmethod
    def load(cls, path=DEFAULT_WEIGHTS):
        z = np.load(path)
        m = cls(z["params"])
        m.meta = json.loads(str(z["meta"]))
        return m


def row_features(A: csr_matrix, dims=None):
    """Per-row features of A on the GPU (torch bfloat16 [n, 32]).  dims: the
    (nz, ny, nx) box of a stencil matrix, or None."""
    import torch
    _declare()
    dev = torch.device("cuda")
    rp = torch.from_numpy(A.row_ptr).to(dev)
    ci = torch.from_numpy(A.cols).to(dev)
    v = torch.from_numpy(np.ascontiguousarray(A.elms, np.float64)).to(dev)
    out = torch.empty((A.n_rows, N_IN), dtype=torch.bfloat16, device=dev)
    nx, ny = (dims[2], dims[1]) if dims is not None else (0, 0)
    _check(_lib().ispm_row_features(A.n_rows, _ptr(rp), _ptr(ci), _ptr(v), nx, ny, _ptr(out),
                                    None))
    return out


def predict_row_controls(model: MLP, A: csr_matrix, dims=None, clip=3.0, clip_scale=0.5):
    """(row_droptol, row_scale) for fastainv_sym_ex, one per row of A."""
    y = model.forward(row_features(A, dims)).cpu().numpy().astype(np.float64)
    tau = BASE_DROPTOL * np.exp2(np.clip(y[:, 0], -clip, clip))
    scale = np.exp(np.clip(y[:, 1], -clip_scale, clip_scale))
    return tau, scale


# ---------------------------------------------------------------- training data

def training_systems(n: int, seed: int = 0, sizes=(32, 64), contrasts=(1e2, 1e4)):
    """Seeded variable-coefficient box stencils: side uniform in `sizes`,
    7- or 27-point, Gaussian-random-field log-coefficients whose contrast
    (max / min coupling, approximately e^(7 sigma)) is log-uniform in
    `contrasts`.  Yields (A, dims, meta) lazily."""
    from . import gen
    rng = np.random.default_rng(seed)
    for k in range(n):
        L = int(rng.integers(sizes[0], sizes[1] + 1))
        points = 7 if rng.random() < 0.5 else 27
        c = 10 ** rng.uniform(math.log10(contrasts[0]), math.log10(contrasts[1]))
        sigma = math.log(c) / 7.0
        corr = float(rng.uniform(4.0, 12.0))
        A = gen.stencil_grf(L, points, corr, sigma, seed * 100000 + k)
        yield A, (L, L, L), {"L": L, "points": points, "contrast": c, "sigma": sigma,
                             "corr": corr, "seed": seed * 100000 + k}


def solve_cost(A, its, nnz_g):
    """Modelled bytes of a mixed-precision solve: iterations x (A and the two
    factor applications, 4-byte values, plus the 17 passes over 4-byte
    vectors of one classic-PCG iteration)."""
    return its * (4.0 * (A.n_nz + 2 * nnz_g) + 68.0 * A.n_rows)


def label_system(A, b, taus=TAUS, tol=1e-10):
    """Plain build + mixed PCG at every drop tolerance of the ladder.
    Returns {tau: (iterations, nnz(G), modelled cost)} and the cost-optimal
    log2(tau / 0.01) (parabolic refinement around the best rung)."""
    res = {}
    for tau in taus:
        G1, G2 = fastainv_sym(A, np.float64, None, 2_000_000_000, tau)
        S = PCGSolver(A, G1, G2, inner=np.float32, tol=tol)
        _, st = S.solve_host(b)
        res[tau] = (int(st["iterations"]), int(G1.n_nz),
                    solve_cost(A, st["iterations"], G1.n_nz) if st["converged"] else math.inf)
    return res, _best_log2(res)


def make_dataset(systems, log=None):
    """Feature rows and targets of labelled systems: [(A, dims, meta, target)]."""
    import torch
    feats, targets = [], []
    for A, dims, meta, y0 in systems:
        f = row_features(A, dims)
        t = torch.zeros((A.n_rows, N_OUT), dtype=torch.float32, device=f.device)
        t[:, 0] = y0
        feats.append(f)
        targets.append(t)
    return torch.cat(feats), torch.cat(targets)


# ---------------------------------------------------------------- the gate

def gate(A, b, model: MLP, dims=None, tol=1e-10, plain=None, log=None):
    """Learned factor vs the plain one (droptol 0.01), both solved with the
    mixed-precision PCG.  The learned factor is accepted only if PCG
    iterations drop and the solve is not slower.  Returns a report dict."""
    import torch
    t0 = time.perf_counter()
    tau, scale = predict_row_controls(model, A, dims)
    t_pred = time.perf_counter() - t0
    t0 = time.perf_counter()
    L1, L2 = fastainv_sym_ex(A, np.float64, tau, scale, 2_000_000_000, BASE_DROPTOL)
    t_build_l = time.perf_counter() - t0
    if plain is None:
        t0 = time.perf_counter()
        P1, P2 = fastainv_sym(A, np.float64, None, 2_000_000_000, BASE_DROPTOL)
        t_build_p = time.perf_counter() - t0
    else:
        (P1, P2), t_build_p = plain

    def timed(G1, G2):
        S = PCGSolver(A, G1, G2, inner=np.float32, tol=tol)
        S.solve_host(b)  # warm-up
        best = None
        for _ in range(3):
            torch.cuda.synchronize()
            t = time.perf_counter()
            x, st = S.solve_host(b)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t
            best = dt if best is None else min(best, dt)
        r = b - A.to_scipy() @ x
        return best, st, float(np.linalg.norm(r) / np.linalg.norm(b))

    tl, sl, rl = timed(L1, L2)
    tp, sp, rp = timed(P1, P2)
    accept = (sl["converged"] and sl["iterations"] < sp["iterations"] and tl <= tp)
    rep = {"accepted": bool(accept),
           "learned": {"iterations": sl["iterations"], "nnz_G": int(L1.n_nz), "solve_s": tl,
                       "true_relres": rl, "build_s": t_build_l, "predict_s": t_pred,
                       "droptol_median": float(np.median(tau)),
                       "droptol_p10_p90": [float(np.percentile(tau, 10)),
                                           float(np.percentile(tau, 90))],
                       "rescale_p10_p90": [float(np.percentile(scale, 10)),
                                           float(np.percentile(scale, 90))]},
           "plain": {"iterations": sp["iterations"], "nnz_G": int(P1.n_nz), "solve_s": tp,
                     "true_relres": rp, "build_s": t_build_p, "droptol": BASE_DROPTOL}}
    if log:
        log(f"[learn] gate: {json.dumps(rep)}")
    return rep


# ---------------------------------------------------------------- drivers

def train(n_systems=96, seed=0, sizes=(32, 48), contrasts=(1e2, 1e4), epochs=30,
          out=DEFAULT_WEIGHTS, log=print, workers=8):
    """Label n_systems training systems with the plain build + solve, fit the
    network on their rows, save the weights."""
    import torch
    from concurrent.futures import ThreadPoolExecutor
    t_start = time.time()
    labelled, meta_rows = [], []
    systems = list(training_systems(n_systems, seed, sizes, contrasts))

    def plain_builds(item):
        A = item[0]
        return {tau: fastainv_sym(A, np.float64, None, 2_000_000_000, tau) for tau in TAUS}

    # the host builds of a system's ladder run on worker threads (the C
    # calls release the GIL); the solves run on the GPU in order
    with ThreadPoolExecutor(max_workers=workers) as ex:
        builds = ex.map(plain_builds, systems)
        for (A, dims, meta), pairs in zip(systems, builds):
            b = A.to_scipy() @ np.random.default_rng(meta["seed"]).uniform(-1, 1, A.n_rows)
            res = {}
            for tau in TAUS:
                G1, G2 = pairs[tau]
                S = PCGSolver(A, G1, G2, inner=np.float32, tol=1e-10)
                _, st = S.solve_host(b)
                res[tau] = (int(st["iterations"]), int(G1.n_nz),
                            solve_cost(A, st["iterations"], G1.n_nz) if st["converged"]
                            else math.inf)
                del S
            y0 = _best_log2(res)
            labelled.append((A, dims, meta, y0))
            meta_rows.append(dict(meta, target=y0,
                                  ladder={str(t): res[t][:2] for t in TAUS}))
            log(f"[learn] system {len(labelled)}/{n_systems} {meta['points']}-pt L={meta['L']} "
                f"contrast {meta['contrast']:.0f}: best log2(tau/0.01) {y0:+.2f} "
                f"{[res[t][0] for t in TAUS]}")
    t_label = time.time() - t_start
    feat, target = make_dataset(labelled)
    model = MLP(seed=seed)
    t0 = time.time()
    hist = model.fit(feat, target, epochs=epochs, log=log)
    t_fit = time.time() - t0
    meta = {"systems": meta_rows, "rows": int(feat.shape[0]), "epochs": epochs,
            "loss": hist, "label_s": t_label, "fit_s": t_fit, "sizes": list(sizes),
            "contrasts": list(contrasts), "taus": list(TAUS)}
    model.save(out, meta)
    log(f"[learn] saved {out}: {feat.shape[0]} rows, final loss {hist[-1]:.5f}, "
        f"labels {t_label:.0f}s, fit {t_fit:.1f}s")
    return model, meta


def _best_log2(res):
    taus = list(res)
    xs = np.log2(np.array(taus) / BASE_DROPTOL)
    cs = np.array([res[t][2] for t in taus])
    order = np.argsort(xs)
    xs, cs = xs[order], cs[order]
    k = int(np.argmin(cs))
    best = float(xs[k])
    if 0 < k < len(xs) - 1 and np.all(np.isfinite(cs[k - 1:k + 2])):
        x0, x1, x2 = xs[k - 1:k + 2]
        y0, y1, y2 = np.log(cs[k - 1:k + 2])
        den = (x0 - x1) * (x0 - x2) * (x1 - x2)
        a = (x2 * (y1 - y0) + x1 * (y0 - y2) + x0 * (y2 - y1)) / den
        bq = (x2 * x2 * (y0 - y1) + x1 * x1 * (y2 - y0) + x0 * x0 * (y1 - y2)) / den
        if a > 0:
            best = float(np.clip(-bq / (2 * a), x0, x2))
    return best


def holdout_system(grid=128, contrast=1e4, seed=9001):
    """Held-out 27-point system: GRF log-coefficients at the given contrast."""
    from . import gen
    sigma = math.log(contrast) / 7.0
    A = gen.stencil_grf(grid, 27, 8.0, sigma, seed)
    b = A.to_scipy() @ np.random.default_rng(seed).uniform(-1, 1, A.n_rows)
    return A, b, (grid, grid, grid)


def main(argv=None):
    import argparse
    import sys
    p = argparse.ArgumentParser(prog="python -m ispm.learn")
    p.add_argument("cmd", choices=["train", "evaluate"])
    p.add_argument("--systems", type=int, default=96)
    p.add_argument("--min-size", type=int, default=32)
    p.add_argument("--max-size", type=int, default=48)
    p.add_argument("--epochs", type=int, default=30)
    p.add_argument("--out", default=DEFAULT_WEIGHTS)
    p.add_argument("--grid", type=int, default=128)
    p.add_argument("--contrast", type=float, default=1e4)
    a = p.parse_args(argv)
    import torch
    torch.cuda.init()
    from . import ispm_initialize
    ispm_initialize()
    log = lambda *m: print(*m, file=sys.stderr, flush=True)
    if a.cmd == "train":
        train(a.systems, sizes=(a.min_size, a.max_size), epochs=a.epochs, out=a.out, log=log)
    else:
        A, b, dims = holdout_system(a.grid, a.contrast)
        rep = gate(A, b, MLP.load(a.out), dims, log=log)
        print(json.dumps(rep))


if __name__ == "__main__":
    main()

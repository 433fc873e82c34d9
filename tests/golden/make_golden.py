"""Generate the golden fixtures of tests/golden/ from the reference's own host
code, compiled in place into oracle/_ref/libispm_ref.so (needs the reference
source tree; run from the repository root):

    python tests/golden/make_golden.py

Writes conversion.npz (csr_to_slell / csr_to_slell_guess_format results),
fastainv.npz (fastainv_sym results) and tuner.npz (DroptolTuner probe
sequences).  Inputs are stored next to outputs, so the fixtures stay valid even
if the generators change.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "ispm-sparse-lib_b200"), os.path.join(ROOT, "oracle")]

import ispm.gen as gen  # noqa: E402
import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

CONV_MATRICES = {
    "poisson6": lambda: gen.poisson7(6),
    "band600": lambda: gen.random_csr(600, 600, 11, mean_len=9, band=24),
    "wide400x900_f32": lambda: gen.random_csr(400, 900, 12, mean_len=12, pair_frac=0.6,
                                              dtype=np.float32),
    "irregular700": lambda: gen.random_csr(700, 700, 13, mean_len=6, max_len=90),
}
CONV_MODES = [(32, 1, 0, 1), (64, 1, 0, 0), (16, 2, 0, 0), (64, 4, 0, 0), (128, 1, 1, 0),
              (256, 1, 1, 1), (256, 2, 1, 0), (32, 1, 0, 0)]


def conversion():
    out = {}
    for name, mk in CONV_MATRICES.items():
        A = mk()
        out[f"{name}/row_ptr"] = A.row_ptr
        out[f"{name}/cols"] = A.cols
        out[f"{name}/elms"] = A.elms
        out[f"{name}/shape"] = np.array([A.n_rows, A.n_cols])
        cases = CONV_MODES + [("guess",)]
        for c in cases:
            if c[0] == "guess":
                r = O.ref_csr_to_slell_guess_format(A.n_rows, A.n_cols, A.row_ptr, A.cols, A.elms)
                key = f"{name}/guess"
            else:
                S, W, V, D = c
                r = O.ref_csr_to_slell(A.n_rows, A.n_cols, A.row_ptr, A.cols, A.elms, S, W, V, D)
                key = f"{name}/S{S}_W{W}_V{V}_D{D}"
            out[f"{key}/meta"] = np.array([r["n_rows"], r["n_cols"], r["n_nz"], r["slice_height"],
                                           r["n_slices"], r["hblock"], int(r["var_height"]),
                                           int(r["diags"])], np.int64)
            out[f"{key}/slice_ptr"] = r["slice_ptr"]
            out[f"{key}/cols"] = r["cols"]
            out[f"{key}/elms"] = r["elms"]
    np.savez_compressed(os.path.join(OUT, "conversion.npz"), **out)


AINV_CASES = [
    ("poisson6_dt0.01_f64", lambda: gen.poisson7(6), 1, 8192000, 0.01),
    ("poisson6_dt0.01_f32", lambda: gen.poisson7(6), 0, 8192000, 0.01),
    ("poisson6_dt0.125_f64", lambda: gen.poisson7(6), 1, 8192000, 0.125),
    ("grf27_6_dt0.01_f64", lambda: gen.stencil_grf(6, 27, 2.0, 1.5, 5), 1, 8192000, 0.01),
    ("grf27_6_trunc_f32", lambda: gen.stencil_grf(6, 27, 2.0, 1.5, 5), 0, 4000, 0.001),
    ("unstr8_dt0.01_f64", lambda: gen.unstructured(8, seed=3), 1, 8192000, 0.01),
]


def fastainv():
    out = {}
    for name, mk, f64, max_elts, dt in AINV_CASES:
        A = mk()
        g1, g2, calls = O.ref_fastainv_sym(A.n_rows, A.row_ptr, A.cols, A.elms, bool(f64),
                                           max_elts, dt)
        out[f"{name}/A_row_ptr"] = A.row_ptr
        out[f"{name}/A_cols"] = A.cols
        out[f"{name}/A_elms"] = A.elms
        out[f"{name}/params"] = np.array([f64, max_elts, dt, calls], np.float64)
        for tag, g in (("G1", g1), ("G2", g2)):
            out[f"{name}/{tag}_row_ptr"] = g[0]
            out[f"{name}/{tag}_cols"] = g[1]
            out[f"{name}/{tag}_elms"] = g[2]
    np.savez_compressed(os.path.join(OUT, "fastainv.npz"), **out)


def tuner_times(d):
    # a smooth bowl in log2(droptol) with its minimum near 2^-6.3
    return 1.0 + (np.log2(d) + 6.3) ** 2


def tuner():
    out = {}
    for name, lo, hi, restart_at in (("default", -10.0, -3.0, 12), ("narrow", -8.0, -5.0, 6)):
        t = O.RefDroptolTuner(lo, hi)
        seq, best, iters = [], [], []
        for k in range(20):
            if k == restart_at:
                t.restart()
            d = t.getDroptol()
            seq.append(d)
            t.noteTime(tuner_times(d))
            best.append(t.getBestDroptol())
            iters.append(t.iterations())
        out[f"{name}/lo_hi_restart"] = np.array([lo, hi, restart_at])
        out[f"{name}/droptols"] = np.array(seq)
        out[f"{name}/best"] = np.array(best)
        out[f"{name}/iterations"] = np.array(iters)
    np.savez_compressed(os.path.join(OUT, "tuner.npz"), **out)


if __name__ == "__main__":
    conversion()
    fastainv()
    tuner()
    for f in ("conversion.npz", "fastainv.npz", "tuner.npz"):
        print(f, os.path.getsize(os.path.join(OUT, f)), "bytes")

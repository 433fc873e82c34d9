"""Achieved bandwidth of the library's kernels against the B200's measured HBM
peak, each timed alone with CUDA events on inputs larger than the 126 MB L2.

  python -m ispm.roofline [--json PATH] [--reps K] [--warm W]
  python -m ispm.roofline --shapes [--json PATH]

For every kernel: its algorithmic bytes per launch (compulsory reads and
writes, no re-reads), the mean launch time after warm-up, achieved GB/s and
the fraction of the peak (MEASURED_PEAKS.json's copy bandwidth when present,
else 6,650 GB/s).  The MLP rows also give tensor-core TFLOP/s against the
measured BF16 peak.  Sizes: the 128^3 27-point system of the headline
workload for the matrix kernels, 2^26-element vectors for the BLAS.

--shapes times the SpMV of the headline solver's operators (A in FP32 and
as the FP16 split, the GPU FSAI factor G and G^T in FP32 and FP16) under
several launch shapes: the default register walk (N = S/4, H = 4), two and
eight rows a thread, and the staged walk (N = S, H = 1), back to back
("warm") and with a 256 MB L2 flush before every launch ("flushed").
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

from . import (F32, F64, csr_matrix, csr_to_slell_guess_format, default_launch_params,
               fsai_sym_gpu, launch_spmv_kernel, sblas, slell_value_map, spmv_plan,
               plan_refresh_values)


def peaks():
    here = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    try:
        m = json.load(open(os.path.join(here, "MEASURED_PEAKS.json")))
        return float(m["hbm_gbs"]), float(m["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


REPS, WARM = 20, 3


def timed(fn, reps=None, warm=None):
    import torch
    reps = REPS if reps is None else min(reps, REPS)
    warm = WARM if warm is None else warm
    for _ in range(warm):
        fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps * 1e-3


def slell_bytes(view, vec_bytes):
    esz = 4 if view.elm_dtype == F32 else 8
    return (4 * view.n_slice_ptr + 4 * view.n_cols_arr + esz * view.n_nz +
            vec_bytes * (view.n_cols + view.n_rows))


def run(log=print):
    import torch
    from . import gen, ispm_initialize
    import ispm.learn as LN
    torch.cuda.init()
    ispm_initialize()
    hbm, bf16, src = peaks()
    rows = []

    def add(name, sec, nbytes, flops=None, note=""):
        r = {"kernel": name, "us": sec * 1e6, "bytes": int(nbytes), "GB/s": nbytes / sec / 1e9,
             "frac_hbm": nbytes / sec / 1e9 / hbm, "note": note}
        if flops:
            r["TFLOP/s"] = flops / sec / 1e12
            r["frac_bf16"] = flops / sec / 1e12 / bf16
        rows.append(r)
        log(f"{name:40s} {r['us']:9.1f} us {r['GB/s']:8.0f} GB/s {r['frac_hbm']:5.2f}"
            + (f"  {r['TFLOP/s']:6.1f} TFLOP/s" if flops else ""))

    dev = torch.device("cuda")
    A = gen.stencil_grf(128, 27, 8.0, 1.5, 0)
    n, nnz = A.n_rows, A.n_nz

    # sliced-ELL SpMV, FP32 and FP64 (the reference's guessed format, the
    # B200 launch heuristic)
    for dt, name in ((np.float32, "spmv FP32 (C2 A, diagonal blocks)"),
                     (np.float64, "spmv FP64 (C2 A, diagonal blocks)")):
        Ad = csr_matrix(n, n, A.row_ptr, A.cols, A.elms.astype(dt))
        H = csr_to_slell_guess_format(Ad)
        D = H.upload()
        p = default_launch_params(D, dt)
        tdt = torch.float32 if dt == np.float32 else torch.float64
        x = torch.rand(n, dtype=tdt, device=dev)
        y = torch.zeros(H.n_rows, dtype=tdt, device=dev)
        add(name, timed(lambda: launch_spmv_kernel(p, D, x, y)),
            slell_bytes(H.view(), 4 if dt == np.float32 else 8))
        del D, H, x, y

    # value refresh: new CSR values scattered into the device matrix
    A32 = csr_matrix(n, n, A.row_ptr, A.cols, A.elms.astype(np.float32))
    plan = spmv_plan(A32, T=np.float32)
    vals = torch.from_numpy(A.elms).to(dev)
    plan_refresh_values(plan, A32, vals)  # builds the map once
    add("value refresh (C2, FP64 -> FP32 slots)", timed(lambda: plan_refresh_values(plan, A32, vals)),
        nnz * (8 + 4 + 4))
    del plan, vals

    # BLAS
    N = 1 << 26
    for tdt, esz, tag in ((torch.float64, 8, "FP64"), (torch.float32, 4, "FP32")):
        x = torch.rand(N, dtype=tdt, device=dev)
        y = torch.rand(N, dtype=tdt, device=dev)
        s = torch.zeros(1, dtype=tdt, device=dev)
        add(f"sblas dot {tag} (n = 2^26)", timed(lambda: sblas.dot(x, y, s, N)), 2 * N * esz)
        del x, y, s
    M = 1 << 22
    v = [torch.rand(M, dtype=torch.float64, device=dev) for _ in range(10)]
    sc = [torch.full((1,), 0.5, dtype=torch.float64, device=dev) for _ in range(5)]
    add("sblas ppcg_update_vectors FP64 (n = 2^22)",
        timed(lambda: sblas.ppcg_update_vectors(*sc, *v, M)), 18 * M * 8)
    del v, sc
    src_v = torch.rand(N, dtype=torch.float64, device=dev)
    dst_v = torch.zeros(N, dtype=torch.float64, device=dev)
    idx = torch.randperm(N, device=dev).to(torch.int32)
    add("sblas copy_indexed FP64 (n = 2^26, random)",
        timed(lambda: sblas.copy_indexed(dst_v, src_v, idx, N)), N * (8 + 4 + 8))
    add("sblas add_indexed FP64 (n = 2^26, random)",
        timed(lambda: sblas.add_indexed(dst_v, src_v, idx, N)), N * (8 + 4 + 8 + 8))
    del src_v, dst_v, idx

    # GPU FSAI build (host pattern set-up included in the wall time)
    t0 = time.perf_counter()
    G1, _ = fsai_sym_gpu(A, np.float64)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    add("fsai_sym_gpu (C2, call wall time)", wall, nnz * 12 + G1.n_nz * 20,
        note="includes host pattern build and copies; fsai_rows_kernel alone in the ncu list")

    # learned drop tolerances: features, MLP forward, loss + gradient
    dims = (128, 128, 128)
    LN.row_features(A, dims)
    rp = torch.from_numpy(A.row_ptr).to(dev)
    ci = torch.from_numpy(A.cols).to(dev)
    vv = torch.from_numpy(A.elms).to(dev)
    feat = torch.empty((n, 32), dtype=torch.bfloat16, device=dev)
    from . import _lib, _ptr, _check
    add("row features (C2)", timed(lambda: _check(_lib().ispm_row_features(
        n, _ptr(rp), _ptr(ci), _ptr(vv), 128, 128, _ptr(feat), None))), nnz * 12 + n * 68)
    net = LN.MLP(seed=0)
    R = 1 << 23
    X = torch.randn((R, 32), device=dev).to(torch.bfloat16)
    T = torch.randn((R, 2), device=dev)
    flops_f = R * 2 * (32 * 64 + 64 * 64 + 64 * 2)
    add("mlp forward (2^23 rows)", timed(lambda: net.forward(X)), R * (64 + 8), flops_f)
    add("mlp loss + gradient (2^23 rows)",
        timed(lambda: net.loss_grad(X, T, want_grad=False), reps=5), R * (64 + 8), 3 * flops_f)
    return {"peak_hbm_gbs": hbm, "peak_bf16_tflops": bf16, "peak_source": src, "rows": rows}


def run_shapes(log=print):
    import torch
    from . import (gen, ispm_initialize, csr_to_slell, device_split_f16, launch_spmv_split,
                   spmv_launch_params, spmv_stage_fault)
    torch.cuda.init()
    ispm_initialize()
    hbm, _, src = peaks()
    dev = torch.device("cuda")
    flush = torch.empty(1 << 26, dtype=torch.float32, device=dev)  # 256 MB > L2
    rows = []

    def timed_flushed(fn, n=10):
        ts = []
        for _ in range(n):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1) * 1e-3)
        return float(np.median(ts))

    def shapes_of(name, view, nbytes, apply, shapes):
        x = torch.rand(view.n_cols, device=dev)
        y = torch.zeros(view.n_rows, device=dev)
        for N, H in shapes:
            p = spmv_launch_params(N, view.slice_height, H, 1, 1)
            f = lambda: apply(p, x, y)
            warm, cold = timed(f), timed_flushed(f)
            r = {"operator": name, "N": N, "S": view.slice_height, "H": H, "bytes": int(nbytes),
                 "us": warm * 1e6, "frac": nbytes / warm / 1e9 / hbm,
                 "us_flushed": cold * 1e6, "frac_flushed": nbytes / cold / 1e9 / hbm}
            rows.append(r)
            log(f"{name:14s} N={N:3d} S={view.slice_height} H={H}: {r['us']:7.2f} us "
                f"{r['frac']:.3f} | flushed {r['us_flushed']:7.2f} us {r['frac_flushed']:.3f}")
        if spmv_stage_fault():
            raise RuntimeError("the staged walk recorded a wait timeout")

    def nbytes_of(view, esz, extra=0):
        return (4 * view.n_slice_ptr + 4 * view.n_cols_arr + esz * view.n_nz +
                4 * (view.n_cols + view.n_rows) + extra)

    A = gen.stencil_grf(128, 27, 8.0, 1.5, 0)
    n = A.n_rows
    A32 = csr_matrix(n, n, A.row_ptr, A.cols, A.elms.astype(np.float32))
    H = csr_to_slell_guess_format(A32)
    D = H.upload()
    S = D.view().slice_height
    regw = [(S // 4, 4), (S // 2, 2), (S // 8, 8), (S, 1)]
    shapes_of("A FP32", D.view(), nbytes_of(D.view(), 4),
              lambda p, x, y: launch_spmv_kernel(p, D, x, y), regw)
    del D, H
    sp = device_split_f16(A)
    v = sp.view()
    shapes_of("A FP16 split", v, nbytes_of(v, 2, 4 * v.n_rows), sp.apply, regw)
    del sp
    G1, G2 = fsai_sym_gpu(A, np.float64)
    for nm, G in (("G", G1), ("G^T", G2)):
        F = csr_matrix(G.n_rows, G.n_cols, G.row_ptr, G.cols, np.asarray(G.elms).astype(np.float32))
        Hf = csr_to_slell(F, 64, 1, 0, 1)
        Df = Hf.upload()
        shapes_of(nm + " FP32", Df.view(), nbytes_of(Df.view(), 4),
                  lambda p, x, y: launch_spmv_kernel(p, Df, x, y), [(16, 4), (32, 2), (8, 8), (64, 1)])
        del Df, Hf
        # FP16 factor: values times a power of two, the product scaled back
        ge = np.asarray(G.elms, np.float64)
        sc = 2.0 ** (14 - int(np.floor(np.log2(np.abs(ge).max()))))
        v16 = (ge * sc).astype(np.float16).astype(np.float32)
        Hh = csr_to_slell(csr_matrix(G.n_rows, G.n_cols, G.row_ptr, G.cols, v16), 64, 1, 0, 1)
        Dh = Hh.upload_f16()
        vh = Dh.view()
        shapes_of(nm + " FP16", vh, nbytes_of(vh, 2),
                  lambda p, x, y: launch_spmv_split(p, vh, None, 1.0 / sc, x, y),
                  [(16, 4), (8, 8), (64, 1)])
        del Dh, Hh
    return {"peak_hbm_gbs": hbm, "peak_source": src, "shapes": rows}


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(prog="python -m ispm.roofline")
    ap.add_argument("--json", default=None)
    ap.add_argument("--reps", type=int, default=20, help="timed launches per kernel")
    ap.add_argument("--warm", type=int, default=3, help="untimed launches per kernel")
    ap.add_argument("--shapes", action="store_true",
                    help="compare SpMV launch shapes on the headline solver's operators")
    a = ap.parse_args(argv)
    global REPS, WARM
    REPS, WARM = max(1, a.reps), max(0, a.warm)
    log = lambda *m: print(*m, file=sys.stderr, flush=True)
    out = run_shapes(log=log) if a.shapes else run(log=log)
    if a.json:
        json.dump(out, open(a.json, "w"), indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()

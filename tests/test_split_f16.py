"""The FP16 split of A that the mixed solver's matrix_f16 option stores.

CPU: ispm_csr_split_f16 against a numpy restatement of its definition
(binary16 rounding of a_ij * scale, nearest even, subnormals kept; the
diagonal moved by the row's rounding of off-diagonal magnitudes), bit for bit;
the split of an M-matrix keeps A's row sums.
GPU: the split-operator SpMV (ispm_launch_spmv_split) against the long-double
product of the same stored values within the FP32 tolerance (1e-6 relative,
norm-wise; every row within gamma_k * sum |terms|), and mixed solves that
store A this way reach the FP64 true-residual target in at most 1.5x the
iterations of the FP32-stored solve.
"""
import numpy as np
import pytest


def split_restated(A):
    """numpy restatement of ispm_csr_split_f16 (sequential row sums, like the
    library, so the FP32 diagonal matches bit for bit)."""
    n = A.row_ptr.size - 1
    rp, ci, v = A.row_ptr, A.cols, np.asarray(A.elms, np.float64)
    rows = np.repeat(np.arange(n), np.diff(rp))
    offm = ci != rows
    amax = np.abs(v[offm]).max(initial=0.0)
    e = int(np.frexp(amax)[1]) if amax > 0 else 14
    sc = 2.0 ** (14 - e)
    h = np.where(offm, v * sc, 0.0).astype(np.float16)
    hv = h.astype(np.float64)
    diag = np.zeros(n, np.float32)
    for i in range(n):
        d = corr = 0.0
        for k in range(rp[i], rp[i + 1]):
            if ci[k] == i:
                d += float(v[k])
            else:
                corr += abs(float(hv[k])) / sc - abs(float(v[k]))
        diag[i] = np.float32(d + corr)
    return h.view(np.uint16), diag, sc


def small_cases(gen, ispm):
    yield "poisson7 8^3", gen.poisson7(8)
    yield "grf 8^3 27-pt", gen.stencil_grf(8, 27, 4.0, 1.5, 2)
    yield "lognormal 6^3 7-pt", gen.lognormal_stencil(6, 7, 1.0, 3)
    # hand-made: values that become subnormal or underflow to zero after
    # scaling, positive couplings, a row without a diagonal entry, an empty row
    rp = np.array([0, 4, 7, 9, 9, 11], np.int32)
    ci = np.array([0, 1, 2, 4, 0, 1, 3, 1, 3, 0, 4], np.int32)
    big = 1000.0
    v = np.array([5.0, -big, big * (1 + 2.0 ** -11), -1e-9,      # row 0
                  -big, 7.0, 3e-4,                               # row 1
                  1.0 + 3 * 2.0 ** -12, 2.0,                     # row 2: no diagonal
                  # row 3 empty
                  -1e-30, 4.0])                                  # row 4
    yield "hand-made", ispm.csr_matrix(5, 5, rp, ci, v)


def test_split_matches_restatement(ispm, gen):
    for name, A in small_cases(gen, ispm):
        off, diag, sc = ispm.csr_split_f16(A)
        off_r, diag_r, sc_r = split_restated(A)
        assert sc == sc_r, name
        assert np.array_equal(off, off_r), name
        assert np.array_equal(diag.view(np.uint32), diag_r.view(np.uint32)), name


def test_split_scale_and_rounding(ispm):
    # largest off-diagonal magnitude (about 1000) lands in [2^13, 2^14): scale
    # 2^4, where binary16 values are 8 apart; 1000.25 and 1000.75 scale to
    # exact ties (16004, 16012), which go to the even neighbours 16000, 16016
    rp = np.array([0, 2, 4], np.int32)
    ci = np.array([0, 1, 0, 1], np.int32)
    A = ispm.csr_matrix(2, 2, rp, ci, np.array([3000.0, -1000.25, -1000.75, 3000.0]))
    off, diag, sc = ispm.csr_split_f16(A)
    assert sc == 16.0
    vals = off.view(np.float16).astype(np.float64) / sc
    assert vals[1] == -1000.0 and vals[2] == -1001.0
    # each diagonal moved by the magnitude its row gained or lost in rounding
    assert diag[0] == np.float32(3000.0 - 0.25) and diag[1] == np.float32(3000.0 + 0.25)


def test_split_keeps_row_sums(ispm, gen):
    """An M-matrix's split differs from it by a weighted graph Laplacian:
    row sums agree up to the FP32 rounding of the diagonal."""
    A = gen.stencil_grf(10, 27, 4.0, 1.5, 5)
    off, diag, sc = ispm.csr_split_f16(A)
    n = A.n_rows
    rows = np.repeat(np.arange(n), np.diff(A.row_ptr))
    offd = A.cols != rows
    split_vals = np.where(offd, off.view(np.float16).astype(np.float64) / sc, 0.0)
    rs_split = np.bincount(rows, split_vals, n) + diag.astype(np.float64)
    rs_a = np.bincount(rows, A.elms, n)
    tol = np.abs(diag.astype(np.float64)) * 2.0 ** -23 + 1e-12 * np.abs(A.elms).max()
    assert np.all(np.abs(rs_split - rs_a) <= tol)
    # and the off-diagonal values are within 2^-11 relative (normal range)
    a_off = np.where(offd, A.elms, 0.0)
    assert np.all(np.abs(split_vals - a_off) <= 2.0 ** -11 * np.abs(a_off) + 2.0 ** -25 / sc)


def test_split_rejects_non_finite(ispm):
    rp = np.array([0, 2, 4], np.int32)
    ci = np.array([0, 1, 0, 1], np.int32)
    A = ispm.csr_matrix(2, 2, rp, ci, np.array([1.0, np.nan, -1.0, 1.0]))
    with pytest.raises(ispm.IspmError):
        ispm.csr_split_f16(A)


# ---------------------------------------------------------------- GPU ----

@pytest.mark.gpu
@pytest.mark.parametrize("mode", [(32, 1, 0, 1), (64, 1, 0, 0), (64, 2, 0, 0), (32, 4, 0, 0),
                                  (256, 1, 1, 0), (128, 1, 1, 1)])
def test_split_spmv_matches_oracle(ispm, oracle, cuda, gen, mode):
    torch = cuda
    from test_spmv_gpu import as_dict
    for A in (gen.stencil_grf(12, 27, 4.0, 1.5, 1), gen.lognormal_stencil(9, 7, 1.0, 4)):
        d = ispm.device_split_f16(A, mode)
        dv, sc = d.view(), d.scale
        n = A.n_rows
        x = np.random.default_rng(7).uniform(-1, 1, n).astype(np.float32)
        y_off, abs_off = oracle.slell_spmv_exact(as_dict(d.host), x)
        dg = d.diag.cpu().numpy().astype(np.float64)
        xp = np.zeros(dv.n_rows)
        xp[:n] = x
        y_ex = y_off / sc + dg * xp
        absrow = abs_off / sc + np.abs(dg * xp)
        k = int(np.diff(A.row_ptr).max()) + 2
        u = 2.0 ** -24
        gamma = k * u / (1 - k * u)
        xt = torch.from_numpy(x).cuda()
        shapes = [ispm.default_launch_params(dv, ispm.F32)]
        if dv.var_height:
            shapes.append(ispm.spmv_launch_params(dv.max_slice_height, dv.max_slice_height,
                                                  1, 1, 1))
        elif dv.slice_height <= 64:
            shapes.append(ispm.spmv_launch_params(64, dv.slice_height, 1, 1, 1))
        if dv.hblock == 1:  # eight rows a thread: one 16-byte element load
            if dv.var_height and dv.min_slice_height >= 8:
                n8 = max(dv.max_slice_height // 8, 4)
                shapes.append(ispm.spmv_launch_params(n8, n8 * 8, 8, 1, 1))
            elif not dv.var_height and dv.slice_height >= 32:
                shapes.append(ispm.spmv_launch_params(dv.slice_height // 8, dv.slice_height,
                                                      8, 1, 1))
        for p in shapes:
            y = torch.full((dv.n_rows + 8,), float("nan"), dtype=torch.float32, device="cuda")
            d.apply(p, xt, y)
            torch.cuda.synchronize()
            yh = y.cpu().numpy()
            assert np.all(np.isnan(yh[dv.n_rows:])), "wrote past the padded rows"
            yh = yh[: dv.n_rows].astype(np.float64)
            err = np.abs(yh - y_ex)
            assert np.all(err <= gamma * absrow + 1e-300), (mode, p.N, p.H, err.max())
            assert np.linalg.norm(err) / np.linalg.norm(absrow) <= 1e-6


@pytest.mark.gpu
def test_split_spmv_rejects_missing_diagonal(ispm, cuda, gen):
    torch = cuda
    A = gen.poisson7(8)
    d = ispm.device_split_f16(A, (32, 1, 0, 1))
    x = torch.zeros(A.n_rows, dtype=torch.float32, device="cuda")
    y = torch.zeros(d.view().n_rows, dtype=torch.float32, device="cuda")
    p = ispm.default_launch_params(d, ispm.F32)
    with pytest.raises(ispm.IspmError):
        ispm.launch_spmv_kernel(p, d, x, y)  # FP16 elements need the split entry


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["c1", "grf"])
def test_split_solver_reaches_target(ispm, cuda, gen, case):
    import scipy.sparse as sp
    A = gen.poisson7(32) if case == "c1" else gen.stencil_grf(32, 27, 8.0, 1.5, 0)
    M = sp.csr_matrix((A.elms, A.cols, A.row_ptr), shape=(A.n_rows, A.n_cols))
    b = M @ np.random.default_rng(0).uniform(-1, 1, A.n_rows)
    its = {}
    for f16 in (False, True):
        S = ispm.PCGSolver(A, inner=np.float32, tol=1e-10, prec="fsai_gpu", matrix_f16=f16)
        x, st = S.solve_host(b)
        assert st["converged"], (case, f16, st)
        assert st["true_relres"] <= 1e-10
        assert np.linalg.norm(b - M @ x) / np.linalg.norm(b) <= 1.05e-10, (case, f16)
        its[f16] = st["iterations"]
    # The split inner matrix costs iterations on some systems (on a B200:
    # within 8% on the 32^3 Poisson system, 134 against 99 on this 32^3 GRF
    # system, 508 against 501 on the 128^3 one); bound the cost.
    assert its[True] <= 1.5 * its[False] + 4, its

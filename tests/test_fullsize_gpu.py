"""Full-size parity: the launches the bench and the solver time, at the
benchmark sizes, against the C oracle.

* 128^3 27-point GRF system (2,097,152 rows, 55,742,968 entries; the bench's
  headline matrix, same generator and seed): A as FP32 and FP64 elements in
  the guessed shape (S = 64, diagonal blocks) at the default launch (the
  staged walk) and at the register walk (N = 64 / H, H rows per thread);
  A's FP16 split; the GPU-built FSAI factor G and its transpose in the
  diagonal-block shapes the solver picks from.  Each product is checked
  against the oracle's long-double slice walk of the same stored matrix:
  FP64 within 1e-14, FP32 within 1e-6 (norm-wise, relative to
  sum |a_ij x_j|), every row within gamma_k * sum |a_ij x_j|.
* Every row of the GPU FSAI factor of that system against the C oracle's
  dense per-row construction (oracle/ispm_oracle.c orc_fsai_rows): the same
  rows, the same pattern, values within 1e-10 relative per row.
* The 192^3 unstructured permuted system (7,077,888 rows) in the shape the
  exhaustive plan picks, through the plan's own launch.
* The headline solve itself: mixed FP32/FP64 PCG with the GPU FSAI to a true
  FP64 residual of 1e-10 on the 128^3 system.
"""
import numpy as np
import pytest

from test_spmv_gpu import as_dict

pytestmark = pytest.mark.gpu

REL32, REL64 = 1e-6, 1e-14


@pytest.fixture(scope="module")
def c2(gen):
    return gen.stencil_grf(128, 27, 8.0, 1.5, 0)


def check(oracle, torch, B, run, T, rel, seed=0, kmax=32):
    """run(x_tensor, y_tensor) computes y = B x on the device."""
    n_cols = B.view().n_cols
    x = np.random.default_rng(seed).uniform(-1, 1, n_cols).astype(T)
    y_ex, absrow = oracle.slell_spmv_exact(as_dict(B), x)
    tdt = torch.float64 if T == np.float64 else torch.float32
    y = torch.full((B.n_rows + 8,), float("nan"), dtype=tdt, device="cuda")
    run(torch.from_numpy(x).cuda(), y)
    torch.cuda.synchronize()
    yh = y.cpu().numpy()
    assert np.all(np.isnan(yh[B.n_rows:])), "wrote past the padded rows"
    yh = yh[: B.n_rows].astype(np.float64)
    err = np.abs(yh - y_ex)
    u = 2.0 ** -53 if T == np.float64 else 2.0 ** -24
    gamma = kmax * u / (1 - kmax * u)
    assert np.all(err <= gamma * absrow + 1e-300), err.max()
    r = np.linalg.norm(err) / np.linalg.norm(absrow)
    assert r <= rel, r
    return r


@pytest.mark.parametrize("T", [np.float32, np.float64], ids=["f32", "f64"])
def test_c2_a_spmv(ispm, oracle, cuda, c2, T):
    A = ispm.csr_matrix(c2.n_rows, c2.n_cols, c2.row_ptr, c2.cols, c2.elms.astype(T))
    B = ispm.csr_to_slell_guess_format(A)
    assert (B.slice_height, B.diags, B.hblock, bool(B.var_height)) == (64, 1, 1, False)
    dB = B.upload()
    rel = REL32 if T == np.float32 else REL64
    # the default shape (the one the bench times), the staged walk, and the
    # register walk at the other rows-per-thread counts
    shapes = [ispm.default_launch_params(dB, T)]
    for N, H in ((64, 1), (16, 4), (32, 2)):
        shapes.append(ispm.spmv_launch_params(N, 64, H, 1, 1))
    for k, p in enumerate(shapes):
        check(oracle, cuda, B, lambda x, y: ispm.launch_spmv_kernel(p, dB, x, y), T, rel,
              seed=k, kmax=28)


def test_c2_a_split_f16(ispm, oracle, cuda, c2):
    torch = cuda
    d = ispm.device_split_f16(c2)
    dv, sc = d.view(), d.scale
    p = ispm.default_launch_params(dv, ispm.F32)
    n = c2.n_rows
    x = np.random.default_rng(2).uniform(-1, 1, n).astype(np.float32)
    y_off, abs_off = oracle.slell_spmv_exact(as_dict(d.host), x)
    dg = d.diag.cpu().numpy().astype(np.float64)
    xp = np.zeros(dv.n_rows)
    xp[:n] = x
    y_ex = y_off / sc + dg * xp
    absrow = abs_off / sc + np.abs(dg * xp)
    gamma = 30 * 2.0 ** -24 / (1 - 30 * 2.0 ** -24)
    y = torch.full((dv.n_rows + 8,), float("nan"), dtype=torch.float32, device="cuda")
    d.apply(p, torch.from_numpy(x).cuda(), y)
    torch.cuda.synchronize()
    yh = y.cpu().numpy()
    assert np.all(np.isnan(yh[dv.n_rows:]))
    err = np.abs(yh[: dv.n_rows].astype(np.float64) - y_ex)
    assert np.all(err <= gamma * absrow + 1e-300), err.max()
    assert np.linalg.norm(err) / np.linalg.norm(absrow) <= REL32


@pytest.fixture(scope="module")
def c2_fsai(ispm, cuda, c2):
    st = {}
    G1, G2 = ispm.fsai_sym_gpu(c2, np.float64, stats=st)
    return G1, G2, st


def test_c2_fsai_values_every_row(ispm, oracle, c2, c2_fsai):
    G1, G2, st = c2_fsai
    rows = np.arange(c2.n_rows, dtype=np.int32)
    orp, oci, ov, jac = oracle.fsai_rows_f64(c2.row_ptr, c2.cols, c2.elms, rows)
    assert st["fallbacks"] == jac == 0
    assert np.array_equal(G1.row_ptr, orp) and np.array_equal(G1.cols, oci)
    gv = np.asarray(G1.elms, np.float64)
    rid = np.repeat(rows, np.diff(orp))
    num = np.sqrt(np.bincount(rid, (gv - ov) ** 2, c2.n_rows))
    den = np.sqrt(np.bincount(rid, ov ** 2, c2.n_rows))
    assert np.all(num <= 1e-10 * den), float((num / den).max())
    # the second factor is the transpose of the first
    import scipy.sparse as sp
    g = sp.csr_matrix((gv, G1.cols, G1.row_ptr), shape=(c2.n_rows, c2.n_cols))
    gt = g.T.tocsr()
    gt.sort_indices()
    assert np.array_equal(gt.indptr, G2.row_ptr) and np.array_equal(gt.indices, G2.cols)
    assert np.array_equal(gt.data, np.asarray(G2.elms, np.float64))


@pytest.mark.parametrize("which", ["G", "Gt"])
@pytest.mark.parametrize("S", [32, 64])
def test_c2_fsai_factor_spmv(ispm, oracle, cuda, c2, c2_fsai, which, S):
    G = c2_fsai[0] if which == "G" else c2_fsai[1]
    F = ispm.csr_matrix(G.n_rows, G.n_cols, G.row_ptr, G.cols,
                        np.asarray(G.elms, np.float64).astype(np.float32))
    B = ispm.csr_to_slell(F, S, 1, 0, 1)
    dB = B.upload()
    for k, p in enumerate((ispm.default_launch_params(dB, np.float32),
                           ispm.spmv_launch_params(S, S, 1, 1, 1))):
        check(oracle, cuda, B, lambda x, y: ispm.launch_spmv_kernel(p, dB, x, y), np.float32,
              REL32, seed=3 + k, kmax=15)


def test_c3_plan_spmv(ispm, oracle, cuda, gen):
    A = gen.unstructured(192, seed=1)
    A32 = ispm.csr_matrix(A.n_rows, A.n_cols, A.row_ptr, A.cols, A.elms.astype(np.float32))
    plan = ispm.spmv_plan(A32, ispm.PLAN_EXHAUSTIVE, T=np.float32)
    B = plan.host_matrix
    check(oracle, cuda, B, lambda x, y: plan.execute_spmv(x, y), np.float32, REL32, seed=4,
          kmax=8)


def test_c2_headline_solve(ispm, oracle, cuda, c2):
    b = oracle.csr_spmv_f64(c2.row_ptr, c2.cols, c2.elms,
                            np.random.default_rng(0).uniform(-1, 1, c2.n_rows))
    S = ispm.PCGSolver(c2, None, None, inner=np.float32, tol=1e-10, prec="fsai_gpu")
    x, st = S.solve_host(b)
    assert st["converged"], st
    r = b - oracle.csr_spmv_f64(c2.row_ptr, c2.cols, c2.elms, x)
    rel = np.linalg.norm(r) / np.linalg.norm(b)
    assert rel <= 1.001e-10, rel
    assert abs(rel - st["true_relres"]) <= 1e-3 * rel + 1e-16

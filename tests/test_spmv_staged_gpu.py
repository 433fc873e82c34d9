"""The staged SpMV walk (launch shape N = S, H = 1 on diagonal-block
matrices: 256-row tiles whose elements and x bands a copy warp moves into
shared memory with bulk copies) against the CPU oracle's long-double slice
walk (cuda/spmv/kernel.h:80-92).

Tiles stage when their windows fit 64 diagonals, 8 bands and the x-area
budget; other tiles read everything from global memory.  These cases drive
each branch: uniform interior tiles, boundary tiles whose slices differ or
carry explicit-column entries, bands reaching past either end of x (zero
fill, a ragged last chunk), bands over the limits, more diagonals than the
staged walk takes, rectangular matrices, x not 16-byte aligned (the launch
takes the register walk), every slice height (512 exceeds a tile: register
walk), both vector types, FP16 split and FP16 factor elements.  After every
launch the kernel's wait-timeout record must read 0.

Tolerances as in test_spmv_gpu: FP64 within 1e-14, FP32 within 1e-6
(norm-wise, relative to sum |a_ij x_j|), and every row within
gamma_k * sum_j |a_ij x_j|.
"""
import numpy as np
import pytest

from test_spmv_gpu import REL, as_dict

pytestmark = pytest.mark.gpu


def multidiag(ispm, n_rows, n_cols, offsets, seed):
    """Rows i with entries at columns i + o (o in offsets) inside [0, n_cols)."""
    rng = np.random.default_rng(seed)
    i = np.arange(n_rows)
    rows, cols = [], []
    for o in sorted(offsets):
        c = i + o
        ok = (c >= 0) & (c < n_cols)
        rows.append(i[ok])
        cols.append(c[ok])
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    order = np.lexsort((c, r))
    r, c = r[order], c[order]
    rp = np.zeros(n_rows + 1, np.int32)
    rp[1:] = np.cumsum(np.bincount(r, minlength=n_rows))
    v = rng.uniform(-1, 1, r.size)
    return ispm.csr_matrix(n_rows, n_cols, rp, c.astype(np.int32), v)


def run_staged(ispm, oracle, torch, A, S, T, E, x_offset=0):
    Ac = ispm.csr_matrix(A.n_rows, A.n_cols, A.row_ptr.copy(), A.cols.copy(),
                         A.elms.astype(E))
    B = ispm.csr_to_slell(Ac, S, 1, 0, 1)
    assert B.diags and not B.var_height
    dB = B.upload()
    x = np.random.default_rng(11).uniform(-1, 1, A.n_cols).astype(T)
    y_ex, absrow = oracle.slell_spmv_exact(as_dict(B), x)
    k = int(np.diff(A.row_ptr).max(initial=0)) + 1
    u = 2.0 ** -53 if T == np.float64 else 2.0 ** -24
    gamma = k * u / (1 - k * u)
    tdt = torch.float64 if T == np.float64 else torch.float32
    # x at an element offset inside a larger buffer: x_offset = 1 leaves it
    # 4 or 8 bytes past a 16-byte boundary
    buf = torch.zeros(A.n_cols + 4, dtype=tdt, device="cuda")
    buf[x_offset: x_offset + A.n_cols] = torch.from_numpy(x).cuda()
    xt = buf[x_offset: x_offset + A.n_cols]
    y = torch.full((B.n_rows + 8,), float("nan"), dtype=tdt, device="cuda")
    ispm.launch_spmv_kernel(ispm.spmv_launch_params(S, S, 1, 1, 1), dB, xt, y)
    torch.cuda.synchronize()
    assert ispm.spmv_stage_fault() == 0
    yh = y.cpu().numpy()
    assert np.all(np.isnan(yh[B.n_rows:])), "wrote past the padded rows"
    yh = yh[: B.n_rows].astype(np.float64)
    assert np.all(np.isfinite(yh)), "rows left unwritten"
    err = np.abs(yh - y_ex)
    assert np.all(err <= gamma * absrow + 1e-300), err.max()
    den = np.linalg.norm(absrow)
    if den > 0:
        assert np.linalg.norm(err) / den <= REL[(T, E)]
    return B


TE = [(np.float64, np.float64), (np.float64, np.float32), (np.float32, np.float32)]


@pytest.mark.parametrize("T,E", TE, ids=["dd", "df", "ff"])
@pytest.mark.parametrize("S", [16, 32, 64, 128, 256, 512])
def test_staged_stencils(ispm, oracle, cuda, gen, S, T, E):
    # 24^3 7-point (13,824 rows) and 20^3 27-point GRF (8,000 rows): interior
    # tiles stage, tiles at the grid's y/z faces mix slices with different
    # diagonal sets, the first and last tiles' bands reach past x
    for A in (gen.poisson7(24), gen.stencil_grf(20, 27, 4.0, 1.5, 2)):
        run_staged(ispm, oracle, cuda, A, S, T, E)


@pytest.mark.parametrize("T,E", TE, ids=["dd", "df", "ff"])
def test_staged_far_apart_diagonals_exceed_budget(ispm, oracle, cuda, T, E):
    # 15 diagonals 700 apart: 15 bands, more than the 8 a tile stages ->
    # interior tiles read everything from global memory
    offs = [700 * k for k in range(-7, 8)]
    A = multidiag(ispm, 20000, 20000, offs, 1)
    run_staged(ispm, oracle, cuda, A, 64, T, E)


@pytest.mark.parametrize("T,E", TE, ids=["dd", "df", "ff"])
def test_staged_many_diagonals(ispm, oracle, cuda, T, E):
    # 70 consecutive diagonals: more than the staged walk's 64
    A = multidiag(ispm, 6000, 6000, list(range(-35, 35)), 2)
    run_staged(ispm, oracle, cuda, A, 32, T, E)
    # 64 exactly, in one band
    A = multidiag(ispm, 6000, 6000, list(range(-32, 32)), 3)
    run_staged(ispm, oracle, cuda, A, 32, T, E)


@pytest.mark.parametrize("T,E", TE, ids=["dd", "df", "ff"])
def test_staged_rectangular_and_ragged_x(ispm, oracle, cuda, T, E):
    # wide (x longer than y), tall (x shorter), and x lengths that are not a
    # multiple of four: the band edges fall back to scalar staging
    for n_rows, n_cols in ((5000, 9003), (9000, 4001), (4096, 4097)):
        A = multidiag(ispm, n_rows, n_cols, [-300, -1, 0, 1, 2, 5, 300, 4000], 4)
        run_staged(ispm, oracle, cuda, A, 64, T, E)


@pytest.mark.parametrize("T,E", TE, ids=["dd", "df", "ff"])
def test_staged_unaligned_x(ispm, oracle, cuda, gen, T, E):
    A = gen.stencil_grf(16, 27, 4.0, 1.5, 5)
    run_staged(ispm, oracle, cuda, A, 32, T, E, x_offset=1)
    run_staged(ispm, oracle, cuda, A, 64, T, E, x_offset=0)


def test_staged_split_operator(ispm, oracle, cuda, gen):
    """FP16-split elements through the staged walk (diagonal added in the
    store epilogue)."""
    torch = cuda
    A = gen.stencil_grf(48, 27, 8.0, 1.5, 0)  # 110,592 rows: the default shape stages
    d = ispm.device_split_f16(A, (64, 1, 0, 1))
    dv, sc = d.view(), d.scale
    p = ispm.spmv_launch_params(64, 64, 1, 1, 1)
    n = A.n_rows
    x = np.random.default_rng(7).uniform(-1, 1, n).astype(np.float32)
    y_off, abs_off = oracle.slell_spmv_exact(as_dict(d.host), x)
    dg = d.diag.cpu().numpy().astype(np.float64)
    xp = np.zeros(dv.n_rows)
    xp[:n] = x
    y_ex = y_off / sc + dg * xp
    absrow = abs_off / sc + np.abs(dg * xp)
    k = int(np.diff(A.row_ptr).max()) + 2
    gamma = k * 2.0 ** -24 / (1 - k * 2.0 ** -24)
    y = torch.full((dv.n_rows + 8,), float("nan"), dtype=torch.float32, device="cuda")
    d.apply(p, torch.from_numpy(x).cuda(), y)
    torch.cuda.synchronize()
    assert ispm.spmv_stage_fault() == 0
    yh = y.cpu().numpy()
    assert np.all(np.isnan(yh[dv.n_rows:]))
    err = np.abs(yh[: dv.n_rows].astype(np.float64) - y_ex)
    assert np.all(err <= gamma * absrow + 1e-300), err.max()
    assert np.linalg.norm(err) / np.linalg.norm(absrow) <= 1e-6


@pytest.mark.parametrize("S", [32, 64])
def test_staged_f16_factor(ispm, oracle, cuda, gen, S):
    """FP16-stored elements times a power of two without a diagonal vector
    (the factor_f16 option's G and G^T): y = inv_scale * (stored sum)."""
    torch = cuda
    A = gen.stencil_grf(40, 27, 8.0, 1.5, 3)
    ge = A.elms.astype(np.float64)
    e = int(np.floor(np.log2(np.abs(ge).max())))
    sc = 2.0 ** (14 - e)
    v16 = (ge * sc).astype(np.float16).astype(np.float32)
    H = ispm.csr_to_slell(ispm.csr_matrix(A.n_rows, A.n_cols, A.row_ptr, A.cols, v16), S, 1, 0, 1)
    dH = H.upload_f16()
    x = np.random.default_rng(9).uniform(-1, 1, A.n_cols).astype(np.float32)
    y_st, ab_st = oracle.slell_spmv_exact(as_dict(H), x)
    y_ex, absrow = y_st / sc, ab_st / sc
    k = int(np.diff(A.row_ptr).max()) + 1
    gamma = k * 2.0 ** -24 / (1 - k * 2.0 ** -24)
    for p in (ispm.spmv_launch_params(S, S, 1, 1, 1), ispm.default_launch_params(dH.view(), ispm.F32)):
        y = torch.full((H.n_rows + 8,), float("nan"), dtype=torch.float32, device="cuda")
        ispm.launch_spmv_split(p, dH.view(), None, 1.0 / sc, torch.from_numpy(x).cuda(), y)
        torch.cuda.synchronize()
        assert ispm.spmv_stage_fault() == 0
        yh = y.cpu().numpy()
        assert np.all(np.isnan(yh[H.n_rows:]))
        err = np.abs(yh[: H.n_rows].astype(np.float64) - y_ex)
        assert np.all(err <= gamma * absrow + 1e-300), (p.N, p.H, err.max())
        assert np.linalg.norm(err) / np.linalg.norm(absrow) <= 1e-6

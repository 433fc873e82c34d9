"""Sliced-ELL SpMV on the GPU against the CPU oracle (cuda/spmv/kernel.h).

Tolerances: FP64 results within 1e-14 relative, FP32 within
1e-6 relative (norm-wise, against the long-double sum of the same stored
values); every row also within the worst-case forward-error bound
gamma_k * sum_j |a_ij x_j| of a k-term sum, whatever the summation order.
The oracle's reference-order emulation (the kernel's own partial sums and
column reduction) is held to the same tolerances.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = {(np.float64, np.float64): 1e-14, (np.float64, np.float32): 1e-14,
       (np.float32, np.float32): 1e-6}


def as_dict(B):
    v = B.view()
    return dict(n_rows=v.n_rows, n_cols=v.n_cols, slice_height=v.slice_height,
                n_slices=v.n_slices, hblock=v.hblock, var_height=v.var_height, diags=v.diags,
                slice_ptr=B.slice_ptr, cols=B.cols, elms=B.elms.copy())


def launches(B, T=None):
    """Every valid launch shape; H = 8 (eight rows a thread, FP32 vectors and
    hblock 1 only) is this library's addition to the reference's 1, 2, 4."""
    v = B.view()
    out = []
    hs = (1, 2, 4, 8) if T == np.float32 and v.hblock == 1 else (1, 2, 4)
    for N in (4, 8, 16, 32, 64, 128, 256, 512, 1024):
        for H in hs:
            S = N * H if v.var_height else v.slice_height
            if v.var_height and (N * H < v.max_slice_height or H > v.min_slice_height):
                continue
            if not v.var_height and not (N >= S // H and S >= H):
                continue
            out.append((N, S, H))
    return out


def check_case(ispm, oracle, torch, A, mode, T, E, seed=0, all_launches=True):
    Ac = ispm.csr_matrix(A.n_rows, A.n_cols, A.row_ptr.copy(), A.cols.copy(),
                         A.elms.astype(E))
    S, W, V, D = mode
    B = ispm.csr_to_slell(Ac, S, W, V, D)
    dB = B.upload()
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, max(A.n_cols, 1)).astype(T)[: A.n_cols]
    m = as_dict(B)
    y_ex, absrow = oracle.slell_spmv_exact(m, x)
    k = max(1, int(np.diff(A.row_ptr).max(initial=0)) + 1)
    u = 2.0 ** -53 if T == np.float64 else 2.0 ** -24
    gamma = k * u / (1 - k * u)
    rel = REL[(T, E)]
    xt = torch.from_numpy(x.copy()).cuda() if A.n_cols else torch.zeros(1, dtype=torch.float64 if T == np.float64 else torch.float32, device="cuda")
    tdt = torch.float64 if T == np.float64 else torch.float32
    todo = launches(B, T) if all_launches else launches(B)[:3]
    assert todo, "no valid launch shape"
    for N, SS, H in todo:
        y = torch.full((B.n_rows + 8,), float("nan"), dtype=tdt, device="cuda")
        p = ispm.spmv_launch_params(N, SS, H, 1, 1)
        ispm.launch_spmv_kernel(p, dB, xt, y)
        torch.cuda.synchronize()
        yh = y.cpu().numpy()
        assert np.all(np.isnan(yh[B.n_rows:])), "wrote past the padded rows"
        yh = yh[: B.n_rows].astype(np.float64)
        assert np.all(np.isfinite(yh)), f"rows left unwritten for N={N} H={H}"
        err = np.abs(yh - y_ex)
        assert np.all(err <= gamma * absrow + 1e-300), (mode, N, H, err.max())
        den = np.linalg.norm(absrow)
        if den > 0:
            assert np.linalg.norm(err) / den <= rel, (mode, N, H)
        # the oracle's emulation of the reference kernel's own summation order
        if H == 8:
            continue
        yk = oracle.slell_spmv_kernel_order(m, x, N, H).astype(np.float64)
        if den > 0:
            assert np.linalg.norm(yk - y_ex) / den <= rel
    return B


MODES_ALL = [(32, 1, 0, 1), (64, 1, 0, 0), (32, 2, 0, 0), (64, 4, 0, 0), (256, 1, 1, 0),
             (256, 1, 1, 1), (128, 2, 1, 0), (16, 1, 0, 1), (512, 1, 0, 0), (128, 4, 1, 0)]
TE = [(np.float64, np.float64), (np.float64, np.float32), (np.float32, np.float32)]


@pytest.fixture(scope="module")
def mats(gen):
    return {
        "poisson7_16": gen.poisson7(16),
        "grf27_12": gen.stencil_grf(12, 27, 4.0, 1.5, 3),
        "band3000": gen.random_csr(3000, 3000, 41, mean_len=10, band=40),
        "odd_pairs1001": gen.random_csr(1001, 1001, 42, mean_len=7, pair_frac=0.9),
        "wide800x2001": gen.random_csr(800, 2001, 43, mean_len=16, pair_frac=0.5),
        "unstructured14": gen.unstructured(14, seed=5),
        "tiny5": gen.random_csr(5, 7, 44, mean_len=3),
    }


@pytest.mark.parametrize("T,E", TE, ids=["dd", "df", "ff"])
@pytest.mark.parametrize("name", ["poisson7_16", "grf27_12", "band3000", "odd_pairs1001",
                                  "wide800x2001", "unstructured14", "tiny5"])
def test_spmv_matches_oracle(ispm, oracle, cuda, mats, name, T, E):
    A = mats[name]
    for mode in MODES_ALL:
        check_case(ispm, oracle, cuda, A, mode, T, E, all_launches=(T, E) != TE[1])


def test_spmv_guess_format_c1(ispm, oracle, cuda, gen):
    # config 1 shape: 32^3 7-point Poisson, S=32 with diagonal blocks
    A = gen.poisson7(32)
    B = check_case(ispm, oracle, cuda, A, (32, 1, 0, 1), np.float64, np.float64)
    assert len(B.cols) == 0
    check_case(ispm, oracle, cuda, A, (32, 1, 0, 1), np.float32, np.float32)


def test_spmv_empty_and_zero_rows(ispm, oracle, cuda):
    Z = ispm.csr_matrix(700, 700, np.zeros(701, np.int32), np.zeros(0, np.int32),
                        np.zeros(0))
    for mode in ((32, 1, 0, 1), (64, 2, 0, 0), (256, 1, 1, 0)):
        Ac = ispm.csr_matrix(700, 700, Z.row_ptr.copy(), Z.cols, Z.elms)
        B = ispm.csr_to_slell(Ac, *mode)
        dB = B.upload()
        x = cuda.ones(700, dtype=cuda.float64, device="cuda")
        y = cuda.full((B.n_rows,), 7.0, dtype=cuda.float64, device="cuda")
        p = ispm.spmv_launch_params(256, 256 if mode[2] else mode[0], 1, 1, 1)
        ispm.launch_spmv_kernel(p, dB, x, y)
        assert float(y.abs().max()) == 0.0


def test_spmv_rejects_invalid_launches(ispm, cuda, gen):
    A = gen.poisson7(8)
    B = ispm.csr_to_slell(A, 32, 1, False, True)
    dB = B.upload()
    x = cuda.ones(B.n_cols, dtype=cuda.float64, device="cuda")
    y = cuda.zeros(B.n_rows, dtype=cuda.float64, device="cuda")
    for N, S, H in ((16, 64, 1), (64, 64, 1), (3, 32, 1), (64, 32, 3), (8, 32, 2)):
        with pytest.raises(ispm.IspmError):
            ispm.launch_spmv_kernel(ispm.spmv_launch_params(N, S, H, 1, 1), dB, x, y)
    xf = cuda.ones(B.n_cols, dtype=cuda.float32, device="cuda")
    yf = cuda.zeros(B.n_rows, dtype=cuda.float32, device="cuda")
    with pytest.raises(ispm.IspmError):  # (float, double) is not instantiated
        ispm.launch_spmv_kernel(ispm.spmv_launch_params(64, 32, 1, 1, 1), dB, xf, yf)


def test_spmv_full_size_properties(ispm, cuda, gen):
    """C2-sized 128^3 27-point matrix: the linearity A(ax + by) = aAx + bAy and
    agreement of FP32/FP64 results, checked on the GPU alone (sizes the CPU
    oracle would take minutes on)."""
    A = gen.stencil_grf(128, 27, 8.0, 1.5, 0)
    B64 = ispm.csr_to_slell_guess_format(ispm.csr_matrix(A.n_rows, A.n_cols, A.row_ptr,
                                                         A.cols, A.elms))
    assert B64.diags and B64.slice_height == 64
    d64 = B64.upload()
    n = A.n_rows
    g = cuda.Generator(device="cuda").manual_seed(0)
    x1 = cuda.rand(n, dtype=cuda.float64, device="cuda", generator=g) - 0.5
    x2 = cuda.rand(n, dtype=cuda.float64, device="cuda", generator=g) - 0.5
    p = ispm.spmv_launch_params(16, 64, 4, 1, 1)
    ys = [cuda.zeros(B64.n_rows, dtype=cuda.float64, device="cuda") for _ in range(3)]
    ispm.launch_spmv_kernel(p, d64, x1, ys[0])
    ispm.launch_spmv_kernel(p, d64, x2, ys[1])
    ispm.launch_spmv_kernel(p, d64, (2.0 * x1 - 3.0 * x2).contiguous(), ys[2])
    lin = (ys[2] - (2.0 * ys[0] - 3.0 * ys[1])).abs().max().item()
    scale = (2 * ys[0].abs() + 3 * ys[1].abs()).max().item()
    assert lin <= 1e-12 * scale
    # the same product on the FP32 copy of the matrix
    A32 = ispm.csr_matrix(A.n_rows, A.n_cols, A.row_ptr, A.cols, A.elms.astype(np.float32))
    B32 = ispm.csr_to_slell(A32, 64, 1, False, True)
    d32 = B32.upload()
    y32 = cuda.zeros(B32.n_rows, dtype=cuda.float32, device="cuda")
    ispm.launch_spmv_kernel(ispm.spmv_launch_params(16, 64, 4, 1, 1), d32,
                            x1.float().contiguous(), y32)
    rel = ((y32.double() - ys[0]).norm() / ys[0].norm()).item()
    assert rel < 1e-4  # differences from rounding A and x to FP32 (cancellation-heavy rows)

"""spmv_plan (plan/plan.h): format from the reference's guess, launch shape
from the B200 heuristic or the exhaustive search; execute_spmv against the
oracle; coefficient refresh and host-matrix change."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check_plan(ispm, oracle, torch, A, plan, T):
    B = plan.host_matrix
    m = dict(n_rows=B.n_rows, n_cols=B.n_cols, slice_height=B.slice_height,
             n_slices=B.n_slices, hblock=B.hblock, var_height=B.var_height, diags=B.diags,
             slice_ptr=B.slice_ptr, cols=B.cols, elms=B.elms.copy())
    x = np.random.default_rng(2).uniform(-1, 1, A.n_cols).astype(T)
    y_ex, absrow = oracle.slell_spmv_exact(m, x)
    tdt = torch.float64 if T == np.float64 else torch.float32
    y = torch.zeros(B.n_rows, dtype=tdt, device="cuda")
    plan.execute_spmv(torch.from_numpy(x).cuda(), y)
    err = np.abs(y.cpu().numpy().astype(np.float64) - y_ex)
    rel = 1e-14 if T == np.float64 else 1e-6
    assert np.linalg.norm(err) <= rel * np.linalg.norm(absrow)
    return y


@pytest.mark.parametrize("T,E", [(np.float64, np.float64), (np.float64, np.float32),
                                 (np.float32, np.float32)], ids=["dd", "df", "ff"])
def test_plan_default_and_exhaustive(ispm, oracle, cuda, gen, T, E):
    for A in (gen.poisson7(20), gen.random_csr(4000, 4000, 51, mean_len=12, pair_frac=0.5)):
        Ae = A.astype(E)
        p = ispm.spmv_plan(Ae, ispm.PLAN_DEFAULT, 0, T=T)
        ref_fmt = ispm.csr_to_slell_guess_format(A.astype(E))
        assert (p.mparams.S, p.mparams.H, p.mparams.V, p.mparams.D) == (
            ref_fmt.slice_height, ref_fmt.hblock, int(ref_fmt.var_height), int(ref_fmt.diags))
        _check_plan(ispm, oracle, cuda, A, p, T)
        px = ispm.spmv_plan(A.astype(E), ispm.PLAN_EXHAUSTIVE, 0, T=T)
        assert px.tuned_seconds > 0
        _check_plan(ispm, oracle, cuda, A, px, T)


def test_plan_coefficient_refresh_and_change(ispm, oracle, cuda, gen):
    A = gen.stencil_grf(12, 27, 4.0, 1.5, 1)
    p = ispm.spmv_plan(A, ispm.PLAN_DEFAULT)
    y0 = _check_plan(ispm, oracle, cuda, A, p, np.float64)
    # update_device_matrix_coefs: edit the host values, refresh the device copy
    h = p.host_matrix
    h.elms[:] *= 2.0
    p.update_device_matrix_coefs()
    x = np.random.default_rng(2).uniform(-1, 1, A.n_cols)
    y = cuda.zeros(h.n_rows, dtype=cuda.float64, device="cuda")
    p.execute_spmv(cuda.from_numpy(x).cuda(), y)
    assert cuda.allclose(y, 2.0 * y0, rtol=1e-14, atol=1e-14)
    # change_host_matrix re-converts with the stored format, upload() moves it
    A2 = gen.stencil_grf(12, 27, 4.0, 1.5, 2)
    p.change_host_matrix(A2)
    p.upload()
    _check_plan(ispm, oracle, cuda, A2, p, np.float64)


def test_plan_without_device(ispm, cuda, gen):
    A = gen.poisson7(8)
    p = ispm.spmv_plan(A, ispm.PLAN_DEFAULT, ispm.SPMV_PLAN_NO_DEVICE)
    assert p.device_matrix is None and p.host_matrix is not None
    x = cuda.ones(A.n_cols, dtype=cuda.float64, device="cuda")
    y = cuda.zeros(p.host_matrix.n_rows, dtype=cuda.float64, device="cuda")
    with pytest.raises(ispm.IspmError):
        p.execute_spmv(x, y)
    p.upload()
    p.execute_spmv(x, y)

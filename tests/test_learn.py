"""Learned drop tolerances, CPU side: the numpy oracle of the MLP (checked
against finite differences of its own unrounded FP64 form), the BF16
rounding it shares with the GPU kernels, and the feature layout.  The
reference has no learned component; the model replaces the search of
fastainv/droptol-tuning.h:4-103."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def lo():
    import learn_oracle
    return learn_oracle


def test_bf16_rounding(lo):
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, -2.5, 0.0, 3e-39],
                 np.float32)
    assert lo.bf16(x)[0] == 1.0
    # exact halfway cases go to even
    assert lo.bf16(np.float32(1.0 + 2 ** -8)) == np.float32(1.0)
    assert lo.bf16(np.float32(1.0 + 3 * 2 ** -8)) == np.float32(1.0 + 2 ** -6)
    assert lo.bf16(np.float32(-2.5)) == np.float32(-2.5)
    assert np.all(lo.from_bf16_bits(lo.bf16_bits(x)) == lo.bf16(x))


def test_oracle_backprop_matches_finite_differences(lo):
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, lo.N_PARAMS)
    X = rng.normal(0, 1, (40, 32))
    T = rng.normal(0, 1, (40, 2))
    Wt = rng.uniform(0.5, 2, (40, 2))
    _, loss, g = lo.forward_backward(p, X, T, Wt, rounding=False)
    idx = rng.choice(lo.N_PARAMS, 60, replace=False)
    idx = np.union1d(idx, [lo.B1, lo.B2 + 3, lo.W3 + 5, lo.B3, lo.B3 + 1])
    for k in idx:
        e = np.zeros(lo.N_PARAMS)
        e[k] = 1e-6
        lp = lo.forward_backward(p + e, X, T, Wt, rounding=False)[1]
        lm = lo.forward_backward(p - e, X, T, Wt, rounding=False)[1]
        fd = (lp - lm) / 2e-6
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(fd), (k, fd, g[k])


def test_oracle_rounded_grad_close_to_exact(lo):
    """The BF16 rounding points perturb the gradient by well under a percent."""
    rng = np.random.default_rng(1)
    p = rng.normal(0, 0.3, lo.N_PARAMS).astype(np.float32)
    X = lo.bf16(rng.normal(0, 1, (256, 32)).astype(np.float32))
    T = rng.normal(0, 1, (256, 2))
    _, l0, g0 = lo.forward_backward(p, X, T, rounding=False)
    _, l1, g1 = lo.forward_backward(p, X, T, rounding=True)
    assert abs(l1 - l0) <= 0.02 * l0
    assert np.linalg.norm(g1 - g0) <= 0.05 * np.linalg.norm(g0)


def test_features_of_poisson(lo, gen):
    A = gen.poisson7(5)
    F = lo.row_features(A.row_ptr, A.cols, A.elms, 5, 5)
    centre = 2 * 25 + 2 * 5 + 2
    f = F[centre]
    assert np.isclose(f[0], np.log(6) / 8) and np.isclose(f[1], 1.0)
    faces = [4, 10, 12, 13, 15, 21]  # (dz,dy,dx) face neighbours in 0..25 numbering
    nb = f[2:28]
    assert np.allclose(nb[faces], 1 / 6) and np.count_nonzero(nb) == 6
    assert f[28] == 0 and f[29] == 0 and np.isclose(f[30], 7 / 27) and f[31] == 1
    corner = F[0]
    assert np.count_nonzero(corner[2:28]) == 3 and np.isclose(corner[1], 0.5)

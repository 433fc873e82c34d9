"""csr_to_slell / csr_to_slell_guess_format: bit-exact against the reference
(formats/conversion.h:338-492), through the committed golden fixtures and,
where oracle/_ref is built, against the reference's code live."""
import os

import numpy as np
import pytest

from conftest import GOLDEN


def _product(ispm, n_rows, n_cols, rp, ci, el, mode):
    A = ispm.csr_matrix(n_rows, n_cols, rp.copy(), ci.copy(), el.copy())
    if mode == "guess":
        B = ispm.csr_to_slell_guess_format(A)
    else:
        S, W, V, D = mode
        B = ispm.csr_to_slell(A, S, W, V, D)
    assert A.n_rows % 512 == 0  # pads the caller's CSR like the reference
    return B


def _same(B, meta, sp, cols, elms):
    assert [B.n_rows, B.n_cols, B.n_nz, B.slice_height, B.n_slices, B.hblock,
            int(B.var_height), int(B.diags)] == list(meta)
    assert np.array_equal(B.slice_ptr, sp)
    assert np.array_equal(B.cols, cols)
    assert B.elms.dtype == elms.dtype
    assert np.array_equal(B.elms.view(np.uint8), elms.view(np.uint8))


def _golden():
    z = np.load(os.path.join(GOLDEN, "conversion.npz"))
    names = sorted({k.split("/")[0] for k in z.files})
    cases = []
    for n in names:
        for k in z.files:
            if k.startswith(n + "/") and k.endswith("/meta"):
                cases.append((n, k[len(n) + 1:-len("/meta")]))
    return z, cases


_Z, _CASES = _golden()


@pytest.mark.parametrize("name,key", _CASES, ids=[f"{a}-{b}" for a, b in _CASES])
def test_conversion_matches_golden(ispm, name, key):
    z = _Z
    n_rows, n_cols = z[f"{name}/shape"]
    rp, ci, el = z[f"{name}/row_ptr"], z[f"{name}/cols"], z[f"{name}/elms"]
    if key == "guess":
        mode = "guess"
    else:
        S, W, V, D = (int(t[1:]) for t in key.split("_"))
        mode = (S, W, V, D)
    B = _product(ispm, int(n_rows), int(n_cols), rp, ci, el, mode)
    _same(B, z[f"{name}/{key}/meta"], z[f"{name}/{key}/slice_ptr"], z[f"{name}/{key}/cols"],
          z[f"{name}/{key}/elms"])


MODES = [(S, W, V, D) for S in (16, 32, 64, 128, 256, 512) for V in (0, 1) for D in (0, 1)
         for W in ((1,) if D else (1, 2, 4))]


def _live_matrices(gen):
    return {
        "poisson7_12": gen.poisson7(12),
        "grf27_10": gen.stencil_grf(10, 27, 3.0, 1.5, 2),
        "unstructured_9": gen.unstructured(9, seed=4),
        "random_band": gen.random_csr(1500, 1500, 21, mean_len=11, band=30),
        "random_wide_f32": gen.random_csr(800, 2000, 22, mean_len=14, pair_frac=0.7,
                                          dtype=np.float32),
        "random_odd_cols": gen.random_csr(1001, 1001, 23, mean_len=5, pair_frac=0.9),
        "tiny": gen.random_csr(5, 7, 24, mean_len=3),
    }


@pytest.fixture(scope="module")
def live(gen):
    return _live_matrices(gen)


@pytest.mark.parametrize("name", ["poisson7_12", "grf27_10", "unstructured_9", "random_band",
                                  "random_wide_f32", "random_odd_cols", "tiny"])
def test_conversion_matches_reference_live(ispm, ref, live, name):
    A = live[name]
    for S, W, V, D in MODES:
        r = ref.ref_csr_to_slell(A.n_rows, A.n_cols, A.row_ptr, A.cols, A.elms, S, W, V, D)
        B = _product(ispm, A.n_rows, A.n_cols, A.row_ptr, A.cols, A.elms, (S, W, V, D))
        _same(B, [r["n_rows"], r["n_cols"], r["n_nz"], r["slice_height"], r["n_slices"],
                  r["hblock"], int(r["var_height"]), int(r["diags"])],
              r["slice_ptr"], r["cols"], r["elms"])
    for ratio in (1, 5, 100):
        r = ref.ref_csr_to_slell_guess_format(A.n_rows, A.n_cols, A.row_ptr, A.cols, A.elms,
                                              ratio)
        Ac = ispm.csr_matrix(A.n_rows, A.n_cols, A.row_ptr.copy(), A.cols.copy(), A.elms.copy())
        B = ispm.csr_to_slell_guess_format(Ac, ratio)
        _same(B, [r["n_rows"], r["n_cols"], r["n_nz"], r["slice_height"], r["n_slices"],
                  r["hblock"], int(r["var_height"]), int(r["diags"])],
              r["slice_ptr"], r["cols"], r["elms"])


def test_min_height_and_empty_matrix(ispm, ref, gen):
    A = gen.random_csr(300, 300, 31, mean_len=4)
    for mh in (4, 8, 16):
        for D in (0, 1):
            r = ref.ref_csr_to_slell(A.n_rows, A.n_cols, A.row_ptr, A.cols, A.elms, 64, 1, 1, D,
                                     mh)
            Ac = ispm.csr_matrix(A.n_rows, A.n_cols, A.row_ptr.copy(), A.cols.copy(),
                                 A.elms.copy())
            B = ispm.csr_to_slell(Ac, 64, 1, True, D, mh)
            assert np.array_equal(B.slice_ptr, r["slice_ptr"])
            assert np.array_equal(B.cols, r["cols"])
    E = ispm.csr_matrix(0, 0, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    B = ispm.csr_to_slell(E, 32, 1, False, True)
    assert B.n_rows == 0 and B.n_slices == 0
    Z = ispm.csr_matrix(700, 700, np.zeros(701, np.int32), np.zeros(0, np.int32), np.zeros(0))
    B = ispm.csr_to_slell(Z, 32, 1, False, True)
    assert B.n_rows == 1024 and B.n_slices == 32 and len(B.elms) == 0


def test_diagonal_extraction_captures_7pt_stencil(ispm, gen):
    # 32^3 Poisson with S=32 and diagonals: every entry lands on a diagonal
    A = gen.poisson7(32)
    B = ispm.csr_to_slell(A, 32, 1, False, True)
    assert B.n_slices == 1024 and len(B.cols) == 0 and len(B.elms) == 225280
    assert len(B.slice_ptr) == 10115

"""Tile records of the staged SpMV walk (ispm_slell_stage_records), checked
on the host: for every staged tile, every (diagonal k, tile row t) reads a
shared-memory word inside the tile's bands that holds x[w_k + t] (zero
outside x), bands are 16-byte aligned the way the kernel copies them, and
tiles whose slices carry different diagonals are not staged.  The same
indexing the kernel does (csrc/spmv_staged.cuh), restated in numpy."""
import numpy as np
import pytest

TILE = 1024


def check_records(B, vw):
    v = B.view()
    S, sp = v.slice_height, B.slice_ptr.astype(np.int64)
    recs = B.stage_records()
    spt = TILE // S
    assert recs.shape == ((v.n_slices + spt - 1) // spt, 96)
    staged = 0
    for tile, r in enumerate(recs):
        b0 = tile * spt
        nsl = min(spt, v.n_slices - b0)
        nds = [(sp[3 * b + 3] - sp[3 * b] - (sp[3 * b + 4] - sp[3 * b + 1])) // S
               for b in range(b0, b0 + nsl)]
        offs = [sp[sp[3 * b + 2]: sp[3 * b + 2] + nds[0]] - (b - b0) * S
                if nds[b - b0] == nds[0] else None for b in range(b0, b0 + nsl)]
        uniform = (1 <= nds[0] <= 64 and all(o is not None and np.array_equal(o, offs[0])
                                             for o in offs))
        if not r[0]:
            continue
        assert uniform, tile
        staged += 1
        nb, total, nd0 = r[1], r[2], r[3]
        assert nd0 == nds[0] and 1 <= nb <= 8 and total % 4 == 0
        # smem word -> x column, built band by band as the kernel copies
        col_of = np.full(total, np.iinfo(np.int64).min)
        for q in range(nb):
            lo, hi, off = r[4 + 3 * q], r[5 + 3 * q], r[6 + 3 * q]
            assert off % 4 == lo % 4 and hi > lo
            c0 = (lo // vw) * vw
            nch = (hi - c0 + vw - 1) // vw
            dst0 = off - (lo - c0)
            assert dst0 >= 0 and dst0 % vw == 0 and dst0 + nch * vw <= total
            col_of[dst0: dst0 + nch * vw] = c0 + np.arange(nch * vw)
        t = np.arange(nsl * S)
        for k in range(nd0):
            w = int(sp[sp[3 * b0 + 2] + k]) - S
            p = r[28 + k] + t
            assert p.min() >= 0 and p.max() < total
            assert np.array_equal(col_of[p], w + t), (tile, k)
    return staged, len(recs)


@pytest.mark.parametrize("S", [16, 32, 64, 128, 256, 512])
def test_stage_records_stencils(ispm, gen, S):
    # grids whose x-lines do not align with the slices (24, 20) stage few or
    # no tiles; a 32^3 grid stages every tile away from its y faces
    for A in (gen.poisson7(24), gen.stencil_grf(20, 27, 4.0, 1.5, 2), gen.poisson7(32)):
        B = ispm.csr_to_slell(A, S, 1, 0, 1)
        for vw in (4, 2):
            staged, n = check_records(B, vw)
    # slices of one x-line (S <= 32 at 32^3) put the y-face lines, which lack
    # the -x-line and +x-line diagonals, into every 1024-row tile of a 32^3
    # grid; at 64^3 half the tiles hold no y-face line
    B = ispm.csr_to_slell(gen.poisson7(64 if S <= 32 else 32), S, 1, 0, 1)
    staged, n = check_records(B, 4)
    assert staged >= n // 2, (staged, n)


def test_stage_records_only_for_the_staged_formats(ispm, gen):
    A = gen.poisson7(10)
    assert ispm.csr_to_slell(A, 64, 1, 0, 0).stage_records().size == 0  # no diagonals
    assert ispm.csr_to_slell(A, 64, 2, 0, 0).stage_records().size == 0  # hblocks
    assert ispm.csr_to_slell(A, 64, 1, 1, 1).stage_records().size == 0  # variable height

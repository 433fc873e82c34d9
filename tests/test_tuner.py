"""DroptolTuner: the probe sequence matches the reference's
(fastainv/droptol-tuning.h:4-103) exactly."""
import os

import numpy as np

from conftest import GOLDEN


def _run(t, restart_at, n=20):
    seq, best, iters = [], [], []
    for k in range(n):
        if k == restart_at:
            t.restart()
        d = t.getDroptol()
        seq.append(d)
        t.noteTime(1.0 + (np.log2(d) + 6.3) ** 2)
        best.append(t.getBestDroptol())
        iters.append(t.iterations())
    return np.array(seq), np.array(best), np.array(iters)


def test_tuner_matches_golden(ispm):
    z = np.load(os.path.join(GOLDEN, "tuner.npz"))
    for name in ("default", "narrow"):
        lo, hi, restart_at = z[f"{name}/lo_hi_restart"]
        seq, best, iters = _run(ispm.DroptolTuner(lo, hi), int(restart_at))
        assert np.array_equal(seq, z[f"{name}/droptols"])
        assert np.array_equal(best, z[f"{name}/best"])
        assert np.array_equal(iters, z[f"{name}/iterations"])


def test_tuner_matches_reference_live(ispm, ref):
    rng = np.random.default_rng(5)
    for trial in range(5):
        lo, hi = -rng.uniform(8, 12), -rng.uniform(1, 4)
        a, b = ispm.DroptolTuner(lo, hi), ref.RefDroptolTuner(lo, hi)
        for k in range(30):
            if k in (10, 21):
                a.restart()
                b.restart()
            if k == 15:
                a.resetPhase()
                b.resetPhase()
            assert a.getDroptol() == b.getDroptol()
            t = float(rng.uniform(0.5, 2.0))
            a.noteTime(t)
            b.noteTime(t)
            assert a.getBestDroptol() == b.getBestDroptol()
            assert a.iterations() == b.iterations()


def test_tuner_converges_to_minimum(ispm):
    t = ispm.DroptolTuner()
    for _ in range(30):
        d = t.getDroptol()
        t.noteTime(1.0 + (np.log2(d) + 6.3) ** 2)
    assert abs(np.log2(t.getBestDroptol()) + 6.3) < 0.05

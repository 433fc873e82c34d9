"""The C++ drop-in headers (include/compat): a caller written only against
the reference's headers and template signatures (tests/cpp/driver_shape.cpp,
in the shape of the reference's foam-extend driver) builds unchanged against
them and links libispm_b200.so.

* CPU: the host part (conversions in three shapes and the format guess, the
  approximate inverse in double and float, a drop-tolerance search) runs, and
  where the reference's source tree is present the same program built
  against the reference's own headers (with its fastainv.cpp compiled in
  place) prints the same lines: every array bit for bit.
* GPU: the device part (upload, both launch_spmv_kernel overloads, an
  unsupported launch that must do nothing, the sblas calls, the DEFAULT and
  EXHAUSTIVE plans and a value update) checks each result against a host
  computation and exits 0.
"""
import os
import subprocess

import pytest

from conftest import ROOT

CPP = os.path.join(ROOT, "tests", "cpp")
BUILD = os.path.join(CPP, "_build")


def _ref_dir():
    return os.environ.get("REF_DIR") or os.path.abspath(os.path.join(ROOT, "..", "reference"))


def _make(target, env=None):
    r = subprocess.run(["make", "-s", "-C", CPP, target], capture_output=True, text=True,
                       env=env)
    assert r.returncode == 0, r.stdout + r.stderr


def _run(name):
    r = subprocess.run([os.path.join(BUILD, name)], capture_output=True, text=True, timeout=600)
    return r.returncode, r.stdout, r.stderr


def test_dropin_host_part_matches_reference_build(ispm):
    _make("compat-host")
    rc, out, err = _run("driver_compat_host")
    assert rc == 0, out + err
    assert "failures 0" in out and "fastainv double ok=1" in out
    ref = _ref_dir()
    if not os.path.exists(os.path.join(ref, "fastainv", "fastainv.cpp")):
        pytest.skip("reference source tree absent: compared with the compat build only")
    env = dict(os.environ, REF_DIR=ref)
    _make("ref-host", env)
    rc2, out2, err2 = _run("driver_ref_host")
    assert rc2 == 0, out2 + err2
    assert out.splitlines() == out2.splitlines()


@pytest.mark.gpu
def test_dropin_device_part(ispm):
    _make("compat-device")
    rc, out, err = _run("driver_compat_device")
    assert rc == 0, out + err
    assert "FAILED" not in out and "failures 0" in out

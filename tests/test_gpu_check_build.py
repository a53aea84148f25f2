"""The check build (libvespa_b200_check.so, -DVB_CHECK): the same kernels
with device bounds checks that skip a bad access and record it instead of
faulting.  Small parity cases run through it in a child process (the library
is chosen once per process) and must equal the oracle with no check failed;
the normal build reports that it has no checks."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECK_LIB = os.path.join(ROOT, "vespa.jl_b200", "libvespa_b200_check.so")


def test_normal_build_has_no_checks(vb):
    assert vb.default_context().check_read() == -1


def test_check_build_parity_without_failed_checks():
    assert os.path.exists(CHECK_LIB), "build it with `make -C vespa.jl_b200/csrc check`"
    env = dict(os.environ, VESPA_B200_LIB=CHECK_LIB)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "check_build_cases.py")],
                       env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["check_build"]
    for name, res in out["cases"].items():
        assert res["check"] == 0, (name, res)
        assert res["same"], (name, res)

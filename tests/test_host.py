"""Host-side logic and the C-ABI surface, without a GPU."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

import vespa_b200 as vb
from vespa_b200 import _lib
from vespa_b200 import problem as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "vespa_b200.h")


def declared_symbols(path=HEADER):
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*int\s+(vb_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    # the ctypes signature table covers the whole header
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)
    assert L.vb_abi_version() == 1


def test_check_build_exports_every_declared_symbol():
    # the device-bounds-check build of the same sources (make ... check)
    path = os.path.join(ROOT, "vespa.jl_b200", "libvespa_b200_check.so")
    assert os.path.exists(path), "build it with `make -C vespa.jl_b200/csrc check`"
    L = C.CDLL(path)
    for n in declared_symbols():
        assert hasattr(L, n), n


def test_library_is_self_contained():
    # no dependency on a CUDA runtime being on the loader path
    import subprocess
    out = subprocess.run(["ldd", _lib.LIB_PATH], capture_output=True, text=True).stdout
    assert "libcudart" not in out


def test_errors_without_device_are_reported_not_raised_in_c():
    L = _lib.load()
    h = C.c_void_p()
    rc = L.vb_ctx_create(0, C.byref(h))
    if rc == 0:  # a GPU is present: nothing to check here
        L.vb_ctx_destroy(h)
        pytest.skip("GPU present")
    assert rc == _lib.VB_ECUDA
    assert "CUDA" in _lib.last_error()
    with pytest.raises(_lib.VespaB200Error):
        _lib.call("vb_ctx_create", 0, C.byref(h))


def test_null_arguments_are_einval():
    L = _lib.load()
    assert L.vb_grid_create(None, None, 0, None) == _lib.VB_EINVAL
    assert L.vb_step(None, 0.1) == _lib.VB_EINVAL
    assert L.vb_compute_dt(None, None) == _lib.VB_EINVAL
    assert L.vb_hllc_faces(None, 0, None, None, None, 1.4, None) == _lib.VB_EINVAL


def test_problem_validation_matches_reference():
    init = lambda x, y, z: (1.0, 0.0, 0.0, 0.0, 1.0)
    ok = dict(name="p", dims=(8,), domain=((0.0, 1.0),), gamma=1.4, bcs=P.Outflow, init=init,
              tfinal=1.0)
    P.Problem(**ok)
    for bad in (dict(gamma=1.0), dict(tfinal=0.0), dict(cfl=0.0), dict(cfl=1.5), dict(dims=(0,)),
                dict(domain=((1.0, 0.0),))):
        with pytest.raises(ValueError):
            P.Problem(**{**ok, **bad})


def test_prng_is_deterministic_and_uniform():
    a = P.uniform01(1, 2, np.arange(100000))
    b = P.uniform01(1, 2, np.arange(100000))
    assert np.array_equal(a, b)
    assert a.min() >= 0.0 and a.max() < 1.0
    assert abs(a.mean() - 0.5) < 0.01
    assert not np.array_equal(a, P.uniform01(1, 3, np.arange(100000)))
    # subsets regenerate identically
    assert np.array_equal(P.uniform01(1, 2, np.arange(500, 600)), a[500:600])


def test_initial_conditions_follow_reference_order():
    prob = P.sod_problem_defaults(400, cfl=0.8)
    U = P.initial_state(prob)
    x = prob.cell_centers()[0]
    assert x[0] == 0.0 + (1.0 - 0.5) * (1.0 / 400)
    assert U.shape == (5, 400)
    assert U[0, 199] == 1.0 and U[0, 200] == 0.125
    assert U[4, 0] == 1.0 / (1.4 - 1.0)
    sm = P.smooth_random_problem((8, 8, 8), seed=3)
    W = P.initial_primitive(sm)
    assert 0.7 <= W[0].min() and W[0].max() <= 1.3
    assert np.abs(W[1:4]).max() <= 0.5
    assert 0.8 <= W[4].min() and W[4].max() <= 1.2
    W2 = P.initial_primitive(P.smooth_random_problem((8, 8), seed=3))
    assert np.all(W2[3] == 0.0)  # planar: vz = 0 keeps the z-momentum exactly 0


def test_riemann_boxes_and_kh():
    sides = {P.riemann_box_problem(i).dims[0] for i in range(64)}
    assert sides <= set(P.BOX_SIDES) and len(sides) >= 4
    small = P.riemann_box_problem(0, side=8)
    W = P.initial_primitive(small)
    assert 0.1 <= W[0].min() and W[0].max() <= 10.0
    assert np.all(np.sqrt(W[1] ** 2 + W[2] ** 2 + W[3] ** 2) <= 2.0 + 1e-12)
    kh = P.kelvin_helmholtz_problem(16)
    Wk = P.initial_primitive(kh)
    assert set(np.unique(Wk[0])) == {1.0, 2.0}


def test_compute_face_fluxes_rejects_other_backends():
    F = np.zeros((2, 5))
    with pytest.raises(TypeError):
        vb.compute_face_fluxes(object(), 1.4, F, F.copy(), F.copy(), [1, 2])


def test_bench_reference_arm_prints_the_contract_line():
    """bench.py --impl reference (the oracle on the host cores) runs without a
    GPU and prints one JSON line with the reference arm's keys."""
    import json
    import subprocess
    import sys
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] in ("port", "reference") and d["cpu_baseline"]["cores"] >= 1
    assert d["unit"] == "Mcell-updates/s" and d["steps"] == 1

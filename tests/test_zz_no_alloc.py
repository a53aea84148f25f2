"""vb_hllc_faces_noalloc: the batched HLLC entry point that allocates nothing.

It exists for callers that own all of the GPU's memory themselves (a pool
allocator that must not see foreign cudaMalloc/cudaFree calls, or memory
reserved up front): its staging buffers live in a fixed array compiled into
the library, capped at VB_NOALLOC_MAX_FACES faces per call.  Its results must
equal the allocating entry point's (vb_hllc_faces) exactly -- the float64 tests
here are bit-for-bit -- on consecutive calls that share that array.

Kept in a file that pytest collects last, and self-contained, so it passes
alone in a fresh process as well as after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

import vespa_b200 as vb
from vespa_b200 import _lib

pytestmark = pytest.mark.gpu

MAX_FACES = 65536  # VB_NOALLOC_MAX_FACES in include/vespa_b200.h


def faces(nf, seed):
    rng = np.random.default_rng(seed)
    WL = np.empty((nf, 5))
    WR = np.empty((nf, 5))
    for W in (WL, WR):
        W[:, 0] = np.exp(rng.uniform(np.log(0.05), np.log(20.0), nf))
        W[:, 1:4] = rng.uniform(-3.0, 3.0, (nf, 3))
        W[:, 4] = np.exp(rng.uniform(np.log(0.01), np.log(10.0), nf))
    q = nf // 8
    WL[:q, 1:4] += 20.0  # supersonic faces: both FL and FR branches
    WR[q:2 * q, 1:4] -= 20.0
    return WL, WR, rng.integers(1, 4, nf).astype(np.int32)


def noalloc(WL, WR, axis, gamma):
    nf = len(axis)
    F = np.full((nf, 5), np.nan)
    rc = _lib.load().vb_hllc_faces_noalloc(nf, _lib.dptr(WL), _lib.dptr(WR), _lib.i32ptr(axis),
                                           gamma, _lib.dptr(F), None)
    _lib.check(rc)
    return F


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls():
    ctx = vb.default_context()  # makes the device current on this thread
    backend = vb.B200Flux(ctx)
    # a full-size call, then a smaller one over the array's stale contents
    for nf, seed, gamma in ((MAX_FACES, 11, 1.4), (3001, 12, 5.0 / 3.0)):
        WL, WR, axis = faces(nf, seed)
        ref = np.zeros((nf, 5))
        vb.compute_face_fluxes(backend, gamma, ref, WL, WR, axis)
        got = noalloc(WL, WR, axis, gamma)
        assert np.array_equal(got, ref), float(np.nanmax(np.abs(got - ref)))


def test_noalloc_rejects_batches_above_the_cap():
    vb.default_context()
    nf = MAX_FACES + 1
    W = np.ones((nf, 5))
    axis = np.ones(nf, dtype=np.int32)
    F = np.zeros((nf, 5))
    rc = _lib.load().vb_hllc_faces_noalloc(nf, _lib.dptr(W), _lib.dptr(W), _lib.i32ptr(axis), 1.4,
                                           _lib.dptr(F), None)
    assert rc == _lib.VB_EINVAL
    assert "VB_NOALLOC_MAX_FACES" in _lib.last_error()
    assert np.all(F == 0.0)

"""The allocation-free closest-hit entry point (pt_trace_closest_static).

It serves callers that cannot allocate device memory (a host whose own pool
allocator owns the device, or code where a cudaMalloc is not allowed): rays
and hits pass through a fixed array that the library holds on every device.

Collected last on purpose: it must give the same hits as pt_trace_closest
and as the oracle's traversal, bit for bit, whether it runs alone or after
every other test of the session, on two calls in a row (the second call
reuses the static array the first one filled), and it rejects more rays than
its array holds without touching the device.
"""
import numpy as np
import pytest

import pathtracingtutorial_b200 as pt
from pathtracingtutorial_b200 import _ffi, scenes

pytestmark = pytest.mark.gpu


def _scene(sa):
    s = sa.scene()
    s.build_accel()
    s.upload_to_device(0)
    return s


def _rays(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d[: n // 50, rng.integers(0, 3)] = 0.0
    return o, d


@pytest.mark.parametrize("name", ["cornell", "spheres"])
def test_static_trace_matches_trace_closest_twice(oracle, name):
    sa = scenes.cornell_box(width=32, height=32) if name == "cornell" else \
        scenes.icosphere_field(n_spheres=40, subdiv=3, width=32, height=18, env_size=(64, 32))
    s = _scene(sa)
    lo, hi = sa.vertices["position"].min(0), sa.vertices["position"].max(0)
    o, d = _rays(pt.STATIC_TRACE_MAX_RAYS, lo, hi, 5)
    ref = pt.trace_closest(s, o, d)
    first = pt.trace_closest_static(s, o, d)
    second = pt.trace_closest_static(s, o, d)
    assert np.array_equal(first.view(np.uint8), ref.view(np.uint8))
    assert np.array_equal(second.view(np.uint8), ref.view(np.uint8))
    assert (ref["prim"] >= 0).mean() > 0.3
    # and the oracle's restatement of the reference's traversal, directly
    prep = oracle.prepare(sa)
    rays = np.zeros((len(o), 8), np.float32)
    rays[:, :3], rays[:, 4:7] = o, d
    orc, _ = oracle.trace(prep.nodes, prep.vertices, prep.faces, rays)
    gpu = np.stack([first["t"], first["prim"].view(np.float32), first["u"], first["v"]], 1)
    assert np.array_equal(gpu.view(np.uint32), orc.view(np.uint32))
    # a smaller call after a full one: only its own rays come back
    o2, d2 = _rays(1000, lo, hi, 6)
    assert np.array_equal(pt.trace_closest_static(s, o2, d2).view(np.uint8), pt.trace_closest(s, o2, d2).view(np.uint8))


def test_static_trace_rejects_oversized_calls():
    s = _scene(scenes.cornell_box(width=16, height=16))
    n = pt.STATIC_TRACE_MAX_RAYS + 1
    rays = np.zeros((n, 8), np.float32)
    hits = np.zeros(n, pt.HIT_DTYPE)
    rc = _ffi.lib().pt_trace_closest_static(s.handle, _ffi.ptr(rays), n, _ffi.ptr(hits))
    assert rc == _ffi.PT_ERR_INVALID
    assert b"at most" in _ffi.lib().pt_last_error()
    assert pt.trace_closest_static(s, np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32)).size == 0

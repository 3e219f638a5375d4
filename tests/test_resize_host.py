"""The host mirror's resizing (_lhl_resize!, src/LHLFactorization.jl:256-292) on the CPU, with
the device library replaced by a recording stand-in: lhl! / lhl_reduce! on a workspace of
another order (test/core_tests.jl:107-112) and lhl_shift! on a shift object of another order
(:306-310) replace the device objects, destroy every old handle exactly once, keep the
workspace's settings, and raise the reference's type errors before resizing anything.
No GPU is involved."""
import ctypes as C
import gc
import itertools

import numpy as np
import pytest
import torch

import lhl_gpu as G


class FakeLib:
    """Creates, views, destroys and records; every other call succeeds and is recorded."""

    def __init__(self):
        self._ids = itertools.count(1)
        self.live, self.created, self.destroyed, self.calls = {}, [], [], []

    @staticmethod
    def _h(h):
        return h.value if isinstance(h, C.c_void_p) else h

    def _new(self, kind, n, out, **kw):
        h = next(self._ids) * 4096
        self.live[h] = dict(kind=kind, n=n, **kw)
        self.created.append(h)
        out._obj.value = h
        return 0

    def lhl_ws_create(self, n, prec, out):
        return self._new("ws", n, out)

    def lhl_ws_create_f32(self, n, prec, out):
        return self._new("ws", n, out)

    def lhl_ws_create_c128(self, n, out):
        return self._new("ws", n, out)

    def lhl_shift_create(self, n, S, out):
        return self._new("sh", n, out, S=S, cplx=0)

    def lhl_shift_create_complex(self, n, S, out):
        return self._new("sh", n, out, S=S, cplx=1)

    def lhl_ws_get_view(self, h, v):
        v._obj.n = self.live[self._h(h)]["n"]
        return 0

    def lhl_shift_get_view(self, h, v):
        d, o = self.live[self._h(h)], v._obj
        o.n, o.nshifts, o.ldg, o.po, o.is_complex = d["n"], d["S"], d["n"] + 4, d["n"] + 8, d["cplx"]
        return 0

    def _destroy(self, h):
        h = self._h(h)
        assert h in self.live, "destroyed twice or never created"
        del self.live[h]
        self.destroyed.append(h)
        return 0

    lhl_ws_destroy = _destroy
    lhl_shift_destroy = _destroy

    def __getattr__(self, name):
        def call(*args):
            self.calls.append((name,) + tuple(self._h(a) for a in args[:2]) + tuple(args[2:]))
            return 0
        return call


@pytest.fixture
def fake(monkeypatch):
    f = FakeLib()
    monkeypatch.setattr(G, "_lib", f)
    monkeypatch.setattr(G, "_stream", lambda s=None: None)
    monkeypatch.setattr(torch.cuda, "current_device", lambda: 0)
    monkeypatch.setattr(torch.Tensor, "is_cuda", property(lambda self: True))
    yield f
    gc.collect()


def J(n):
    return torch.as_tensor(np.asfortranarray(np.eye(n)))


def test_reduce_into_a_workspace_of_another_order(fake):
    ws = G.LHLWorkspace(4)
    ws.set_probes(True)
    ws.set_barrier_limit_ns(123)
    h0, s0 = ws._h.value, ws.shift._h.value
    assert G.lhl_(ws, J(6)) is ws
    assert ws.n == 6 and ws.shift.n == 6 and ws.reduced
    h1 = ws._h.value
    assert h1 not in (h0, s0) and h0 in fake.destroyed and s0 in fake.destroyed
    assert ("lhl_ws_set_probes", h1, 1) in fake.calls
    assert ("lhl_ws_set_barrier_limit_ns", h1, 123) in fake.calls
    assert fake.calls[-1][:2] == ("lhl_reduce", h1)
    # the same order keeps the device objects
    n_created = len(fake.created)
    G.lhl_reduce_(ws, J(6), True)
    assert len(fake.created) == n_created and ws._h.value == h1
    del ws
    gc.collect()
    assert not fake.live


def test_shift_object_takes_the_workspace_order(fake):
    ws = G.LHLWorkspace(5)
    sh = G.LHLShift(3, 2)
    old = sh._h.value
    assert G.lhl_shift_(sh, ws, 1.0, -0.1) is sh
    assert sh.n == 5 and sh.nshifts == 2 and sh.ldg == 9 and old in fake.destroyed
    assert fake.calls[-1][:3] == ("lhl_shift", sh._h.value, ws._h.value)
    # the reference's type errors come first and leave the shift object as it was
    sh2 = G.LHLShift(3)
    h2 = sh2._h.value
    with pytest.raises(G.ArgumentError):
        G.lhl_shift_(sh2, ws, 1.0, -0.1j)
    assert sh2.n == 3 and sh2._h.value == h2
    wc = G.LHLWorkspace(4, dtype=torch.complex128)
    with pytest.raises(G.ArgumentError):
        G.lhl_shift_(sh2, wc, 1.0, -0.1)
    assert sh2.n == 3
    # a complex shift object resizes and stays complex
    shc = G.LHLShift(2, 1, complex=True)
    G.lhl_shift_(shc, wc, 1.0, -0.1j)
    assert shc.n == 4 and shc.is_complex and fake.calls[-1][0] == "lhl_shift_complex"
    del ws, sh, sh2, wc, shc
    gc.collect()
    assert not fake.live

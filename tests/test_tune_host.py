"""The autotuner's host logic on the CPU (lhl_gpu/tune.py): workload keys, the JSON cache, and
the choice among timed trials, with a stand-in for torch's CUDA events; and the C ABI's
launch-shape table (host-only calls)."""
import ctypes
import os
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, "lhl.jl_b200"))


class _FakeTorch:
    """torch.cuda's events and synchronize, with scripted durations: each timed call of fn
    returns the next value of `durations` as its elapsed time."""

    def __init__(self, durations):
        self.durations = list(durations)
        outer = self

        class _Ev:
            def __init__(self, enable_timing=False):
                self.t = None

            def record(self, stream=None):
                pass

            def elapsed_time(self, other):
                return outer.durations.pop(0)

        class _Cuda:
            Event = _Ev

            @staticmethod
            def synchronize():
                pass

            @staticmethod
            def current_stream():
                return None

        self.cuda = _Cuda


def test_keys_bucket_orders_by_powers_of_two():
    from lhl_gpu import tune as T
    assert T.order_bucket(1) == 16 and T.order_bucket(400) == 512 and T.order_bucket(2048) == 2048
    assert T.order_bucket(2049) == 4096
    k = T.workload_key("NVIDIA B200", True, 8192, "mixed", 32)
    assert k == "NVIDIA B200|complex|n8192|mixed|r32"
    assert T.workload_key("d", False, 300, "plain", 1) == T.workload_key("d", False, 400, "plain", 1)


def test_cache_round_trip(tmp_path):
    from lhl_gpu import tune as T
    p = str(tmp_path / "tuning.json")
    assert T.load_cache(p) == {}
    c = T.record({}, "k", {"refine": ["gmres", 4, 3], "shift_variant": [3, 0]})
    T.save_cache(c, p)
    got = T.lookup("ignored", False, 1, "x", 1, path=p)
    assert got is None  # another key
    assert T.load_cache(p)["k"]["refine"] == ["gmres", 4, 3]
    assert "measured" in T.load_cache(p)["k"]


def test_refine_choice_is_the_fastest_accepted_one():
    from lhl_gpu import tune as T
    cands = [("fixed", 16), ("gmres", 6, 3), ("gmres", 4, 4)]
    # per candidate: one warm-up run (untimed) then reps = 2 timed runs
    fake = _FakeTorch([9.0, 8.0, 3.0, 2.5, 5.0, 4.0])
    accepted = iter([True, False, True])  # the fastest (gmres 6,3) misses the tolerance
    runs = []
    best, trials = T.tune_refine(fake, "mixed", lambda ch: runs.append(ch), lambda: next(accepted), reps=2,
                                 candidates=cands)
    assert best == ("gmres", 4, 4)
    assert [t["ms"] for t in trials] == [8.0, 2.5, 4.0]
    assert [t["ok"] for t in trials] == [True, False, True]
    assert len(runs) == 9  # (warm-up + 2) per candidate


def test_refine_choice_none_when_nothing_reaches_the_target():
    from lhl_gpu import tune as T
    fake = _FakeTorch([1.0, 1.0])
    best, trials = T.tune_refine(fake, "plain", lambda ch: None, lambda: False, reps=1,
                                 candidates=[("fixed", 4), ("gmres", 4, 3)])
    assert best is None and len(trials) == 2


def test_shift_shape_table_on_the_host():
    L = ctypes.CDLL(os.path.join(REPO, "lhl.jl_b200", "liblhl_gpu.so"))
    T, E = ctypes.c_int(), ctypes.c_int()
    shapes = {}
    for cplx in (0, 1):
        v = 1
        while L.lhl_shift_variant_shape(cplx, v, ctypes.byref(T), ctypes.byref(E)) == 0:
            shapes[(cplx, v)] = (T.value, E.value)
            v += 1
        assert v > 1
        assert L.lhl_shift_variant_shape(cplx, 0, ctypes.byref(T), ctypes.byref(E)) == 1
    assert shapes[(0, 1)] == (256, 1) and shapes[(1, 5)] == (1024, 8)
    assert all(t in (256, 512, 1024) and e >= 1 for t, e in shapes.values())
    L.lhl_ws_set_shift_variant.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    assert L.lhl_ws_set_shift_variant(None, 1, 0) == 1  # null workspace: ArgumentError


def test_python_lists_the_shapes_that_cover_an_order():
    import lhl_gpu as G
    v = G.shift_variants(False, 2048)
    assert v and all(G.shift_variant_shape(False, k)[0] * G.shift_variant_shape(False, k)[1] >= 2048 for k in v)
    assert 1 not in v  # 256 x 1 does not cover 2048
    assert G.shift_variants(True, 8192) == [5, 9, 10]  # 1024 x 8, 512 x 16, 256 x 32

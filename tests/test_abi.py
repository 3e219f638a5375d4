"""CPU-side checks of the drop-in boundary: the library builds, loads without a GPU and
exports every entry point include/lhl_gpu.h declares; the host mirror rejects bad
arguments before touching the device."""
import ctypes
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "lhl_gpu.h")
LIB = os.path.join(REPO, "lhl.jl_b200", "liblhl_gpu.so")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:int|const char\*)\s+(lhl_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_api():
    names = declared_functions()
    for must in ("lhl_ws_create", "lhl_reduce", "lhl_shift", "lhl_shift_batched", "lhl_ldiv", "lhl_refine",
                 "lhl_applyZ", "lhl_applyZinv"):
        assert must in names


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        import importlib.util
        spec = importlib.util.spec_from_file_location("lhl_build", os.path.join(REPO, "lhl.jl_b200", "build.py"))
        m = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(m)
        m.build()
    L = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    L.lhl_version.restype = ctypes.c_char_p
    assert b"sm_100a" in L.lhl_version()


def test_null_handles_rejected_on_host():
    L = ctypes.CDLL(LIB)
    vp = ctypes.c_void_p
    assert L.lhl_ws_destroy(vp(0)) == 1
    assert L.lhl_shift_destroy(vp(0)) == 1
    L.lhl_ws_create.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.POINTER(vp)]
    h = vp()
    assert L.lhl_ws_create(-1, 0, ctypes.byref(h)) == 2        # DimensionMismatch
    assert L.lhl_ws_create(4, 7, ctypes.byref(h)) == 1         # ArgumentError: precision
    L.lhl_ldiv.argtypes = [vp, vp, vp, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, vp]
    assert L.lhl_ldiv(vp(0), vp(0), vp(0), 1, 1, 1, vp(0)) == 1
    # the later entry points refuse null handles the same way, before any device call
    i64, i32, d = ctypes.c_int64, ctypes.c_int, ctypes.c_double
    L.lhl_ldiv_f32.argtypes = [vp, vp, vp, i64, i64, i64, vp]
    assert L.lhl_ldiv_f32(vp(0), vp(0), vp(0), 1, 1, 1, vp(0)) == 1
    L.lhl_reduce_f32.argtypes = [vp, vp, i64, i32, vp]
    assert L.lhl_reduce_f32(vp(0), vp(0), 1, 1, vp(0)) == 1
    L.lhl_ws_import.argtypes = [vp] * 9
    assert L.lhl_ws_import(*([vp(0)] * 9)) == 1
    L.lhl_ws_set_probes.argtypes = [vp, i32]
    assert L.lhl_ws_set_probes(vp(0), 1) == 1
    L.lhl_ws_create_f32.argtypes = [i64, i32, ctypes.POINTER(vp)]
    assert L.lhl_ws_create_f32(-1, 0, ctypes.byref(h)) == 2
    assert L.lhl_ws_create_f32(4, 7, ctypes.byref(h)) == 1
    L.lhl_refine_gmres.argtypes = [vp, vp, vp, i64, vp, i64, vp, i64, vp, vp, i64, i64, d, i32, i32, i32, vp]
    assert L.lhl_refine_gmres(vp(0), vp(0), vp(0), 1, vp(0), 1, vp(0), 1, vp(0), vp(0), 1, 1, 1e-10, 1, 3, 1,
                              vp(0)) == 1
    # LHLWorkspace{ComplexF64}: order checked on the host, null handles refused
    L.lhl_ws_create_c128.argtypes = [i64, ctypes.POINTER(vp)]
    assert L.lhl_ws_create_c128(-1, ctypes.byref(h)) == 2
    assert L.lhl_ws_create_c128(8193, ctypes.byref(h)) == 2
    assert L.lhl_ws_create_c128(4, None) == 1
    L.lhl_reduce_c128.argtypes = [vp, vp, i64, i32, vp]
    assert L.lhl_reduce_c128(vp(0), vp(0), 1, 1, vp(0)) == 1
    # refinement with the caller's system matrix
    L.lhl_refine_system.argtypes = [vp, vp, i64, vp, i64, vp, i64, vp, i64, vp, vp, i64, d, i32, vp]
    assert L.lhl_refine_system(vp(0), vp(0), 0, vp(0), 1, vp(0), 1, vp(0), 1, vp(0), vp(0), 1, 0.0, 1, vp(0)) == 1
    L.lhl_refine_system_gmres.argtypes = [vp, vp, i64, vp, i64, vp, i64, vp, i64, vp, vp, i64, d, i32, i32, i32, vp]
    assert L.lhl_refine_system_gmres(vp(0), vp(0), 0, vp(0), 1, vp(0), 1, vp(0), 1, vp(0), vp(0), 1, 0.0, 1, 3, 1,
                                     vp(0)) == 1


def handle_functions():
    """(name, ctypes argument types) of every declared entry point whose first argument is a
    workspace, shift object or batch handle, read from the header."""
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    scalars = {"int64_t": ctypes.c_int64, "int": ctypes.c_int, "double": ctypes.c_double,
               "uint64_t": ctypes.c_uint64}
    out = []
    for name, params in re.findall(r"\bint\s+(lhl_\w+)\s*\(([^)]*)\)\s*;", src):
        params = [p.strip() for p in params.split(",")]
        if params[0].split()[0] not in ("lhl_ws_t", "lhl_shift_t", "lhl_batch_t"):
            continue
        types = []
        for p in params:
            ty = p.replace("const ", "").split()[0]
            types.append(ctypes.c_void_p if ("*" in p or ty.startswith("lhl_")) else scalars[ty])
        out.append((name, types))
    return out


def test_every_handle_entry_point_refuses_a_null_handle():
    """LHL_ERR_ARG from every call on a null handle, other arguments zero or one, before any
    device call (the library is loaded here without a GPU)."""
    L = ctypes.CDLL(LIB)
    fns = handle_functions()
    assert len(fns) >= 30
    for name, types in fns:
        f = getattr(L, name)
        f.argtypes = types
        args = [None if t is ctypes.c_void_p else t(0.0 if t is ctypes.c_double else 1) for t in types]
        assert f(*args) == 1, name


def test_creators_check_sizes_and_pointers_on_host():
    """Shift objects, batches and the allocation-free reduction: DimensionMismatch for bad
    orders, counts or leading dimensions, ArgumentError for null pointers, before any device
    call."""
    C = ctypes
    L = C.CDLL(LIB)
    vp, i64, i32 = C.c_void_p, C.c_int64, C.c_int
    h = vp()
    for name in ("lhl_shift_create", "lhl_shift_create_complex", "lhl_shift_create_f32", "lhl_shift_create_complex64"):
        f = getattr(L, name)
        f.argtypes = [i64, i64, C.POINTER(vp)]
        assert f(-1, 1, C.byref(h)) == 2 and f(4, -1, C.byref(h)) == 2 and f(4, 1, None) == 1, name
    L.lhl_batch_create.argtypes = [i64, vp, i64, C.POINTER(vp)]
    ok_ns = (i64 * 2)(4, 5)
    assert L.lhl_batch_create(2, C.cast((i64 * 2)(4, -3), vp), 1, C.byref(h)) == 2
    assert L.lhl_batch_create(2, C.cast(ok_ns, vp), -1, C.byref(h)) == 2
    assert L.lhl_batch_create(0, C.cast(ok_ns, vp), 1, C.byref(h)) == 2
    assert L.lhl_batch_create(2, None, 1, C.byref(h)) == 1
    assert L.lhl_batch_create(2, C.cast(ok_ns, vp), 1, None) == 1
    L.lhl_reduce_noalloc.argtypes = [i64, vp, i64, i32] + [vp] * 8
    assert L.lhl_reduce_noalloc(-1, None, 1, 1, *([None] * 8)) == 2
    assert L.lhl_reduce_noalloc(8, None, 8, 1, *([None] * 8)) == 1
    assert L.lhl_reduce_noalloc(8, 1, 4, 1, *([1] * 7), None) == 2      # ldj < n
    assert L.lhl_reduce_noalloc(2000, 1, 2000, 1, *([1] * 7), None) == 2  # above its order limit
    # J sharing bytes with factors (or factors with Ht) is refused before anything is queued
    assert L.lhl_reduce_noalloc(8, 4096, 8, 1, 4096 + 8, 1 << 20, 1, 1, 1, 1, 1, None) == 1
    assert L.lhl_reduce_noalloc(8, 4096, 8, 1, 1 << 20, (1 << 20) + 64, 1, 1, 1, 1, 1, None) == 1


def test_configs_are_seeded_and_shaped():
    import sys
    sys.path.insert(0, os.path.join(REPO, "lhl.jl_b200"))
    from lhl_gpu import configs
    c1 = configs.config1()
    assert c1["J"].shape == (400, 400) and c1["J"].flags.f_contiguous
    assert list(-c1["tau"]) == [0.01, 0.013, 0.021]
    c2a, c2b = configs.config2(8), configs.config2(8)
    assert (c2a["J"] == c2b["J"]).all() and (c2a["tau"] == c2b["tau"]).all()
    assert (-c2a["tau"] >= 1e-4).all() and (-c2a["tau"] <= 1e-1).all()


def test_launch_settings_are_cached_per_device():
    """A kernel's dynamic shared-memory opt-in belongs to one device's context, and SM counts and
    cooperative grid sizes are per device: a launcher that cached them in one process-wide
    variable would launch with the wrong settings once a process switches devices.  Every such
    cache in the CUDA sources is an array indexed by the device ordinal."""
    csrc = os.path.join(REPO, "lhl.jl_b200", "csrc")
    scalar_cache = re.compile(r"^\s*static\s+(?:bool|int|size_t|unsigned)\s+\w+\s*(?:=\s*[^;{]+)?;", re.M)
    bad = []
    for name in sorted(os.listdir(csrc)):
        if not name.endswith((".cu", ".cuh")):
            continue
        src = open(os.path.join(csrc, name)).read()
        bad += [f"{name}: {m.group(0).strip()}" for m in scalar_cache.finditer(src)]
        # a dynamic shared-memory opt-in outside the per-device helper sits in a per-device branch
        for m in re.finditer(r"cudaFuncSetAttribute\(", src):
            head = src[max(0, m.start() - 600):m.start()]
            if name != "internal.cuh" and "_of[dev]" not in head and "MAX_DEVICES" not in head:
                bad.append(f"{name}: cudaFuncSetAttribute outside a per-device cache")
    assert not bad, bad

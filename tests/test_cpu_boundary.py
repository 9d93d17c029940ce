"""CPU-only checks of the C ABI library and the host logic (no GPU calls)."""
import ctypes
import os
import re
import subprocess

import numpy as np

import cublox_b200 as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    syms = set()
    for name in os.listdir(os.path.join(ROOT, "include")):
        if name.endswith(".h"):
            src = open(os.path.join(ROOT, "include", name)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            syms |= set(re.findall(r"\b(cublox_[a-z0-9_]+)\s*\(", src))
    return syms


def test_library_exports_every_header_symbol():
    syms = header_symbols()
    assert len(syms) >= 30
    out = subprocess.check_output(["nm", "-D", "--defined-only", C.LIB_PATH], text=True)
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = sorted(syms - exported)
    assert not missing, missing
    lib = C.lib()
    for s in syms:
        getattr(lib, s)


def test_library_is_built_for_sm100a_only():
    """The build's nvcc flags name one target, sm_100a (native code, no PTX
    for other targets); the GPU suite checks the loaded kernels' binary
    version on the device."""
    from cublox_b200 import build as B
    gencodes = [B.NVCC_FLAGS[i + 1] for i, f in enumerate(B.NVCC_FLAGS) if f == "-gencode"]
    assert gencodes == ["arch=compute_100a,code=sm_100a"]
    assert not any(f.startswith("-arch") for f in B.NVCC_FLAGS)


def test_noalloc_rejects_voxel_counts_above_int32_before_any_device_call():
    """2 * half + 1 is formed in 64-bit arithmetic: a half size of 2^30
    (2 * half + 1 > INT_MAX) is refused as out of range, not wrapped."""

    class MapView(ctypes.Structure):
        _fields_ = [
            ("occ", ctypes.c_void_p), ("cnt", ctypes.c_void_p), ("hit", ctypes.c_void_p),
            ("half_map_size", ctypes.c_int * 3), ("origin_index", ctypes.c_int * 3),
            ("resolution", ctypes.c_float), ("origin_at_center", ctypes.c_int),
            ("max_range", ctypes.c_float), ("l_hit", ctypes.c_float), ("l_miss", ctypes.c_float),
            ("l_min", ctypes.c_float), ("l_max", ctypes.c_float),
        ]

    L = C.lib()
    fn = L.cublox_integrate_noalloc
    fn.argtypes = [ctypes.POINTER(MapView), ctypes.c_void_p, ctypes.c_int,
                   ctypes.POINTER(ctypes.c_float), ctypes.c_void_p]
    L.cublox_noalloc_last_error.restype = ctypes.c_char_p
    so = (ctypes.c_float * 3)(0.0, 0.0, 0.0)
    for half in ([1 << 30, 1, 1], [1, 1, (1 << 30) - 1], [40000, 40000, 1]):
        view = MapView()
        view.occ = view.cnt = view.hit = 1  # never dereferenced: refused first
        view.half_map_size[:] = half
        view.resolution = 0.1
        assert fn(ctypes.byref(view), None, 0, so, None) == C.ERR_RANGE, half
        assert b"above int32" in L.cublox_noalloc_last_error()


def test_version_and_error_string():
    assert C.lib().cublox_version().startswith(b"cublox_b200")
    assert isinstance(C.lib().cublox_last_error(), bytes)


def test_null_arguments_are_rejected_without_a_gpu():
    L = C.lib()
    assert L.cublox_grid_update(None, None, None, None, 0, None) == C.ERR_INVALID
    assert L.cublox_grid_recenter(None, None, None) == C.ERR_INVALID
    assert L.cublox_grid_destroy(None) == C.OK
    out = ctypes.c_void_p()
    half = (ctypes.c_int * 3)(40000, 40000, 40000)
    o = (ctypes.c_float * 3)(0, 0, 0)
    # voxel count above int32 is refused before any device call (Grid.cpp:44-50)
    assert L.cublox_grid_create(half, 0.1, 0, 0, 0.0, o, None, ctypes.byref(out)) == C.ERR_RANGE
    assert b"exceeds int32" in L.cublox_last_error()


def test_yaml_log_odds_bits():
    bits = [np.float32(v).view(np.uint32) for v in C.yaml_log_odds()]
    assert bits == [0x400C9F53, 0xBD23DC91, 0xBFFF07F3, 0x4079139A, 0xBB831205, 0x3FDE076A]

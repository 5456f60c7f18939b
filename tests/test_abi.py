"""The C ABI: the libraries load and export every symbol their headers declare; calls that need
a GPU fail with an error status (no CPU fallback) when there is none. CPU only."""
import ctypes
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gir_(?:dev|gen|write)\w*)\s*\(", text)))


def test_dev_library_exports_header(pkg):
    lib = pkg.native.dev_lib()
    names = declared("gir_dev.h")
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(pkg.native.DEV_SYMBOLS)


def test_gen_library_exports_header(pkg):
    lib = pkg.native.gen_lib()
    names = declared("gir_gen.h")
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(pkg.native.GEN_SYMBOLS)


def test_create_without_device_fails_loudly(pkg):
    """With no GPU, gir_dev_create returns GIR_ERR_NODEVICE (never a CPU result)."""
    lib = pkg.native.dev_lib()
    fb = np.zeros(3, np.int32)
    h = ctypes.c_void_p()
    rc = lib.gir_dev_create(pkg.native.ptr(fb), None, pkg.native.ptr(fb), None, 2, 0, None, ctypes.byref(h))
    if rc == 0:  # a GPU is present (the GPU box)
        lib.gir_dev_destroy(h)
    else:
        assert rc == 9, rc
        assert b"CUDA" in lib.gir_dev_last_error(None)


def test_bad_arguments_are_rejected_before_the_device(pkg):
    lib = pkg.native.dev_lib()
    h = ctypes.c_void_p()
    assert lib.gir_dev_create(None, None, None, None, 5, 0, None, ctypes.byref(h)) == 1
    fb = np.zeros(3, np.int32)
    assert lib.gir_dev_create(pkg.native.ptr(fb), None, pkg.native.ptr(fb), None, -1, 0, None, ctypes.byref(h)) == 1
    assert lib.gir_dev_load(b"/nonexistent/dir/", ctypes.byref(h)) == 4
    assert lib.gir_dev_build(None, 1) == 1
    assert lib.gir_dev_bfs(None, None, 0, None) == 1
    assert lib.gir_dev_destroy(None) == 0


def test_loader_size_mismatch_is_malformed(pkg, tmp_path):
    d = str(tmp_path) + "/"
    np.array([0, 1, 2], np.int32).tofile(d + "fw_begin.bin")
    np.array([1, 0], np.int32).tofile(d + "fw_adjacent.bin")
    np.array([0, 1, 1, 2], np.int32).tofile(d + "bw_begin.bin")
    np.array([1, 0], np.int32).tofile(d + "bw_adjacent.bin")
    h = ctypes.c_void_p()
    assert pkg.native.dev_lib().gir_dev_load(d.encode(), ctypes.byref(h)) == 5

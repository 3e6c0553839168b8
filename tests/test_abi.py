"""The C-ABI library builds for sm_100a, loads, and exports every symbol include/tarang_gpu.h
declares (CPU: no compute calls)."""

import ctypes
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?(?:int|void|double|char)\s*\**\s*(tg_\w+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def test_header_declares_api():
    names = declared_functions()
    for must in ("tg_ctx_create", "tg_step", "tg_compute_nlin", "tg_time_advance", "tg_flux",
                 "tg_shell_to_shell", "tg_shell_spectrum", "tg_forward_transform", "tg_server_submit"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    from tarang_b200 import _lib
    names = declared_functions()
    missing = [n for n in names if getattr(lib, n, None) is None]
    assert not missing, f"not exported: {missing}"
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\s[T]\s+(tg_\w+)", out))
    assert set(names) <= exported


def test_build_targets_sm100a():
    from tarang_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_config_default_without_gpu(lib):
    from tarang_b200 import _lib
    cfg = _lib.tg_config()
    lib.tg_config_default(ctypes.byref(cfg))
    assert list(cfg.N) == [64, 64, 64] and cfg.scheme == 4 and cfg.dealias == 1
    assert ctypes.sizeof(_lib.tg_config) == 168

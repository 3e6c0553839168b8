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
    assert ctypes.sizeof(_lib.tg_config) == 224 and cfg.rb_temp_grad == 1.0
    assert cfg.hyper_nu == 0.0 and cfg.hyper_eta == 0.0 and cfg.hyper_kappa == 0.0   # hyper terms off


def test_struct_layouts_match_header(tmp_path):
    """The ctypes mirrors have the sizes and field offsets that a C compiler gives the header."""
    from tarang_b200 import _lib
    structs = [_lib.tg_config, _lib.tg_server_config, _lib.tg_request, _lib.tg_request_status,
               _lib.tg_server_stats, _lib.tg_kernel_stat, _lib.tg_batch_stat, _lib.tg_slab_info]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "tarang_gpu.h"', 'int main(void) {']
    for s in structs:
        n = s.__name__
        lines.append(f'  printf("{n} %zu\\n", sizeof({n}));')
        for f, _ in s._fields_:
            lines.append(f'  printf("{n}.{f} %zu\\n", offsetof({n}, {f}));')
    lines += ['  return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines())
    for s in structs:
        n = s.__name__
        assert int(got[n]) == ctypes.sizeof(s), n
        for f, _ in s._fields_:
            assert int(got[f"{n}.{f}"]) == getattr(s, f).offset, f"{n}.{f}"


def test_request_bytes_without_gpu(lib):
    """tg_request_bytes is host arithmetic: affine in the batch size, errors for bad configs."""
    from tarang_b200 import _lib
    from tarang_b200.serving import request_bytes
    cfg = dict(N=(64, 64, 64))
    b1, b2, b3 = (request_bytes(cfg, b) for b in (1, 2, 3))
    assert b3 - b2 == b2 - b1 > 0
    assert request_bytes(dict(N=(64, 64, 64), precision="FP32"), 1) < b1
    try:
        request_bytes(dict(N=(64, 64, 64), dt=-1.0))
        raise AssertionError("negative dt accepted")
    except _lib.TarangError as e:
        assert e.code == _lib.TG_ERR_ARG


def test_energy_noalloc_rejects_bad_arguments_without_gpu(lib):
    """Argument checks of the allocation-free energy reduction run before any CUDA call: more
    fields than its fixed scratch holds, fields not on a 16-byte boundary (they are read as
    16-byte complex values), an output not on an 8-byte boundary."""
    from tarang_b200 import _lib
    n3 = (ctypes.c_int * 3)(16, 16, 16)
    kf = (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    ok16 = ctypes.c_void_p(4096)   # never dereferenced: each call is rejected before any launch
    assert lib.tg_energy_noalloc(ok16, 9, n3, kf, 1, ok16, None) == _lib.TG_ERR_ARG
    assert lib.tg_energy_noalloc(ok16, 0, n3, kf, 1, ok16, None) == _lib.TG_ERR_ARG
    assert lib.tg_energy_noalloc(ctypes.c_void_p(4096 + 8), 3, n3, kf, 1, ok16, None) == _lib.TG_ERR_ARG
    assert lib.tg_energy_noalloc(ok16, 3, n3, kf, 1, ctypes.c_void_p(4096 + 4), None) == _lib.TG_ERR_ARG
    odd = (ctypes.c_int * 3)(16, 16, 15)
    assert lib.tg_energy_noalloc(ok16, 3, odd, kf, 1, ok16, None) == _lib.TG_ERR_ARG


def test_cpp_mirror_header_builds_and_links(tmp_path):
    """include/tarang_b200.hpp compiles with g++ (C++17, warnings as errors) and a driver written
    against it links with the library (no GPU needed to build)."""
    from tarang_b200 import _lib
    _lib.load()
    lib_dir = os.path.dirname(_lib.LIB_PATH)
    exe = str(tmp_path / "ifluid_driver")
    cmd = ["g++", "-std=c++17", "-O0", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "ifluid_driver.cc"), "-L" + lib_dir, "-ltarang_gpu",
           "-Wl,-rpath," + lib_dir, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr

"""The C-ABI library loads and exports every symbol include/fmm_gpu.h
declares; without a GPU its entry points fail with a status code (no CPU
fallback, no crash)."""
import ctypes
import os
import re

import pytest
from conftest import ROOT

import fmmgpu


def header_symbols():
    src = open(os.path.join(ROOT, "include", "fmm_gpu.h")).read()
    return sorted(set(re.findall(r"FMM_API\s+[\w\s\*]*?\b(fmm_\w+)\s*\(", src)))


def test_header_lists_match_binding():
    assert header_symbols() == sorted(fmmgpu.EXPORTED)


def test_library_exports_all_symbols():
    if not os.path.exists(fmmgpu.LIB_PATH):
        pytest.fail(f"{fmmgpu.LIB_PATH} not built: run __graft_entry__.build() or make -C nbody-fmm_b200")
    lib = ctypes.CDLL(fmmgpu.LIB_PATH)
    for name in header_symbols():
        assert hasattr(lib, name), name


def test_strerror_and_defaults_without_gpu():
    L = fmmgpu.load_library()
    assert L.fmm_strerror(fmmgpu.FMM_ERR_NONFINITE_INPUT) == b"non-finite position or mass"
    cfg = fmmgpu.FmmConfig()
    assert L.fmm_config_default(ctypes.byref(cfg)) == 0
    assert (cfg.dim, cfg.p, cfg.leaf_cap, cfg.G) == (3, 8, 64, 1.0)
    assert L.fmm_config_default(None) == fmmgpu.FMM_ERR_INVALID_ARGUMENT


def test_create_rejects_bad_config():
    L = fmmgpu.load_library()
    cfg = fmmgpu.FmmConfig()
    L.fmm_config_default(ctypes.byref(cfg))
    cfg.dim = 4
    h = ctypes.c_void_p()
    assert L.fmm_create(ctypes.byref(cfg), ctypes.byref(h)) == fmmgpu.FMM_ERR_INVALID_ARGUMENT
    cfg.dim = 3
    cfg.p = 99
    assert L.fmm_create(ctypes.byref(cfg), ctypes.byref(h)) == fmmgpu.FMM_ERR_INVALID_ARGUMENT
    cfg.p = 8
    assert cfg.adaptive_leaf == 0  # the default: the reference's uniform targets
    cfg.adaptive_leaf = -1
    assert L.fmm_create(ctypes.byref(cfg), ctypes.byref(h)) == fmmgpu.FMM_ERR_INVALID_ARGUMENT


def test_no_cpu_fallback_without_gpu():
    """On a machine without a GPU, creating a context fails loudly."""
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(fmmgpu.FmmError):
        fmmgpu.Context()


def test_binding_structs_match_header(tmp_path):
    """The ctypes mirrors of the header's structs have the C layout: the
    same size and the same offset for every field, as the C compiler lays
    them out from include/fmm_gpu.h."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    mirrors = {"fmm_config": fmmgpu.FmmConfig, "fmm_stats": fmmgpu.FmmStats,
               "fmm_tune_result": fmmgpu.FmmTuneResult}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "fmm_gpu.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'  printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(ln.split() for ln in subprocess.run([str(exe)], capture_output=True, text=True,
                                                   check=True).stdout.splitlines())
    for cname, py in mirrors.items():
        assert int(got[cname]) == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(py, f).offset, f"{cname}.{f}"

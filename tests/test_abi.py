"""The C ABI: the library builds, loads and exports every entry point the
public headers declare; the product never reaches into the oracle."""
import os
import re
import subprocess

import pytest

from conftest import PKG, REPO
from op2b import build, lib as L


def _header_functions():
    names = set()
    for h in os.listdir(os.path.join(REPO, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(REPO, "include", h)).read()
        if "extern \"C\"" not in text:
            continue
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        body = text[text.index("extern \"C\""):]
        for m in re.finditer(r"^\s*[A-Za-z_][\w \*]*?\b(op\w+)\s*\(", body, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_builds_and_loads():
    path = build.build()
    assert os.path.exists(path)
    L.load(path)


def test_every_declared_symbol_is_exported():
    path = build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    declared = _header_functions()
    assert declared, "no declarations parsed"
    missing = sorted(declared - exported)
    assert not missing, f"declared but not exported: {missing}"
    # the ctypes binding covers the same entry points
    assert set(L.exported_symbols()) <= exported


def test_product_does_not_use_the_oracle():
    for root, _, files in os.walk(PKG):
        for f in files:
            if f.endswith((".py", ".cpp", ".cu", ".h", ".cuh")):
                text = open(os.path.join(root, f), errors="ignore").read()
                assert "import oracle" not in text and "from oracle" not in text, f
                assert "liboracle" not in text, f


def test_sm100a_only_build_flags():
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)


def test_init_without_device_fails_loudly():
    import ctypes
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    L.load()
    with pytest.raises(L.Op2Error):
        L.op_init()
    assert L.load().op2b_status() != 0
    # a loop without op_init is refused, not run on the host
    arr = (L.op_arg * 1)()
    assert L.load().op_par_loop_c(b"save_soln", None, 0, arr) != 0
    assert "op_init" in L.load().op2b_last_error().decode()
    del ctypes

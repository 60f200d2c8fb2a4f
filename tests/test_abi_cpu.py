"""The C-ABI library builds, loads without a GPU and exports every declared symbol."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fpsg.h")


def declared(header: str) -> set[str]:
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(fpsg_[a-z_0-9]+)\s*\(", text))


def test_header_and_python_binding_agree(engine_lib):
    assert declared(HEADER) == set(engine_lib.EXPORTS)


def test_library_exports_every_declared_symbol(engine_lib):
    so = engine_lib.LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (fpsg_\w+)", out))
    missing = declared(HEADER) - exported
    assert not missing, missing


def test_library_loads_and_reports_version(engine_lib):
    L = engine_lib.load()
    assert L.fpsg_version().decode().startswith("fpsg")


def test_null_context_is_rejected(engine_lib):
    L = engine_lib.load()
    assert L.fpsg_set_memory_cap(None, 0) == engine_lib.ERR_INVALID
    assert L.fpsg_set_grad_memory(None, 0) == engine_lib.ERR_INVALID
    assert L.fpsg_num_trajectories(None) == 0
    assert L.fpsg_last_error(None) is not None


def test_create_without_device_fails_cleanly(engine_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    L = engine_lib.load()
    h = ctypes.c_void_p()
    rc = L.fpsg_create(ctypes.byref(h), 0, 0)
    assert rc == engine_lib.ERR_NO_DEVICE
    assert not h.value

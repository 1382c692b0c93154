"""The C-ABI library loads without a GPU and exports every symbol that
include/r2.h declares; host-only entry points behave on CPU."""
import ctypes as C
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "r2.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(r2_[a-z0-9_]+)\s*\(", src)))


def test_header_symbols_exported():
    from renderer2_b200 import _native as N
    names = _declared()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(N.lib, n)]
    assert not missing, missing


def test_status_strings_and_version():
    from renderer2_b200 import _native as N
    assert N.lib.r2_status_string(0) == b"R2_OK"
    assert N.lib.r2_status_string(8) == b"R2_ERR_UNSUPPORTED"
    assert N.lib.r2_version() >= 100


def test_no_device_reported_without_gpu():
    import torch
    from renderer2_b200 import _native as N
    from renderer2_b200 import filter as F, scenes
    if torch.cuda.is_available():
        return
    mesh = scenes.icosphere(1, 0.0, 1)
    try:
        F.FilterScene(mesh, F.material())
        raise AssertionError("expected R2_ERR_NO_DEVICE")
    except N.R2Error as e:
        assert e.name == "R2_ERR_NO_DEVICE"


def test_generator_capacity_checked():
    from renderer2_b200 import _native as N
    pos = np.zeros(3, np.float32)
    idx = np.zeros(3, np.uint32)
    st = N.lib.r2_gen_icosphere(2, 0.0, 1, N.ptr(pos), pos.size, N.ptr(idx), idx.size, None, None, None)
    assert N.lib.r2_status_string(st) == b"R2_ERR_INVALID_ARGUMENT"

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


def test_workload_generators_do_not_load_the_library():
    """The CPU baseline builds the benchmark's inputs with the seeded numpy
    generators; the GPU library must stay unloaded in that process."""
    import subprocess
    import sys
    code = ("import bench, sys\n"
            "desc, cam, prm = bench.render_workload()\n"
            "mesh, mat, fprm, vs = bench.filter_workload()\n"
            "maps = open('/proc/self/maps').read()\n"
            "sys.exit(3 if 'librenderer2' in maps else 0)\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr

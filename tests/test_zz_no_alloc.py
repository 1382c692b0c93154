"""The allocation-free filter entry point, r2_filter_scene_run_static.

Callers that must not allocate device memory while filtering (a frame loop
under a fixed memory budget with no allocation after start-up, an application
that owns all device memory through its own pool, or a latency-bound caller
that cannot afford the synchronisation an allocation may imply) filter
through r2_filter_scene_run_static, which keeps its voxel work
list and queue counters in a fixed scratch array inside the library instead
of allocating them.  This file is collected last so that a failure here
cannot hide another test's result; it must pass in a fresh process as well as
after the other tests.  The output must equal that of r2_filter_scene_run
(the allocating entry point) on two calls in a row, since the shared scratch
keeps the previous call's contents.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from renderer2_b200 import _native as N  # noqa: E402
from renderer2_b200 import filter as F  # noqa: E402
from renderer2_b200 import scenes  # noqa: E402

N.lib.r2_filter_scene_run_static.restype = C.c_int
N.lib.r2_filter_scene_run_static.argtypes = [C.c_void_p] * 7


def _run_static(sc, g, prm, out, wide):
    N.check(N.lib.r2_filter_scene_run_static(sc.handle, C.byref(g), C.byref(prm), C.c_void_p(out.data_ptr()),
                                             C.c_void_p(wide.data_ptr()), None, None))


def test_static_scratch_matches_allocating_entry_twice():
    mesh = scenes.icosphere(4, 0.05, 1)
    mat = F.material()
    sc = F.FilterScene(mesh, mat)
    for n, spv, seed in [(32, 64, 0), (24, 33, 9)]:
        prm = F.params(samples_per_voxel=spv, iterations=10, seed=seed)
        g = sc.grid(scenes.voxel_size_for(mesh, n))
        nvox = int(np.prod(np.array(g.num_voxels[:], np.int64)))
        ref_out = torch.empty(nvox * 32, dtype=torch.uint8, device="cuda")
        ref_wide = torch.empty(nvox * 20, dtype=torch.float32, device="cuda")
        sc.run(g, prm, ref_out.data_ptr(), ref_wide.data_ptr())
        for _ in range(2):  # two calls in a row over the same shared scratch
            out = torch.full((nvox * 32,), 0xAB, dtype=torch.uint8, device="cuda")
            wide = torch.full((nvox * 20,), -7.0, dtype=torch.float32, device="cuda")
            _run_static(sc, g, prm, out, wide)
            torch.cuda.synchronize()
            assert torch.equal(out, ref_out)
            assert torch.equal(wide, ref_wide)
    sc.close()


def test_static_null_stream_orders_calls_on_different_scenes():
    """Two scenes filtered back to back with stream NULL: the calls run in
    order on the legacy default stream, so the second call cannot overwrite
    the shared work list while the first one still reads it."""
    meshes = [scenes.icosphere(4, 0.05, 1), scenes.icosphere(3, 0.08, 7)]
    mat = F.material()
    scs = [F.FilterScene(m, mat) for m in meshes]
    grids = [sc.grid(scenes.voxel_size_for(m, n)) for sc, m, n in zip(scs, meshes, (40, 36))]
    prms = [F.params(samples_per_voxel=64, iterations=10, seed=3), F.params(samples_per_voxel=48, iterations=6)]
    refs, outs = [], []
    for sc, g, prm in zip(scs, grids, prms):
        nvox = int(np.prod(np.array(g.num_voxels[:], np.int64)))
        ro = torch.empty(nvox * 32, dtype=torch.uint8, device="cuda")
        rw = torch.empty(nvox * 20, dtype=torch.float32, device="cuda")
        sc.run(g, prm, ro.data_ptr(), rw.data_ptr())
        refs.append((ro, rw))
        outs.append((torch.full((nvox * 32,), 0xCD, dtype=torch.uint8, device="cuda"),
                     torch.full((nvox * 20,), -3.0, dtype=torch.float32, device="cuda")))
    torch.cuda.synchronize()
    for _ in range(2):
        for sc, g, prm, (o, w) in zip(scs, grids, prms, outs):  # no synchronisation between the calls
            _run_static(sc, g, prm, o, w)
        torch.cuda.synchronize()
        for (ro, rw), (o, w) in zip(refs, outs):
            assert torch.equal(o, ro)
            assert torch.equal(w, rw)
    for sc in scs:
        sc.close()


def test_static_scratch_rejects_oversized_grid():
    mesh = scenes.icosphere(2, 0.05, 1)
    sc = F.FilterScene(mesh, F.material())
    g = sc.grid(scenes.voxel_size_for(mesh, 128))  # 128^3 = 2,097,152 voxels > 2^20
    out = torch.empty(32, dtype=torch.uint8, device="cuda")
    wide = torch.empty(20, dtype=torch.float32, device="cuda")
    with pytest.raises(N.R2Error) as e:
        _run_static(sc, g, F.params(), out, wide)
    assert e.value.name == "R2_ERR_UNSUPPORTED"
    sc.close()

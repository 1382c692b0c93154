"""The request loop: every job's result is the same alone and in a mix of
concurrent render and filter jobs (bit for bit: random streams depend on
pixel, sample and seed only), admission respects the HBM budget, and a job
larger than the budget is rejected."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from renderer2_b200 import _native as N  # noqa: E402
from renderer2_b200 import filter as F  # noqa: E402
from renderer2_b200 import raytracer as R  # noqa: E402
from renderer2_b200 import render_scenes as RS  # noqa: E402
from renderer2_b200 import scenes  # noqa: E402
from renderer2_b200 import serving as S  # noqa: E402


@pytest.fixture(scope="module")
def world(tmp_path_factory):
    desc1, _ = RS.icosphere_scene()
    desc1 = dict(desc1)
    desc1["env"] = RS.lognormal_env(64, 32, 1.0, 2)
    sc1 = RS.build_scene(desc1)
    # a media scene: a filtered icosphere with the brick grid
    out = tmp_path_factory.mktemp("serve")
    ico = scenes.icosphere(3, 0.08, 4)
    mat = F.material(diffuse=(0.8, 0.5, 0.3), specular=(0.9, 0.9, 0.9), alpha=0.35, ior=1.5)
    paths, _ = F.run_filtering(ico, mat, F.params(samples_per_voxel=16, iterations=5,
                                                  min_voxel_size=scenes.voxel_size_for(ico, 24)), out, "ico")
    desc2 = {"media": [(paths[0], (0, 0, 0), (10, 10, 10), (0, 0, 0), (0, 1, 0), (1, 1, 1))],
             "shapes": [(R.CIRCLE, (0, -1.3, 0), 40.0, (0, 1, 0), F.material(diffuse=(0.6, 0.6, 0.6), alpha=0.5))],
             "env": RS.lognormal_env(32, 16, 0.7, 3)}
    sc2 = RS.build_scene(desc2)
    leaves = scenes.foliage(20_000, 6, 0.7, 9)
    fmat = F.material(diffuse=(0.1, 0.6, 0.1), specular=(0.04, 0.04, 0.04), alpha=0.5, ior=1.5)
    fs = F.FilterScene(leaves, fmat)
    yield {"sc1": sc1, "sc2": sc2, "fs": fs, "leaves": leaves, "fmat": fmat}
    sc1.close()
    sc2.close()
    fs.close()


def _jobs(w):
    """(kind, args) of a mixed job list with various sizes."""
    cams = [R.camera(64, 48, 45.0, (0, 0, 3)), R.camera(96, 96, 50.0, (0.5, 0.3, 3.2)),
            R.camera(40, 30, 60.0, (0.3, 0.6, 3.2))]
    jobs = []
    for k in range(9):
        if k % 3 == 2:
            vs = scenes.voxel_size_for(w["leaves"], 24 + 8 * (k % 2))
            prm = F.params(samples_per_voxel=32, iterations=6, seed=k)
            jobs.append(("filter", w["fs"].grid(vs), prm))
        else:
            sc = w["sc1"] if k % 2 == 0 else w["sc2"]
            prm = R.params(2 + k % 3, 6, 100 + k, brick_grid=(k % 4 == 1))
            jobs.append(("render", sc, cams[k % 3], prm))
    return jobs


def _alone(w, job):
    if job[0] == "render":
        _, sc, cam, prm = job
        return sc.render(cam, prm)
    _, g, prm = job
    nvox = int(np.prod(np.array(g.num_voxels[:], np.int64)))
    out = torch.empty(nvox * 32, dtype=torch.uint8, device="cuda")
    w["fs"].run(g, prm, out.data_ptr())
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_results_same_alone_and_in_the_mix(world):
    jobs = _jobs(world)
    alone = [_alone(world, j) for j in jobs]
    srv = S.Server(slots=4, hbm_budget=8 << 30)
    handles = []
    for j in jobs:
        handles.append(srv.submit_render(*j[1:]) if j[0] == "render" else srv.submit_filter(world["fs"], *j[1:]))
    for h, ref in zip(handles, alone):
        assert srv.wait(h, 120.0)
        got = h.out if h.kind == "render" else h.out.view(np.uint8).reshape(-1)
        assert np.array_equal(got.reshape(ref.shape), ref), f"job {h.id} differs"
        t = h.times
        assert t[0] <= t[1] <= t[2]
    st = srv.stats()
    assert st["done"] == len(jobs) and st["queued"] == 0 and st["bytes_admitted"] == 0
    srv.close()


def test_budget_serialises_and_rejects(world):
    cam = R.camera(128, 128, 45.0, (0, 0, 3))
    prm = R.params(2, 6, 7)
    ref = world["sc1"].render(cam, prm)
    one_job = S.Server.render_bytes(world["sc1"], cam, prm)
    assert one_job >= 128 * 128 * (5 * 16 + 6 * 16 + 16 + 12 + 8 + 12)  # at least the wave state of one sample
    srv = S.Server(slots=4, hbm_budget=int(one_job * 1.5))  # at most one such job admitted at a time
    hs = [srv.submit_render(world["sc1"], cam, prm) for _ in range(4)]
    for h in hs:
        assert srv.wait(h, 120.0)
        assert np.array_equal(h.out, ref)
    ts = sorted((h.times[1], h.times[2]) for h in hs)
    for (s0, e0), (s1, e1) in zip(ts, ts[1:]):
        assert s1 >= e0 - 1e-6  # admitted one after the other
    with pytest.raises(N.R2Error) as e:
        srv.submit_render(world["sc1"], R.camera(1024, 1024), prm)
    assert e.value.status == 5  # R2_ERR_ADMISSION_REJECTED
    srv.close()


def test_wait_timeout_reports_pending(world):
    srv = S.Server(slots=1, hbm_budget=8 << 30)
    cam = R.camera(512, 512, 45.0, (0, 0, 3))
    h = srv.submit_render(world["sc1"], cam, R.params(64, 8, 1))
    assert not srv.wait(h, 0.0)  # a frame of 16M paths is still running
    assert srv.wait(h, 300.0)
    assert np.isfinite(h.out).all() and h.out.mean() > 0
    srv.close()


def test_render_batch_matches_single_frames(world):
    """One captured graph holding a wave of every frame (the same scene twice
    with other cameras, a media scene with both tracking modes) gives every
    frame bit for bit, run twice."""
    cams = [R.camera(64, 48, 45.0, (0, 0, 3)), R.camera(96, 96, 50.0, (0.5, 0.3, 3.2)),
            R.camera(40, 30, 60.0, (0.3, 0.6, 3.2)), R.camera(48, 64, 40.0, (0.2, 0.1, 3.0))]
    scs = [world["sc1"], world["sc2"], world["sc1"], world["sc2"]]
    prms = [R.params(3, 6, 11), R.params(3, 8, 12, brick_grid=True), R.params(3, 5, 13), R.params(3, 8, 14)]
    refs = [s.render(c, p) for s, c, p in zip(scs, cams, prms)]
    frames = [torch.empty((c.height, c.width, 3), dtype=torch.float32, device="cuda") for c in cams]
    b = R.RenderBatch(scs, cams, prms, [f.data_ptr() for f in frames])
    for _ in range(2):
        ms = b.run()
        assert ms > 0
        for f, ref in zip(frames, refs):
            assert np.array_equal(f.cpu().numpy(), ref)
    b.close()


def test_render_batch_rejects_mixed_sample_counts(world):
    cam = R.camera(16, 16)
    f = torch.empty((16, 16, 3), dtype=torch.float32, device="cuda")
    with pytest.raises(N.R2Error) as e:
        R.RenderBatch([world["sc1"], world["sc1"]], [cam, cam], [R.params(2), R.params(3)],
                      [f.data_ptr(), f.data_ptr()])
    assert e.value.name == "R2_ERR_INVALID_ARGUMENT"

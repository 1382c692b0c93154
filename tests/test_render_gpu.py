"""GPU parity of the wavefront path tracer against the CPU oracle.

The oracle runs each path start to finish (like the reference's megakernel)
with the same Philox streams, so the GPU frame must match it pixel for pixel
up to the rounding of acos/atan2/sin inside the environment lookup; and a
low-spp GPU frame must lie within 3 sigma of a high-spp oracle estimate.
"""
import numpy as np
import pytest

import flip
import oracle_lib as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from renderer2_b200 import filter as F  # noqa: E402
from renderer2_b200 import raytracer as R  # noqa: E402
from renderer2_b200 import render_scenes as RS  # noqa: E402
from renderer2_b200 import scenes  # noqa: E402

PIX_REL = 1e-4   # per-pixel relative tolerance (libm vs CUDA acos/atan2/sin in the env lookup)
PIX_FRAC = 0.999  # fraction of pixels that must meet it


def _gpu_frame(desc, cam, spp, depth, seed):
    sc = RS.build_scene(desc)
    img = sc.render(cam, R.params(spp, depth, seed))
    sc.close()
    return img.reshape(-1, 3)


def _agree(g, o):
    tol = PIX_REL * np.maximum(1.0, np.abs(o))
    ok = np.all(np.abs(g - o) <= tol, axis=1)
    return ok.mean()


def test_small_icosphere_matches_oracle():
    desc, _ = RS.icosphere_scene()
    cam = R.camera(64, 64, 45.0, (0, 0, 3), (0, 0, 0), (0, 1, 0))
    g = _gpu_frame(desc, cam, 8, 8, 0)
    o = O.render(desc, cam, 8, 8, 0)
    assert np.isfinite(g).all()
    frac = _agree(g, o)
    assert frac >= PIX_FRAC, f"only {frac:.4f} of pixels agree"
    assert np.abs(g.mean(0) - o.mean(0)).max() < 1e-4


def test_shapes_and_lognormal_env_match_oracle():
    mesh = scenes.icosphere(3, 0.05, 7)
    desc = {
        "meshes": [(mesh, F.material(diffuse=(0.7, 0.4, 0.2), specular=(1, 1, 1), alpha=0.15, ior=1.5),
                    RS.translate43(0.0, 0.2, 0.0))],
        "shapes": [(R.SPHERE, (1.6, 0.0, -0.5), 0.6, (1, 0, 0),
                    F.material(diffuse=(0.2, 0.8, 0.3), specular=(0.5, 0.5, 0.5), alpha=0.6, ior=1.33,
                               diffuse_roughness=0.5)),
                   (R.CIRCLE, (0.0, -1.1, 0.0), 3.4e38, (0, 1, 0),
                    F.material(diffuse=(0.3, 0.3, 0.3), specular=(0.9, 0.9, 0.9), alpha=0.99, ior=1.2,
                               diffuse_roughness=0.99))],
        "env": RS.lognormal_env(64, 32, 1.5, 9),
    }
    cam = R.camera(48, 40, 60.0, (0.5, 1.0, 4.0), (0.0, 0.0, 0.0), (0, 1, 0))
    g = _gpu_frame(desc, cam, 6, 6, 5)
    o = O.render(desc, cam, 6, 6, 5)
    frac = _agree(g, o)
    assert frac >= PIX_FRAC, f"only {frac:.4f} of pixels agree"


def test_deep_paths_rr_match_oracle():
    # depth > 4 exercises Russian roulette; albedo near 1 keeps paths alive
    mesh = scenes.icosphere(2, 0.3, 3)
    desc = {"meshes": [(mesh, F.material(diffuse=(0.95, 0.95, 0.95), specular=(1, 1, 1), alpha=0.5, ior=1.5),
                        RS.translate43(0, 0, 0))],
            "shapes": [(R.CIRCLE, (0.0, -1.2, 0.0), 50.0, (0, 1, 0), F.material(diffuse=(0.9, 0.9, 0.9), alpha=0.3))],
            "env": RS.lognormal_env(32, 16, 0.5, 1)}
    cam = R.camera(32, 32, 50.0, (0, 0.5, 3.5), (0, 0, 0), (0, 1, 0))
    g = _gpu_frame(desc, cam, 4, 12, 3)
    o = O.render(desc, cam, 4, 12, 3)
    assert _agree(g, o) >= PIX_FRAC


def test_three_sigma_against_high_spp_oracle():
    desc, _ = RS.icosphere_scene()
    desc = dict(desc)
    desc["env"] = RS.lognormal_env(32, 16, 1.0, 4)
    cam = R.camera(24, 24, 45.0, (0, 0, 3), (0, 0, 0), (0, 1, 0))
    spp_g, spp_o = 64, 4096
    g = _gpu_frame(desc, cam, spp_g, 8, 101)
    o, var = O.render(desc, cam, spp_o, 8, 7, want_var=True)
    sigma = np.sqrt(var / spp_g + var / spp_o) + 1e-7
    z = np.abs(g - o) / sigma
    within = (z <= 3.0).mean()
    assert within >= 0.98, f"{within:.4f} of pixel channels within 3 sigma"
    # mean LDR-FLIP of the 64-spp frame against the 4096-spp estimate
    # (x / (1 + x), gamma 2.2): Monte Carlo noise only
    ldr = lambda f: (np.asarray(f).reshape(24, 24, 3) / (1.0 + np.asarray(f).reshape(24, 24, 3))) ** (1 / 2.2)
    mf = flip.mean_flip(ldr(o), ldr(g))
    print(f"mean FLIP 64 spp vs 4096 spp: {mf:.4f}")
    assert mf < 0.1


def test_device_entry_matches_host_entry_and_is_deterministic():
    desc, _ = RS.icosphere_scene()
    cam = R.camera(40, 30, 45.0, (0, 0, 3), (0, 0, 0), (0, 1, 0))
    sc = RS.build_scene(desc)
    a = sc.render(cam, R.params(4, 8, 2))
    buf = torch.empty(40 * 30 * 3, dtype=torch.float32, device="cuda")
    st = sc.render_device(cam, R.params(4, 8, 2), buf.data_ptr())
    torch.cuda.synchronize()
    b = buf.cpu().numpy().reshape(30, 40, 3)
    c = sc.render(cam, R.params(4, 8, 2))
    sc.close()
    assert np.array_equal(a, b) and np.array_equal(a, c)
    assert st[0] == 40 * 30 * 4


def test_device_rebuild_gives_the_same_frame():
    """r2_scene_rebuild rebuilds the triangle BVH from the resident triangles
    and re-gathers the shading data: the frames before and after, on the
    scene's stream and on a caller's stream, are bit-identical."""
    desc, _ = RS.icosphere_grid_scene()
    cam = R.camera(48, 40, 45.0, (0, 0, 24), (0, 0, 0), (0, 1, 0))
    sc = RS.build_scene(desc)
    prm = R.params(2, 8, 4)
    a = sc.render(cam, prm)
    sc.rebuild()
    b = sc.render(cam, prm)
    s = torch.cuda.Stream()
    sc.rebuild(s.cuda_stream)
    c = sc.render(cam, prm)
    sc.close()
    assert np.array_equal(a, b) and np.array_equal(a, c)


def test_frame_does_not_depend_on_the_bvh_method():
    """Closest hits (ties to the lower triangle) and shadow visibility do not
    depend on the hierarchy, so scenes built with the PLOC and with the Karras
    tree render the same frame bit for bit."""
    desc, _ = RS.icosphere_grid_scene()
    cam = R.camera(64, 48, 45.0, (0, 0, 24), (0, 0, 0), (0, 1, 0))
    prm = R.params(4, 8, 9)
    frames = []
    try:
        for method in (R.BVH_PLOC, R.BVH_KARRAS):
            R.set_bvh_method(method)
            assert R.bvh_method() == method
            sc = RS.build_scene(desc)
            frames.append(sc.render(cam, prm))
            sc.close()
    finally:
        R.set_bvh_method(R.BVH_AUTO)
    assert np.array_equal(frames[0], frames[1])


def test_set_vertices_matches_a_scene_built_from_the_moved_meshes():
    """r2_scene_set_vertices + r2_scene_rebuild on a committed scene give the
    frame of a scene built from scratch with the moved geometry, bit for bit;
    the unmoved vertices give back the original frame."""
    desc, _ = RS.icosphere_grid_scene()
    cam = R.camera(48, 40, 45.0, (0, 0, 24), (0, 0, 0), (0, 1, 0))
    prm = R.params(2, 8, 9)
    sc = RS.build_scene(desc)
    a = sc.render(cam, prm)
    moved = {"meshes": [(m, mat, RS.translate43(float(t[9]) + 0.7, float(t[10]) - 0.4, 1.5))
                        for m, mat, t in desc["meshes"]], "shapes": [], "env": desc["env"]}
    pos, nrm = RS.world_vertices(moved)
    sc.set_vertices(pos, nrm)
    sc.rebuild()
    b = sc.render(cam, prm)
    ref = RS.build_scene(moved)
    c = ref.render(cam, prm)
    ref.close()
    pos0, nrm0 = RS.world_vertices(desc)
    sc.set_vertices(pos0, nrm0)
    sc.rebuild()
    d = sc.render(cam, prm)
    from renderer2_b200 import _native as N
    with pytest.raises(N.R2Error):
        sc.set_vertices(pos0[:-1], None)  # vertex count must match
    sc.close()
    assert not np.array_equal(a, b)
    assert np.array_equal(b, c)
    assert np.array_equal(a, d)


def test_render_rejects_bad_arguments():
    desc, _ = RS.icosphere_scene()
    sc = RS.build_scene(desc)
    from renderer2_b200 import _native as N
    with pytest.raises(N.R2Error):
        sc.render(R.camera(8, 8), R.params(0, 8, 0))
    with pytest.raises(N.R2Error):
        sc.render(R.camera(8, 8), R.params(1, 100, 0))
    sc.close()


def test_launch_tuning_never_changes_the_frame():
    """Refill thresholds and visit rounds of the persistent traversals (and the
    autotuner's choice) give the same frame bit for bit."""
    desc, _ = RS.icosphere_grid_scene()
    cam = R.camera(96, 80, 45.0, (0, 0, 24), (0, 0, 0), (0, 1, 0))
    prm = R.params(2, 8, 5)
    sc = RS.build_scene(desc)
    sc.set_tuning(R.tuning(wave_paths=96 * 80))  # one sample per wave
    ref = sc.render(cam, prm)
    for visits, refill, wave, top, srt in [(1, 1, 0, 0, 1), (3, 32, 96 * 80, 64, 0), (1000, 5, 2 * 96 * 80, 256, 1),
                                           (64, 16, 1 << 24, 7, 1)]:
        sc.set_tuning(R.tuning(trav_visits=visits, trav_refill=refill, wave_paths=wave, top_nodes=top, sort_rays=srt))
        assert sc.get_tuning().as_tuple() == (0, visits, refill, wave, 0, 0, 0, top, srt)
        assert sc.wave_samples(cam, prm) == (2 if wave != 96 * 80 else 1)
        assert np.array_equal(sc.render(cam, prm), ref), (visits, refill, wave, top, srt)
    t = sc.autotune(cam, prm)
    assert 1 <= t.trav_refill <= 32 and t.trav_visits >= 1
    assert sc.get_tuning().as_tuple() == t.as_tuple()
    assert np.array_equal(sc.render(cam, prm), ref)
    from renderer2_b200 import _native as N
    with pytest.raises(N.R2Error):
        sc.set_tuning(R.tuning(trav_refill=33))
    with pytest.raises(N.R2Error):
        sc.set_tuning(R.tuning(top_nodes=257))
    with pytest.raises(N.R2Error):
        sc.set_tuning(R.tuning(sort_rays=2))
    sc.close()

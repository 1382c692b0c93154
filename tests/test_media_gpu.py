"""GPU parity of heterogeneous SGGX media against the CPU oracle.

A displaced icosphere is filtered on the GPU into two LODs of NanoVDB +
brick-grid files; scenes place those media (with and without an instance
transform) over a ground disc under a lognormal environment map.  The oracle
reads the same files through its own NanoVDB tree walk and brick-grid reader
and runs each path start to finish with the same Philox streams and the same
tracking logarithm, so GPU and oracle frames agree pixel for pixel up to the
rounding of acos/atan2/sin inside the environment lookup (values only, never
path decisions).  Both tracking modes are covered: the global majorant
(sampleInternal / trInternal) and the brick-grid DDA (sampleDDA / trDDA).
"""
import numpy as np
import pytest

import flip
import oracle_lib as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from renderer2_b200 import _native as N  # noqa: E402
from renderer2_b200 import filter as F  # noqa: E402
from renderer2_b200 import raytracer as R  # noqa: E402
from renderer2_b200 import render_scenes as RS  # noqa: E402
from renderer2_b200 import scenes  # noqa: E402

PIX_REL = 1e-4
PIX_FRAC = 0.995
SIGMA_A = (0.0, 0.0, 0.0)
SIGMA_S = (10.0, 10.0, 10.0)  # sigma_t = 10, the filter's SigmaT


@pytest.fixture(scope="module")
def lods(tmp_path_factory):
    out = tmp_path_factory.mktemp("filtering")
    mesh = scenes.icosphere(3, 0.08, 4)
    mat = F.material(diffuse=(0.8, 0.5, 0.3), specular=(0.9, 0.9, 0.9), alpha=0.35, ior=1.5)
    vs = scenes.voxel_size_for(mesh, 24)
    prm = F.params(samples_per_voxel=32, iterations=10, min_voxel_size=vs, lods=2)
    paths, st = F.run_filtering(mesh, mat, prm, out, "sphere")
    assert len(paths) == 2 and st[2] > 0
    return paths


def _desc(path, pos=(0.0, 0.0, 0.0), ori=(0.0, 1.0, 0.0), scl=(1.0, 1.0, 1.0), ground=True):
    d = {"media": [(path, SIGMA_A, SIGMA_S, pos, ori, scl)],
         "shapes": [], "env": RS.lognormal_env(32, 16, 0.7, 3)}
    if ground:
        d["shapes"].append((R.CIRCLE, (0.0, -1.3, 0.0), 40.0, (0, 1, 0),
                            F.material(diffuse=(0.6, 0.6, 0.6), specular=(0.5, 0.5, 0.5), alpha=0.6, ior=1.3,
                                       diffuse_roughness=0.4)))
    return d


def _gpu(desc, cam, spp, depth, seed, dda):
    sc = RS.build_scene(desc)
    img = sc.render(cam, R.params(spp, depth, seed, brick_grid=dda))
    sc.close()
    return img.reshape(-1, 3)


def _agree(g, o):
    tol = PIX_REL * np.maximum(1.0, np.abs(o))
    return np.all(np.abs(g - o) <= tol, axis=1).mean()


@pytest.mark.parametrize("dda", [False, True])
def test_medium_frame_matches_oracle(lods, dda):
    desc = _desc(lods[0])
    cam = R.camera(40, 32, 50.0, (0.3, 0.6, 3.2), (0.0, 0.0, 0.0), (0, 1, 0))
    g = _gpu(desc, cam, 4, 6, 3, dda)
    o = O.render(desc, cam, 4, 6, 3, flags=1 if dda else 0)
    assert np.isfinite(g).all()
    frac = _agree(g, o)
    assert frac >= PIX_FRAC, f"only {frac:.4f} of pixels agree"
    # the medium is visible: it darkens the env seen straight through it
    empty = _gpu({"shapes": desc["shapes"], "env": desc["env"]}, cam, 4, 6, 3, False)
    centre = (np.arange(40 * 32) % 40 > 12) & (np.arange(40 * 32) % 40 < 28)
    assert np.abs(g[centre] - empty[centre]).mean() > 1e-3


def test_medium_instance_transform_and_coarse_lod_match_oracle(lods):
    # LOD 1 (twice the voxel size), moved, scaled and rotated (+Y -> +X)
    desc = _desc(lods[1], pos=(0.2, 0.1, -0.3), ori=(1.0, 0.0, 0.0), scl=(1.4, 1.4, 1.4))
    cam = R.camera(36, 36, 55.0, (0.0, 0.8, 3.5), (0.1, 0.0, -0.2), (0, 1, 0))
    for dda in (False, True):
        g = _gpu(desc, cam, 3, 8, 9, dda)
        o = O.render(desc, cam, 3, 8, 9, flags=1 if dda else 0)
        frac = _agree(g, o)
        assert frac >= PIX_FRAC, f"dda={dda}: only {frac:.4f} of pixels agree"


@pytest.mark.parametrize("g", [0.0, 0.45, -0.6])
def test_medium_henyey_greenstein_matches_oracle(lods, g):
    # a Medium with a "G" key: Henyey-Greenstein phase function, SGGX payload albedo
    desc = _desc(lods[0])
    desc["media"] = [desc["media"][0] + (g,)]
    cam = R.camera(32, 32, 50.0, (0.3, 0.6, 3.2), (0.0, 0.0, 0.0), (0, 1, 0))
    gi = _gpu(desc, cam, 3, 6, 21, True)
    o = O.render(desc, cam, 3, 6, 21, flags=1)
    frac = _agree(gi, o)
    assert frac >= PIX_FRAC, f"g={g}: only {frac:.4f} of pixels agree"


def test_medium_three_sigma_against_high_spp_oracle(lods):
    desc = _desc(lods[0], ground=False)
    cam = R.camera(16, 16, 45.0, (0.0, 0.0, 3.0), (0.0, 0.0, 0.0), (0, 1, 0))
    spp_g, spp_o = 256, 4096
    g = _gpu(desc, cam, spp_g, 8, 101, True)
    o, var = O.render(desc, cam, spp_o, 8, 7, want_var=True, flags=1)
    sigma = np.sqrt(var / spp_g + var / spp_o) + 1e-7
    within = (np.abs(g - o) / sigma <= 3.0).mean()
    assert within >= 0.97, f"{within:.4f} of pixel channels within 3 sigma"
    # mean LDR-FLIP of the 256-spp frame against the 4096-spp estimate (x / (1 + x), gamma 2.2)
    ldr = lambda f: (np.asarray(f).reshape(16, 16, 3) / (1.0 + np.asarray(f).reshape(16, 16, 3))) ** (1 / 2.2)
    mf = flip.mean_flip(ldr(o), ldr(g))
    print(f"mean FLIP 256 spp vs 4096 spp: {mf:.4f}")
    assert mf < 0.1


def test_medium_loading_errors(lods, tmp_path):
    sc = R.Scene()
    with pytest.raises(N.R2Error) as e:
        sc.add_medium(str(tmp_path / "missing_0.500000"), SIGMA_A, SIGMA_S)
    assert e.value.status == 3  # R2_ERR_IO
    with pytest.raises(N.R2Error) as e:
        sc.add_medium(str(tmp_path / "no_voxel_size"), SIGMA_A, SIGMA_S)
    assert e.value.status in (2, 3)
    with pytest.raises(N.R2Error):
        sc.add_medium(lods[0], (0, 0, 0), (0, 0, 0))  # sigma_t = 0
    sc.close()


def test_medium_tuning_out_of_range_is_rejected(lods):
    sc = RS.build_scene(_desc(lods[0]))
    with pytest.raises(N.R2Error):
        sc.set_tuning(R.tuning(media_rounds=33))
    sc.close()


def test_medium_tracking_tuning_never_changes_the_frame(lods):
    desc = _desc(lods[0])
    cam = R.camera(32, 28, 50.0, (0.3, 0.6, 3.2), (0.0, 0.0, 0.0), (0, 1, 0))
    sc = RS.build_scene(desc)
    prm = R.params(3, 8, 17, brick_grid=True)
    ref = sc.render(cam, prm)
    for steps, visits, refill, wave, rounds, blocks in [(1, 2, 1, 32 * 28, 1, 1), (64, 7, 32, 3 * 32 * 28, 32, 64),
                                                        (8, 32, 8, 32 * 28, 5, 3)]:
        sc.set_tuning(R.tuning(steps, visits, refill, wave, rounds, blocks))
        assert sc.wave_samples(cam, prm) == wave // (32 * 28)
        assert np.array_equal(sc.render(cam, prm), ref), (steps, visits, refill, wave, rounds, blocks)
    t = sc.autotune(cam, prm)
    assert t.track_steps >= 1 and 1 <= t.media_rounds <= 32
    assert np.array_equal(sc.render(cam, prm), ref)
    sc.close()


@pytest.mark.parametrize("dda", [False, True])
def test_tracking_step_bound_ends_paths_with_timeout_status(lods, dda):
    """A tracking loop that reaches its step bound ends its path instead of
    spinning: the kernels return, count the paths they ended, and the
    synchronous render reports R2_ERR_DEVICE_TIMEOUT with that count (no hang,
    no trap).  The bound is lowered from 2^20 to 2 steps through the launch
    tuning; the context stays usable and the default bound renders the same
    frame as before."""
    desc = _desc(lods[0])
    cam = R.camera(32, 28, 50.0, (0.3, 0.6, 3.2), (0.0, 0.0, 0.0), (0, 1, 0))
    sc = RS.build_scene(desc)
    prm = R.params(2, 8, 5, brick_grid=dda)
    ref = sc.render(cam, prm)
    for rounds in (1, 32):  # the persistent tracker, and the queued rounds walked to the end
        sc.set_tuning(R.tuning(media_rounds=rounds, track_limit=2))
        with pytest.raises(N.R2Error) as e:
            sc.render(cam, prm)
        assert e.value.name == "R2_ERR_DEVICE_TIMEOUT"
        ended = int(str(e.value).split(":", 1)[1].split()[0])
        assert 0 < ended <= 2 * 32 * 28 * 2 * 8 * 3, str(e.value)
    sc.set_tuning(R.tuning())
    assert np.array_equal(sc.render(cam, prm), ref)
    with pytest.raises(N.R2Error):
        sc.set_tuning(R.tuning(track_limit=(1 << 20) + 1))
    sc.close()

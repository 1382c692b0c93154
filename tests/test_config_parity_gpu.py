"""GPU parity at the benchmark configurations' own sizes.

* Filter at scale (500k leaf quads = 1M triangles, 256 samples per voxel,
  20 iterations) on the full 256^3 and 512^3 grids, checked against the FP64
  oracle on z-slabs through the grid's centre: hit counts bit-exact, density
  and SGGX entries within 1e-4 relative, payload within one LSB; the FP16
  payload's error against FP64 stated and bounded by half a binary16 ulp.
* The small configuration's full frame (256x256, 16 spp, depth 8, white
  environment) and a 64-row band of the surface configuration's frame
  (1024x1024, 64 spp, depth 8, 327,680 triangles, lognormal environment)
  against the oracle with the same random streams.
* 3 sigma: the small configuration's scene rendered at 64x64 and 64 spp
  against a 4096-spp oracle estimate.
"""
import numpy as np
import pytest

import oracle_lib as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from renderer2_b200 import _native as N  # noqa: E402
from renderer2_b200 import filter as F  # noqa: E402
from renderer2_b200 import raytracer as R  # noqa: E402
from renderer2_b200 import render_scenes as RS  # noqa: E402
from renderer2_b200 import scenes  # noqa: E402
from test_filter_gpu import _compare  # noqa: E402

PIX_REL = 1e-4
PIX_FRAC = 0.999


@pytest.fixture(scope="module")
def foliage_1m():
    mesh = scenes.foliage(500_000, 20, 0.7, 4)
    mat = F.material(diffuse=(0.1, 0.6, 0.1), specular=(0.04, 0.04, 0.04), alpha=0.5, ior=1.5)
    return mesh, mat


@pytest.mark.parametrize("n,slices", [(256, 4), (512, 1)])
def test_filter_at_scale_slab_parity(foliage_1m, n, slices):
    mesh, mat = foliage_1m
    prm = F.params(samples_per_voxel=256, iterations=20)
    sc = F.FilterScene(mesh, mat)
    g = sc.grid(scenes.voxel_size_for(mesh, n))
    nx, ny, nz = g.num_voxels[:]
    nvox = nx * ny * nz
    out = torch.empty(nvox * 32, dtype=torch.uint8, device="cuda")
    wide = torch.empty(nvox * 20, dtype=torch.float32, device="cuda")
    f16 = torch.empty(nvox * 8, dtype=torch.float16, device="cuda")
    sc.run(g, prm, out.data_ptr(), wide.data_ptr(), f16.data_ptr())
    torch.cuda.synchronize()
    z0 = nz // 2 - slices // 2
    v0, v1 = z0 * nx * ny, (z0 + slices) * nx * ny
    gc = out.view(nvox, 32)[v0:v1].cpu().numpy()
    gw = wide.view(nvox, 20)[v0:v1].cpu().numpy().astype(np.float64)
    gh = f16.view(nvox, 8)[v0:v1].cpu().numpy().astype(np.float64)
    sc.close()
    del out, wide, f16
    ow, oc = O.filter_voxels(mesh, O.material_from(mat), N.identity43(), O.grid_from(g), O.params_from(prm), v0, v1)
    h = ow[:, 17] > 0
    assert h.sum() > 1000
    _compare(gw, gc, ow, oc)
    fin = h & np.isfinite(ow[:, 0])
    rel_d = np.abs(gh[fin, 0] - ow[fin, 0]) / np.abs(ow[fin, 0])
    scale = np.max(np.abs(ow[fin, 1:4]), axis=1, keepdims=True)
    rel_s = np.abs(gh[fin, 1:7] - ow[fin, 1:7]) / scale
    print(f"{n}^3 z-slab of {slices}: {int(h.sum())} voxels with hits; FP16 payload vs FP64: "
          f"density {rel_d.max():.3e}, S {rel_s.max():.3e} (max relative)")
    assert rel_d.max() <= 2.0 ** -11 * 1.01
    assert rel_s.max() <= 2.0 ** -11 * 1.01


def _agree(g, o):
    tol = PIX_REL * np.maximum(1.0, np.abs(o))
    return np.all(np.abs(g - o) <= tol, axis=1).mean()


def test_small_config_full_frame_matches_oracle():
    desc, cam = RS.icosphere_scene()  # 256x256, icosphere sub 4, GGX 0.3 albedo 0.8, white environment
    assert (cam.width, cam.height) == (256, 256)
    sc = RS.build_scene(desc)
    g = sc.render(cam, R.params(16, 8, 0)).reshape(-1, 3)
    sc.close()
    o = O.render(desc, cam, 16, 8, 0)
    frac = _agree(g, o)
    print(f"256x256 16 spp: {frac:.5f} of pixels within 1e-4")
    assert frac >= PIX_FRAC
    assert np.abs(g.mean(0) - o.mean(0)).max() < 1e-5


def test_surface_config_band_matches_oracle():
    desc, cam = RS.icosphere_grid_scene()  # 1024x1024, 64 meshes, lognormal environment
    assert (cam.width, cam.height) == (1024, 1024)
    prm = R.params(64, 8, 0)
    sc = RS.build_scene(desc)
    sc.autotune(cam, prm)  # the benchmark's launch tuning: the frame does not depend on it
    g = sc.render(cam, prm).reshape(-1, 3)
    sc.close()
    row0 = 480
    p0, p1 = row0 * 1024, (row0 + 64) * 1024
    o = O.render(desc, cam, 64, 8, 0, p0, p1)
    gb = g[p0:p1]
    rel = (np.abs(gb - o) / np.maximum(1.0, np.abs(o))).max(axis=1)
    q = {t: float((rel <= t).mean()) for t in (1e-4, 1e-3, 1e-2)}
    print(f"1024x1024 64 spp, rows {row0}..{row0 + 63}: fraction of pixels within 1e-4 / 1e-3 / 1e-2: "
          f"{q[1e-4]:.5f} / {q[1e-3]:.5f} / {q[1e-2]:.5f}, max {rel.max():.2e}")
    # The environment here is lognormal(0, 1.5): neighbouring texels differ by
    # orders of magnitude, so the last-bit differences of CUDA's and libm's
    # acos/atan2/sin in the environment lookup move a bilinear lookup by more
    # than 1e-4 of the pixel in a few tenths of a percent of the pixels.
    assert q[1e-4] >= 0.995
    assert q[1e-3] >= 0.9995
    band = np.abs(gb.mean(0) - o.mean(0)) / np.abs(o.mean(0))
    assert band.max() <= 1e-4


def test_three_sigma_small_config_64x64():
    """Per pixel and channel, |GPU(64 spp) - oracle(4096 spp)| <= 3 sigma with
    sigma^2 = var/64 + var/4096 from the oracle's sample variance.  For
    Gaussian errors 99.73 % of the 12,288 values fall inside; the bound allows
    four binomial standard deviations below that (99.54 %)."""
    desc, _ = RS.icosphere_scene()
    cam = R.camera(64, 64, 45.0, (0, 0, 3), (0, 0, 0), (0, 1, 0))
    sc = RS.build_scene(desc)
    g = sc.render(cam, R.params(64, 8, 101)).reshape(-1, 3)
    sc.close()
    o, var = O.render(desc, cam, 4096, 8, 7, want_var=True)
    sigma = np.sqrt(var / 64 + var / 4096)
    z = np.abs(g - o) / np.maximum(sigma, 1e-12)
    z[(sigma == 0) & (g == o)] = 0.0
    within = (z <= 3.0).mean()
    n = z.size
    bound = 0.9973 - 4.0 * np.sqrt(0.0027 * 0.9973 / n)
    print(f"64x64: {within:.5f} of {n} pixel channels within 3 sigma (bound {bound:.5f})")
    assert within >= bound

"""Drop-in boundary on the GPU: a config.json run gives the frames and files
of the lower-level entry points it is built from, the output stage agrees with
the oracle's, and the `r2 <config.json>` tool writes the same image."""
import os
import struct
import subprocess
import zlib

import numpy as np
import pytest

import oracle_lib as O
from test_pipeline_cpu import _pipeline_files

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from renderer2_b200 import filter as F  # noqa: E402
from renderer2_b200 import pipeline as P  # noqa: E402
from renderer2_b200 import raytracer as R  # noqa: E402
from renderer2_b200 import render_scenes as RS  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _hand_scene(tmp_path, mesh):
    """The scene of _pipeline_files built through r2_scene_* calls."""
    env = P.read_hdr(tmp_path / "env.hdr")
    mat = P.obj_info(tmp_path / "assets", "sphere.obj")[3]  # the material the importer derived from the MTL
    return {"meshes": [(mesh, mat, RS.translate43(0, 0, 0))],
            "shapes": [(R.CIRCLE, (0, -1.2, 0), 3.4e38, (0, 1, 0),
                        F.material(diffuse=(0.5, 0.5, 0.5), specular=(0.2, 0.2, 0.2), alpha=0.5, ior=1.3,
                                   diffuse_roughness=0.3)),
                       (R.SPHERE, (1.5, 0, 0), 0.4, (0, 1, 0),
                        F.material(diffuse=(0.2, 0.7, 0.2), specular=(1, 1, 1), alpha=0.2, ior=1.5))],
            "env": env}


def test_config_render_equals_scene_render(tmp_path):
    mesh = _pipeline_files(tmp_path)
    cfg = P.Config(tmp_path / "config.json")
    lin, by = cfg.render(spp=4, max_depth=8, seed=5)
    desc = _hand_scene(tmp_path, mesh)
    sc = RS.build_scene(desc)
    cam = R.camera(48, 32, 50.0, (0.3, 0.5, 3.5), (0, 0, 0), (0, 1, 0))
    ref = sc.render(cam, R.params(4, 8, 5, brick_grid=True))
    sc.close()
    assert np.array_equal(lin, ref)
    # the bytes are the output stage of that frame
    _, tb = P.tonemap(lin, 2.0)
    assert np.array_equal(by, tb)
    # a second render reuses the resident scene and is deterministic
    lin2, _ = cfg.render(spp=4, max_depth=8, seed=5)
    assert np.array_equal(lin, lin2)
    cfg.close()


def test_tonemap_matches_oracle():
    rng = np.random.default_rng(3)
    lin = rng.lognormal(-1.0, 1.5, (45, 70, 3)).astype(np.float32)
    lin[3, 4] = 0.0
    for gamma in (2.0, 2.2, 1.0):
        g_out, g_by = P.tonemap(lin, gamma)
        o_out, o_by = O.tonemap(lin, gamma)
        assert np.allclose(g_out, o_out, rtol=2e-6, atol=1e-7)
        d = np.abs(g_by.astype(int) - o_by.astype(int))
        assert d.max() <= 1 and (d == 0).mean() > 0.999


def test_config_filter_run_equals_direct_filter(tmp_path):
    mesh = _pipeline_files(tmp_path, mesh_mask=("FILTER",), filter_active=True)
    cfg = P.Config(tmp_path / "config.json")
    st = cfg.filter_run(tmp_path / "filtering")
    assert st[0] == 2 and st[2] > 0
    mat = P.obj_info(tmp_path / "assets", "sphere.obj")[3]
    prm = F.params(samples_per_voxel=16, iterations=5, min_voxel_size=float(np.float32(0.12)), lods=2)
    paths, st2 = F.run_filtering(mesh, mat, prm, tmp_path / "direct", "sphere")
    assert list(st[:3]) == list(st2[:3])  # LODs, voxels, active voxels (st[3] is a time)
    for p in paths:
        q = p.replace(str(tmp_path / "direct"), str(tmp_path / "filtering"))
        for ext in (".nvdb", ".brickgrid"):
            assert open(p + ext, "rb").read() == open(q + ext, "rb").read()
    cfg.close()


def _read_png(path):
    raw = open(path, "rb").read()
    pos, idat, dims = 8, b"", None
    while pos < len(raw):
        n = struct.unpack(">I", raw[pos:pos + 4])[0]
        typ, body = raw[pos + 4:pos + 8], raw[pos + 8:pos + 8 + n]
        if typ == b"IHDR":
            dims = struct.unpack(">II", body[:8])
        elif typ == b"IDAT":
            idat += body
        pos += 12 + n
    w, h = dims
    return np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + 3 * w)[:, 1:].reshape(h, w, 3)


def test_cli_writes_the_frame(tmp_path):
    _pipeline_files(tmp_path)
    exe = os.path.join(ROOT, "renderer2_b200", "_lib", "r2")
    r = subprocess.run([exe, str(tmp_path / "config.json"), "--spp", "2", "--seed", "9"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    img = _read_png(tmp_path / "output.png")
    cfg = P.Config(tmp_path / "config.json")
    lin, by = cfg.render(spp=2, max_depth=50, seed=9)
    cfg.close()
    assert np.array_equal(img, by[::-1])  # written top row first
    hdr = P.read_hdr(tmp_path / "output.hdr")
    m = lin[::-1].max(axis=2, keepdims=True)
    assert np.all(np.abs(hdr - lin[::-1]) <= m / 128.0 + 1e-30)
    Image = pytest.importorskip("PIL.Image")
    with Image.open(tmp_path / "output.jpg") as im:  # quality 100, as the reference writes it
        jpg = np.asarray(im.convert("RGB")).astype(np.float64)
    assert jpg.shape == img.shape and np.abs(jpg - img).mean() < 3.0

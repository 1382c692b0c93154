"""Textured materials (OBJ map_Kd / map_Ks / map_Bump / map_d) against the CPU
oracle: albedo and glossy colours from texture maps (glossy from the albedo's
luma when the specular colour is dark), tangent-space normal maps, and
opacity cut-outs (from map_d, or from the albedo's alpha channel) that every
ray ignores, camera, extension and shadow rays alike.  The same scene through
config.json + OBJ/MTL + PNG files renders the same frame."""
import math
import os

import numpy as np
import pytest

import oracle_lib as O

torch = pytest.importorskip("torch")
Image = pytest.importorskip("PIL.Image")
pytestmark = pytest.mark.gpu

from renderer2_b200 import _native as N  # noqa: E402
from renderer2_b200 import filter as F  # noqa: E402
from renderer2_b200 import raytracer as R  # noqa: E402
from renderer2_b200 import render_scenes as RS  # noqa: E402
from renderer2_b200 import scenes  # noqa: E402

PIX_REL = 1e-4
PIX_FRAC = 0.995  # libm vs CUDA acos/atan2/sin in the environment lookup


def _quad(c, ex, ey, nrm):
    c, ex, ey = (np.asarray(v, np.float32) for v in (c, ex, ey))
    pos = np.stack([c - ex - ey, c + ex - ey, c + ex + ey, c - ex + ey]).astype(np.float32)
    idx = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    nr = np.tile(np.asarray(nrm, np.float32), (4, 1))
    uv = np.array([[0, 1], [2, 1], [2, -1], [0, -1]], np.float32)  # repeats: wrap addressing
    return F.Mesh(pos, idx, nr), uv


def _sphere_uv(mesh):
    p = mesh.positions / np.linalg.norm(mesh.positions, axis=1, keepdims=True)
    u = np.arctan2(p[:, 2], p[:, 0]) / (2 * math.pi) + 0.5
    v = np.arccos(np.clip(p[:, 1], -1, 1)) / math.pi
    return np.stack([u * 3, v * 2], 1).astype(np.float32)


def _maps(d):
    rng = np.random.default_rng(5)
    yy, xx = np.mgrid[0:48, 0:64]
    checker = ((xx // 8 + yy // 8) % 2).astype(np.float32)
    alb = np.stack([0.2 + 0.7 * checker, 0.3 + 0.4 * (xx / 63), 0.8 - 0.6 * checker], -1)
    Image.fromarray((alb * 255).astype(np.uint8)).save(d / "albedo.png")
    nx, ny = 0.5 * np.sin(xx / 4.0), 0.5 * np.cos(yy / 5.0)
    n = np.stack([nx, ny, np.ones_like(nx)], -1)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    Image.fromarray(((n * 0.5 + 0.5) * 255).astype(np.uint8)).save(d / "normal.png")
    spec = rng.integers(40, 255, (16, 16, 3), dtype=np.uint8)
    Image.fromarray(spec).save(d / "spec.png")
    stripes = np.where((xx // 6) % 3 == 0, 0, 255).astype(np.uint8)
    Image.fromarray(stripes).save(d / "opacity.png")  # map_d: the red channel
    rgba = np.concatenate([(alb * 255).astype(np.uint8),
                           np.where((xx - 32) ** 2 + (yy - 24) ** 2 < 15 ** 2, 0, 255).astype(np.uint8)[..., None]], -1)
    Image.fromarray(rgba, "RGBA").save(d / "albedo_rgba.png")  # alpha channel: a round hole
    return {k: str(d / f) for k, f in [("albedo", "albedo.png"), ("normal", "normal.png"), ("spec", "spec.png"),
                                        ("opacity", "opacity.png"), ("albedo_rgba", "albedo_rgba.png")]}


def _desc(maps):
    ground, guv = _quad((0, -1, 0), (3, 0, 0), (0, 0, 3), (0, 1, 0))
    wall, wuv = _quad((0.2, 0.1, -0.6), (0.9, 0, 0), (0, 0.9, 0), (0, 0, 1))
    ico = scenes.icosphere(3, 0.0, 2)
    dark = F.material(diffuse=(0.5, 0.5, 0.5), specular=(0.01, 0.5, 0.5), alpha=0.35, ior=1.5)  # glossy from luma
    bright = F.material(diffuse=(0.5, 0.5, 0.5), specular=(0.9, 0.9, 0.9), alpha=0.2, ior=1.4)
    m_ico = RS.translate43(-0.9, -0.3, 0.3)
    m_ico[0] = m_ico[4] = m_ico[8] = 0.6
    return {
        "meshes": [
            (ground, dark, RS.translate43(0, 0, 0), {"uv": guv, "albedo": maps["albedo"], "normal": maps["normal"]}),
            (wall, bright, RS.translate43(0, 0, 0), {"uv": wuv, "albedo": maps["albedo_rgba"]}),
            (ico, bright, m_ico, {"uv": _sphere_uv(ico), "albedo": maps["albedo"], "specular": maps["spec"],
                                  "alpha": maps["opacity"], "normal": maps["normal"]}),
        ],
        "shapes": [],
        "env": RS.lognormal_env(64, 32, 1.0, 4),
    }


def _agree(g, o):
    tol = PIX_REL * np.maximum(1.0, np.abs(o))
    return np.all(np.abs(g - o) <= tol, axis=1).mean()


def test_textured_frame_matches_oracle(tmp_path):
    desc = _desc(_maps(tmp_path))
    cam = R.camera(64, 48, 50.0, (0.4, 0.8, 3.2), (0.0, -0.3, 0.0), (0, 1, 0))
    sc = RS.build_scene(desc)
    g = sc.render(cam, R.params(4, 6, 11)).reshape(-1, 3)
    sc.close()
    o = O.render(desc, cam, 4, 6, 11)
    assert np.isfinite(g).all()
    frac = _agree(g, o)
    assert frac >= PIX_FRAC, f"only {frac:.4f} of pixels agree"


def test_textures_change_the_frame_where_they_should(tmp_path):
    """Maps are used: the frame differs from the untextured one, and the
    cut-outs let the environment through where the opaque version is lit."""
    maps = _maps(tmp_path)
    desc = _desc(maps)
    plain = {"meshes": [m[:3] for m in desc["meshes"]], "shapes": [], "env": desc["env"]}
    cam = R.camera(48, 48, 50.0, (0.4, 0.8, 3.2), (0.0, -0.3, 0.0), (0, 1, 0))
    prm = R.params(2, 4, 3)
    a, b = RS.build_scene(desc), RS.build_scene(plain)
    ga, gb = a.render(cam, prm), b.render(cam, prm)
    a.close()
    b.close()
    assert np.abs(ga - gb).mean() > 1e-3


def test_textured_mesh_arguments_checked(tmp_path):
    maps = _maps(tmp_path)
    mesh, uv = _quad((0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1))
    sc = R.Scene()
    with pytest.raises(N.R2Error):  # not a PNG file
        (tmp_path / "t.jpg").write_bytes(b"\xff\xd8\xff")
        sc.add_mesh_textured(mesh, F.material(), uv, albedo=str(tmp_path / "t.jpg"))
    with pytest.raises(N.R2Error):
        sc.add_mesh_textured(mesh, F.material(), uv, albedo=str(tmp_path / "missing.png"))
    sc.add_mesh_textured(mesh, F.material(), uv, albedo=maps["albedo"])
    sc.close()


def test_obj_with_texture_maps_renders_the_same_frame(tmp_path):
    """config.json + OBJ (vt) + MTL (map_Kd, map_Bump, map_d) + PNG files give
    the frame of the same scene built through the array entry points."""
    from renderer2_b200 import pipeline as P
    maps = _maps(tmp_path)
    ground, guv = _quad((0, -1, 0), (3, 0, 0), (0, 0, 3), (0, 1, 0))
    lines = ["mtllib m.mtl", "usemtl tex"]
    lines += [f"v {x} {y} {z}" for x, y, z in ground.positions]
    lines += [f"vt {u} {v}" for u, v in guv]
    lines += [f"vn {x} {y} {z}" for x, y, z in ground.normals]
    lines += [f"f {a + 1}/{a + 1}/{a + 1} {b + 1}/{b + 1}/{b + 1} {c + 1}/{c + 1}/{c + 1}" for a, b, c in ground.indices]
    (tmp_path / "g.obj").write_text("\n".join(lines) + "\n")
    (tmp_path / "m.mtl").write_text("newmtl tex\nKd 0.5 0.5 0.5\nKs 0.01 0.5 0.5\nNs 20\nNi 1.5\n"
                                    "map_Kd albedo.png\nmap_Bump -bm 1.0 normal.png\nmap_d opacity.png\n")
    from test_pipeline_cpu import _write_env
    _write_env(tmp_path / "env.hdr", 16, 8, 2)
    objs = [{"Type": "Mesh", "Directory": str(tmp_path), "Filename": "g.obj", "Pos": [0, 0, 0],
             "Orientation": [0, 1, 0], "Scaling": [1, 1, 1], "Mask": ["RENDER"]}]
    P.write_config(tmp_path / "config.json", objs, str(tmp_path / "env.hdr"), str(tmp_path / "scene.json"),
                   40, 30, 2, fov=50.0, cam_pos=(0.3, 1.5, 3.5))
    cfg = P.Config(tmp_path / "config.json")
    lin, _ = cfg.render(spp=2, max_depth=8, seed=4)
    cfg.close()
    mat = P.obj_info(tmp_path, "g.obj")[3]
    desc = {"meshes": [(ground, mat, RS.translate43(0, 0, 0),
                        {"uv": guv, "albedo": maps["albedo"], "normal": maps["normal"], "alpha": maps["opacity"]})],
            "shapes": [], "env": P.read_hdr(tmp_path / "env.hdr")}
    sc = RS.build_scene(desc)
    cam = R.camera(40, 30, 50.0, (0.3, 1.5, 3.5), (0, 0, 0), (0, 1, 0))
    g = sc.render(cam, R.params(2, 8, 4, brick_grid=True))
    sc.close()
    assert np.abs(g).sum() > 0
    assert np.array_equal(g, lin)


def test_textured_filter_matches_oracle(tmp_path):
    """The filter over textured leaves: diffuse(tc), glossy(tc) from the
    albedo's luma, the normal-mapped normal, and the opacity map's holes,
    against the FP64 oracle on the same texels."""
    from test_filter_gpu import _compare, _gpu_filter_scene
    maps = _maps(tmp_path)
    leaves = scenes.foliage(3000, 6, 0.7, 8)
    # each leaf quad (4 vertices) spans the texture once
    q = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    uv = np.tile(q, (leaves.nverts // 4 + 1, 1))[:leaves.nverts]
    tex = {"uv": uv, "albedo": maps["albedo"], "normal": maps["normal"], "alpha": maps["opacity"]}
    mat = F.material(diffuse=(0.1, 0.6, 0.1), specular=(0.01, 0.3, 0.3), alpha=0.5, ior=1.5)
    prm = F.params(samples_per_voxel=64, iterations=10)
    vs = scenes.voxel_size_for(leaves, 16)
    sc = F.FilterScene(leaves, mat, None, tex)
    g, gc, gw = _gpu_filter_scene(sc, prm, vs)
    sc.close()
    ow, oc = O.filter_voxels(leaves, O.material_from(mat), N.identity43(), O.grid_from(g), O.params_from(prm),
                             tex=tex)
    _compare(gw, gc, ow, oc)
    # the holes matter: fewer hits than the same leaves without the opacity map
    sc2 = F.FilterScene(leaves, mat, None, {k: v for k, v in tex.items() if k != "alpha"})
    _, _, gw2 = _gpu_filter_scene(sc2, prm, vs)
    sc2.close()
    assert gw[:, 17].sum() < gw2[:, 17].sum()


def test_textured_instances_match_oracle(tmp_path):
    """A textured, alpha-mapped, normal-mapped mesh placed twice (one asset,
    two instances, rotated and non-uniformly scaled) beside textured
    world-space meshes: the two-level scene against the oracle's."""
    desc = _desc(_maps(tmp_path))
    ico = desc["meshes"][2]
    desc["meshes"].append((ico[0], ico[1], RS.trs43((0.9, -0.35, 0.2), (0.3, 1.0, 0.2, 0.7), (0.5, 0.65, 0.55)),
                           ico[3]))
    assert RS.mesh_groups(desc) == [[2, 3]]
    cam = R.camera(64, 48, 50.0, (0.4, 0.8, 3.2), (0.0, -0.3, 0.0), (0, 1, 0))
    sc = RS.build_scene(desc)
    g = sc.render(cam, R.params(4, 6, 12)).reshape(-1, 3)
    sc.close()
    o = O.render(desc, cam, 4, 6, 12)
    assert np.isfinite(g).all()
    frac = _agree(g, o)
    assert frac >= PIX_FRAC, f"only {frac:.4f} of pixels agree"

"""Drop-in boundary on CPU: config.json / scenedescription.json loading, the
OBJ/MTL importer, Radiance .hdr reading (flat and run-length scanlines) and
writing, and the PNG writer.  None of these calls needs a GPU."""
import json
import math
import struct
import zlib

import numpy as np
import pytest

from renderer2_b200 import _native as N
from renderer2_b200 import pipeline as P
from renderer2_b200 import scenes


def _write_env(path, w=8, h=4, seed=0):
    rgb = np.random.default_rng(seed).lognormal(0.0, 1.0, (h, w, 3)).astype(np.float32)
    P.write_hdr(path, rgb)
    return rgb


def test_obj_import_materials_and_counts(tmp_path):
    a = scenes.icosphere(1, 0.0, 1)
    b = scenes.icosphere(2, 0.1, 2)
    P.write_obj(tmp_path, "two", [(a, (0.8, 0.5, 0.2), (1, 1, 1), 2.0 / 0.3 ** 2 - 2.0, 1.0),
                                  (b, (0.1, 0.2, 0.3), (0.5, 0.5, 0.5), 50.0, 1.33)])
    ns, nv, nt, m = P.obj_info(tmp_path, "two.obj")
    assert ns == 2
    assert nt == a.ntris + b.ntris
    assert nv == a.nverts + b.nverts  # shared (position, normal) corners are joined
    # CMaterial(aiMaterial*): alpha = (2/(Ns+2))^0.5, eta_t = 1.5 when Ni == 1, Oren-Nayar roughness 0
    assert abs(m.alpha_x - 0.3) < 1e-6 and m.alpha_x == m.alpha_y
    assert m.eta_i == 1.0 and m.eta_t == 1.5 and m.diffuse_roughness == 0.0
    assert np.allclose(m.diffuse[:], [0.8, 0.5, 0.2]) and np.allclose(m.specular[:], [1, 1, 1])


def test_obj_flat_normals_quads_and_negative_indices(tmp_path):
    (tmp_path / "q.obj").write_text(
        "# quad without normals, negative indices\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf -4 -3 -2 -1\n"
        "v 0 0 1\nv 1 0 1\nv 0 1 1\nf 5/1 6/2 7/3\n")
    ns, nv, nt, m = P.obj_info(tmp_path, "q.obj")
    assert (ns, nt) == (1, 3)
    assert nv == 9  # generated flat normals: one vertex per face corner
    # no material: the importer's default (Kd 0.6, Ks 0, Ns 0 -> alpha 1, Ni 1 -> 1.5)
    assert np.allclose(m.diffuse[:], 0.6) and m.alpha_x == 1.0 and m.eta_t == 1.5


def test_obj_rejects_bad_index(tmp_path):
    (tmp_path / "bad.obj").write_text("v 0 0 0\nv 1 0 0\nf 1 2 3\n")
    with pytest.raises(N.R2Error) as e:
        P.obj_info(tmp_path, "bad.obj")
    assert e.value.status == 3


def test_hdr_round_trip(tmp_path):
    rgb = _write_env(tmp_path / "e.hdr", 13, 7, 3)
    back = P.read_hdr(tmp_path / "e.hdr")
    assert back.shape == rgb.shape
    # RGBE keeps 8 mantissa bits of the largest channel
    m = rgb.max(axis=2, keepdims=True)
    assert np.all(np.abs(back - rgb) <= m / 128.0 + 1e-30)


def _rle_scanline(vals):
    out = bytearray()
    i = 0
    while i < len(vals):
        run = 1
        while i + run < len(vals) and vals[i + run] == vals[i] and run < 127:
            run += 1
        if run >= 3:
            out += bytes([128 + run, vals[i]])
            i += run
        else:
            j = i
            lit = []
            while j < len(vals) and len(lit) < 128 and not (j + 2 < len(vals) and vals[j] == vals[j + 1] == vals[j + 2]):
                lit.append(vals[j])
                j += 1
            out += bytes([len(lit)]) + bytes(lit)
            i = j
    return bytes(out)


def test_hdr_run_length_scanlines(tmp_path):
    w, h = 40, 3
    rng = np.random.default_rng(7)
    px = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    px[:, 10:30, :] = px[:, 10:11, :]  # long runs
    px[1, :, 3] = 0                    # exponent 0 -> black
    data = bytearray(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y %d +X %d\n" % (h, w))
    for y in range(h):
        data += bytes([2, 2, w >> 8, w & 255])
        for c in range(4):
            data += _rle_scanline(list(px[y, :, c]))
    (tmp_path / "r.hdr").write_bytes(bytes(data))
    back = P.read_hdr(tmp_path / "r.hdr")
    e = px[..., 3].astype(np.int32)
    f = np.where(e == 0, 0.0, np.ldexp(1.0, e - 136)).astype(np.float32)
    exp = px[..., :3].astype(np.float32) * f[..., None]
    assert np.array_equal(back, exp)


def test_png_writer_decodes(tmp_path):
    rgb = np.random.default_rng(1).integers(0, 256, (37, 300, 3), dtype=np.uint8)  # > 64 KiB of rows
    P.write_png(tmp_path / "o.png", rgb, flip_vertical=True)
    raw = (tmp_path / "o.png").read_bytes()
    assert raw[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, dims = 8, b"", None
    while pos < len(raw):
        n = struct.unpack(">I", raw[pos:pos + 4])[0]
        typ = raw[pos + 4:pos + 8]
        body = raw[pos + 8:pos + 8 + n]
        assert struct.unpack(">I", raw[pos + 8 + n:pos + 12 + n])[0] == zlib.crc32(typ + body)
        if typ == b"IHDR":
            dims = struct.unpack(">IIBBBBB", body)
        elif typ == b"IDAT":
            idat += body
        pos += 12 + n
    assert dims == (300, 37, 8, 2, 0, 0, 0)
    rows = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(37, 1 + 900)
    assert np.all(rows[:, 0] == 0)
    assert np.array_equal(rows[:, 1:].reshape(37, 300, 3), rgb[::-1])


@pytest.mark.parametrize("w,h", [(64, 48), (37, 29)])
def test_jpg_writer_decodes(tmp_path, w, h):
    """output.jpg as the reference writes it (quality 100, flipped): a baseline
    JPEG that an independent decoder (Pillow) reads back to within JPEG's
    rounding of the original, on a smooth image and on noise, also when the
    size is not a multiple of the 8x8 block."""
    Image = pytest.importorskip("PIL.Image")
    yy, xx = np.mgrid[0:h, 0:w]
    smooth = np.stack([xx * 255 // max(w - 1, 1), yy * 255 // max(h - 1, 1), (xx + yy) % 256], -1).astype(np.uint8)
    noise = np.random.default_rng(3).integers(0, 256, (h, w, 3), dtype=np.uint8)
    for img, tol in ((smooth, 3.0), (noise, 6.0)):
        P.write_jpg(tmp_path / "o.jpg", img, flip_vertical=True, quality=100)
        with Image.open(tmp_path / "o.jpg") as im:
            assert im.format == "JPEG" and im.size == (w, h) and im.mode == "RGB"
            back = np.asarray(im.convert("RGB")).astype(np.float64)
        err = np.abs(back - img[::-1].astype(np.float64))
        assert err.mean() < tol / 3 and err.max() <= 8 * tol, (err.mean(), err.max())
    # lower quality: coarser but still close on the smooth image
    P.write_jpg(tmp_path / "q50.jpg", smooth, quality=50)
    with Image.open(tmp_path / "q50.jpg") as im:
        back = np.asarray(im.convert("RGB")).astype(np.float64)
    assert np.abs(back - smooth).mean() < 6.0
    with pytest.raises(N.R2Error):
        P.write_jpg(tmp_path / "bad.jpg", smooth, quality=0)


@pytest.mark.parametrize("mode,kw", [("RGB", {}), ("RGBA", {}), ("L", {}), ("LA", {}), ("P", {}), ("1", {}),
                                     ("RGB", {"compress_level": 0}), ("RGBA", {"compress_level": 1}),
                                     ("I;16", {}), ("P4", {"bits": 4})])
def test_png_reader_matches_pillow(tmp_path, mode, kw):
    """Texture maps: every PNG colour type and filter Pillow writes decodes to
    the same RGBA bytes Pillow reads (16-bit samples: the high byte)."""
    Image = pytest.importorskip("PIL.Image")
    rng = np.random.default_rng(7)
    h, w = 37, 53
    base = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    base[:, :20] = np.linspace(0, 255, 20, dtype=np.uint8)[None, :, None]  # smooth part: the filters matter
    if mode == "P4":
        im = Image.fromarray(base[..., :3]).quantize(16)
        mode = "P"
    elif mode == "I;16":
        im = Image.fromarray((base[..., 0].astype(np.uint16) * 257 + 3).astype(np.uint16))
    elif mode == "1":
        im = Image.fromarray(base[..., 0] > 127)
    elif mode == "P":
        im = Image.fromarray(base[..., :3]).quantize(200)
    else:
        im = Image.fromarray(base[..., :len(mode)] if len(mode) > 1 else base[..., 0], mode)
    im.save(tmp_path / "t.png", **{k: v for k, v in kw.items() if k != "bits"}, **({"bits": 4} if "bits" in kw else {}))
    got, ch = P.read_png(tmp_path / "t.png")
    with Image.open(tmp_path / "t.png") as ref:
        if ref.mode == "I;16" or ref.mode == "I":
            exp = np.asarray(ref).astype(np.uint32) >> 8
            exp = np.stack([exp, exp, exp, np.full_like(exp, 255)], -1).astype(np.uint8)
        else:
            exp = np.asarray(ref.convert("RGBA"))
    assert got.shape == (h, w, 4)
    assert np.array_equal(got, exp)
    assert ch == {"RGB": 3, "RGBA": 4, "L": 1, "LA": 2, "P": 3, "1": 1, "I;16": 1}[mode]


def test_png_reader_rejects_bad_files(tmp_path):
    (tmp_path / "x.png").write_bytes(b"not a png")
    with pytest.raises(N.R2Error):
        P.read_png(tmp_path / "x.png")
    with pytest.raises(N.R2Error):
        P.read_png(tmp_path / "missing.png")


def _pipeline_files(tmp_path, mesh_mask=("RENDER",), filter_active=False):
    mesh = scenes.icosphere(2, 0.05, 1)
    P.write_obj(tmp_path / "assets", "sphere", [(mesh, (0.8, 0.8, 0.8), (1, 1, 1), 2.0 / 0.3 ** 2 - 2.0, 1.5)])
    _write_env(tmp_path / "env.hdr")
    objs = [
        {"Type": "Mesh", "Directory": str(tmp_path / "assets"), "Filename": "sphere.obj", "Pos": [0, 0, 0],
         "Orientation": [0, 1, 0], "Scaling": [1, 1, 1], "Mask": list(mesh_mask)},
        {"Type": "Circle", "Pos": [0, -1.2, 0], "Radius": 3.4e38, "Normal": [0, 1, 0],
         "DiffuseReflection": [0.5, 0.5, 0.5], "DiffuseRoughness": 0.3, "SpecularReflection": [0.2, 0.2, 0.2],
         "AlphaX": 0.5, "AlphaY": 0.5, "EtaI": 1.0, "EtaT": 1.3},
        {"Type": "Sphere", "Pos": [1.5, 0, 0], "Radius": 0.4, "Normal": [0, 1, 0],
         "DiffuseReflection": [0.2, 0.7, 0.2], "DiffuseRoughness": 0.0, "SpecularReflection": [1, 1, 1],
         "AlphaX": 0.2, "AlphaY": 0.2, "EtaI": 1.0, "EtaT": 1.5, "Mask": ["RENDER"]},
        {"Type": "Unknown"},
    ]
    P.write_config(tmp_path / "config.json", objs, str(tmp_path / "env.hdr"), str(tmp_path / "scene.json"),
                   48, 32, 4, fov=50.0, cam_pos=(0.3, 0.5, 3.5), filter_active=filter_active,
                   min_voxel_size=0.12, lods=2, samples_per_voxel=16, iterations=5)
    return mesh


def test_config_load_and_info(tmp_path):
    mesh = _pipeline_files(tmp_path)
    cfg = P.Config(tmp_path / "config.json")
    i = cfg.info()
    assert (i.frame_width, i.frame_height, i.channels, i.samples) == (48, 32, 3, 4)
    assert i.gamma == 2.0 and i.use_brick_grid == 1 and i.filter_active == 0
    assert (i.env_width, i.env_height) == (8, 4)
    assert (i.n_meshes, i.n_shapes, i.n_media) == (1, 2, 0)
    assert i.n_triangles == mesh.ntris
    assert i.filter.lods == 2 and i.filter.samples_per_voxel == 16 and i.filter.estimation_iterations == 5
    assert abs(i.filter.min_voxel_size - 0.12) < 1e-7 and i.filter.clip_rays == 1
    assert i.camera.width == 48 and math.isclose(i.camera.fov_deg, 50.0) and list(i.camera.pos) == [
        np.float32(0.3), np.float32(0.5), np.float32(3.5)]
    cfg.close()


@pytest.mark.parametrize("drop", [("General", "Gamma"), ("Filtering", "ClipRays"), ("Camera", "Up"),
                                  ("Scene", "Envmap")])
def test_config_missing_key_rejected(tmp_path, drop):
    _pipeline_files(tmp_path)
    text = (tmp_path / "config.json").read_text()
    cfg = json.loads(text[text.index("{"):])
    del cfg[drop[0]][drop[1]]
    (tmp_path / "config.json").write_text(json.dumps(cfg))
    with pytest.raises(N.R2Error) as e:
        P.Config(tmp_path / "config.json")
    assert e.value.status == 2 and drop[1] in str(e.value)


def test_scene_object_missing_field_rejected(tmp_path):
    _pipeline_files(tmp_path)
    objs = json.loads((tmp_path / "scene.json").read_text().split("\n", 1)[1])
    del objs[1]["AlphaY"]
    (tmp_path / "scene.json").write_text(json.dumps(objs))
    with pytest.raises(N.R2Error) as e:
        P.Config(tmp_path / "config.json")
    assert e.value.status == 2 and "AlphaY" in str(e.value)

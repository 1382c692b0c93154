"""GPU parity of the SGGX filter against the CPU oracle.

Bar (from the build's contract): BVH leaf assignment, voxel indexing and the
active topology are bit-exact; SGGX coefficients and densities within 1e-4
relative of the FP64 oracle; the quantised payload within one LSB.
"""
import numpy as np
import pytest

import oracle_lib as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from renderer2_b200 import _native as N  # noqa: E402
from renderer2_b200 import filter as F  # noqa: E402
from renderer2_b200 import scenes  # noqa: E402

REL_TOL = 1e-4  # SGGX / density tolerance against FP64
I43 = N.identity43()


def _world(mesh, m2w):
    m = np.asarray(m2w, np.float32).reshape(4, 3)
    p = mesh.positions.astype(np.float32)
    # glm mat4x3 * vec4(p, 1), same left-to-right float32 accumulation as the library
    out = np.empty_like(p)
    for r in range(3):
        acc = m[0, r] * p[:, 0]
        acc = (acc + m[1, r] * p[:, 1]).astype(np.float32)
        acc = (acc + m[2, r] * p[:, 2]).astype(np.float32)
        acc = (acc + m[3, r] * np.float32(1.0)).astype(np.float32)
        out[:, r] = acc
    return out


def _gpu_filter(mesh, mat, prm, vs, m2w=I43, fp16=False):
    sc = F.FilterScene(mesh, mat, m2w)
    g = sc.grid(vs)
    nvox = int(np.prod(np.array(g.num_voxels[:], np.int64)))
    out = torch.empty(nvox * 32, dtype=torch.uint8, device="cuda")
    wide = torch.empty(nvox * 20, dtype=torch.float32, device="cuda")
    f16 = torch.empty(nvox * 8, dtype=torch.float16, device="cuda") if fp16 else None
    st = np.zeros(3)
    sc.run(g, prm, out.data_ptr(), wide.data_ptr(), f16.data_ptr() if fp16 else 0, stats=st)
    torch.cuda.synchronize()
    res = (g, out.cpu().numpy().reshape(nvox, 32), wide.cpu().numpy().reshape(nvox, 20).astype(np.float64), st)
    if fp16:
        res = res + (f16.cpu().numpy().reshape(nvox, 8).astype(np.float64),)
    sc.close()
    return res


def _gpu_filter_scene(sc, prm, vs):
    """(grid, compact, wide) of one LOD of an existing filter scene."""
    g = sc.grid(vs)
    nvox = int(np.prod(np.array(g.num_voxels[:], np.int64)))
    out = torch.empty(nvox * 32, dtype=torch.uint8, device="cuda")
    wide = torch.empty(nvox * 20, dtype=torch.float32, device="cuda")
    sc.run(g, prm, out.data_ptr(), wide.data_ptr())
    torch.cuda.synchronize()
    return g, out.cpu().numpy().reshape(nvox, 32), wide.cpu().numpy().reshape(nvox, 20).astype(np.float64)


def _compare(gw, gc, ow, oc):
    # topology and hit counts: bit-exact
    assert np.array_equal(gw[:, 17], ow[:, 17]), "hit counts differ"
    assert np.array_equal(gw[:, 0] > 0, ow[:, 0] > 0), "active topology differs"
    h = ow[:, 17] > 0
    # density: relative to FP64 (both infinite when every ray hit)
    gd, od = gw[h, 0], ow[h, 0]
    fin = np.isfinite(od)
    assert np.array_equal(np.isfinite(gd), fin)
    rel = np.abs(gd[fin] - od[fin]) / np.abs(od[fin])
    assert rel.max(initial=0) <= REL_TOL, f"density rel err {rel.max()}"
    # SGGX entries: relative to the matrix scale max(S_ii)
    scale = np.max(np.abs(ow[h, 1:4]), axis=1, keepdims=True)
    serr = np.abs(gw[h, 1:7] - ow[h, 1:7]) / scale
    assert serr.max(initial=0) <= REL_TOL, f"S rel err {serr.max()}"
    # other means
    assert np.abs(gw[h, 7:13] - ow[h, 7:13]).max(initial=0) < 1e-5
    assert np.abs(gw[h, 13:16] - ow[h, 13:16]).max(initial=0) < 1e-5
    assert np.abs(gw[h, 16] - ow[h, 16]).max(initial=0) < 1e-5
    # payload: density float, u16/u8 fields within 1 LSB, ior half identical
    gcv = gc.view(N.VOXEL_DTYPE).reshape(-1)
    ocv = oc.view(N.VOXEL_DTYPE).reshape(-1)
    for f in ["sigma", "r", "normal"]:
        d = np.abs(gcv[f].astype(np.int64) - ocv[f].astype(np.int64))
        assert d.max(initial=0) <= 1, f
    for f in ["diffuse", "specular"]:
        d = np.abs(gcv[f].astype(np.int64) - ocv[f].astype(np.int64))
        assert d.max(initial=0) <= 1, f
    assert np.array_equal(gcv["ior"], ocv["ior"])
    assert np.array_equal(gcv["density"][~h], ocv["density"][~h])


def _oracle(mesh, mat, prm, g, m2w=I43):
    return O.filter_voxels(mesh, O.material_from(mat), m2w, O.grid_from(g), O.params_from(prm))


@pytest.fixture(params=[0, 1], ids=["ploc", "karras"])
def bvh_method(request):
    """Both hierarchies of the builder, on the GPU and in the oracle."""
    N.check(N.lib.r2_set_bvh_method(request.param))
    O.lib.orc_set_bvh_method(request.param)
    yield request.param
    N.check(N.lib.r2_set_bvh_method(-1))
    O.lib.orc_set_bvh_method(-1)


@pytest.mark.parametrize("mesh_kind", ["ico4", "foliage", "foliage_big", "single", "pair", "dupes"])
def test_bvh_bit_exact(mesh_kind, bvh_method):
    if mesh_kind == "ico4":
        mesh = scenes.icosphere(4, 0.05, 1)
    elif mesh_kind == "foliage":
        mesh = scenes.foliage(3000, 5, 0.7, 4)
    elif mesh_kind == "foliage_big":  # 80k triangles: many sort blocks and two scan partitions per pass
        mesh = scenes.foliage(40000, 20, 0.7, 9)
    elif mesh_kind == "single":
        mesh = F.Mesh(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), np.array([[0, 1, 2]], np.uint32),
                      np.tile(np.array([0, 0, 1], np.float32), (3, 1)))
    elif mesh_kind == "pair":
        mesh = F.Mesh(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]], np.float32),
                      np.array([[0, 1, 2], [1, 3, 2]], np.uint32), np.tile(np.array([0, 0, 1], np.float32), (4, 1)))
    else:  # many triangles sharing one centroid: duplicate Morton codes
        base = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
        pos = np.concatenate([base] * 200)
        mesh = F.Mesh(pos, np.arange(600, dtype=np.uint32).reshape(200, 3),
                      np.tile(np.array([0, 0, 1], np.float32), (600, 1)))
    sc = F.FilterScene(mesh, F.material(), I43)
    nodes, order, height = sc.bvh()
    sc.close()
    onodes, oorder, _, oheight = O.build_bvh(_world(mesh, I43), mesh.indices)
    assert np.array_equal(order, oorder)
    assert height == oheight
    assert np.array_equal(nodes, onodes)


def test_filter_small_icosphere_parity():
    """Plain small case: icosphere sub 4 (5,120 tris), 32^3, 64 samples/voxel, 10 iterations."""
    mesh = scenes.icosphere(4, 0.05, 1)
    mat = F.material()
    prm = F.params(samples_per_voxel=64, iterations=10)
    vs = scenes.voxel_size_for(mesh, 32)
    g, gc, gw, st = _gpu_filter(mesh, mat, prm, vs)
    assert list(g.num_voxels) == [32, 32, 32]
    ow, oc = _oracle(mesh, mat, prm, g)
    _compare(gw, gc, ow, oc)
    assert st[0] == 32 ** 3 and 0 < st[1] < st[0]
    # every voxel the classifier culled has no hits in the oracle
    assert (ow[:, 17] > 0).sum() <= st[1]


@pytest.mark.parametrize("spv,clip,iters,n", [(1, True, 0, 6), (33, True, 20, 9), (64, False, 10, 10),
                                               (1024, True, 3, 5), (256, True, 20, 7)])
def test_filter_variants(spv, clip, iters, n):
    mesh = scenes.icosphere(3, 0.05, 2)
    mat = F.material(diffuse=(0.2, 0.5, 0.9), specular=(0.3, 0.3, 0.3), alpha=0.7, ior=1.33)
    prm = F.params(samples_per_voxel=spv, iterations=iters, clip_rays=clip, seed=11)
    vs = scenes.voxel_size_for(mesh, n)
    g, gc, gw, _ = _gpu_filter(mesh, mat, prm, vs)
    ow, oc = _oracle(mesh, mat, prm, g)
    _compare(gw, gc, ow, oc)


def test_filter_transformed_object():
    mesh = scenes.icosphere(3, 0.05, 5)
    mat = F.material()
    prm = F.params(samples_per_voxel=48, iterations=10, seed=3)
    m2w = np.array([0.5, 0, 0, 0, 0.5, 0, 0, 0, 0.5, 1.0, -2.0, 0.25], np.float32)
    vs = 0.06
    g, gc, gw, _ = _gpu_filter(mesh, mat, prm, vs, m2w)
    ow, oc = _oracle(mesh, mat, prm, g, m2w)
    _compare(gw, gc, ow, oc)


def test_filter_foliage_parity():
    mesh = scenes.foliage(20000, 20, 0.7, 4)
    mat = F.material(diffuse=(0.1, 0.6, 0.1), specular=(0.04, 0.04, 0.04), alpha=0.5, ior=1.5)
    prm = F.params(samples_per_voxel=128, iterations=20)
    g, gc, gw, st = _gpu_filter(mesh, mat, prm, scenes.voxel_size_for(mesh, 24))
    ow, oc = _oracle(mesh, mat, prm, g)
    _compare(gw, gc, ow, oc)


def test_host_entry_matches_device_entry():
    mesh = scenes.icosphere(3, 0.05, 1)
    mat = F.material()
    prm = F.params(samples_per_voxel=32, iterations=5)
    vs = scenes.voxel_size_for(mesh, 12)
    g1, vox, wide = F.filter_mesh(mesh, mat, prm, vs, wide=True)
    g2, gc, gw, _ = _gpu_filter(mesh, mat, prm, vs)
    assert vox.tobytes() == gc.tobytes()
    assert np.array_equal(wide.astype(np.float64), gw)


def test_counting_build_gives_the_same_payload_and_consistent_counts():
    """The counting build of the sampling kernel writes the same voxels and
    counts spv rays per candidate voxel, at least one node visit per ray."""
    leaves = scenes.foliage(20_000, 6, 0.7, 5)
    mat = F.material(diffuse=(0.1, 0.6, 0.1), alpha=0.5)
    prm = F.params(samples_per_voxel=48, iterations=4)
    sc = F.FilterScene(leaves, mat)
    g = sc.grid(scenes.voxel_size_for(leaves, 24))
    nvox = int(np.prod(np.array(g.num_voxels[:], np.int64)))
    a = torch.empty(nvox * 32, dtype=torch.uint8, device="cuda")
    b = torch.empty(nvox * 32, dtype=torch.uint8, device="cuda")
    st = np.zeros(3)
    sc.run(g, prm, a.data_ptr(), stats=st)
    rays, nodes, tris = sc.count(g, prm, b.data_ptr())
    torch.cuda.synchronize()
    sc.close()
    assert torch.equal(a, b)
    assert rays == int(st[1]) * 48 and rays > 0
    assert nodes >= rays and tris > 0


def test_candidate_lists_and_per_ray_traversal_both_match_the_oracle():
    """A voxel with at most 512 candidate triangles tests them all with the
    warp's lanes in step (one BVH walk per voxel); a voxel with more traces
    every ray through the BVH.  The counting build shows which path ran (inner
    nodes visited against rays), and both give the oracle's hits bit for bit."""
    mat = F.material(diffuse=(0.1, 0.6, 0.1), alpha=0.5)
    prm = F.params(samples_per_voxel=256, iterations=4)
    cases = [(scenes.icosphere(4, 0.05, 1), 32, False),  # ~10 candidates per voxel
             (scenes.foliage(20_000, 6, 0.7, 5), 5, True)]  # thousands per voxel
    for mesh, n, per_ray in cases:
        vs = scenes.voxel_size_for(mesh, n)
        g, gc, gw, st = _gpu_filter(mesh, mat, prm, vs)
        ow, oc = _oracle(mesh, mat, prm, g)
        _compare(gw, gc, ow, oc)
        sc = F.FilterScene(mesh, mat)
        nvox = int(np.prod(np.array(g.num_voxels[:], np.int64)))
        b = torch.empty(nvox * 32, dtype=torch.uint8, device="cuda")
        rays, nodes, tris = sc.count(sc.grid(vs), prm, b.data_ptr())
        torch.cuda.synchronize()
        sc.close()
        assert rays == int(st[1]) * 256 and rays > 0
        if per_ray:
            assert nodes >= rays, (nodes, rays)
        else:  # a few dozen nodes per voxel against 256 rays
            assert nodes * 2 < rays, (nodes, rays)
            assert tris % 256 == 0  # every ray of a voxel tests the voxel's whole list


def test_filter_output_does_not_depend_on_the_bvh_method():
    """Closest hits do not depend on the hierarchy (ties go to the lower
    triangle), and neither does anything the filter sums, so the PLOC and the
    Karras trees give the same payload and records bit for bit, on the
    candidate-list path (fine grid) and the traversal path (coarse grid)."""
    mat = F.material(diffuse=(0.1, 0.6, 0.1), specular=(0.04, 0.04, 0.04), alpha=0.5, ior=1.5)
    prm = F.params(samples_per_voxel=128, iterations=10)
    leaves = scenes.foliage(20_000, 6, 0.7, 5)
    try:
        for n in (48, 6):
            outs = []
            for method in (0, 1):
                N.check(N.lib.r2_set_bvh_method(method))
                g, gc, gw, _ = _gpu_filter(leaves, mat, prm, scenes.voxel_size_for(leaves, n))
                outs.append((gc, gw))
            assert np.array_equal(outs[0][0], outs[1][0]), n
            assert np.array_equal(outs[0][1], outs[1][1]), n
    finally:
        N.check(N.lib.r2_set_bvh_method(-1))


def test_fp16_payload_error_stated():
    mesh = scenes.icosphere(4, 0.05, 1)
    mat = F.material()
    prm = F.params(samples_per_voxel=64, iterations=10)
    g, gc, gw, st, f16 = _gpu_filter(mesh, mat, prm, scenes.voxel_size_for(mesh, 32), fp16=True)
    ow, _ = _oracle(mesh, mat, prm, g)
    h = (ow[:, 17] > 0) & np.isfinite(ow[:, 0])
    rel_d = np.abs(f16[h, 0] - ow[h, 0]) / np.abs(ow[h, 0])
    scale = np.max(np.abs(ow[h, 1:4]), axis=1, keepdims=True)
    rel_s = np.abs(f16[h, 1:7] - ow[h, 1:7]) / scale
    # binary16 has an 11-bit significand: half-ulp relative error 2^-11 ~ 4.9e-4
    assert rel_d.max() <= 2.0 ** -11 * 1.01
    assert rel_s.max() <= 2.0 ** -11 * 1.01


def test_invalid_arguments_rejected():
    mesh = scenes.icosphere(1, 0.0, 1)
    sc = F.FilterScene(mesh, F.material(), I43)
    g = sc.grid(0.5)
    out = torch.empty(int(np.prod(g.num_voxels[:])) * 32, dtype=torch.uint8, device="cuda")
    with pytest.raises(N.R2Error) as e:
        sc.run(g, F.params(samples_per_voxel=2000), out.data_ptr())
    assert e.value.name == "R2_ERR_UNSUPPORTED"
    with pytest.raises(N.R2Error):
        sc.grid(-1.0)
    sc.close()

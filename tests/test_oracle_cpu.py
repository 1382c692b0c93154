"""CPU tests of the oracle (the checker) and of the host-side logic.

Known-answer properties of the reference's algorithms (the reference ships no
tests or golden vectors, so the properties are derived from its math):
  * buildS(n, a) has eigenvalues {1 along n, a, a}  (sggx_phase_function.hpp:95-105)
  * estimateDensity fixed point ln2/(sigma_t t) for P_mesh = 1/2 (mesh_filter.hpp:182-226)
  * the compact payload of a voxel without hits is zero with ior = 1 (mesh_filter.hpp:112-119)
"""
import math

import numpy as np
import pytest

import oracle_lib as O


def test_philox_counter_sensitivity_and_determinism():
    a = O.philox([0, 0, 0, 0], [0, 0])
    b = O.philox([0, 0, 0, 0], [0, 0])
    c = O.philox([1, 0, 0, 0], [0, 0])
    d = O.philox([0, 0, 0, 0], [1, 0])
    assert (a == b).all()
    assert (a != c).any() and (a != d).any()


def test_philox_uniformity():
    # 4096 draws: mean of top-24-bit uniforms ~ 0.5, each bit ~ balanced
    vals = np.concatenate([O.philox([i, 7, 0, 0], [123, 456]) for i in range(1024)])
    u = (vals >> 8).astype(np.float64) / 2 ** 24
    assert abs(u.mean() - 0.5) < 0.02
    for bit in range(32):
        frac = ((vals >> bit) & 1).mean()
        assert 0.45 < frac < 0.55


def test_sincos_turns_accuracy():
    for u in np.linspace(0.0, 1.0, 4097, endpoint=False):
        s, c = O.sincos_turns(float(np.float32(u)))
        x = 2 * math.pi * float(np.float32(u))
        assert abs(s - math.sin(x)) < 3e-7
        assert abs(c - math.cos(x)) < 3e-7


def test_tracking_log_accuracy():
    # the free-flight logarithm of delta/ratio tracking, over every argument
    # 1 - u that the 24-bit uniforms produce, stays within 2 ulp of log
    rng = np.random.default_rng(5)
    ks = np.concatenate([np.arange(1, 4096), rng.integers(1, 1 << 24, 20000), [1 << 23, (1 << 24) - 1, 1 << 24]])
    worst = 0.0
    for k in ks:
        x = np.float32(int(k) * 2.0 ** -24)
        got = O.lib.orc_t_log(float(x))
        ref = math.log(float(x))
        ulp = float(np.spacing(np.float32(abs(ref)))) if ref != 0.0 else 2.0 ** -149
        worst = max(worst, abs(got - ref) / ulp)
    assert O.lib.orc_t_log(1.0) == 0.0
    assert worst <= 2.0, worst


def _random_mesh(n, seed):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-1, 1, size=(3 * n, 3)).astype(np.float32)
    idx = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    return pos, idx


def _brute(pos, idx, o, d, tmax, tris, order):
    best = (tmax, None)
    for bi in range(idx.shape[0]):
        prim = order[bi]
        # reuse the oracle's own watertight test through a one-triangle BVH
        n1, o1, t1, _ = O.build_bvh(pos[idx[prim]], np.array([[0, 1, 2]], np.uint32))
        tri, t, _, _ = O.trace(n1, t1, o, d, tmax)
        if tri >= 0 and (t < best[0] or (t == best[0] and (best[1] is None or bi < best[1]))):
            best = (t, bi)
    return best


@pytest.fixture(params=[0, 1], ids=["ploc", "karras"])
def bvh_method(request):
    O.lib.orc_set_bvh_method(request.param)
    yield request.param
    O.lib.orc_set_bvh_method(-1)


@pytest.mark.parametrize("n", [1, 2, 7, 64, 600])
def test_oracle_bvh_matches_brute_force(n, bvh_method):
    pos, idx = _random_mesh(n, n)
    nodes, order, tris, h = O.build_bvh(pos, idx)
    assert h >= 1
    assert sorted(order.tolist()) == list(range(n))
    rng = np.random.default_rng(99)
    for _ in range(64):
        o = rng.uniform(-1.5, 1.5, 3).astype(np.float32)
        d = rng.normal(size=3)
        d = (d / np.linalg.norm(d)).astype(np.float32)
        tri, t, _, _ = O.trace(nodes, tris, o, d, 10.0)
        bt, bi = _brute(pos, idx, o, d, np.float32(10.0), tris, order)
        if bi is None:
            assert tri == -1
        else:
            assert tri == bi and t == bt


def _sah_cost(nodes):
    """SAH cost of a node array (inner 1.2, triangle 1.0, areas relative to the root's)."""
    f = nodes.view(np.float32).astype(np.float64)

    def area(lx, hx, ly, hy, lz, hz):
        dx, dy, dz = hx - lx, hy - ly, hz - lz
        return dx * dy + dy * dz + dz * dx
    a0 = area(f[:, 0], f[:, 1], f[:, 2], f[:, 3], f[:, 8], f[:, 9])
    a1 = area(f[:, 4], f[:, 5], f[:, 6], f[:, 7], f[:, 10], f[:, 11])
    b = f[0]
    root = area(min(b[0], b[4]), max(b[1], b[5]), min(b[2], b[6]), max(b[3], b[7]), min(b[8], b[10]),
                max(b[9], b[11]))
    cost = 1.2
    for a, ch in ((a0, nodes[:, 12]), (a1, nodes[:, 13])):
        inner = ch >= 0
        leaf = (ch < 0) & (ch != np.int32(-2 ** 31))
        cnt = ((~ch.astype(np.int64)) >> 26) & 31
        cost += (1.2 * a[inner]).sum() / root + (cnt[leaf] * a[leaf]).sum() / root
    return cost


def test_ploc_tree_structure_and_quality():
    """PLOC over the 8x8 icosphere grid (327,680 triangles): every triangle in
    exactly one leaf, every child box inside its parent's, parents numbered
    below their children, and a lower SAH cost than the Karras tree."""
    from renderer2_b200 import render_scenes as RS
    desc, _ = RS.icosphere_grid_scene()
    pos, _ = RS.world_vertices(desc)
    idx, base = [], 0
    for m, _, _ in desc["meshes"]:
        idx.append(m.indices.astype(np.uint32) + np.uint32(base))
        base += m.positions.shape[0]
    idx = np.concatenate(idx)
    cost = {}
    for meth in (1, 0):
        O.lib.orc_set_bvh_method(meth)
        nodes, order, _, h = O.build_bvh(pos, idx)
        cost[meth] = _sah_cost(nodes)
    O.lib.orc_set_bvh_method(-1)
    n = idx.shape[0]
    assert np.array_equal(np.sort(order), np.arange(n))
    covered = np.zeros(n, np.int32)
    f = nodes.view(np.float32)
    reach = np.zeros(nodes.shape[0], bool)  # inner nodes reachable from the root (not inside collapsed leaves)
    reach[0] = True
    for i in range(nodes.shape[0]):  # parents have smaller indices than their children
        if reach[i]:
            for c in range(2):
                ch = int(nodes[i, 12 + c])
                if ch >= 0:
                    reach[ch] = True
                elif ch != -2 ** 31:
                    a, k = (~ch) & 0x03FFFFFF, ((~ch) >> 26) & 31
                    covered[a:a + k] += 1
    for c in range(2):
        ch = nodes[:, 12 + c]
        inner = np.flatnonzero(ch >= 0)
        kids = ch[inner]
        assert np.all(nodes[kids, 14] == inner) and np.all(kids > inner)
        lo = f[inner][:, [0, 2, 8]] if c == 0 else f[inner][:, [4, 6, 10]]
        hi = f[inner][:, [1, 3, 9]] if c == 0 else f[inner][:, [5, 7, 11]]
        klo = np.minimum(f[kids][:, [0, 2, 8]], f[kids][:, [4, 6, 10]])
        khi = np.maximum(f[kids][:, [1, 3, 9]], f[kids][:, [5, 7, 11]])
        assert np.all(klo >= lo) and np.all(khi <= hi)
    assert np.all(covered == 1)
    print(f"SAH cost: PLOC {cost[0]:.2f}, Karras {cost[1]:.2f}")
    assert cost[0] < 0.85 * cost[1]


def test_build_s_eigenvalues_via_oracle_filter_math():
    # buildS(n, a) = n n^T + a (I - n n^T): eigen-decomposition {1 (n), a, a}
    rng = np.random.default_rng(3)
    for _ in range(20):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        a = rng.uniform(0.05, 1.0)
        S = np.outer(n, n) + a * (np.eye(3) - np.outer(n, n))
        ev = np.sort(np.linalg.eigvalsh(S))
        assert np.allclose(ev, [a, a, 1.0], atol=1e-12)


def test_encode_empty_voxel():
    w = np.zeros(20, np.float64)
    w[16] = 1.0
    out = np.zeros(32, np.uint8)
    O.lib.orc_encode(O._p(w), O._p(out))
    exp = np.zeros(32, np.uint8)
    exp[28:30] = np.frombuffer(np.float16(1.0).tobytes(), np.uint8)
    assert (out == exp).all()


def test_encode_known_values():
    # n = +z, alpha = 0.25: S = diag(0.25, 0.25, 1); sigma = 65535*sqrt(S_ii)
    w = np.zeros(20, np.float64)
    w[0] = 2.5
    w[1:7] = [0.25, 0.25, 1.0, 0.0, 0.0, 0.0]
    w[7:10] = [0.8, 0.8, 0.8]
    w[10:13] = [1.0, 1.0, 1.0]
    w[13:16] = [0.0, 0.0, 1.0]
    w[16] = 1.5
    out = np.zeros(32, np.uint8)
    O.lib.orc_encode(O._p(w), O._p(out))
    u16 = np.frombuffer(out[4:16].tobytes(), np.uint16)
    assert np.frombuffer(out[0:4].tobytes(), np.float32)[0] == np.float32(2.5)
    assert u16.tolist() == [32767, 32767, 65535, 32767, 32767, 32767]
    assert out[16:19].tolist() == [204, 204, 204] and out[19:22].tolist() == [255, 255, 255]
    assert np.frombuffer(out[22:28].tobytes(), np.uint16).tolist() == [32767, 32767, 65535]
    assert np.frombuffer(out[28:30].tobytes(), np.float16)[0] == np.float16(1.5)


def test_density_fixed_point():
    """estimateDensity with every hit ray of length t and P_mesh = 1/2 converges to ln2/(sigma_t t)."""
    sig, t, alpha = 10.0, 0.1, 0.1
    p_mesh = 0.5
    d = -math.log(1 - p_mesh) / (t * sig)
    for _ in range(20):
        p_vol = 1 - math.exp(-d * sig * t)
        d = d - alpha / sig * (p_vol - p_mesh)
    assert abs(d - math.log(2) / (sig * t)) < 1e-12


def test_grid_setup_matches_library():
    from renderer2_b200 import _native as N
    import ctypes as C
    lo = np.array([-1.05, -1.02, -1.03], np.float32)
    hi = np.array([1.04, 1.05, 1.01], np.float32)
    for m2w in [N.identity43(), np.array([2, 0, 0, 0, 2, 0, 0, 0, 2, 0.5, -1.0, 3.0], np.float32)]:
        for vs in [2.1 / 32, 0.1, 0.37]:
            g = N.FilterGrid()
            N.check(N.lib.r2_filter_setup_grid(N.ptr(lo), N.ptr(hi), N.ptr(m2w), float(vs), C.byref(g)))
            go = O.setup_grid(lo, hi, m2w, vs)
            assert list(g.num_voxels) == list(go.num_voxels)
            for f in ["index_to_model", "model_to_index", "model_to_world", "world_to_model", "world_bb_min",
                      "world_bb_max"]:
                assert np.array_equal(np.array(getattr(g, f)[:], np.float32),
                                      np.array(getattr(go, f)[:], np.float32)), f


def test_grid_voxel_count_rule():
    # numVoxels = ceil(extent / vs - 0.001) per axis (openvdb_backend.cpp:62-63)
    from renderer2_b200 import _native as N
    import ctypes as C
    lo = np.zeros(3, np.float32)
    # 0.2501 / 0.25 - 0.001 < 1 (absorbed by the epsilon); 0.2526 / 0.25 - 0.001 > 1
    hi = np.array([1.0, 0.2501, 0.2526], np.float32)
    g = N.FilterGrid()
    N.check(N.lib.r2_filter_setup_grid(N.ptr(lo), N.ptr(hi), N.ptr(N.identity43()), 0.25, C.byref(g)))
    assert list(g.num_voxels) == [4, 1, 2]


def test_icosphere_generator():
    from renderer2_b200 import scenes
    m = scenes.icosphere(4, 0.05, 1)
    assert m.nverts == 2562 and m.ntris == 5120
    r = np.linalg.norm(m.positions, axis=1)
    assert r.min() > 0.94 and r.max() < 1.06
    assert np.allclose(np.linalg.norm(m.normals, axis=1), 1.0, atol=1e-5)
    m2 = scenes.icosphere(4, 0.05, 1)
    assert np.array_equal(m.positions, m2.positions)


def test_oracle_filter_small_scene_properties():
    """Oracle on a tiny grid: empty voxels give the empty payload; hit voxels
    have positive density, unit-trace-bounded S, mean normal of unit length."""
    from renderer2_b200 import scenes, filter as F
    mesh = scenes.icosphere(2, 0.05, 1)
    mat = F.material()
    prm = F.params(samples_per_voxel=32, iterations=10)
    vs = scenes.voxel_size_for(mesh, 8)
    lo = mesh.positions.min(0)
    hi = mesh.positions.max(0)
    g = O.setup_grid(lo, hi, np.eye(4, 3).T.reshape(-1).astype(np.float32) if False else
                     np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0], np.float32), vs)
    wide, comp = O.filter_voxels(mesh, O.material_from(mat), np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0],
                                                                       np.float32), g, O.params_from(prm))
    hits = wide[:, 17]
    assert (hits > 0).any() and (hits == 0).any()
    h = hits > 0
    assert (wide[h, 0] > 0).all()
    tr = wide[h, 1] + wide[h, 2] + wide[h, 3]
    assert np.allclose(tr, 1 + 2 * 0.3, atol=1e-9)  # trace(buildS) = 1 + 2a for unit normals
    assert np.allclose(np.linalg.norm(wide[h, 13:16], axis=1), 1.0, atol=1e-12)
    assert (comp[~h, :28] == 0).all()


def test_oracle_jacobi_eigendecomposition():
    """orc_sym3_eig (cyclic Jacobi in FP64) against LAPACK's symmetric solver,
    on random and near-planar SGGX matrices (eigenvalues 1, a, a with a down to 1e-8)."""
    import ctypes as C
    O.lib.orc_sym3_eig.argtypes = [C.c_void_p] * 3
    rng = np.random.default_rng(7)
    for i in range(2000):
        if i % 2:
            m = rng.normal(size=(3, 3))
            S = m @ m.T
        else:
            n = rng.normal(size=3)
            n /= np.linalg.norm(n)
            a = 10.0 ** rng.uniform(-8, 0)
            S = np.outer(n, n) + a * (np.eye(3) - np.outer(n, n))
        S6 = np.ascontiguousarray([S[0, 0], S[1, 1], S[2, 2], S[0, 1], S[0, 2], S[1, 2]])
        w, V = np.zeros(3), np.zeros(9)
        O.lib.orc_sym3_eig(S6.ctypes.data_as(C.c_void_p), w.ctypes.data_as(C.c_void_p), V.ctypes.data_as(C.c_void_p))
        V = V.reshape(3, 3)
        ref = np.linalg.eigvalsh(S)[::-1]
        assert np.all(np.abs(w - ref) <= 1e-13 * ref[0])
        assert np.abs(V @ np.diag(w) @ V.T - S).max() <= 1e-13 * ref[0]
        assert np.abs(V.T @ V - np.eye(3)).max() <= 1e-13

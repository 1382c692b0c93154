"""FP64 eigendecomposition of the filtered SGGX matrices, and the optional
projection that keeps near-planar voxels invertible.

A voxel crossed by one flat leaf averages buildS(n, alpha) = n n^T +
alpha (I - n n^T): eigenvalues 1, alpha, alpha.  With alpha near 0 the matrix
is near rank one, det(S) ~ alpha^2, and the phase function's
D(w) = 1/(pi sqrt|det S| (w^T S^-1 w)^2) (sggx_phase_function.hpp:107-117)
divides by almost nothing.  The filter decomposes each voxel's mean S in FP64
with Jacobi rotations (r2_filter_scene_run_eig) and, with
r2_filter_params.sggx_projection, stores V diag(max(w, floor w0)) V^T instead.

Bar: eigenvalues within 1e-4 (relative to the largest) of the oracle's FP64
decomposition of its FP64-accumulated S; V diag(w) V^T reproduces the stored
S within 1e-4; the projection off leaves every output bit unchanged; with it
on, the stored and the decoded payload S have det > 0 and a finite D in every
direction, and agree with the oracle's projected S within 1e-4.
"""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from renderer2_b200 import _native as N  # noqa: E402
from renderer2_b200 import filter as F  # noqa: E402
from renderer2_b200 import scenes  # noqa: E402

REL = 1e-4
O.lib.orc_sym3_eig.argtypes = [C.c_void_p] * 3


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _full(S6):
    xx, yy, zz, xy, xz, yz = (S6[..., k] for k in range(6))
    return np.stack([np.stack([xx, xy, xz], -1), np.stack([xy, yy, yz], -1), np.stack([xz, yz, zz], -1)], -2)


def _oracle_eig(S6):
    w = np.zeros((len(S6), 3))
    V = np.zeros((len(S6), 9))
    for i, s in enumerate(np.ascontiguousarray(S6, np.float64)):
        s = np.ascontiguousarray(s)
        wi, vi = np.zeros(3), np.zeros(9)
        O.lib.orc_sym3_eig(_p(s), _p(wi), _p(vi))
        w[i], V[i] = wi, vi
    return w, V.reshape(-1, 3, 3)


def _leaves(alpha):
    mesh = scenes.foliage(1500, 4, 0.7, 21)
    mat = F.material(diffuse=(0.2, 0.6, 0.1), specular=(0.05, 0.05, 0.05), alpha=alpha, ior=1.5)
    return mesh, mat, scenes.voxel_size_for(mesh, 24)


def _run(mesh, mat, prm, vs, eig=True):
    sc = F.FilterScene(mesh, mat)
    g = sc.grid(vs)
    nvox = int(np.prod(np.array(g.num_voxels[:], np.int64)))
    out = torch.empty(nvox * 32, dtype=torch.uint8, device="cuda")
    wide = torch.empty(nvox * 20, dtype=torch.float32, device="cuda")
    if eig:
        e = torch.full((nvox * 12,), np.nan, dtype=torch.float32, device="cuda")
        sc.run_eig(g, prm, out.data_ptr(), e.data_ptr(), wide.data_ptr())
    else:
        sc.run(g, prm, out.data_ptr(), wide.data_ptr())
    torch.cuda.synchronize()
    res = (g, out.cpu().numpy().reshape(nvox, 32), wide.cpu().numpy().reshape(nvox, 20).astype(np.float64))
    if eig:
        res = res + (e.cpu().numpy().reshape(nvox, 12).astype(np.float64),)
    sc.close()
    return res


def _decoded_S(compact):
    v = compact.view(N.VOXEL_DTYPE).reshape(-1)
    sig = v["sigma"].astype(np.float64) / 65535.0
    r = v["r"].astype(np.float64) / 65535.0 * 2.0 - 1.0
    return np.stack([sig[:, 0] ** 2, sig[:, 1] ** 2, sig[:, 2] ** 2, r[:, 0] * sig[:, 0] * sig[:, 1],
                     r[:, 1] * sig[:, 0] * sig[:, 2], r[:, 2] * sig[:, 1] * sig[:, 2]], 1)


def _D_finite(S6, rng):
    """det(S) and whether D(w) is finite and positive in float32 over 64 random
    directions, with inverse(S) = adj(S) / det(S) as glm forms it."""
    M = _full(np.asarray(S6, np.float64)).astype(np.float32)
    a, b, c = M[:, 0, 0], M[:, 0, 1], M[:, 0, 2]
    d, e, f = M[:, 1, 1], M[:, 1, 2], M[:, 2, 2]
    adj = np.stack([np.stack([d * f - e * e, c * e - b * f, b * e - c * d], -1),
                    np.stack([c * e - b * f, a * f - c * c, b * c - a * e], -1),
                    np.stack([b * e - c * d, b * c - a * e, a * d - b * b], -1)], -2).astype(np.float32)
    det = (a * (d * f - e * e) - b * (b * f - e * c) + c * (b * e - d * c)).astype(np.float32)
    w = rng.normal(size=(64, 3)).astype(np.float32)
    w /= np.linalg.norm(w, axis=1, keepdims=True)
    with np.errstate(all="ignore"):
        inv = (adj / det[:, None, None]).astype(np.float32)
        q = np.einsum("kj,nji,ki->nk", w, inv, w).astype(np.float32)
        D = np.float32(1.0) / (np.float32(np.pi) * np.sqrt(np.abs(det))[:, None] * q * q)
    return det.astype(np.float64), np.isfinite(D).all(axis=1) & (D > 0).all(axis=1)


@pytest.mark.parametrize("alpha", [0.3, 1e-3])
def test_eigendecomposition_matches_fp64_oracle(alpha):
    mesh, mat, vs = _leaves(alpha)
    prm = F.params(samples_per_voxel=64, iterations=10, seed=2)
    g, out, wide, eig = _run(mesh, mat, prm, vs)
    _, out0, wide0 = _run(mesh, mat, prm, vs, eig=False)
    assert np.array_equal(out, out0) and np.array_equal(wide, wide0)  # the decomposition changes no output
    h = wide[:, 17] > 0
    assert h.sum() > 200
    assert np.all(eig[~h] == 0.0)
    w, V = eig[h, :3], eig[h, 3:].reshape(-1, 3, 3).transpose(0, 2, 1)  # columns are eigenvectors
    assert np.all(w[:, 0] >= w[:, 1]) and np.all(w[:, 1] >= w[:, 2])
    assert np.abs(np.einsum("nij,nik->njk", V, V) - np.eye(3)).max() < 1e-6
    R = np.einsum("nij,nj,nkj->nik", V, w, V)
    S = _full(wide[h, 1:7])
    assert (np.abs(R - S).max(axis=(1, 2)) / w[:, 0]).max() <= REL
    ow, _ = O.filter_voxels(mesh, O.material_from(mat), I43(), O.grid_from(g), O.params_from(prm))
    assert np.array_equal(ow[:, 17], wide[:, 17])
    w64, V64 = _oracle_eig(ow[h, 1:7])
    assert (np.abs(w - w64).max(axis=1) / w64[:, 0]).max() <= REL
    if alpha < 0.01:  # near-planar voxels are present: the two small eigenvalues are ~alpha
        assert (w64[:, 2] / w64[:, 0] < 2e-3).sum() > 50


def I43():
    return N.identity43()


def test_projection_keeps_near_planar_voxels_invertible():
    mesh, mat, vs = _leaves(0.0)  # perfectly flat leaves: single-leaf voxels have S = n n^T, det 0
    rng = np.random.default_rng(5)
    plain = F.params(samples_per_voxel=64, iterations=10, seed=4)
    g, out0, wide0, _ = _run(mesh, mat, plain, vs)
    h = wide0[:, 17] > 0
    det0, ok0 = _D_finite(wide0[h, 1:7], rng)
    assert (~ok0 | (det0 <= 1e-12)).sum() > 50  # the problem the projection addresses
    prj = F.params(samples_per_voxel=64, iterations=10, seed=4, sggx_projection=True, sggx_floor=1e-3)
    _, out1, wide1, eig1 = _run(mesh, mat, prj, vs)
    assert np.array_equal(wide1[:, 17], wide0[:, 17])
    assert np.array_equal(wide1[:, 0], wide0[:, 0])  # density untouched
    assert np.array_equal(eig1, _run(mesh, mat, plain, vs)[3])  # eigen output is of the mean S before projection
    for S6 in (wide1[h, 1:7], _decoded_S(out1)[h]):
        det, ok = _D_finite(S6, rng)
        assert np.all(det > 0.0) and np.all(ok)
    ow, _ = O.filter_voxels(mesh, O.material_from(mat), I43(), O.grid_from(g), O.params_from(prj))
    w64, _ = _oracle_eig(ow[h, 1:7])
    assert np.all(w64[:, 2] >= 1e-3 * w64[:, 0] * (1 - 1e-9))
    err = np.abs(wide1[h, 1:7] - ow[h, 1:7]).max(axis=1) / w64[:, 0]
    assert err.max() <= REL


def test_eig_entry_rejects_bad_arguments():
    mesh, mat, vs = _leaves(0.3)
    sc = F.FilterScene(mesh, mat)
    g = sc.grid(vs)
    nvox = int(np.prod(np.array(g.num_voxels[:], np.int64)))
    out = torch.empty(nvox * 32, dtype=torch.uint8, device="cuda")
    with pytest.raises(N.R2Error):
        sc.run(g, F.params(sggx_projection=True, sggx_floor=1.5), out.data_ptr())
    with pytest.raises(N.R2Error):
        N.check(N.lib.r2_filter_scene_run_eig(sc.handle, C.byref(g), C.byref(F.params()), C.c_void_p(out.data_ptr()),
                                              None, None, None, None, None))
    sc.close()

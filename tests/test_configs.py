"""Mesh generation and workload construction (CPU)."""
import numpy as np

from preprocess_src_b200 import configs, mesh


def test_icosphere_sizes_and_winding():
    for k, (nv, ne) in {2: (162, 320), 3: (642, 1280), 4: (2562, 5120)}.items():
        v, f = mesh.rbc_shape(k)
        assert v.shape == (nv, 3) and f.shape == (ne, 3)
        a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
        n = np.cross(b - a, c - a)
        assert np.all(np.einsum("ij,ij->i", n, (a + b + c) / 3.0) > 0)   # outward


def test_evans_fung_volume():
    v, f = mesh.rbc_shape(4)
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    vol = np.einsum("ij,ij->i", (a + b + c) / 3.0, np.cross(b - a, c - a)).sum() / 6.0 * 7.82 ** 3
    assert 740 < vol < 760
    assert abs(np.abs(v[:, :2]).max() - 1.0) < 1e-12


def test_rotation_is_proper_and_orthonormal():
    rng = np.random.default_rng(0)
    for _ in range(10):
        R = mesh.random_rotation(rng)
        assert np.allclose(R @ R.T, np.eye(3), atol=1e-12)
        assert abs(np.linalg.det(R) - 1) < 1e-12


def test_single_cell_duct_layout():
    case = configs.single_cell_duct()
    assert (case.nx, case.ny, case.nz) == (32, 32, 68)
    assert case.fluid_nodes() == 64 * 30 * 30
    x = case.xr.reshape(-1, 3).mean(axis=0)
    assert np.allclose(x, [0.5, 0.5, 0.5], atol=0.2)


def test_dense_suspension_placement():
    case = configs.dense_suspension()
    assert case.ncell == 200 and case.vertex == 2562 and case.element == 5120
    assert case.fluid_nodes() == 256 * 126 * 126
    x = case.xr.reshape(case.ncell, case.vertex, 3)
    c = x.mean(axis=1)
    LZ = case.params["LZ"]
    d = c[:, None, :] - c[None, :, :]
    d[..., 2] -= LZ * np.round(d[..., 2] / LZ)
    dist = np.sqrt((d ** 2).sum(-1)) + np.eye(case.ncell) * 1e9
    assert dist.min() > 2 * 7.82
    # every vertex inside the half-way walls with the stencil margin
    half = (case.nx - 1) / 2.0 - 1.0
    assert np.abs(x[..., 0]).max() < half - 2 and np.abs(x[..., 1]).max() < half - 2
    assert 0.03 < case.meta["hematocrit"] < 0.045


def test_duct_bc_shape():
    bc = configs.duct_bc(6, 5, 9).reshape(9, 5, 6)
    assert (bc[2:7, 1:4, 1:5] == configs.COMP).all()
    assert (bc[[0, 1, 7, 8]][:, 1:4, 1:5] == configs.BUFF).all()
    assert (bc[:, 0, :] == configs.WALL).all() and (bc[:, :, -1] == configs.WALL).all()

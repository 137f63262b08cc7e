"""The FP64 oracle against known answers and invariants (CPU only).

The reference ships no tests or golden vectors; these pin the oracle with
analytic results and conservation laws, and tests/test_golden.py pins it
against outputs of the reference's own kernels.
"""
import dataclasses
import math

import numpy as np
import pytest

from preprocess_src_b200 import configs, mesh


def test_rest_state_is_invariant(oracle_mod):
    case = configs.duct_case("rest", 16, 10, 10, g=0.0)
    o = oracle_mod.Oracle(case)
    f0 = o.fn.copy()
    o.step(3)
    m = np.repeat(case.bc == configs.COMP, 19)
    assert np.abs(o.fn[m] - f0[m]).max() < 1e-15


def test_mass_is_conserved(oracle_mod):
    case = configs.small_duct(g=1e-4)
    o = oracle_mod.Oracle(case)
    m = case.bc == configs.COMP
    mass0 = o.fn.reshape(-1, 19)[m].sum()
    o.step(30)
    mass1 = o.fn.reshape(-1, 19)[m].sum()
    assert abs(mass1 - mass0) / mass0 < 1e-13


def _duct_series(y, z, a, b, G, mu, terms=60):
    """Laminar flow in a rectangular duct |y| < a, |z| < b (Boussinesq series),
    body force density G, viscosity mu."""
    u = np.zeros_like(y)
    for k in range(terms):
        n = 2 * k + 1
        beta = n * math.pi / (2 * a)
        u += ((-1) ** k / n ** 3) * (1 - np.cosh(beta * z) / np.cosh(beta * b)) * np.cos(beta * y)
    return 16 * a * a * G / (mu * math.pi ** 3) * u


def test_duct_flow_known_answer(oracle_mod):
    """Steady body-force-driven duct flow against the series solution; the
    reference's own known-answer check is the commented-out Poiseuille error
    of etc.cu:76-108."""
    width, g = 12, 1e-5
    case = configs.duct_case("duct_known_answer", 8, width, width, g=g)
    o = oracle_mod.Oracle(case)
    o.step(3000)
    nx = ny = width
    wn = o["wn"].reshape(case.nz, ny, nx)[case.nz // 2]
    # half-way walls half a node inside the wall nodes: fluid nodes 1..w-2, walls at 0.5, w-1.5
    coords = np.arange(nx) - (nx - 1) / 2.0
    Y, X = np.meshgrid(coords, coords, indexing="ij")
    half = (width - 2) / 2.0
    nu = (o.p.tau - 0.5) / 3.0
    exact = _duct_series(X, Y, half, half, g, nu)
    inner = (np.abs(X) < half) & (np.abs(Y) < half)
    err = np.linalg.norm((wn - exact)[inner]) / np.linalg.norm(exact[inner])
    assert err < 0.02, err


def test_spread_partition_of_unity(oracle_mod):
    """The delta function sums to 1: the lattice force equals the vertex force
    sum, including vertices whose stencil wraps the periodic z boundary."""
    case = configs.small_duct()
    o = oracle_mod.Oracle(case)
    rng = np.random.default_rng(0)
    for k in ("cfx", "cfy", "cfz"):
        o.a[k][:] = rng.standard_normal(o.a[k].size)
    o.a["z"][:5] = o.p.zmax - 0.3     # near the periodic end
    o.ibm_st1()
    m = case.bc == configs.COMP
    for k, c in (("fx", "cfx"), ("fy", "cfy"), ("fz", "cfz")):
        assert abs(o.a[k][m].sum() - o.a[c].sum()) < 1e-10


def test_skalak_force_vanishes_on_reference_shape(oracle_mod):
    case = configs.small_duct(subdiv=3, radius=6.0)
    o = oracle_mod.Oracle(case)
    assert o.stress() == 0
    f = np.concatenate([o["cfx"], o["cfy"], o["cfz"]])
    assert np.abs(f).max() < 1e-10


def test_skalak_isotropic_stretch_load(oracle_mod):
    """A sphere stretched uniformly by lam carries the isotropic tension of the
    reference's law, tau = (lam^2 - 1) + C lam^2 (lam^4 - 1) (from
    stress.cu:94-96 with g = lam^2 G), so the load is the Laplace pressure
    2 tau / r, inward: f_i = -(2 tau / r) n_i ds_i."""
    R, lam, C = 6.0, 1.002, 100.0
    v, f = mesh.icosphere(3)
    case = configs.duct_case("sphere", 32, 24, 24, centers_duct=[(16.0, 11.5, 11.5)], subdiv=3, radius=R, C=C)
    center = configs.duct_to_ref((16.0, 11.5, 11.5), case.nx, case.ny, case.nz)
    case.xr = (v * R + center).reshape(-1)
    case.tri = f
    o = oracle_mod.Oracle(case)
    x = (o["xd"].reshape(-1, 3) - center) * lam + center
    o.a["xd"][:] = x.reshape(-1)
    assert o.stress() == 0
    force = np.stack([o["cfx"], o["cfy"], o["cfz"]], axis=1)
    nrm = (x - center) / np.linalg.norm(x - center, axis=1, keepdims=True)
    tau = (lam * lam - 1) + C * lam * lam * (lam ** 4 - 1)
    r = R * lam
    # nodal area of the one-ring / 3
    tri_area = 0.5 * np.linalg.norm(np.cross(x[f[:, 1]] - x[f[:, 0]], x[f[:, 2]] - x[f[:, 0]]), axis=1)
    ds = np.zeros(len(x))
    for k in range(3):
        np.add.at(ds, f[:, k], tri_area / 3.0)
    expected = -(2 * tau / r) * nrm * ds[:, None]
    # discretisation error of a subdivision-3 sphere: ~0.7% in the mean load,
    # ~4% pointwise; both fall about 4x per subdivision level
    err = np.linalg.norm(force - expected) / np.linalg.norm(expected)
    assert err < 0.05, err
    load = np.einsum("ij,ij->i", force, nrm) / ds
    assert abs(load.mean() / (-2 * tau / r) - 1) < 0.015
    assert np.all(load < 0)


def test_volume_correction_restores_volume(oracle_mod):
    case = configs.small_duct(subdiv=3, radius=6.0)
    o = oracle_mod.Oracle(case)
    c = o["gx"][:3].copy()
    for k, d in (("x", 0), ("y", 1), ("z", 2)):
        o.a[k][:] = (o.a[k] - c[d]) * 1.002 + c[d]
    vol, _ = o.volumes()
    assert abs(vol[0] / o["volume0"][0] - 1) > 1e-3
    it = o.volume_correction()
    vol, _ = o.volumes()
    assert it > 0
    assert abs(vol[0] / o["volume0"][0] - 1) < 1e-5


def test_link_tables(oracle_mod):
    case = configs.small_duct(subdiv=2)
    o = oracle_mod.Oracle(case)
    nln, ln, lo = o["nln"], o["ln"].reshape(-1, 7), o["lo"].reshape(-1, 7)
    x = o["xd"].reshape(-1, 3)
    g = x.mean(axis=0)
    assert set(nln.tolist()) <= {5, 6}
    for j in range(case.vertex):
        k = nln[j]
        assert list(lo[j, :k + 1]) == sorted(list(ln[j, :k]) + [j])
        # one-ring ordered counter-clockwise about the outward direction
        for s in range(k):
            a, b = x[ln[j, s]] - x[j], x[ln[j, (s + 1) % k]] - x[j]
            assert np.dot(np.cross(a, b), x[j] - g) > 0


def test_drive_schedule(oracle_mod):
    """FLOWSTART/FREQ drive (lbm.cu:1030-1035): zero before flowstart."""
    case = configs.duct_case("drive", 8, 10, 10, g=1e-4)
    case.params["flowstart"] = 5
    o = oracle_mod.Oracle(case)
    o.step(5)
    assert np.abs(o["wn"]).max() == 0.0
    o.step(1)
    assert o["wn"].max() > 0.0


def _bend_energy(x, y, z, tri, br):
    """(2 / sqrt 3) BR sum over edge-neighbour pairs of (1 - cos theta), theta
    the angle between the two outward triangle normals."""
    p = np.stack([x, y, z], axis=1)
    n = np.cross(p[tri[:, 1]] - p[tri[:, 0]], p[tri[:, 2]] - p[tri[:, 0]])
    n /= np.linalg.norm(n, axis=1)[:, None]
    edges = {}
    for e, t in enumerate(tri):
        for a in range(3):
            edges.setdefault(tuple(sorted((t[a], t[(a + 1) % 3]))), []).append(e)
    pairs = np.array([v for v in edges.values() if len(v) == 2])
    cos = np.einsum("ij,ij->i", n[pairs[:, 0]], n[pairs[:, 1]])
    return 2.0 / math.sqrt(3.0) * br * float((1.0 - cos).sum())


def test_bending_force_is_energy_gradient(oracle_mod):
    """stress.cu:448-578 with spontaneous angle 0 (init1.cu:849-850): the
    four-point forces are minus the gradient of (2/sqrt 3) BR sum (1 - cos
    theta) over edge-neighbour pairs; they have no net force or torque."""
    case = configs.small_duct(subdiv=2, radius=5.0, br=0.05, Gs=1e-3)
    rng = np.random.default_rng(5)
    o = oracle_mod.Oracle(case)
    for k in ("x", "y", "z"):   # bending reads cel->x: perturb it after the setup
        o[k][:] += rng.normal(scale=0.15, size=case.vertex)
    for k in ("cfx", "cfy", "cfz"):
        o[k][:] = 0.0
    oracle_mod.lib().orc_bend(oracle_mod.C.byref(o.p), oracle_mod.C.byref(o.s))
    f = np.stack([o["cfx"], o["cfy"], o["cfz"]], axis=1)
    assert np.abs(f).max() > 1e-3
    assert np.abs(f.sum(axis=0)).max() <= 1e-12 * np.abs(f).max() * case.vertex
    pos = np.stack([o["x"], o["y"], o["z"]], axis=1)
    torque = np.cross(pos - pos.mean(axis=0), f).sum(axis=0)
    assert np.abs(torque).max() <= 1e-10 * np.abs(f).max() * case.vertex
    h = 1e-6
    for i in rng.choice(case.vertex, 8, replace=False):
        for d in range(3):
            xp, xm = [pos[:, c].copy() for c in range(3)], [pos[:, c].copy() for c in range(3)]
            xp[d][i] += h
            xm[d][i] -= h
            g = (_bend_energy(*xp, case.tri, 0.05) - _bend_energy(*xm, case.tri, 0.05)) / (2 * h)
            assert abs(-g - f[i, d]) <= 1e-6 * np.abs(f).max(), (i, d, -g, f[i, d])


def _signed_angles(x, y, z, tri):
    """cos and sin of the dihedral angle of every edge-neighbour pair, sin
    signed by the centroid test of stress.cu:527 (symmetric in the pair)."""
    p = np.stack([x, y, z], axis=1)
    n = np.cross(p[tri[:, 1]] - p[tri[:, 0]], p[tri[:, 2]] - p[tri[:, 0]])
    t = p[tri].mean(axis=1)
    edges = {}
    for e, tr in enumerate(tri):
        for a in range(3):
            edges.setdefault(tuple(sorted((tr[a], tr[(a + 1) % 3]))), []).append(e)
    pairs = np.array([v for v in edges.values() if len(v) == 2])
    n1, n2 = n[pairs[:, 0]], n[pairs[:, 1]]
    cos = np.einsum("ij,ij->i", n1, n2) / np.linalg.norm(n1, axis=1) / np.linalg.norm(n2, axis=1)
    sgn = np.where(np.einsum("ij,ij->i", n1 - n2, t[pairs[:, 0]] - t[pairs[:, 1]]) >= 0.0, 1.0, -1.0)
    return cos, sgn * np.sqrt(np.clip(1.0 - cos * cos, 0.0, None))


def test_spontaneous_bending_angles(oracle_mod):
    """Bending about the initial shape's dihedral angles (init1.cu:797-848,
    kept instead of the override of 849-850): no force on the initial shape;
    on a perturbed shape the four-point forces are minus the gradient of
    (2/sqrt 3) BR sum (1 - cos(theta - theta0)) over edge-neighbour pairs."""
    case = configs.small_duct(subdiv=2, radius=5.0, br=0.05, Gs=1e-3, bend_spont=1)
    o = oracle_mod.Oracle(case)
    assert o.a["s0"].std() > 0.05   # an RBC shape: the angles differ from edge to edge

    def bend(oo):
        for k in ("cfx", "cfy", "cfz"):
            oo[k][:] = 0.0
        oracle_mod.lib().orc_bend(oracle_mod.C.byref(oo.p), oracle_mod.C.byref(oo.s))
        return np.stack([oo["cfx"], oo["cfy"], oo["cfz"]], axis=1)

    flat = oracle_mod.Oracle(case, bend_spont=False)
    f_flat = bend(flat)
    assert np.abs(bend(o)).max() <= 1e-12 * np.abs(f_flat).max()
    xr = case.xr.reshape(-1, 3)
    c0, s0 = _signed_angles(xr[:, 0], xr[:, 1], xr[:, 2], case.tri)
    rng = np.random.default_rng(6)
    for k in ("x", "y", "z"):
        o[k][:] += rng.normal(scale=0.15, size=case.vertex)
    f = bend(o)
    assert np.abs(f).max() > 1e-3
    assert np.abs(f.sum(axis=0)).max() <= 1e-12 * np.abs(f).max() * case.vertex
    pos = np.stack([o["x"], o["y"], o["z"]], axis=1)
    coef = 2.0 / math.sqrt(3.0) * 0.05

    def energy(q):
        cos, sin = _signed_angles(q[0], q[1], q[2], case.tri)
        return coef * float((1.0 - cos * c0 - sin * s0).sum())

    h = 1e-6
    for i in rng.choice(case.vertex, 8, replace=False):
        for d in range(3):
            xp, xm = [pos[:, c].copy() for c in range(3)], [pos[:, c].copy() for c in range(3)]
            xp[d][i] += h
            xm[d][i] -= h
            g = (energy(xp) - energy(xm)) / (2 * h)
            assert abs(-g - f[i, d]) <= 1e-6 * np.abs(f).max(), (i, d, -g, f[i, d])


@pytest.mark.parametrize("walls", [0, 1])
def test_shear_mode_reaches_the_couette_profile(oracle_mod, walls):
    """CapsuleSHEARFLOW without cells: from rest, walls moving from step 1 on
    (FLOWSTART = 1), the flow between the half-way walls becomes the linear
    Couette profile u_z(y) = sr y (both walls at -/+ sr LY/2) or sr (y + LY/2)
    (top wall at sr LY), which half-way bounce-back holds exactly."""
    from preprocess_src_b200 import configs
    case = configs.shear_case("couette_8x16x8", 8, 16, 8, sr=1e-3, walls=walls, flowstart=1)
    o = oracle_mod.Oracle(case)
    o.step(4000)
    nx, ny, nz = case.nx, case.ny, case.nz
    w = o["wn"].reshape(nz, ny, nx)[2:nz - 2, 2:ny - 2, 2:nx - 2]
    LY = ny - 4
    y = -LY / 2 - 1.5 + np.arange(2, ny - 2)
    exact = 1e-3 * (y if walls == 0 else y + LY / 2)
    assert np.abs(w - exact[None, :, None]).max() <= 1e-9 * np.abs(exact).max()
    assert np.abs(o["un"]).max() <= 1e-12 and np.abs(o["vn"]).max() <= 1e-12


def test_tube_interpolated_bounce_back_beats_the_staircase(oracle_mod):
    """Circular tube of radius 7.3 (lbm_cylinder.cu): steady Poiseuille flow
    u(r) = g (R^2 - r^2) / (4 nu).  The interpolated bounce-back on the circle
    lands within 1.5 % (relative L2) and well below the half-way staircase's
    error (8 % here; doubling R brings the interpolated error to 0.09 %)."""
    from preprocess_src_b200 import configs
    R, g = 7.3, 1e-5
    errs = {}
    for interp in (False, True):
        case = configs.tube_case("tube", 6, R, interp=interp, g=g)
        o = oracle_mod.Oracle(case)
        o.step(6000)
        nx, ny, nz = case.nx, case.ny, case.nz
        w = o["wn"].reshape(nz, ny, nx)[nz // 2]
        x = np.arange(nx) - (nx - 1) / 2.0
        y = np.arange(ny) - (ny - 1) / 2.0
        r2 = x[None, :] ** 2 + y[:, None] ** 2
        m = case.bc.reshape(nz, ny, nx)[nz // 2] == configs.COMP
        exact = g / (4 * (1.0 / 6.0)) * (R * R - r2)
        errs[interp] = np.sqrt(((w - exact)[m] ** 2).sum() / (exact[m] ** 2).sum())
    assert errs[True] <= 0.015 and errs[True] <= 0.25 * errs[False], errs


def test_oracle_per_cell_membrane_coefficients(oracle_mod):
    """The oracle's per-cell rgs and BR (a second cell population on the same
    mesh, cel->rg_w and cel->br_w of init3.cu:91-92): each cell's stress()
    force is the one of a single population with that cell's coefficients."""
    from preprocess_src_b200 import configs
    case = configs.duct_case("percell", 24, 20, 20, centers_duct=[(6.0, 9.8, 10.1), (17.0, 10.2, 9.7)],
                             subdiv=2, radius=4.0, seed=5, g=4e-5, Gs=2e-3)
    o0 = oracle_mod.Oracle(case)
    o0.step(4)   # deformed cells

    def forces(o):
        assert o.stress() == 0
        return np.stack([o["cfx"], o["cfy"], o["cfz"]])

    def at(rgs=None, br=None, cell_rgs=None, cell_br=None):
        p = dict(case.params)
        if rgs is not None:
            p["rgs"] = rgs
        if br is not None:
            p["br"] = br
        o = oracle_mod.Oracle(dataclasses.replace(case, params=p), init_fluid=False, cell_rgs=cell_rgs,
                              cell_br=cell_br)
        for k in ("x", "y", "z", "xd", "nd", "volume0", "gx"):
            o.a[k][:] = o0.a[k]
        return forces(o)

    V = case.vertex
    mixed = at(cell_rgs=[1.0, 2.5], cell_br=[0.0, 0.02])
    np.testing.assert_array_equal(mixed[:, :V], at(rgs=1.0, br=0.0)[:, :V])
    np.testing.assert_array_equal(mixed[:, V:], at(rgs=2.5, br=0.02)[:, V:])
    assert np.abs(mixed[:, V:] - at(rgs=1.0)[:, V:]).max() > 1e-6


def test_volume_fraction_invariants(oracle_mod):
    """Front tracking (fronttrack.cu) gives the cells' indicator: its sum over
    the fluid is the cell volume, it vanishes on walls and its BUFF planes
    hold their periodic images; THINC/WLIC (thincwlic.cu) moves it through
    faces only, so the sum stays."""
    case = configs.duct_case("vof", 24, 20, 20, centers_duct=[(3.0, 9.5, 9.5)], subdiv=3, radius=5.0, seed=3,
                             g=4e-5, Gs=2e-3, vof_k=10, lambda1=5.0)
    o = oracle_mod.Oracle(case)
    m = case.bc == configs.COMP
    vf = o["vf"].reshape(case.nz, case.ny, case.nx).copy()
    assert o.s.vof_iters > 0
    assert abs(o["vf"][m].sum() - o["volume0"][0]) <= 0.01 * o["volume0"][0]
    assert not o["vf"][case.bc == configs.WALL].any()
    np.testing.assert_allclose(vf[:2][:, 1:-1, 1:-1], vf[-4:-2][:, 1:-1, 1:-1], rtol=0, atol=1e-9)   # to the solve's tolerance
    total = o["vf"][m].sum()
    o.step(9)   # THINC/WLIC every step, no solve before step 10
    assert abs(o["vf"][m].sum() - total) <= 1e-11 * total
    assert np.abs(o["vf"] - vf.reshape(-1)).max() > 1e-4   # it moved

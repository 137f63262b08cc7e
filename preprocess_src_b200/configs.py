"""Workloads in the reference's own frame and layout.

The workloads are square ducts, periodic along the flow axis, with half-way
bounce-back walls on the four sides, driven by a body force along the flow,
with red cells (Skalak, C = 100) suspended in the flow.  They are described in
"duct" coordinates: flow axis X (periodic, length ``flow``), cross-section
Y x Z with wall nodes at Y = 0, Ly-1 and Z = 0, Lz-1.

The reference's CapsuleCHANNELFLOW mode is periodic along its z axis with two
BUFF planes at each end (init1.cu:207-234) and drives the flow along z
(lbm.cu:1030-1035).  So duct (X, Y, Z) maps to reference (z, x, y): nx = Ly,
ny = Lz, nz = flow + 4, and a duct lattice point (X, Y, Z) sits at reference
physical position (Y - (nx-1)/2, Z - (ny-1)/2, X + 2 - (nz-1)/2) in lattice
units (dx = dt = 1, init1.cu:207-234).  The map is a cyclic axis permutation,
a proper rotation, so triangle winding is preserved.

Parameters in lattice units: Cr = dx = dt = 1, tau = 3 Df + 1/2, a body
acceleration g maps to the reference macro P = g/2 (the force density is
2 rho P, lbm.cu:1116,1134), the shear modulus Gs maps to B = Gs/2 (the IB force
density is 2 rho B F with F normalised by Gs, stress.cu:96, lbm.cu:1117,1135).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import mesh as _mesh

COMP, BUFF, WALL = 0, 1, 2


@dataclass
class Case:
    name: str
    params: dict
    bc: np.ndarray              # [nx*ny*nz] int32, reference layout
    tri: np.ndarray             # [E,3] int32 local connectivity shared by all cells
    xr: np.ndarray              # [3*nv] AoS initial (= reference) positions
    ncell: int
    vertex: int
    element: int
    steps: int = 1
    meta: dict = field(default_factory=dict)

    @property
    def nx(self): return self.params["nx"]

    @property
    def ny(self): return self.params["ny"]

    @property
    def nz(self): return self.params["nz"]

    @property
    def n(self): return self.nx * self.ny * self.nz

    def fluid_nodes(self) -> int:
        return int((self.bc == COMP).sum())

    def ele_global(self) -> np.ndarray:
        """Reference cel->eleH: [3*N*E] global vertex ids (init1.cu:673-690)."""
        off = (np.arange(self.ncell, dtype=np.int64) * self.vertex)[:, None, None]
        return (self.tri[None, :, :].astype(np.int64) + off).reshape(-1).astype(np.int32)


def duct_bc(nx: int, ny: int, nz: int) -> np.ndarray:
    """Square duct: WALL on the cross-section rim, COMP inside, BUFF in the two
    end planes at each z end over fluid columns (init1.cu:219-234 with a square
    instead of a circular section)."""
    bc = np.full((nz, ny, nx), COMP, dtype=np.int32)
    rim = np.zeros((ny, nx), dtype=bool)
    rim[0, :] = rim[-1, :] = True
    rim[:, 0] = rim[:, -1] = True
    bc[:, rim] = WALL
    for z in (0, 1, nz - 2, nz - 1):
        bc[z][~rim] = BUFF
    return bc.reshape(-1)


def base_params(nx: int, ny: int, nz: int, *, tau=1.0, g=1e-6, Gs=5e-4, C=100.0, br=0.0, storage=0,
                membrane_fp64=0, solver_iters=0, residual=1e-13, itrmax=2000, flow=0, sr=0.0, walls=0,
                flowstart=0, bend_spont=0, lambda1=1.0, vof_k=0, vof_residual=1e-10, vof_itrmax=20000, M=1,
                rk_order=4) -> dict:
    LX, LZ = float(nx - 4), float(nz - 4)
    return dict(nx=nx, ny=ny, nz=nz, dx=1.0, dt=1.0, tau=float(tau), Cr=1.0, P=g / 2.0, B=Gs / 2.0,
                flowstart=int(flowstart), freq=math.inf, LX=LX, LZ=LZ, xmin=-LX / 2, xmax=LX / 2, zmin=-LZ / 2,
                zmax=LZ / 2, C=float(C), rgs=1.0, law=0, br=float(br), M=int(M), rk_order=int(rk_order),
                storage=storage,
                membrane_fp64=membrane_fp64, solver_iters=solver_iters, residual=residual,
                itrmax=itrmax, device=-1, flow=int(flow), sr=float(sr), walls=int(walls), tube_r=0.0,
                bend_spont=int(bend_spont), lambda1=float(lambda1), vof_k=int(vof_k),
                vof_residual=float(vof_residual), vof_itrmax=int(vof_itrmax))


def duct_to_ref(p, nx: int, ny: int, nz: int) -> np.ndarray:
    """Duct lattice coordinates (X, Y, Z) -> reference physical (x, y, z)."""
    p = np.asarray(p, dtype=np.float64)
    return np.array([p[1] - (nx - 1) / 2.0, p[2] - (ny - 1) / 2.0, p[0] + 2.0 - (nz - 1) / 2.0])


def duct_case(name: str, flow: int, Ly: int, Lz: int, *, centers_duct=(), subdiv=3, radius=7.82,
              seed=0, steps=1, **kw) -> Case:
    nx, ny, nz = Ly, Lz, flow + 4
    params = base_params(nx, ny, nz, **kw)
    shape, tri = _mesh.rbc_shape(subdiv)
    rng = np.random.default_rng(seed)
    cells = [_mesh.place(shape, _mesh.random_rotation(rng), radius, duct_to_ref(c, nx, ny, nz))
             for c in centers_duct]
    xr = np.concatenate(cells).reshape(-1) if cells else np.zeros(0)
    return Case(name=name, params=params, bc=duct_bc(nx, ny, nz), tri=tri.astype(np.int32), xr=xr,
                ncell=len(cells), vertex=len(shape), element=len(tri), steps=steps,
                meta=dict(seed=seed, subdiv=subdiv, radius=radius, flow=flow, Ly=Ly, Lz=Lz))


def suspension_case(name: str, flow: int, Ly: int, Lz: int, ncell: int, *, subdiv=4, radius=7.82,
                    seed=0, gap=1.0, wall_margin=2.5, steps=1, **kw) -> Case:
    """Cells placed by random sequential addition of bounding spheres (no
    overlap), orientations uniform on SO(3)."""
    nx, ny, nz = Ly, Lz, flow + 4
    params = base_params(nx, ny, nz, **kw)
    shape, tri = _mesh.rbc_shape(subdiv)
    rb = radius * _mesh.bounding_radius(shape)
    rng = np.random.default_rng(seed)
    # half-way walls sit half a node inside the outermost wall nodes
    hx = (nx - 1) / 2.0 - 1.0 - rb - wall_margin
    hy = (ny - 1) / 2.0 - 1.0 - rb - wall_margin
    LZ = params["LZ"]
    centers = _mesh.random_sequential_addition(ncell, rb, [-hx, -hy, -LZ / 2], [hx, hy, LZ / 2], gap, rng,
                                               periodic_z=LZ)
    cells = [_mesh.place(shape, _mesh.random_rotation(rng), radius, c) for c in centers]
    xr = np.concatenate(cells).reshape(-1)
    fluid_vol = (nx - 2) * (ny - 2) * (nz - 4)
    hct = ncell * _cell_volume(shape, tri) * radius ** 3 / fluid_vol
    return Case(name=name, params=params, bc=duct_bc(nx, ny, nz), tri=tri.astype(np.int32), xr=xr,
                ncell=ncell, vertex=len(shape), element=len(tri), steps=steps,
                meta=dict(seed=seed, subdiv=subdiv, radius=radius, flow=flow, Ly=Ly, Lz=Lz,
                          hematocrit=hct))


def split_cells(case: Case, nred: int) -> tuple[Case, Case]:
    """The first nred cells of case as the red cells and the rest as a white
    cell population on the same mesh: (red case, white-cell case).  The
    white-cell case carries only the mesh (its lattice is case's)."""
    nv = nred * case.vertex
    red = Case(name=case.name + "_red", params=dict(case.params), bc=case.bc, tri=case.tri,
               xr=case.xr[:3 * nv].copy(), ncell=nred, vertex=case.vertex, element=case.element,
               steps=case.steps, meta=dict(case.meta))
    white = Case(name=case.name + "_white", params=dict(case.params), bc=case.bc, tri=case.tri,
                 xr=case.xr[3 * nv:].copy(), ncell=case.ncell - nred, vertex=case.vertex,
                 element=case.element, steps=case.steps, meta=dict(case.meta))
    return red, white


def sphere_cells(case: Case, centers_ref, *, subdiv=2, radius=4.0, seed=0) -> Case:
    """Spherical cells (init3.cu's SPHERE shape: an icosphere) of the given
    radius at reference-frame centres, as a white-cell population for case's
    lattice."""
    shape, tri = _mesh.icosphere(subdiv)
    rng = np.random.default_rng(seed)
    cells = [_mesh.place(shape, _mesh.random_rotation(rng), radius, np.asarray(c, dtype=np.float64))
             for c in centers_ref]
    xr = np.concatenate(cells).reshape(-1)
    return Case(name=case.name + "_spheres", params=dict(case.params), bc=case.bc, tri=tri.astype(np.int32),
                xr=xr, ncell=len(cells), vertex=len(shape), element=len(tri), steps=case.steps,
                meta=dict(subdiv=subdiv, radius=radius, seed=seed))


def _cell_volume(v: np.ndarray, f: np.ndarray) -> float:
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    return float(np.einsum("ij,ij->i", (a + b + c) / 3.0, np.cross(b - a, c - a)).sum() / 6.0)


# ---- the named workloads ----------------------------------------------------

def single_cell_duct(**kw) -> Case:
    """64 x 32 x 32 duct, tau = 1, g = 1e-6, one subdivision-3 cell (642 vertices,
    1280 triangles) of radius 7.82 centred at duct (32, 16, 16), Gs = 5e-4,
    C = 100, 1000 steps."""
    kw.setdefault("seed", 1)
    return duct_case("single_cell_duct_64x32x32", 64, 32, 32, centers_duct=[(32.0, 16.0, 16.0)],
                     subdiv=3, steps=1000, **kw)


def tube_bc(nx: int, ny: int, nz: int, R: float) -> np.ndarray:
    """Circular tube (init1.cu:219-234): COMP where sqrt(x^2 + y^2) <= R in
    the cross-section, BUFF over those columns in the two end planes at each z
    end, WALL elsewhere."""
    x = np.arange(nx) - (nx - 1) / 2.0
    y = np.arange(ny) - (ny - 1) / 2.0
    inside = (x[None, :] ** 2 + y[:, None] ** 2) <= R * R
    bc = np.full((nz, ny, nx), WALL, dtype=np.int32)
    bc[:, inside] = COMP
    for z in (0, 1, nz - 2, nz - 1):
        bc[z][inside] = BUFF
    return bc.reshape(-1)


def tube_case(name: str, flow: int, R: float, *, interp=True, centers=(), subdiv=3, radius=5.0, seed=0,
              steps=1, **kw) -> Case:
    """Circular tube of radius R along z (the reference channel's own
    cross-section, init1.cu:219-234), periodic in z; interp selects the
    interpolated bounce-back on the circle (lbm_cylinder.cu) instead of
    half-way bounce-back on the staircase."""
    n = int(math.ceil(2 * R)) + 3
    nx = ny = n + (n % 2 == 0)
    nz = flow + 4
    params = base_params(nx, ny, nz, **kw)
    params["tube_r"] = float(R) if interp else 0.0
    shape, tri = _mesh.rbc_shape(subdiv)
    rng = np.random.default_rng(seed)
    cells = [_mesh.place(shape, _mesh.random_rotation(rng), radius, np.asarray(c, dtype=np.float64)) for c in centers]
    xr = np.concatenate(cells).reshape(-1) if cells else np.zeros(0)
    return Case(name=name, params=params, bc=tube_bc(nx, ny, nz, R), tri=tri.astype(np.int32), xr=xr,
                ncell=len(cells), vertex=len(shape), element=len(tri), steps=steps,
                meta=dict(R=R, interp=interp, flow=flow, seed=seed, subdiv=subdiv, radius=radius))


def shear_bc(nx: int, ny: int, nz: int) -> np.ndarray:
    """CapsuleSHEARFLOW box (init1.cu:133-187): COMP inside, BUFF in the two x
    and z layers at each end between the walls, WALL in the two rows beyond
    each y wall."""
    bc = np.full((nz, ny, nx), WALL, dtype=np.int32)
    bc[:, 2:ny - 2, :] = BUFF
    bc[2:nz - 2, 2:ny - 2, 2:nx - 2] = COMP
    return bc.reshape(-1)


def shear_case(name: str, LX: int, LY: int, LZ: int, *, centers=(), sr=1e-3, walls=0, subdiv=3, radius=6.0,
               seed=0, steps=1, **kw) -> Case:
    """Shear flow (CapsuleSHEARFLOW): an LX x LY x LZ box periodic in x and z
    between y walls moving along z at -/+ sr LY / 2 (walls = 0) or with the top
    wall at sr LY (walls = 1); cells centred at the given reference-frame
    positions (origin at the box centre)."""
    nx, ny, nz = LX + 4, LY + 4, LZ + 4
    kw.setdefault("g", 0.0)
    params = base_params(nx, ny, nz, flow=1, sr=sr, walls=walls, **kw)
    shape, tri = _mesh.rbc_shape(subdiv)
    rng = np.random.default_rng(seed)
    cells = [_mesh.place(shape, _mesh.random_rotation(rng), radius, np.asarray(c, dtype=np.float64)) for c in centers]
    xr = np.concatenate(cells).reshape(-1) if cells else np.zeros(0)
    return Case(name=name, params=params, bc=shear_bc(nx, ny, nz), tri=tri.astype(np.int32), xr=xr,
                ncell=len(cells), vertex=len(shape), element=len(tri), steps=steps,
                meta=dict(seed=seed, subdiv=subdiv, radius=radius, LX=LX, LY=LY, LZ=LZ, sr=sr, walls=walls))


def capillary_batch(n: int = 512, seed: int = 4, lengths=tuple(range(48, 129, 16)), **kw) -> list:
    """n independent capillaries (config 4): square 32 x 32 ducts of length L
    drawn uniformly from {48, 64, ..., 128}, one subdivision-3 cell each at the
    duct centre with a uniform random orientation, Gs log-uniform in
    [1e-4, 2e-3], g uniform in [5e-7, 2e-6], tau = 1, FP32.  All draws come from
    one seeded generator in capillary order."""
    rng = np.random.default_rng(seed)
    cases = []
    for i in range(n):
        L = int(rng.choice(lengths))
        Gs = float(np.exp(rng.uniform(np.log(1e-4), np.log(2e-3))))
        g = float(rng.uniform(5e-7, 2e-6))
        cases.append(duct_case(f"capillary{i:03d}_{L}x32x32", L, 32, 32, centers_duct=[(L / 2.0, 16.0, 16.0)],
                               subdiv=3, seed=int(rng.integers(1 << 31)), g=g, Gs=Gs, steps=2000, **kw))
    return cases


def dense_suspension(**kw) -> Case:
    """256 x 128 x 128 duct, 200 subdivision-4 cells (2562 vertices, 5120
    triangles each) of radius 7.82 placed by random sequential addition,
    Gs = 5e-4, C = 100, 5000 steps."""
    kw.setdefault("seed", 2)
    return suspension_case("dense_suspension_256x128x128_200rbc", 256, 128, 128, 200, subdiv=4,
                           steps=5000, **kw)


def small_duct(subdiv=2, radius=5.0, flow=32, width=20, ncell=1, **kw) -> Case:
    """Small case for oracle-sized parity tests."""
    kw.setdefault("seed", 3)
    if ncell == 1:
        c = [(flow / 2.0 + 0.3, width / 2.0 - 0.2, width / 2.0 + 0.4)]
    else:
        c = [(flow * (k + 0.5) / ncell, width / 2.0 + 0.3 * k, width / 2.0 - 0.2 * k) for k in range(ncell)]
    return duct_case(f"small_duct_{flow}x{width}x{width}_{ncell}c_s{subdiv}", flow, width, width,
                     centers_duct=c, subdiv=subdiv, radius=radius, **kw)

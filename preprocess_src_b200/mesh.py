"""Red-cell surface meshes and their placement.

The reference reads its meshes from ``./cell/icosa_div/icosa_div%d_cal.dat``
and ``./cell/rbc_div/rbc_div%d_cal.dat`` (init1.cu:490-519), files that are not
part of the reference.  They are generated here: a unit icosphere refined by
midpoint subdivision (each triangle -> 4, vertices pushed back to the sphere),
then the Evans-Fung map to the biconcave disc

    z = +-0.5 R sqrt(1 - rho^2) (0.207 + 2.003 rho^2 - 1.123 rho^4),  rho = r / R.

On the unit sphere sqrt(1 - rho^2) = |z|, so the map is z -> 0.5 z (...).
Triangles are wound outward, (x_b - x_a) x (x_c - x_a) pointing out of the
cell, which the reference's volume (volume_correction.cu:166-198) and one-ring
ordering (init2.cu:92-166) rely on.

Placement follows cel_init (init1.cu:626-669): unit shape, rotation, scale by
the radius, translate.  The reference draws three Euler angles from
``srand(time(NULL))``; here rotations are drawn uniformly on SO(3) from a
seeded generator so runs are reproducible.
"""
from __future__ import annotations

import numpy as np

_PHI = (1.0 + 5.0 ** 0.5) / 2.0


def icosahedron() -> tuple[np.ndarray, np.ndarray]:
    v = np.array([[-1, _PHI, 0], [1, _PHI, 0], [-1, -_PHI, 0], [1, -_PHI, 0],
                  [0, -1, _PHI], [0, 1, _PHI], [0, -1, -_PHI], [0, 1, -_PHI],
                  [_PHI, 0, -1], [_PHI, 0, 1], [-_PHI, 0, -1], [-_PHI, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
                  [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
                  [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                  [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int32)
    return v, f


def icosphere(subdiv: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: 10*4^k + 2 vertices, 20*4^k triangles, outward winding."""
    v, f = icosahedron()
    verts = [tuple(p) for p in v]
    for _ in range(subdiv):
        cache: dict[tuple[int, int], int] = {}

        def mid(a: int, b: int) -> int:
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                p = (np.asarray(verts[a]) + np.asarray(verts[b])) * 0.5
                p /= np.linalg.norm(p)
                cache[key] = len(verts)
                verts.append(tuple(p))
            return cache[key]

        nf = []
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        f = np.asarray(nf, dtype=np.int32)
    v = np.asarray(verts, dtype=np.float64)
    return v, orient_outward(v, f)


def orient_outward(v: np.ndarray, f: np.ndarray) -> np.ndarray:
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    n = np.cross(b - a, c - a)
    out = np.einsum("ij,ij->i", n, (a + b + c) / 3.0 - v.mean(axis=0)) < 0
    f = f.copy()
    f[out, 1], f[out, 2] = f[out, 2].copy(), f[out, 1].copy()
    return f


def evans_fung(v: np.ndarray) -> np.ndarray:
    """Unit sphere -> unit-radius Evans-Fung biconcave disc (symmetry axis z)."""
    rho2 = np.clip(v[:, 0] ** 2 + v[:, 1] ** 2, 0.0, 1.0)
    out = v.copy()
    out[:, 2] = 0.5 * v[:, 2] * (0.207 + 2.003 * rho2 - 1.123 * rho2 ** 2)
    return out


def rbc_shape(subdiv: int) -> tuple[np.ndarray, np.ndarray]:
    v, f = icosphere(subdiv)
    return evans_fung(v), f


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    """Uniform rotation on SO(3) from a random unit quaternion (Shoemake)."""
    u1, u2, u3 = rng.random(3)
    q = np.array([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2), np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                  np.sqrt(u1) * np.sin(2 * np.pi * u3), np.sqrt(u1) * np.cos(2 * np.pi * u3)])
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def place(shape: np.ndarray, rot: np.ndarray, radius: float, center) -> np.ndarray:
    return (shape @ rot.T) * radius + np.asarray(center, dtype=np.float64)


def bounding_radius(shape: np.ndarray) -> float:
    return float(np.linalg.norm(shape, axis=1).max())


def random_sequential_addition(n: int, radius: float, lo, hi, gap: float, rng: np.random.Generator,
                               periodic_z: float | None = None, max_tries: int = 200000) -> np.ndarray:
    """Centres of n non-overlapping spheres of the given radius (plus gap) inside
    the box [lo, hi], periodic along z with period ``periodic_z`` if given."""
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    dmin = 2.0 * radius + gap
    centers = np.empty((0, 3))
    tries = 0
    while len(centers) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError(f"random sequential addition placed only {len(centers)} of {n} cells")
        c = lo + (hi - lo) * rng.random(3)
        if len(centers):
            d = centers - c
            if periodic_z:
                d[:, 2] -= periodic_z * np.round(d[:, 2] / periodic_z)
            if (np.einsum("ij,ij->i", d, d) < dmin * dmin).any():
                continue
        centers = np.vstack([centers, c])
    return centers


def write_reference_dat(path: str, v: np.ndarray, f: np.ndarray) -> None:
    """The reference's mesh file format (init1.cu:490-519): 'V E', V lines of
    x y z, then 3E vertex ids."""
    with open(path, "w") as fh:
        fh.write(f"{len(v)} {len(f)}\n")
        for p in v:
            fh.write(f"{p[0]:.17e} {p[1]:.17e} {p[2]:.17e}\n")
        for t in f:
            fh.write(f"{t[0]} {t[1]} {t[2]}\n")

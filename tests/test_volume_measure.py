"""The volume correction measures a cell's volume and area per triangle as
(a + b + c) . c / 18 and |c| / 2 with c = (b - a) x (c - a) (tri_measure in
preprocess_src_b200/csrc/rbc_internal.cuh); the reference forms the unit normal
n = c / |c|, dS = |c| / 2 and the centroid r = (a + b + c) / 3 and sums
(r . n) dS / 3 and dS (volume_correction.cu:138-200, 246-281).  The two are the
same quantities; this checks, on the host in FP64, that they agree to rounding
on the meshes the workloads use, placed far from the origin as cells in a duct
are."""
import numpy as np

from preprocess_src_b200 import mesh


def reference_form(p, tri):
    a, b, c = p[tri[:, 0]], p[tri[:, 1]], p[tri[:, 2]]
    cr = np.cross(b - a, c - a)
    nc = np.sqrt((cr * cr).sum(1))
    n = cr / nc[:, None]
    ds = nc / 2.0
    r = (a + b + c) / 3.0
    return (1.0 / 3.0 * (r * n).sum(1) * ds).sum(), ds.sum()


def division_free_form(p, tri):
    a, b, c = p[tri[:, 0]], p[tri[:, 1]], p[tri[:, 2]]
    cr = np.cross(b - a, c - a)
    return ((a + b + c) * cr).sum(1).sum() / 18.0, np.sqrt((cr * cr).sum(1)).sum() / 2.0


def test_division_free_measure_equals_reference_form():
    rng = np.random.default_rng(3)
    for subdiv in (2, 3, 4):
        shape, tri = mesh.rbc_shape(subdiv)
        for _ in range(3):
            p = mesh.place(shape, mesh.random_rotation(rng), 7.82, rng.uniform(-100.0, 100.0, 3))
            p = np.asarray(p, dtype=np.float64).reshape(-1, 3)
            v_ref, a_ref = reference_form(p, tri)
            v_new, a_new = division_free_form(p, tri)
            assert v_ref > 0 and a_ref > 0
            # measured: volume 0 to 4.6e-16 relative (the cell ~100 lattice units from the
            # origin), area equal (halving is exact)
            assert abs(v_new - v_ref) <= 5e-15 * abs(v_ref), (subdiv, v_new, v_ref)
            assert abs(a_new - a_ref) <= 1e-15 * a_ref, (subdiv, a_new, a_ref)

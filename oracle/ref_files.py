"""The reference's restart and output files, restated in numpy.

TEST INFRASTRUCTURE ONLY: the checker for the library's file writers and
readers (csrc/ref_files.cu).  Byte layouts follow etc.cu of the reference for
a run with red cells (N_R), white cells (N_W) or both, no cytoadhesion; the
white cells' fields carry the suffix "_w" as in the reference:

  restart.bin   output_data etc.cu:738-781 / restart_file etc.cu:164-270
  cell%04d.bin  etc.cu:566-600 (one block per population, red first)
  prof%04d.bin  etc.cu:547-560
  center.dat    OutputCapsuleCenter / InputCapsuleCenter etc.cu:110-160
                (red cells' lines, then the white cells', each counted from 0)

and the output-interval averages those files carry: fem->tp, the principal
tensions of calc_tension (stress.cu:76-118), and fem->qi, the load of
substitute_load (stress.cu:280-300).
"""
from __future__ import annotations

import numpy as np


def expand2pow2(n: int) -> int:
    """etc.cu:425-446"""
    cnt = 0
    while n > 1:
        if n % 2 == 1:
            n += 1
        n //= 2
        cnt += 1
    return 2 ** cnt


def _cell_block(N: int, V: int, E: int, sfx: str):
    mn = expand2pow2(3 * V)
    lay = [(k + sfx, np.float64, N * V) for k in ("x", "y", "z")]
    lay += [(k + sfx, np.float64, N) for k in ("rx", "ry", "rz")]
    lay += [(k + sfx, np.float64, N * V) for k in ("u", "v", "w")]
    lay += [("qi" + sfx, np.float64, N * mn), ("tp" + sfx, np.float64, N * E * 2)]
    return lay


def restart_layout(n: int, N: int, V: int, E: int, Nw: int = 0, Vw: int = 0, Ew: int = 0):
    """(name, dtype, count) in file order; N, V, E the red cells', Nw, Vw, Ew
    the white cells'."""
    lay = [("iter", np.int32, 1), ("fnum", np.int32, 1), ("fn", np.float64, 19 * n)]
    lay += [(k, np.float64, n) for k in ("dm", "um", "vm", "wm", "vf", "vf2")]
    if N > 0:
        lay += _cell_block(N, V, E, "")
    if Nw > 0:
        lay += _cell_block(Nw, Vw, Ew, "_w")
    return lay


def _read(path, lay) -> dict:
    raw = open(path, "rb").read()
    out, off = {}, 0
    for name, dt, cnt in lay:
        nb = np.dtype(dt).itemsize * cnt
        if off + nb > len(raw):
            raise ValueError(f"{path}: too short at {name}")
        out[name] = np.frombuffer(raw, dtype=dt, count=cnt, offset=off).copy()
        off += nb
    if off != len(raw):
        raise ValueError(f"{path}: {len(raw) - off} bytes beyond the layout")
    return out


def _write(path, lay, fields: dict):
    with open(path, "wb") as f:
        for name, dt, cnt in lay:
            a = np.ascontiguousarray(fields.get(name, np.zeros(cnt)), dtype=dt).reshape(-1)
            if a.size != cnt:
                raise ValueError(f"{name}: {a.size} values, layout has {cnt}")
            f.write(a.tobytes())


def read_restart(path, n, N, V, E, Nw=0, Vw=0, Ew=0) -> dict:
    return _read(path, restart_layout(n, N, V, E, Nw, Vw, Ew))


def write_restart(path, n, N, V, E, fields: dict, Nw=0, Vw=0, Ew=0):
    """fields: any subset of the layout's names; the rest are zeros."""
    _write(path, restart_layout(n, N, V, E, Nw, Vw, Ew), fields)


def cell_layout(N, V, E, sfx=""):
    return ([(k + sfx, np.int32, 1) for k in ("N", "V", "E")]
            + [(k + sfx, np.float64, N * V) for k in ("x", "y", "z", "u", "v", "w")]
            + [("qi" + sfx, np.float64, N * V * 3), ("tp" + sfx, np.float64, N * E * 2),
               ("ele" + sfx, np.int32, N * E * 3)])


def read_cell_file(path, blocks: int = 1) -> dict:
    """blocks = 2 for a file with red and white cells (the second block's
    names carry "_w"); a run with white cells only writes one block."""
    raw_len = len(open(path, "rb").read())
    lay, off = [], 0
    for b in range(blocks):
        N, V, E = (int(v) for v in np.fromfile(path, dtype=np.int32, count=3, offset=off))
        blk = cell_layout(N, V, E, "_w" if b else "")
        lay += blk
        off += sum(np.dtype(dt).itemsize * c for _, dt, c in blk)
        if off > raw_len:
            raise ValueError(f"{path}: too short for block {b}")
    return _read(path, lay)


def prof_layout(n):
    return ([("iter", np.int32, 1)] + [(k, np.float64, n) for k in ("dm", "um", "vm", "wm", "vf", "vf2")]
            + [("bc", np.int32, n)])


def read_prof_file(path, n) -> dict:
    return _read(path, prof_layout(n))


def write_center(path, gx):
    """gx: [3 N] AoS, as cel->gx."""
    g = np.asarray(gx, dtype=np.float64).reshape(-1, 3)
    with open(path, "w") as f:
        for c, (a, b, d) in enumerate(g):
            f.write("%d %e %e %e \n" % (c, a, b, d))


def read_center(path) -> np.ndarray:
    rows = [line.split() for line in open(path) if line.strip()]
    return np.array([[float(r[1]), float(r[2]), float(r[3])] for r in rows]).reshape(-1)


def principal_tensions(xd, nd, ele, E, C, LX, LZ) -> np.ndarray:
    """The step value of fem->tp [N E 2] (calc_tension, stress.cu:29-118): xd
    AoS [3 nv] positions, nd [4 ne] reference contravariant metric, ele global
    vertex ids [3 ne]."""
    x = np.asarray(xd).reshape(-1, 3)
    e = np.asarray(ele).reshape(-1, 3)
    v1 = x[e[:, 1]] - x[e[:, 0]]
    v2 = x[e[:, 2]] - x[e[:, 0]]
    for v in (v1, v2):
        v[:, 0] -= LX * np.where(v[:, 0] > LX / 2, 1, np.where(v[:, 0] < -LX / 2, -1, 0))
        v[:, 2] -= LZ * np.where(v[:, 2] > LZ / 2, 1, np.where(v[:, 2] < -LZ / 2, -1, 0))
    l1 = (v1 * v1).sum(1)
    l2 = (v2 * v2).sum(1)
    i12 = (v1 * v2).sum(1)
    dv12 = l1 * l2 - i12 * i12
    n = np.asarray(nd).reshape(-1, 4)
    dn12 = n[:, 0] * n[:, 3] - n[:, 1] * n[:, 2]
    i1 = n[:, 0] * l1 + n[:, 1] * i12 + n[:, 2] * i12 + n[:, 3] * l2 - 2.0
    i2 = dv12 * dn12 - 1.0
    root = np.sqrt(np.abs((i1 + 2.0) ** 2 - 4.0 * (i2 + 1.0)))
    l12, l22 = 0.5 * (i1 + 2.0 + root), 0.5 * (i1 + 2.0 - root)
    l11, l21 = np.sqrt(l12), np.sqrt(l22)
    tp = np.empty((len(e), 2))
    tp[:, 0] = l11 / l21 * (l12 - 1.0 + C * l22 * i2)
    tp[:, 1] = l21 / l11 * (l22 - 1.0 + C * l12 * i2)
    return tp.reshape(-1)

"""The numpy restatement of the reference's file layouts (no GPU)."""
import numpy as np

from oracle import ref_files as RF


def test_expand2pow2_matches_etc_cu():
    # etc.cu:425-446 rounds up to a power of two by halving with round-up
    assert [RF.expand2pow2(n) for n in (1, 2, 3, 486, 1926, 7686)] == [1, 2, 4, 512, 2048, 8192]


def test_restart_layout_round_trip(tmp_path):
    n, N, V, E = 40, 2, 12, 20
    rng = np.random.default_rng(0)
    f = {name: (rng.integers(0, 100, cnt) if dt == np.int32 else rng.standard_normal(cnt))
         for name, dt, cnt in RF.restart_layout(n, N, V, E)}
    RF.write_restart(tmp_path / "r.bin", n, N, V, E, f)
    size = (tmp_path / "r.bin").stat().st_size
    assert size == 8 + 8 * (19 * n + 6 * n + 6 * N * V + 3 * N + N * RF.expand2pow2(3 * V) + 2 * N * E)
    g = RF.read_restart(tmp_path / "r.bin", n, N, V, E)
    for k in f:
        np.testing.assert_array_equal(g[k], f[k])


def test_center_file_format(tmp_path):
    RF.write_center(tmp_path / "c.dat", [1.0, -2.5, 3.25e-3, 4.0, 5.0, 6.0])
    assert (tmp_path / "c.dat").read_text().splitlines()[0] == "0 1.000000e+00 -2.500000e+00 3.250000e-03 "
    np.testing.assert_allclose(RF.read_center(tmp_path / "c.dat"), [1.0, -2.5, 3.25e-3, 4.0, 5.0, 6.0])


def test_restart_layout_with_white_cells(tmp_path):
    """output_data (etc.cu:738-781): the white cells' block follows the red
    cells' with the same field order; a run with white cells only has no red
    block."""
    n, N, V, E, Nw, Vw, Ew = 30, 2, 12, 20, 3, 42, 80
    names = [k for k, _, _ in RF.restart_layout(n, N, V, E, Nw, Vw, Ew)]
    red = ["x", "y", "z", "rx", "ry", "rz", "u", "v", "w", "qi", "tp"]
    assert names == ["iter", "fnum", "fn", "dm", "um", "vm", "wm", "vf", "vf2"] + red + [k + "_w" for k in red]
    cnt = dict((k, c) for k, _, c in RF.restart_layout(n, N, V, E, Nw, Vw, Ew))
    assert cnt["qi_w"] == Nw * RF.expand2pow2(3 * Vw) and cnt["tp_w"] == 2 * Nw * Ew and cnt["rx_w"] == Nw
    only_w = [k for k, _, _ in RF.restart_layout(n, 0, 0, 0, Nw, Vw, Ew)]
    assert only_w[9:] == [k + "_w" for k in red]
    rng = np.random.default_rng(1)
    f = {k: rng.standard_normal(c) for k, dt, c in RF.restart_layout(n, N, V, E, Nw, Vw, Ew) if dt == np.float64}
    RF.write_restart(tmp_path / "r.bin", n, N, V, E, f, Nw, Vw, Ew)
    g = RF.read_restart(tmp_path / "r.bin", n, N, V, E, Nw, Vw, Ew)
    for k in f:
        np.testing.assert_array_equal(g[k], f[k])


def test_cell_file_blocks(tmp_path):
    """cell%04d.bin (etc.cu:566-600): one self-describing block per population."""
    rng = np.random.default_rng(2)
    blocks = []
    for (N, V, E), sfx in (((2, 12, 20), ""), ((1, 42, 80), "_w")):
        lay = RF.cell_layout(N, V, E, sfx)
        vals = {k: (np.array([dict(N=N, V=V, E=E)[k[0]]], np.int32) if c == 1 and dt == np.int32
                    else rng.integers(0, 50, c).astype(dt) if dt == np.int32 else rng.standard_normal(c))
                for k, dt, c in lay}
        blocks.append((lay, vals))
    with open(tmp_path / "c.bin", "wb") as fh:
        for lay, vals in blocks:
            for k, dt, c in lay:
                fh.write(np.asarray(vals[k], dtype=dt).tobytes())
    got = RF.read_cell_file(tmp_path / "c.bin", blocks=2)
    for _, vals in blocks:
        for k, v in vals.items():
            np.testing.assert_array_equal(got[k], v)


def _file_golden():
    from pathlib import Path

    from tests.golden.make_golden import FILE_NAMES, file_cases
    out = []
    for name, case in file_cases().items():
        p = Path(__file__).resolve().parent / "golden" / f"{name}.npz"
        if p.exists():
            out.append((name, case, np.load(p), FILE_NAMES))
    return out


def test_layouts_match_the_reference_writers_files(tmp_path):
    """Files written by the reference's own output_data (etc.cu:449-790,
    compiled from the reference sources; fixture made by make_golden.py
    run-files): the numpy layouts parse every byte of them, and restart.bin and
    center%04d.dat written back from the parsed fields are the same bytes."""
    cases = _file_golden()
    if not cases:
        import pytest
        pytest.skip("no output-file fixture")
    for name, case, g, names in cases:
        n, N, V, E = case.n, case.ncell, case.vertex, case.element
        paths = {}
        for k in names:
            paths[k] = tmp_path / k.replace("/", "_")
            paths[k].write_bytes(g[f"file_{k}"].tobytes())
        fnum, steps = int(g["fnum"]), int(g["steps"])
        r = RF.read_restart(paths["restart.bin"], n, N, V, E)
        assert int(r["iter"][0]) == steps and int(r["fnum"][0]) == fnum
        RF.write_restart(tmp_path / "again.bin", n, N, V, E, r)
        assert (tmp_path / "again.bin").read_bytes() == paths["restart.bin"].read_bytes()
        prof = RF.read_prof_file(paths[f"prof{fnum:04d}.bin"], n)
        assert int(prof["iter"][0]) == steps
        np.testing.assert_array_equal(prof["bc"], case.bc)
        np.testing.assert_array_equal(prof["dm"], r["dm"])   # the same host copies in both files
        cell = RF.read_cell_file(paths[f"cell/cell{fnum:04d}.bin"])
        assert (int(cell["N"][0]), int(cell["V"][0]), int(cell["E"][0])) == (N, V, E)
        np.testing.assert_array_equal(cell["ele"], case.ele_global())
        for k in ("x", "y", "z", "u", "v", "w"):
            np.testing.assert_array_equal(cell[k], r[k])
        gx = RF.read_center(paths[f"center{fnum:04d}.dat"])
        assert gx.size == 3 * N
        RF.write_center(tmp_path / "center.dat", gx)
        assert (tmp_path / "center.dat").read_text() == paths[f"center{fnum:04d}.dat"].read_text()

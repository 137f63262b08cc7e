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

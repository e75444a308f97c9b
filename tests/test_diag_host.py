"""Host side of the diagnostics: the paneled real*4 writer and the oracle's CFL
restatement on states with known answers."""
import numpy as np

from oracle.oracle import EARTH_GRAV, EARTH_RADIUS, Oracle


def test_paneled_writer_records_and_layout(tmp_path):
    from ch_swe_b200.diag import read_paneled, write_paneled
    rng = np.random.default_rng(3)
    f1 = rng.standard_normal((6, 9, 9))
    f2 = rng.standard_normal((6, 9, 9))
    p = str(tmp_path / "h.dat")
    write_paneled(p, f2, rec=2)
    write_paneled(p, f1, rec=1)
    raw = np.fromfile(p, dtype="<f4")
    assert raw.size == 2 * 6 * 9 * 9
    # i fastest, then j, then panel: element (t, j, i) of record 1 at t*81 + j*9 + i
    assert raw[2 * 81 + 4 * 9 + 7] == np.float32(f1[2, 4, 7])
    assert np.array_equal(read_paneled(p, (6, 9, 9), rec=2), f2.astype(np.float32))


def test_oracle_diag_known_answers(oracle_built):
    N, dt, c = 16, 300.0, 2.5
    o = Oracle(N)
    h, u, v = o.zeros()
    h[:] = c
    hmin, hmax, cg, cx, cy = o.diag(h, u, v, dt)
    dx = EARTH_RADIUS * (np.pi / 2) / N
    assert hmin == c and hmax == c
    assert abs(cg - np.sqrt(EARTH_GRAV / dx ** 2 * c) * dt) < 1e-12 * cg
    assert cx == 0.0 and cy == 0.0
    # a solid-body rotation: the advective CFL is u0 dt / dx up to the metric factors
    axis = (0.0, 0.0, 1.0)
    u0 = 20.0
    h, u, v = o.ts2(u0=u0, h_mean=1000.0, axis=axis, linear_mode=True)
    _, _, _, cx, cy = o.diag(h, u, v, dt)
    assert 0.5 * u0 * dt / dx < max(cx, cy) < 2.0 * u0 * dt / dx


def test_write_latlon_records(tmp_path):
    """write_latlon: record rec holds the real*4 field, longitude fastest, and earlier
    records are kept."""
    from ch_swe_b200.diag import write_latlon
    path = str(tmp_path / "h.dat")
    a = np.arange(5 * 8, dtype=np.float64).reshape(5, 8) * 0.5
    b = -a
    write_latlon(path, a, rec=1)
    write_latlon(path, b, rec=3)
    raw = np.fromfile(path, dtype="<f4").reshape(-1, 5, 8)
    assert raw.shape[0] == 3
    np.testing.assert_array_equal(raw[0], a.astype("<f4"))
    np.testing.assert_array_equal(raw[2], b.astype("<f4"))

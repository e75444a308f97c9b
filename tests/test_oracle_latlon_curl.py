"""The oracle's lat-lon regrid of a cell-centre field (output_curl's curl.dat): the ECS_O
halo of width 2 -- the o-point exchange, the rows of virtual cells interpolated along
the neighbours' grid lines and the six special points of every cube corner -- and the
cubic stencils on the cell-centre mesh.  Pinned by: no stencil reads a halo cell that
the procedure leaves unfilled (the fields are NaN-poisoned); a smooth field converges at
the interpolation's order, at the cube corners too (a wrong corner formula leaves an
O(1) or O(h) error there); the regridded curl of a solid-body rotation converges to its
exact vorticity."""
import numpy as np
import pytest

from oracle.oracle import EARTH_RADIUS, Oracle


def _grid(N):
    nlat, nlon = 2 * N + 1, 4 * N
    phi = -0.5 * np.pi + np.arange(nlat) * np.pi / (nlat - 1)
    lam = np.arange(nlon) * 2 * np.pi / nlon
    P, L = np.meshgrid(phi, lam, indexing="ij")
    return np.cos(P) * np.cos(L), np.cos(P) * np.sin(L), np.sin(P)


def _cell_centres(N):
    from ch_swe_b200.testcases import mesh_geometry
    r, _, _ = mesh_geometry(N, "o")
    return r


def test_smooth_field_converges_and_reads_only_filled_cells(oracle_built):
    errs, corner = [], []
    for N in (16, 32, 64):
        r = _cell_centres(N)
        f = r[..., 2] + 0.3 * r[..., 0] * r[..., 1] + 0.2 * r[..., 0] ** 3
        out = Oracle(N).latlon_o(f)
        assert not np.isnan(out).any(), N
        x, y, z = _grid(N)
        e = np.abs(out - (z + 0.3 * x * y + 0.2 * x ** 3))
        errs.append(e.max())
        # points within two cells of a cube corner (|x| = |y| = |z| = 1/sqrt 3)
        near = np.min([np.abs(np.abs(x) - 1 / np.sqrt(3)) + np.abs(np.abs(y) - 1 / np.sqrt(3)) +
                       np.abs(np.abs(z) - 1 / np.sqrt(3))], axis=0) < 3 * np.pi / (2 * N)
        assert near.any()
        corner.append(e[near].max())
    assert errs[0] / errs[1] > 6 and errs[1] / errs[2] > 6, errs
    assert corner[0] / corner[1] > 6 and corner[1] / corner[2] > 6, corner


def test_curl_of_solid_body_rotation_converges(oracle_built):
    axis = np.array([np.sin(0.7), 0.0, np.cos(0.7)])
    u0 = 20.0
    errs = []
    for N in (16, 64):
        o = Oracle(N)
        _, u, v = o.ts2(u0=u0, h_mean=1000.0, axis=tuple(axis))
        out = o.latlon_curl(u, v)
        x, y, z = _grid(N)
        exact = 2 * u0 / EARTH_RADIUS * (x * axis[0] + y * axis[1] + z * axis[2])
        errs.append(np.abs(out - exact).max() / (2 * u0 / EARTH_RADIUS))
    # the curl's own order near 2 in the max norm (the SBP closures), kept by the regrid
    assert errs[1] < 0.15 * errs[0], errs
    assert errs[1] < 1e-3


@pytest.mark.parametrize("nlat,nlon", [(37, 50), (5, 8)])
def test_other_grids(oracle_built, nlat, nlon):
    N = 16
    r = _cell_centres(N)
    out = Oracle(N).latlon_o(r[..., 2], nlat, nlon)
    assert out.shape == (nlat, nlon) and not np.isnan(out).any()
    phi = -0.5 * np.pi + np.arange(nlat) * np.pi / (nlat - 1)
    assert np.abs(out - np.sin(phi)[:, None]).max() < 1e-4

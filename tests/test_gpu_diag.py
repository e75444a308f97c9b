"""GPU diagnostics (swe_diag through the C ABI) against the oracle's restatement of
swm_output_diag_t's CFL and extrema."""
import numpy as np
import pytest

from tests.conftest import gpu_available

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu(lib_built, oracle_built):
    if not gpu_available():
        pytest.fail("no CUDA device: the -m gpu tests need a B200")


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_diag_matches_oracle(precision, tol):
    from ch_swe_b200 import create_domain, create_stvec_swm
    from ch_swe_b200.diag import SwmOutputDiag
    from oracle.oracle import Oracle
    N, dt = 24, 450.0
    o = Oracle(N, h_mean=1000.0)
    h = o.gaussian(lam0=0.4, phi0=0.3, d0=0.3, amp=5.0)[0] - 1.0
    _, u, v = o.ts2(u0=30.0, h_mean=1000.0, axis=(0.3, 0.0, 0.95), linear_mode=True)
    ref = o.diag(h, u, v, dt)
    dom = create_domain(N, precision=precision, h_mean=1000.0, n_members=2)
    st = create_stvec_swm(dom)
    st.upload(h, u, v, member=1)
    st.upload(h * 0, u * 0, v * 0, member=0)
    d = SwmOutputDiag(dom).diagnostics(st, dt, member=1)
    got = (d["h_min"], d["h_max"], d["cfl_gravity"], d["cfl_adv_x"], d["cfl_adv_y"])
    for g, r, name in zip(got, ref, ("h_min", "h_max", "cfl_gravity", "cfl_adv_x", "cfl_adv_y")):
        assert abs(g - r) <= tol * max(abs(r), 1e-30), (name, g, r)
    d0 = SwmOutputDiag(dom).diagnostics(st, dt, member=0)
    assert d0["h_max"] == 0.0 and d0["cfl_adv_x"] == 0.0
    dom.destroy()


def _energy_state(o, seed):
    """A state with h > 0 everywhere (the enstrophy divides by h on the cell centres) and
    a rotated wind, plus seeded noise on every field so that the duplicated panel-edge
    copies disagree and the curl SAT terms matter."""
    rng = np.random.default_rng(seed)
    h, u, v = o.ts2(u0=30.0, h_mean=3000.0, axis=(0.3, 0.0, 0.95))
    h = h + o.gaussian(lam0=0.4, phi0=0.3, d0=0.3, amp=50.0)[0]
    return h + rng.standard_normal(h.shape), u + rng.standard_normal(u.shape), v + rng.standard_normal(v.shape)


def _gpu_diag(N, precision, order, state, operator="linear"):
    from ch_swe_b200 import create_domain, create_stvec_swm
    from ch_swe_b200.diag import SwmOutputDiag
    dom = create_domain(N, precision=precision, h_mean=1000.0, n_members=2, sbp_order=order, operator=operator)
    st = create_stvec_swm(dom)
    st.upload(*state, member=1)
    st.upload(*(x * 0 + 1.0 for x in state), member=0)
    diag = SwmOutputDiag(dom)
    e = diag.calc_energies(st, member=1)
    curl = diag.curl(st, member=1)
    e0 = diag.calc_energies(st, member=0)
    dom.destroy()
    return (e["te"], e["ke"], e["pe"], e["enstrophy"]), curl, e0


@pytest.mark.parametrize("order", [42, 21, 63])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_energies_and_curl_match_oracle(order, precision, tol):
    """swe_energies / swe_curl against the oracle's calc_energies / curl_ch_sbp_sat_*:
    relative to each quantity (the curl in the max norm over the field's max)."""
    from oracle.oracle import Oracle
    N = 24
    o = Oracle(N, h_mean=1000.0, axis=(0.0, 0.0, 1.0), sbp_order=order)
    st = _energy_state(o, 40 + order)
    ref = o.energies(*st)
    ref_curl = o.curl(st[1], st[2])
    got, curl, e0 = _gpu_diag(N, precision, order, st)
    for g, r, name in zip(got, ref, ("te", "ke", "pe", "enstrophy")):
        assert abs(g - r) <= tol * abs(r), (order, precision, name, g, r)
    err = np.abs(curl - ref_curl).max() / np.abs(ref_curl).max()
    assert err < tol, (order, precision, err)
    # member 0 holds constant fields (h = u = v = 1): each member is read on its own
    ref0 = o.energies(*(np.ones_like(x) for x in st))
    for g, r, name in zip((e0["te"], e0["ke"], e0["pe"], e0["enstrophy"]), ref0, ("te", "ke", "pe", "enstrophy")):
        assert abs(g - r) <= tol * abs(r), ("member 0", name, g, r)


def test_energies_advective_domain_fp64():
    """The diagnostics of an advective-operator context (SBP 4-2)."""
    from oracle.oracle import Oracle
    N = 20
    o = Oracle(N, h_mean=1000.0)
    st = _energy_state(o, 7)
    ref = o.energies(*st)
    got, curl, _ = _gpu_diag(N, "fp64", 42, st, operator="advective")
    for g, r in zip(got, ref):
        assert abs(g - r) <= 1e-12 * abs(r)
    assert np.abs(curl - o.curl(st[1], st[2])).max() <= 1e-12 * np.abs(curl).max()


def test_curl_solid_body_rotation_large_cube():
    """At C192 (beyond the oracle's sizes): the curl of a solid-body rotation about a
    tilted axis is 2 u0 / a (r . axis) on the cell centres up to the SBP 4-2
    truncation error (about 2e-5 of its maximum at this size)."""
    from ch_swe_b200 import create_domain, create_stvec_swm
    from ch_swe_b200.diag import SwmOutputDiag
    from ch_swe_b200.testcases import mesh_geometry, williamson2
    N, u0, H = 192, 20.0, 1000.0
    axis = np.array([np.sin(0.7), 0.0, np.cos(0.7)])
    dom = create_domain(N, precision="fp64", h_mean=H, rotation_axis=tuple(axis))
    st = create_stvec_swm(dom)
    st.upload(*williamson2(N, u0=u0, h_mean=H, axis=axis))
    curl = SwmOutputDiag(dom).curl(st)
    r, _, _ = mesh_geometry(N, "o")
    exact = 2 * u0 / dom.planet_radius * (r @ axis)
    assert np.abs(curl - exact).max() < 1e-4 * np.abs(exact).max()
    dom.destroy()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
@pytest.mark.parametrize("grid", [None, (37, 50)])
def test_latlon_regrid_matches_oracle(precision, tol, grid):
    """swe_regrid_latlon of h against the oracle's latlon_regrid_t (ECS_xy halo of width 2,
    cubic stencil), for a state whose duplicated panel-edge copies disagree (the halo
    averages them), on the outputer's default 2N+1 x 4N grid and on another one."""
    from ch_swe_b200 import create_domain, create_stvec_swm
    from ch_swe_b200.diag import LatlonOutputer
    from oracle.oracle import Oracle
    N = 24
    o = Oracle(N)
    rng = np.random.default_rng(11)
    h = o.gaussian(lam0=1.0, phi0=0.4, d0=0.5, amp=100.0)[0] + rng.standard_normal((6, N + 1, N + 1))
    _, u, v = o.zeros()
    nlat, nlon = grid if grid else (None, None)
    ref = o.latlon(h, nlat, nlon)
    dom = create_domain(N, precision=precision, n_members=2)
    st = create_stvec_swm(dom)
    st.upload(h, u, v, member=1)
    st.upload(h * 0, u, v, member=0)
    out = LatlonOutputer(dom, nlat, nlon)
    got = out.regrid(st, member=1)
    assert got.shape == ref.shape
    assert np.abs(got - ref).max() <= tol * np.abs(ref).max()
    assert np.abs(out.regrid(st, member=0)).max() == 0.0
    dom.destroy()


def test_latlon_regrid_large_cube_converges(tmp_path):
    """At C192: the regridded Gaussian hill matches the analytic field to the cubic
    interpolation error, and the record written is its real*4 image."""
    from ch_swe_b200 import create_domain, create_stvec_swm
    from ch_swe_b200.diag import LatlonOutputer
    from ch_swe_b200.testcases import gaussian_hill
    N = 192
    dom = create_domain(N, precision="fp64")
    st = create_stvec_swm(dom)
    st.upload(*gaussian_hill(N, lam0=1.0, phi0=0.4, d0=0.5, amp=1.0))
    out = LatlonOutputer(dom)
    path = str(tmp_path / "h.dat")
    f = out.write(st, path, rec=2)
    nlat, nlon = f.shape
    phi = -np.pi / 2 + np.arange(nlat) * np.pi / (nlat - 1)
    lam = np.arange(nlon) * 2 * np.pi / nlon
    P, L = np.meshgrid(phi, lam, indexing="ij")
    c0 = (np.cos(0.4) * np.cos(1.0), np.cos(0.4) * np.sin(1.0), np.sin(0.4))
    d = np.clip(np.cos(P) * np.cos(L) * c0[0] + np.cos(P) * np.sin(L) * c0[1] + np.sin(P) * c0[2], -1, 1)
    exact = np.exp(-(np.arccos(d) / 0.5) ** 2)
    assert np.abs(f - exact).max() < 1e-7
    raw = np.fromfile(path, dtype="<f4")
    assert raw.size == 2 * nlat * nlon
    np.testing.assert_array_equal(raw[nlat * nlon:].reshape(nlat, nlon), f.astype("<f4"))
    dom.destroy()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_latlon_wind_regrid_matches_oracle(precision, tol):
    """swe_regrid_latlon_wind against the oracle's latlon_regrid_vec_t (Ch to vertex
    interpolation, covariant ecs_xy_vec halo, cubic stencils, rotation to lat-lon
    components), for a wind whose duplicated panel-edge copies disagree."""
    from ch_swe_b200 import create_domain, create_stvec_swm
    from ch_swe_b200.diag import LatlonVecOutputer
    from oracle.oracle import Oracle
    N = 24
    o = Oracle(N)
    rng = np.random.default_rng(12)
    h, u, v = o.ts2(u0=20.0, h_mean=1000.0, axis=(0.3, 0.0, 0.95))
    u = u + 0.1 * rng.standard_normal(u.shape)
    v = v + 0.1 * rng.standard_normal(v.shape)
    ref_u, ref_v = o.latlon_vec(u, v)
    dom = create_domain(N, precision=precision)
    st = create_stvec_swm(dom).upload(h, u, v)
    gu, gv = LatlonVecOutputer(dom).regrid(st)
    s = max(np.abs(ref_u).max(), np.abs(ref_v).max())
    assert np.abs(gu - ref_u).max() <= tol * s and np.abs(gv - ref_v).max() <= tol * s
    dom.destroy()


def test_latlon_wind_solid_body_rotation_large_cube(tmp_path):
    """At C192: the regridded wind of a solid-body rotation about a tilted axis is the
    exact eastward / northward wind away from the poles to the interpolation error."""
    from ch_swe_b200 import create_domain, create_stvec_swm
    from ch_swe_b200.diag import LatlonVecOutputer
    from ch_swe_b200.testcases import williamson2
    N, u0 = 192, 20.0
    axis = np.array([np.sin(0.7), 0.0, np.cos(0.7)])
    dom = create_domain(N, precision="fp64")
    st = create_stvec_swm(dom).upload(*williamson2(N, u0=u0, h_mean=1000.0, axis=axis))
    out = LatlonVecOutputer(dom)
    uo, vo = out.write(st, str(tmp_path / "u.dat"), str(tmp_path / "v.dat"))
    nlat, nlon = uo.shape
    phi = -np.pi / 2 + np.arange(nlat) * np.pi / (nlat - 1)
    lam = np.arange(nlon) * 2 * np.pi / nlon
    P, L = np.meshgrid(phi, lam, indexing="ij")
    r = np.stack([np.cos(P) * np.cos(L), np.cos(P) * np.sin(L), np.sin(P)], -1)
    vel = u0 * np.cross(axis, r)
    iv = np.stack([-np.sin(L), np.cos(L), 0 * L], -1)
    jv = np.stack([-np.sin(P) * np.cos(L), -np.sin(P) * np.sin(L), np.cos(P)], -1)
    inner = slice(1, nlat - 1)
    assert np.abs(uo - (vel * iv).sum(-1))[inner].max() < 1e-3 * u0
    assert np.abs(vo - (vel * jv).sum(-1))[inner].max() < 1e-3 * u0
    raw = np.fromfile(str(tmp_path / "v.dat"), dtype="<f4").reshape(nlat, nlon)
    np.testing.assert_array_equal(raw, vo.astype("<f4"))
    dom.destroy()


@pytest.mark.parametrize("operator,order", [("linear", 42), ("advective", 42), ("linear", 63)])
def test_latlon_div_regrid_matches_oracle(operator, order):
    """The div.dat field of output_div: the model's divergence of the contravariant wind
    (div_ch_sbp_sat_<order>_proj) regridded like h, against the oracle's co2contra, div
    and lat-lon regrid; for the advective context too, whose tendency is not -H div."""
    from ch_swe_b200 import create_domain, create_stvec_swm
    from ch_swe_b200.diag import LatlonOutputer
    from oracle.oracle import Oracle
    N = 24
    o = Oracle(N, sbp_order=order)
    rng = np.random.default_rng(3)
    h, u, v = o.ts2(u0=20.0, h_mean=1000.0, axis=(0.3, 0.0, 0.95))
    u = u + rng.standard_normal(u.shape)
    v = v + rng.standard_normal(v.shape)
    ref = o.latlon(o.div(*o.co2contra(u, v)))
    dom = create_domain(N, precision="fp64", operator=operator, sbp_order=order, n_members=2)
    st = create_stvec_swm(dom)
    st.upload(h + 1000.0, u, v, member=1)
    st.upload(h + 1000.0, 0 * u, 0 * v, member=0)
    out = LatlonOutputer(dom)
    got = out.regrid_div(st, member=1)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.abs(out.regrid_div(st, member=0)).max() == 0.0
    dom.destroy()


@pytest.mark.parametrize("precision,tol,order,grid", [("fp64", 1e-12, 42, None), ("fp64", 1e-12, 21, (37, 50)),
                                                      ("fp64", 1e-12, 63, None), ("fp32", 1e-5, 42, None)])
def test_latlon_curl_regrid_matches_oracle(precision, tol, order, grid):
    """The curl.dat field of output_curl: curl_ch_sbp_sat_<order> of the covariant wind on
    the cell centres, its ECS_O halo (exchange, virtual rows, the six special points of
    each cube corner) and the cubic stencils on the cell-centre mesh, against the
    oracle, for a wind whose panel-edge copies disagree."""
    from ch_swe_b200 import create_domain, create_stvec_swm
    from ch_swe_b200.diag import LatlonOutputer
    from oracle.oracle import Oracle
    N = 24
    o = Oracle(N, sbp_order=order)
    rng = np.random.default_rng(21)
    h, u, v = o.ts2(u0=20.0, h_mean=1000.0, axis=(0.3, 0.0, 0.95))
    u = u + rng.standard_normal(u.shape)
    v = v + rng.standard_normal(v.shape)
    nlat, nlon = grid if grid else (None, None)
    ref = o.latlon_curl(u, v, nlat, nlon)
    dom = create_domain(N, precision=precision, sbp_order=order, n_members=2)
    st = create_stvec_swm(dom)
    st.upload(h, u, v, member=1)
    st.upload(h, 0 * u, 0 * v, member=0)
    out = LatlonOutputer(dom, nlat, nlon)
    got = out.regrid_curl(st, member=1)
    assert got.shape == ref.shape
    assert np.abs(got - ref).max() <= tol * np.abs(ref).max()
    assert np.abs(out.regrid_curl(st, member=0)).max() == 0.0
    dom.destroy()


def test_latlon_curl_solid_body_rotation_large_cube():
    """At C192: the regridded curl of a solid-body rotation is its exact vorticity
    2 u0 / a (r . axis) to the discretisation error, near the cube corners too."""
    from ch_swe_b200 import create_domain, create_stvec_swm
    from ch_swe_b200.diag import LatlonOutputer
    from ch_swe_b200.testcases import williamson2
    from oracle.oracle import EARTH_RADIUS
    N, u0 = 192, 20.0
    axis = np.array([np.sin(0.7), 0.0, np.cos(0.7)])
    dom = create_domain(N, precision="fp64")
    st = create_stvec_swm(dom).upload(*williamson2(N, u0=u0, h_mean=1000.0, axis=axis))
    f = LatlonOutputer(dom).regrid_curl(st)
    nlat, nlon = f.shape
    phi = -np.pi / 2 + np.arange(nlat) * np.pi / (nlat - 1)
    lam = np.arange(nlon) * 2 * np.pi / nlon
    P, L = np.meshgrid(phi, lam, indexing="ij")
    rdot = np.cos(P) * np.cos(L) * axis[0] + np.cos(P) * np.sin(L) * axis[1] + np.sin(P) * axis[2]
    exact = 2 * u0 / EARTH_RADIUS * rdot
    assert np.abs(f - exact).max() < 1e-3 * 2 * u0 / EARTH_RADIUS
    dom.destroy()

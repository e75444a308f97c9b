"""ctypes wrapper of the CPU FP64 oracle (oracle/swe_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU legs of ``bench.py`` as the checker.  The product path never imports it.

State arrays use the packed host layout of the drop-in boundary: for each of the
six panels, Fortran order p(i, j) with i fastest and halos stripped:
  h : xy mesh, (6, N+1, N+1)   [panel, j, i]
  u : y  mesh, (6, N+1, N)     covariant alpha-component
  v : x  mesh, (6, N,   N+1)   covariant beta-component
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

EARTH_RADIUS = 0.6371229e7       # const_mod.f90:7
EARTH_GRAV = 9.80616             # const_mod.f90:6
EARTH_OMEGA = 2.0 * np.pi / (23 * 60 * 60 + 56 * 60 + 4)   # const_mod.f90:8-9

_dp = ctypes.POINTER(ctypes.c_double)


def build() -> str:
    """Compile the oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double, _dp, ctypes.c_int]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_apply.argtypes = [ctypes.c_void_p] + [_dp] * 6
        L.orc_rk4.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, ctypes.c_double, ctypes.c_int]
        L.orc_grad.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        L.orc_co2contra.argtypes = [ctypes.c_void_p] + [_dp] * 4
        L.orc_coriolis.argtypes = [ctypes.c_void_p] + [_dp] * 4
        L.orc_div.argtypes = [ctypes.c_void_p] + [_dp] * 3
        L.orc_integrals.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp]
        L.orc_dot.restype = ctypes.c_double
        L.orc_dot.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.orc_init_gaussian.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, _dp, _dp, _dp]
        L.orc_init_ts2.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _dp, ctypes.c_int,
                                   _dp, _dp, _dp]
        L.orc_metric.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp]
        L.orc_sync_weights.argtypes = [ctypes.c_void_p] + [_dp] * 4
        L.orc_halo_probe.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, ctypes.c_int, _dp, _dp]
        L.orc_sbp1d.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.orc_set_operator.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_set_orography.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_c_grad.argtypes = [ctypes.c_void_p] * 4
        L.orc_c_div.argtypes = [ctypes.c_void_p] * 4
        L.orc_c_co2contra.argtypes = [ctypes.c_void_p] * 5
        L.orc_c_weights.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.orc_c_halo_probe.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                       ctypes.c_void_p, ctypes.c_void_p]
        L.orc_set_sbp_order.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_diag.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, ctypes.c_double, _dp]
        L.orc_sbp1d_ord.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.orc_curl.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        L.orc_energies.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp]
        L.orc_ah_apply.argtypes = [ctypes.c_void_p] + [_dp] * 6
        L.orc_ah_rk4.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, ctypes.c_double, ctypes.c_int]
        L.orc_ah_integrals.argtypes = [ctypes.c_void_p] + [_dp] * 5
        L.orc_diff_apply.argtypes = [ctypes.c_void_p] + [_dp] * 6 + [ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.orc_lap_ah.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_int]
        L.orc_diff_step.argtypes = [ctypes.c_void_p] + [_dp] * 3 + [ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                                                  ctypes.c_double, ctypes.c_int]
        L.orc_latlon_vec.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.orc_latlon_xy.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_int, _dp]
        L.orc_latlon_o.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_int, _dp]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def shapes(N: int):
    return (6, N + 1, N + 1), (6, N + 1, N), (6, N, N + 1)


class Oracle:
    """FP64 CPU restatement of the linear Ch shallow-water operator (SBP 4-2, 2-1 or 6-3) and RK4."""

    OPERATORS = {"linear": 0, "advective": 1}

    def __init__(self, N: int, radius: float = EARTH_RADIUS, grav: float = EARTH_GRAV,
                 omega: float = EARTH_OMEGA, h_mean: float = 1000.0, axis=(0.0, 0.0, 1.0),
                 coriolis_constant: bool = False, operator: str = "linear", sbp_order: int = 42):
        """operator: 'linear' (linear_swm_operator) or 'advective' (advective_swm_operator,
        covariant Ch branch: up4 mass flux and up4 vector advection).  sbp_order: 42, 21
        or 63 (N >= 16), the order of the Ch difference, interpolation and quadrature
        operators (the _sbp_sat_42 / _21 / _63 operator names of the reference's
        factories)."""
        self.N = N
        self.radius, self.grav, self.omega, self.h_mean = radius, grav, omega, h_mean
        self.axis = np.ascontiguousarray(axis, dtype=np.float64)
        self._c = lib().orc_create(N, radius, grav, omega, h_mean, _p(self.axis), int(coriolis_constant))
        if not self._c:
            raise ValueError(f"oracle: unsupported N={N} (need N >= 8)")
        self.operator = operator
        lib().orc_set_operator(self._c, self.OPERATORS[operator])
        self.sbp_order = int(sbp_order)
        if lib().orc_set_sbp_order(self._c, self.sbp_order) != 0:
            raise ValueError(f"oracle: unsupported SBP order {sbp_order} (21, 42, or 63 with N >= 16)")

    def __del__(self):
        c = getattr(self, "_c", None)
        if c:
            lib().orc_destroy(c)
            self._c = None

    def zeros(self):
        sh, su, sv = shapes(self.N)
        return np.zeros(sh), np.zeros(su), np.zeros(sv)

    def diag(self, h, u, v, dt: float):
        """(h_min, h_max, gravity-wave CFL, advective CFL x, y) of swm_output_diag_t."""
        out = np.zeros(5)
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (h, u, v)]
        lib().orc_diag(self._c, _p(a[0]), _p(a[1]), _p(a[2]), float(dt), _p(out))
        return tuple(out)

    def curl(self, u, v):
        """Curl of the covariant (u, v) on the cell centres (curl_ch_sbp_sat_*): shape (6, N, N)."""
        out = np.zeros((6, self.N, self.N))
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (u, v)]
        lib().orc_curl(self._c, _p(a[0]), _p(a[1]), _p(out))
        return out

    # Ah staggering (linear operator, SBP 4-2): h, u, v all (6, N+1, N+1) on the xy mesh
    def ah_apply(self, h, u, v):
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (h, u, v)]
        out = [np.zeros_like(a[0]) for _ in range(3)]
        lib().orc_ah_apply(self._c, *(_p(x) for x in a), *(_p(x) for x in out))
        return tuple(out)

    def ah_rk4(self, h, u, v, dt: float, nsteps: int):
        a = [np.array(x, dtype=np.float64, order="C") for x in (h, u, v)]
        lib().orc_ah_rk4(self._c, *(_p(x) for x in a), float(dt), int(nsteps))
        return tuple(a)

    # diffusion on the Ah staggering (hordiff_vec_xyz_Ah_sbp_21_narrow for u, v and
    # hordiff_scalar_Ah_sbp_21_narrow for h; lap_order 21)
    def diff_apply(self, h, u, v, uv_coeff: float, h_coeff: float, lap_order: int = 21):
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (h, u, v)]
        out = [np.zeros_like(a[0]) for _ in range(3)]
        rc = lib().orc_diff_apply(self._c, *(_p(x) for x in a), *(_p(x) for x in out), int(lap_order),
                                  float(uv_coeff), float(h_coeff))
        if rc != 0:
            raise ValueError(f"no {lap_order} narrow Laplacian diffusion in the oracle")
        return tuple(out)

    def lap_ah(self, f, lap_order: int = 21):
        a = np.ascontiguousarray(f, dtype=np.float64)
        out = np.zeros_like(a)
        if lib().orc_lap_ah(self._c, _p(a), _p(out), int(lap_order)) != 0:
            raise ValueError(f"no {lap_order} narrow Laplacian in the oracle")
        return out

    def diff_step(self, h, u, v, dt: float, uv_coeff: float, h_coeff: float, nsteps: int = 1, lap_order: int = 21):
        a = [np.array(x, dtype=np.float64, order="C") for x in (h, u, v)]
        rc = lib().orc_diff_step(self._c, *(_p(x) for x in a), float(dt), int(lap_order), float(uv_coeff),
                                 float(h_coeff), int(nsteps))
        if rc != 0:
            raise ValueError(f"no {lap_order} narrow Laplacian diffusion in the oracle")
        return tuple(a)

    def ah_integrals(self, h, u, v):
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (h, u, v)]
        m = ctypes.c_double()
        e = ctypes.c_double()
        lib().orc_ah_integrals(self._c, *(_p(x) for x in a), ctypes.byref(m), ctypes.byref(e))
        return m.value, e.value

    def latlon(self, f, nlat=None, nlon=None):
        """Cubic lat-lon regrid of an xy field (latlon_outputer_t, default grid 2N+1 x 4N):
        shape (nlat, nlon)."""
        nlat = 2 * self.N + 1 if nlat is None else int(nlat)
        nlon = 4 * self.N if nlon is None else int(nlon)
        out = np.zeros((nlat, nlon))
        lib().orc_latlon_xy(self._c, _p(np.ascontiguousarray(f, dtype=np.float64)), nlat, nlon, _p(out))
        return out

    def latlon_o(self, f, nlat=None, nlon=None):
        """Cubic lat-lon regrid of a cell-centre field (6, N, N) on its ECS_O halo of width
        2 (the curl output of output_curl): shape (nlat, nlon)."""
        nlat = 2 * self.N + 1 if nlat is None else int(nlat)
        nlon = 4 * self.N if nlon is None else int(nlon)
        out = np.zeros((nlat, nlon))
        lib().orc_latlon_o(self._c, _p(np.ascontiguousarray(f, dtype=np.float64)), nlat, nlon, _p(out))
        return out

    def latlon_curl(self, u, v, nlat=None, nlon=None):
        """curl.dat of output_curl: the curl of the covariant Ch wind on the cell centres,
        regridded to the lat-lon grid."""
        return self.latlon_o(self.curl(u, v), nlat, nlon)

    def latlon_vec(self, u, v, nlat=None, nlon=None):
        """Cubic lat-lon regrid of the covariant Ch wind (latlon_vec_outputer_t): the
        eastward and northward components, each (nlat, nlon)."""
        nlat = 2 * self.N + 1 if nlat is None else int(nlat)
        nlon = 4 * self.N if nlon is None else int(nlon)
        uo = np.zeros((nlat, nlon))
        vo = np.zeros((nlat, nlon))
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (u, v)]
        lib().orc_latlon_vec(self._c, _p(a[0]), _p(a[1]), nlat, nlon, _p(uo), _p(vo))
        return uo, vo

    def energies(self, h, u, v):
        """(TE, KE, PE, enstrophy) of swm_output_diag_t%calc_energies (covariant u, v)."""
        out = np.zeros(4)
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (h, u, v)]
        lib().orc_energies(self._c, _p(a[0]), _p(a[1]), _p(a[2]), _p(out))
        return tuple(out)

    def gaussian(self, lam0=np.pi, phi0=0.0, d0=0.25, amp=1.0):
        h, u, v = self.zeros()
        lib().orc_init_gaussian(self._c, lam0, phi0, d0, amp, _p(h), _p(u), _p(v))
        return h, u, v

    # ---- C staggering (h on the cell centres, u on the x mesh, v on the y mesh)
    def c_shapes(self):
        N = self.N
        return (6, N, N), (6, N, N + 1), (6, N + 1, N)

    def c_grad(self, h):
        """grad_c_sbp_sat_<order>: (gx on x, gy on y) of h on the cell centres."""
        _, sx, sy = self.c_shapes()
        gx, gy = np.zeros(sx), np.zeros(sy)
        lib().orc_c_grad(self._c, _p(np.ascontiguousarray(h, dtype=np.float64)), _p(gx), _p(gy))
        return gx, gy

    def c_div(self, ut, vt):
        """div_c_sbp_sat_<order> of (ut on x, vt on y), on the cell centres."""
        so, _, _ = self.c_shapes()
        d = np.zeros(so)
        lib().orc_c_div(self._c, _p(np.ascontiguousarray(ut, dtype=np.float64)),
                        _p(np.ascontiguousarray(vt, dtype=np.float64)), _p(d))
        return d

    def c_co2contra(self, u, v):
        """co2contra_c_sbp<order>_new: contravariant (ut on x, vt on y) of covariant (u, v)."""
        _, sx, sy = self.c_shapes()
        ut, vt = np.zeros(sx), np.zeros(sy)
        lib().orc_c_co2contra(self._c, _p(np.ascontiguousarray(u, dtype=np.float64)),
                              _p(np.ascontiguousarray(v, dtype=np.float64)), _p(ut), _p(vt))
        return ut, vt

    def c_weights(self, mesh: int):
        """SBP quadrature weights J hx hy Ax Ay on the C meshes: 0 = o, 1 = x, 2 = y."""
        w = np.zeros(self.c_shapes()[mesh])
        lib().orc_c_weights(self._c, int(mesh), _p(w))
        return w

    def c_halo_probe(self, kind: int, f, f2=None, w: int = 3):
        """The C exchanges' halos: kind 0 o-point scalar (width 3), 1 C vector (width 3)."""
        N = self.N
        if kind == 0:
            out = np.zeros((6, N + 2 * w, N + 2 * w))
            lib().orc_c_halo_probe(self._c, 0, _p(np.ascontiguousarray(f, dtype=np.float64)), None, w, _p(out), None)
            return out
        o1 = np.zeros((6, N + 2 * w, N + 1 + 2 * w))
        o2 = np.zeros((6, N + 1 + 2 * w, N + 2 * w))
        lib().orc_c_halo_probe(self._c, 1, _p(np.ascontiguousarray(f, dtype=np.float64)),
                               _p(np.ascontiguousarray(f2, dtype=np.float64)), w, _p(o1), _p(o2))
        return o1, o2

    def set_orography(self, h_surf):
        """Orography of the advective operator (packed like h), or None."""
        if h_surf is None:
            lib().orc_set_orography(self._c, None)
        else:
            self._hs = np.ascontiguousarray(h_surf, dtype=np.float64)
            lib().orc_set_orography(self._c, _p(self._hs))

    def ts2(self, u0, h_mean, axis=(0.0, 0.0, 1.0), linear_mode=False):
        h, u, v = self.zeros()
        ax = np.ascontiguousarray(axis, dtype=np.float64)
        lib().orc_init_ts2(self._c, u0, h_mean, _p(ax), int(linear_mode), _p(h), _p(u), _p(v))
        return h, u, v

    def apply(self, h, u, v):
        dh, du, dv = self.zeros()
        lib().orc_apply(self._c, _p(np.ascontiguousarray(h)), _p(np.ascontiguousarray(u)),
                        _p(np.ascontiguousarray(v)), _p(dh), _p(du), _p(dv))
        return dh, du, dv

    def rk4(self, h, u, v, dt, nsteps=1):
        h, u, v = (np.array(x, dtype=np.float64, order="C") for x in (h, u, v))
        lib().orc_rk4(self._c, _p(h), _p(u), _p(v), dt, int(nsteps))
        return h, u, v

    def grad(self, h):
        _, gx, gy = self.zeros()
        lib().orc_grad(self._c, _p(np.ascontiguousarray(h)), _p(gx), _p(gy))
        return gx, gy

    def co2contra(self, u, v):
        _, ut, vt = self.zeros()
        lib().orc_co2contra(self._c, _p(np.ascontiguousarray(u)), _p(np.ascontiguousarray(v)), _p(ut), _p(vt))
        return ut, vt

    def coriolis(self, ut, vt):
        _, cu, cv = self.zeros()
        lib().orc_coriolis(self._c, _p(np.ascontiguousarray(ut)), _p(np.ascontiguousarray(vt)), _p(cu), _p(cv))
        return cu, cv

    def div(self, ut, vt):
        d, _, _ = self.zeros()
        lib().orc_div(self._c, _p(np.ascontiguousarray(ut)), _p(np.ascontiguousarray(vt)), _p(d))
        return d

    def integrals(self, h, u, v):
        m = ctypes.c_double()
        e = ctypes.c_double()
        lib().orc_integrals(self._c, _p(np.ascontiguousarray(h)), _p(np.ascontiguousarray(u)),
                            _p(np.ascontiguousarray(v)), ctypes.byref(m), ctypes.byref(e))
        return m.value, e.value

    def dot(self, mesh: int, a, b=None):
        a = np.ascontiguousarray(a, dtype=np.float64)
        if b is None:
            return lib().orc_dot(self._c, mesh, _p(a), None)
        return lib().orc_dot(self._c, mesh, _p(a), _p(np.ascontiguousarray(b, dtype=np.float64)))

    def metric(self, mesh: int, what: int):
        """mesh 0 xy, 1 y (u), 2 x (v), 3 o (centres); what 0 J, 1-3 Q1-Q3, 4 f J^2 (f on o),
        5-7 the unit position vector's x, y, z."""
        shp = (6, self.N, self.N) if mesh == 3 else shapes(self.N)[mesh]
        out = np.empty(shp)
        lib().orc_metric(self._c, mesh, what, _p(out))
        return out

    def sync_weights(self):
        n = self.N + 1
        qb, qt, ql, qr = (np.empty(n) for _ in range(4))
        lib().orc_sync_weights(self._c, _p(qb), _p(qt), _p(ql), _p(qr))
        return qb, qt, ql, qr

    def halo_probe(self, kind: int, f, f2=None, w: int = 3):
        """Run one reference exchange on packed field(s); return haloed arrays
        (6, ny+2w, nx+2w) with NaN where nothing was written."""
        N = self.N
        if kind in (0, 1):
            nx = ny = N + 1
            nx2, ny2 = nx, ny
        else:
            nx, ny, nx2, ny2 = N, N + 1, N + 1, N
        out = np.empty((6, ny + 2 * w, nx + 2 * w))
        out2 = np.empty((6, ny2 + 2 * w, nx2 + 2 * w))
        f = np.ascontiguousarray(f, dtype=np.float64)
        f2p = _p(np.ascontiguousarray(f2, dtype=np.float64)) if f2 is not None else None
        lib().orc_halo_probe(self._c, kind, _p(f), f2p, w, _p(out), _p(out2))
        return (out, out2) if kind != 0 else out


def sbp1d(op: int, n: int, x, order: int = 42) -> np.ndarray:
    """One-dimensional SBP operator (order 42, 21 or 63) on one line (0 i2c diff, 1 c2i diff,
    both without SAT, 2 i2c interpolation, 3 c2i interpolation)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    nout = n if op in (0, 2) else n + 1
    out = np.empty(nout)
    lib().orc_sbp1d_ord(int(order), op, n, _p(x), _p(out))
    return out

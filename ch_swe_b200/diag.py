"""Diagnostics and output of a shallow-water state: the swm_output_diag_t checks
(CFL numbers, h extrema, mass, energies, enstrophy, curl), the lat-lon outputer of h
and the paneled single-precision writer
(src/models/shallow_water/output_and_diag/swm_output_diag_mod.f90,
src/outputer/latlon_outputer_mod.f90, src/outputer/master_paneled_outputer_mod.f90)."""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from ._lib import check


class SwmOutputDiag:
    """swm_output_diag_t for a device state: print_CFL_diag and the h extrema and
    mass of print_integrals_diag (swm_output_diag_mod.f90:110-171)."""

    def __init__(self, domain):
        self.domain = domain

    def diagnostics(self, state, dt: float, member: int = 0) -> dict:
        """h_min, h_max, the gravity-wave CFL and the advective CFL numbers (x, y)."""
        out = (ctypes.c_double * 5)()
        check(_lib.load().swe_diag(self.domain.ctx, state.handle, int(member), float(dt), out), self.domain.ctx,
              "swe_diag")
        return {"h_min": out[0], "h_max": out[1], "cfl_gravity": out[2], "cfl_adv_x": out[3], "cfl_adv_y": out[4]}

    def calc_energies(self, state, member: int = 0) -> dict:
        """TE, KE, PE and the potential enstrophy of calc_energies (swm_output_diag_mod.f90:186-234)
        for covariant (u, v), computed on the device in FP64."""
        out = (ctypes.c_double * 4)()
        check(_lib.load().swe_energies(self.domain.ctx, state.handle, int(member), out), self.domain.ctx,
              "swe_energies")
        return {"te": out[0], "ke": out[1], "pe": out[2], "enstrophy": out[3]}

    def curl(self, state, member: int = 0) -> np.ndarray:
        """Curl of the covariant (u, v) on the cell centres (curl_ch_sbp_sat_*): (6, N, N), FP64."""
        N = self.domain.N
        out = np.empty((6, N, N))
        check(_lib.load().swe_curl(self.domain.ctx, state.handle, int(member),
                                   out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), self.domain.ctx, "swe_curl")
        return out

    def print_integrals_diag(self, state, member: int = 0) -> str:
        """The line of print_integrals_diag (swm_output_diag_mod.f90:155-183): h extrema, mass,
        TE, KE, PE and enstrophy."""
        d = self.diagnostics(state, 0.0, member)
        mass, _ = state_integrals(self.domain, state, member)
        e = self.calc_energies(state, member)
        vals = [("hmin = ", d["h_min"]), (" hmax = ", d["h_max"]), (" mass = ", mass), (" TE = ", e["te"]),
                (" KE = ", e["ke"]), (" PE = ", e["pe"]), (" Enstrophy = ", e["enstrophy"])]
        line = "".join(f"{k}{v:24.16E}" for k, v in vals)
        print(line)
        return line

    def print_cfl_diag(self, state, dt: float, member: int = 0) -> str:
        d = self.diagnostics(state, dt, member)
        line = (f"Gravity waves CFL-max = {d['cfl_gravity']:15.7f}, Advective CFL-max (x,y) = "
                f"{d['cfl_adv_x']:15.7f}{d['cfl_adv_y']:15.7f}")
        print(line)
        return line


def state_integrals(domain, state, member: int = 0):
    """(mass, linear energy) of swe_integrals for one member."""
    m = ctypes.c_double()
    e = ctypes.c_double()
    check(_lib.load().swe_integrals(domain.ctx, state.handle, int(member), ctypes.byref(m), ctypes.byref(e)),
          domain.ctx, "swe_integrals")
    return m.value, e.value


class LatlonOutputer:
    """latlon_outputer_t for h (latlon_outputer_mod.f90:30-53): the cubic regrid on the
    device (swe_regrid_latlon) onto nlat x nlon points (default 2N+1 x 4N, as
    create_swm_output_diag sets them) and one real*4 direct-access record per write."""

    def __init__(self, domain, nlat: int | None = None, nlon: int | None = None):
        self.domain = domain
        self.nlat = 2 * domain.N + 1 if nlat is None else int(nlat)
        self.nlon = 4 * domain.N if nlon is None else int(nlon)

    def regrid(self, state, member: int = 0) -> np.ndarray:
        """h on the lat-lon grid, (nlat, nlon) in FP64, longitude fastest."""
        out = np.empty((self.nlat, self.nlon))
        check(_lib.load().swe_regrid_latlon(self.domain.ctx, state.handle, int(member), 0, self.nlat, self.nlon,
                                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
              self.domain.ctx, "swe_regrid_latlon")
        return out

    def write(self, state, path: str, rec: int = 1, member: int = 0) -> np.ndarray:
        """Record rec (1-based) of `path`: the regridded h as real*4, longitude fastest."""
        f = self.regrid(state, member)
        write_latlon(path, f, rec)
        return f

    def regrid_div(self, state, member: int = 0) -> np.ndarray:
        """The divergence of the wind (the div.dat field of output_div: the model's
        div_ch_sbp_sat_<order>_proj of the contravariant wind) on the lat-lon grid."""
        out = np.empty((self.nlat, self.nlon))
        check(_lib.load().swe_regrid_latlon(self.domain.ctx, state.handle, int(member), 1, self.nlat, self.nlon,
                                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
              self.domain.ctx, "swe_regrid_latlon (div)")
        return out

    def regrid_curl(self, state, member: int = 0) -> np.ndarray:
        """The curl of the covariant wind (the curl.dat field of output_curl:
        curl_ch_sbp_sat_<order> on the cell centres, regridded from the ECS_O halo) on
        the lat-lon grid."""
        out = np.empty((self.nlat, self.nlon))
        check(_lib.load().swe_regrid_latlon(self.domain.ctx, state.handle, int(member), 2, self.nlat, self.nlon,
                                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
              self.domain.ctx, "swe_regrid_latlon (curl)")
        return out


class LatlonVecOutputer:
    """latlon_vec_outputer_t for the covariant Ch wind (latlon_outputer_mod.f90:55-85): the
    regrid on the device (swe_regrid_latlon_wind) to eastward / northward components on
    nlat x nlon points (default 2N+1 x 4N) and one real*4 record per file per write."""

    def __init__(self, domain, nlat: int | None = None, nlon: int | None = None):
        self.domain = domain
        self.nlat = 2 * domain.N + 1 if nlat is None else int(nlat)
        self.nlon = 4 * domain.N if nlon is None else int(nlon)

    def regrid(self, state, member: int = 0):
        """(u, v) on the lat-lon grid, each (nlat, nlon) in FP64, longitude fastest."""
        u = np.empty((self.nlat, self.nlon))
        v = np.empty((self.nlat, self.nlon))
        dp = ctypes.POINTER(ctypes.c_double)
        check(_lib.load().swe_regrid_latlon_wind(self.domain.ctx, state.handle, int(member), self.nlat, self.nlon,
                                                 u.ctypes.data_as(dp), v.ctypes.data_as(dp)),
              self.domain.ctx, "swe_regrid_latlon_wind")
        return u, v

    def write(self, state, path_u: str, path_v: str, rec: int = 1, member: int = 0):
        u, v = self.regrid(state, member)
        write_latlon(path_u, u, rec)
        write_latlon(path_v, v, rec)
        return u, v


def write_latlon(path: str, field: np.ndarray, rec: int = 1) -> None:
    """One record of latlon_outputer_t%write: real(f_latlon, 4) with f_latlon(Nlon, Nlat),
    longitude fastest, record length nlat * nlon values.  field: (nlat, nlon)."""
    a = np.ascontiguousarray(field, dtype="<f4")
    if a.ndim != 2:
        raise ValueError("expected a (nlat, nlon) field")
    mode = "r+b" if os.path.exists(path) else "wb"
    with open(path, mode) as f:
        f.seek((int(rec) - 1) * a.nbytes)
        f.write(a.tobytes())


def write_paneled(path: str, field: np.ndarray, rec: int = 1) -> None:
    """master_paneled_outputer_t%write for one level: record rec (1-based) of a
    direct-access file holds the six panels of the field as real*4, i fastest, then j,
    then panel (master_paneled_outputer_mod.f90:32-77).  field: (6, ny, nx)."""
    a = np.ascontiguousarray(field, dtype="<f4")
    if a.ndim != 3 or a.shape[0] != 6:
        raise ValueError("expected a (6, ny, nx) panel field")
    reclen = a.nbytes
    mode = "r+b" if os.path.exists(path) else "wb"
    with open(path, mode) as f:
        f.seek((int(rec) - 1) * reclen)
        f.write(a.tobytes())


def read_paneled(path: str, shape, rec: int = 1) -> np.ndarray:
    """Record rec of a file written by write_paneled (or by the reference's writer)."""
    shape = tuple(shape)
    n = int(np.prod(shape))
    with open(path, "rb") as f:
        f.seek((int(rec) - 1) * n * 4)
        return np.frombuffer(f.read(n * 4), dtype="<f4").reshape(shape).copy()

"""Host-side mirror of the reference's operator_t / stvec_t / timescheme_t API for
the shallow-water hot path, backed by libchswe.so.

Names, arguments and error behaviour follow the reference (paths relative to the
ch_swe source tree):

* ``create_domain``        ~ create_domain            (src/domain/domain_factory_mod.f90:55-147)
* ``create_stvec_swm``     ~ create_stvec_swm         (src/models/shallow_water/stvec/stvec_swm_factory_mod.f90:15-36)
* ``StvecSwm.assign/update`` ~ stvec_t%assign/update  (src/stvec/stvec_flexible_mod.f90:196-306)
* ``create_swm_operator``  ~ create_swm_operator      (src/models/shallow_water/operator/operator_swm_factory_mod.f90:14-57)
* ``OperatorSwmLin.apply`` ~ operator_swm_lin_t%apply (.../operator_swm_lin_mod.f90:66-108)
* ``create_timescheme``    ~ create_timescheme        (src/time_schemes/timescheme_factory_mod.f90:21-52)
* ``Rk4.step``             ~ rk4_t%step               (src/time_schemes/rk4_mod.f90:20-42)

Where the reference calls ``parcomm_global%abort`` these raise ``SweError``
(device/library failures) or ``ValueError`` (unknown names, bad configuration).
Host arrays use the packed per-panel Fortran layout documented in include/chswe.h.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import SweCfg, SweError, check, dptr

EARTH_RADIUS = 0.6371229e7                                   # const_mod.f90:7
EARTH_GRAV = 9.80616                                         # const_mod.f90:6
EARTH_OMEGA = 2.0 * np.pi / (23 * 60 * 60 + 56 * 60 + 4)     # const_mod.f90:8-9

# operator names accepted by the Ch / SBP 4-2 linear operator (gen_config_linear.sh:37-64)
LINEAR_CH42_NAMES = {
    "div_op_name": "div_ch_sbp_sat_42_proj",
    "grad_op_name": "grad_ch_sbp_sat_42",
    "coriolis_op_name": "coriolis_Ch_sbp42",
    "co2contra_op_name": "co2contra_ch_sbp42",
    "quadrature_name": "SBP_C42_quadrature",
}
# the same operator with the SBP 2-1 Ch operators (the _21 names of the same factories)
LINEAR_CH21_NAMES = {
    "div_op_name": "div_ch_sbp_sat_21_proj",
    "grad_op_name": "grad_ch_sbp_sat_21",
    "coriolis_op_name": "coriolis_Ch_sbp21",
    "co2contra_op_name": "co2contra_ch_sbp21",
    "quadrature_name": "SBP_C21_quadrature",
}
# ... and with the SBP 6-3 Ch operators (the _63 names)
LINEAR_CH63_NAMES = {
    "div_op_name": "div_ch_sbp_sat_63_proj",
    "grad_op_name": "grad_ch_sbp_sat_63",
    "coriolis_op_name": "coriolis_Ch_sbp63",
    "co2contra_op_name": "co2contra_ch_sbp63",
    "quadrature_name": "SBP_C63_quadrature",
}
LINEAR_NAMES_BY_ORDER = {42: LINEAR_CH42_NAMES, 21: LINEAR_CH21_NAMES, 63: LINEAR_CH63_NAMES}
# the linear operator on the Ah staggering (gen_config_linear.sh:9-36), per SBP order
LINEAR_AH_NAMES_BY_ORDER = {
    order: {
        "div_op_name": f"div_ah_sbp_proj_{order}",
        "grad_op_name": f"grad_ah_sbp_proj_{order}",
        "coriolis_op_name": "coriolis_colocated",
        "co2contra_op_name": "co2contra_colocated",
        "quadrature_name": f"SBP_Ah{order}_quadrature",
    }
    for order in (42, 21, 63)
}
LINEAR_AH42_NAMES = LINEAR_AH_NAMES_BY_ORDER[42]
STAGGERINGS = {"Ch": _lib.SWE_STAG_CH, "Ah": _lib.SWE_STAG_AH, "C": _lib.SWE_STAG_C}
# advective_swm_operator, covariant Ch (gen_config.sh Ch template with UPSTREAM_ORDER up4),
# per SBP order of its Ch operators
ADVECTIVE_NAMES_BY_ORDER = {
    order: dict(names, vector_advection_op_name="vector_advection_Ch_up4_cov", massflux_op_name="massflux_ch_up4")
    for order, names in LINEAR_NAMES_BY_ORDER.items()
}
ADVECTIVE_CH42_NAMES = ADVECTIVE_NAMES_BY_ORDER[42]
OPERATORS = {"linear": _lib.SWE_OP_LINEAR, "advective": _lib.SWE_OP_ADVECTIVE}


def state_shapes(N: int, members: int | None = None, staggering: str = "Ch"):
    """Packed host shapes of (h, u, v) for one member (or a batch of members): on Ch,
    h on the vertices, u on the y points, v on the x points; on Ah all on the vertices;
    on C h on the cell centres, u on the x points, v on the y points."""
    if staggering == "Ah":
        sh = [(6, N + 1, N + 1)] * 3
    elif staggering == "C":
        # h on the cell centres, u on the x points, v on the y points
        sh = [(6, N, N), (6, N, N + 1), (6, N + 1, N)]
    else:
        sh = [(6, N + 1, N + 1), (6, N + 1, N), (6, N, N + 1)]
    if members is None:
        return tuple(sh)
    return tuple((members,) + s for s in sh)


@dataclass
class Domain:
    """Cubed-sphere domain with Ch (default) or Ah staggering; owns the device context."""
    N: int
    precision: str = "fp64"
    n_members: int = 1
    planet_radius: float = EARTH_RADIUS
    omega: float = EARTH_OMEGA
    rotation_axis: tuple = (0.0, 0.0, 1.0)
    coriolis_constant: bool = False
    grav: float = EARTH_GRAV
    h_mean: float = 1000.0
    horizontal_staggering: str = "Ch"
    operator: str = "linear"          # the operator the context runs: 'linear' or 'advective'
    sbp_order: int = 42               # SBP order of the Ch operators: 42, or 21 / 63 (linear operator)
    _ctx: int = field(default=None, repr=False)

    def __post_init__(self):
        if self.horizontal_staggering not in STAGGERINGS:
            raise ValueError("domain_factory_mod, unsupported horizontal staggering: " + self.horizontal_staggering)
        if self.horizontal_staggering in ("Ah", "C") and self.operator != "linear":
            raise ValueError(f"the {self.horizontal_staggering} staggering is built for the linear operator")
        if self.horizontal_staggering == "C" and self.sbp_order != 42:
            raise ValueError("the C staggering is built for SBP 4-2")
        if self.precision not in ("fp64", "fp32"):
            raise ValueError("precision must be 'fp64' or 'fp32'")
        if self.operator not in OPERATORS:
            raise ValueError(f"operator must be one of {sorted(OPERATORS)}")
        if self.sbp_order not in (42, 21, 63):
            raise ValueError("sbp_order must be 42, 21 or 63")
        if self.sbp_order == 63 and self.N < 16:
            raise ValueError("SBP 6-3 needs N >= 16")
        L = _lib.load()
        cfg = SweCfg()
        check(L.swe_cfg_default(ctypes.byref(cfg)))
        cfg.N = int(self.N)
        cfg.precision = _lib.SWE_FP64 if self.precision == "fp64" else _lib.SWE_FP32
        cfg.n_members = int(self.n_members)
        cfg.radius = float(self.planet_radius)
        cfg.grav = float(self.grav)
        cfg.omega = float(self.omega)
        for d in range(3):
            cfg.rotation_axis[d] = float(self.rotation_axis[d])
        cfg.coriolis_constant = int(bool(self.coriolis_constant))
        cfg.h_mean = float(self.h_mean)
        cfg.operator_kind = OPERATORS[self.operator]
        cfg.sbp_order = int(self.sbp_order)
        cfg.staggering = STAGGERINGS[self.horizontal_staggering]
        ctx = ctypes.c_void_p()
        check(L.swe_ctx_create(ctypes.byref(cfg), ctypes.byref(ctx)), None, "swe_ctx_create")
        self._ctx = ctx.value

    @property
    def ctx(self):
        if not self._ctx:
            raise SweError("domain was destroyed")
        return self._ctx

    def synchronize(self):
        check(_lib.load().swe_synchronize(self.ctx), self.ctx, "swe_synchronize")

    def launch_count(self) -> int:
        return int(_lib.load().swe_launch_count(self.ctx))

    def set_stream(self, stream_ptr: int | None):
        check(_lib.load().swe_set_stream(self.ctx, stream_ptr), self.ctx, "swe_set_stream")

    # tile size of the stage kernels (17, 25 or 33) and its autotuner
    TILES = (17, 25, 33)

    @property
    def tile(self) -> int:
        t = ctypes.c_int()
        check(_lib.load().swe_get_tile(self.ctx, ctypes.byref(t)), self.ctx, "swe_get_tile")
        return t.value

    @tile.setter
    def tile(self, value: int):
        check(_lib.load().swe_set_tile(self.ctx, int(value)), self.ctx, "swe_set_tile")

    # built stage-kernel configurations: (tile edge, resident blocks per SM, runs)
    KERNEL_CONFIGS = tuple((t, o, r) for r in (0, 1)
                           for t, o in ((17, 3), (17, 4), (25, 2), (25, 3), (25, 4), (33, 2), (33, 3)))
    # the fused stage (linear operator, Ch, SBP 4-2): (maximal tile rows, blocks per SM, 2)
    FUSED_CONFIGS = {"fp32": ((17, 4, 2), (25, 3, 2), (33, 2, 2)), "fp64": ((17, 2, 2), (25, 1, 2))}

    @property
    def kernel_config(self) -> tuple:
        """(tile edge, resident blocks per SM, runs) of the stage kernels; runs 1: each
        thread evaluates runs of consecutive outputs along a stencil; runs 2: the fused
        stage (contravariant components computed in the stage kernel, TMA-loaded tiles of
        at most 26 columns and `tile` rows)."""
        t, o, r = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(_lib.load().swe_get_kernel_config(self.ctx, ctypes.byref(t), ctypes.byref(o), ctypes.byref(r)),
              self.ctx, "swe_get_kernel_config")
        return t.value, o.value, r.value

    @kernel_config.setter
    def kernel_config(self, value):
        """(tile, blocks per SM) or (tile, blocks per SM, runs); runs defaults to 0."""
        runs = int(value[2]) if len(value) > 2 else 0
        check(_lib.load().swe_set_kernel_config(self.ctx, int(value[0]), int(value[1]), runs), self.ctx,
              "swe_set_kernel_config")

    def autotune(self, nreps: int = 20) -> dict:
        """Time RK4 steps for every tile size, keep the fastest; returns {tile: ms per step}."""
        best = ctypes.c_int()
        ms = (ctypes.c_double * 3)()
        check(_lib.load().swe_autotune(self.ctx, int(nreps), ctypes.byref(best), ms), self.ctx, "swe_autotune")
        return {t: ms[k] for k, t in enumerate(self.TILES)}

    def set_diffusion(self, operator=None):
        """The driver loop's diffusion (shallow_water_mod.f90:112-118) inside the RK4 steps:
        every RK4 step of this domain is followed by one explicit_Eul1 step of the
        OperatorSwmDiff with the same dt, captured in the same graphs; None turns it off."""
        if operator is None:
            rc = _lib.load().swe_set_diffusion(self.ctx, 0, 0.0, 0.0)
        else:
            rc = _lib.load().swe_set_diffusion(self.ctx, operator.lap_order, operator.uv_coeff, operator.h_coeff)
        check(rc, self.ctx, "set diffusion")

    def destroy(self):
        if self._ctx:
            _lib.load().swe_ctx_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def create_domain(N: int, **kw) -> Domain:
    return Domain(N=N, **kw)


class StvecSwm:
    """stvec_swm_t on the device: fields h (xy), u (y), v (x) for every member."""

    def __init__(self, domain: Domain):
        self.domain = domain
        p = ctypes.c_void_p()
        check(_lib.load().swe_stvec_create(domain.ctx, ctypes.byref(p)), domain.ctx, "swe_stvec_create")
        self._p = p.value

    @property
    def handle(self):
        return self._p

    def __del__(self):
        p = getattr(self, "_p", None)
        try:
            if p and self.domain._ctx:
                _lib.load().swe_stvec_destroy(p)
                self._p = None
        except Exception:   # interpreter shutdown: the module globals may be gone already
            pass

    # -- transfers ------------------------------------------------------
    def upload(self, h, u, v, member: int | None = 0):
        N, stag = self.domain.N, self.domain.horizontal_staggering
        arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (h, u, v)]
        L = _lib.load()
        if member is None:
            for a, s in zip(arrs, state_shapes(N, self.domain.n_members, stag)):
                if a.shape != s:
                    raise ValueError(f"expected shape {s}, got {a.shape}")
            rc = L.swe_stvec_upload_all(self._p, *(dptr(a) for a in arrs))
        else:
            for a, s in zip(arrs, state_shapes(N, None, stag)):
                if a.shape != s:
                    raise ValueError(f"expected shape {s}, got {a.shape}")
            rc = L.swe_stvec_upload(self._p, int(member), *(dptr(a) for a in arrs))
        check(rc, self.domain.ctx, "swe_stvec_upload")
        return self

    def download(self, member: int | None = 0):
        N, stag = self.domain.N, self.domain.horizontal_staggering
        L = _lib.load()
        if member is None:
            out = [np.empty(s) for s in state_shapes(N, self.domain.n_members, stag)]
            rc = L.swe_stvec_download_all(self._p, *(dptr(a) for a in out))
        else:
            out = [np.empty(s) for s in state_shapes(N, None, stag)]
            rc = L.swe_stvec_download(self._p, int(member), *(dptr(a) for a in out))
        check(rc, self.domain.ctx, "swe_stvec_download")
        return tuple(out)

    # -- stvec algebra (stvec_flexible_mod.f90:196-306) ------------------
    def assign(self, s1, v1, s2=None, v2=None, domain=None):
        self._check(v1, v2)
        rc = _lib.load().swe_stvec_assign(self._p, float(s1), v1._p, float(s2 or 0.0), v2._p if v2 else None)
        check(rc, self.domain.ctx, "stvec assign")
        return self

    def update(self, s1, v1, s2=None, v2=None, domain=None):
        self._check(v1, v2)
        rc = _lib.load().swe_stvec_update(self._p, float(s1), v1._p, float(s2 or 0.0), v2._p if v2 else None)
        check(rc, self.domain.ctx, "stvec update")
        return self

    def create_similar(self) -> "StvecSwm":
        return StvecSwm(self.domain)

    def copy_to(self, dst: "StvecSwm", domain=None):
        dst.assign(1.0, self)
        return dst

    def device_view(self):
        ptr = ctypes.c_void_p()
        nb = ctypes.c_size_t()
        prec = ctypes.c_int()
        pitch = ctypes.c_int()
        check(_lib.load().swe_stvec_device_view(self._p, ctypes.byref(ptr), ctypes.byref(nb), ctypes.byref(prec),
                                                ctypes.byref(pitch)), self.domain.ctx, "device_view")
        return ptr.value, nb.value, prec.value, pitch.value

    def _check(self, v1, v2):
        for v in (v1, v2):
            if v is not None and (not isinstance(v, StvecSwm) or v.domain is not self.domain):
                raise ValueError("stvec algebra between different domains")


def create_stvec_swm(domain: Domain, halo_width: int = 8, halo_width_z: int = 0) -> StvecSwm:
    """Halo widths are accepted for interface parity; device states carry no halo."""
    return StvecSwm(domain)


class OperatorSwmLin:
    """operator_swm_lin_t: linear SWE on the Ch grid with SBP 4-2 operators."""

    def __init__(self, domain: Domain, h_mean: float, grav: float):
        self.domain = domain
        self.h_mean = float(h_mean)
        self.grav = float(grav)
        for m in range(domain.n_members):
            check(_lib.load().swe_set_member_h_mean(domain.ctx, m, self.h_mean), domain.ctx, "h_mean")

    def set_member_h_mean(self, member: int, h_mean: float):
        check(_lib.load().swe_set_member_h_mean(self.domain.ctx, int(member), float(h_mean)),
              self.domain.ctx, "h_mean")

    def apply(self, vout: StvecSwm, vin: StvecSwm, domain: Domain | None = None):
        if not isinstance(vout, StvecSwm):
            raise ValueError("swm operator failure: vout of wrong type")
        if not isinstance(vin, StvecSwm):
            raise ValueError("swm operator failure: vin of wrong type")
        check(_lib.load().swe_operator_apply(self.domain.ctx, vout.handle, vin.handle), self.domain.ctx,
              "operator apply")

    def contravariant(self, vout: StvecSwm, vin: StvecSwm, domain: Domain | None = None):
        """vout.u, vout.v = contravariant components of vin (co2contra_operator_t%transform)."""
        check(_lib.load().swe_operator_contravariant(self.domain.ctx, vout.handle, vin.handle), self.domain.ctx,
              "co2contra")

    def integrals(self, state: StvecSwm, member: int = 0):
        """FP64 SBP-quadrature mass and linear energy of one member."""
        m = ctypes.c_double()
        e = ctypes.c_double()
        check(_lib.load().swe_integrals(self.domain.ctx, state.handle, int(member), ctypes.byref(m),
                                        ctypes.byref(e)), self.domain.ctx, "integrals")
        return m.value, e.value


def create_swm_operator(grav: float, config: dict, domain: Domain, orography_generator=None):
    """operator_swm_factory_mod.f90:33-55: 'linear_swm_operator' or 'advective_swm_operator'
    (covariant Ch, up4 mass flux and vector advection).  The operator kind is fixed
    when the domain's device context is created (create_domain(..., operator=...))."""
    kind = config.get("swm_operator_type")
    if kind == "linear_swm_operator":
        if "h_mean" not in config:
            raise ValueError("linear_swm_operator requires h_mean")
        names, want_op = LINEAR_NAMES_BY_ORDER[domain.sbp_order], "linear"
        if domain.horizontal_staggering == "Ah":
            names = LINEAR_AH_NAMES_BY_ORDER[domain.sbp_order]
    elif kind == "advective_swm_operator":
        if config.get("v_components_type", "covariant") != "covariant":
            raise ValueError("advective_swm_operator: only v_components_type = 'covariant' is built for Ch")
        names, want_op = ADVECTIVE_NAMES_BY_ORDER[domain.sbp_order], "advective"
    else:
        raise ValueError(f"unknown swm_op_type: {kind}")
    for key, want in names.items():
        got = config.get(key, want)
        if got != want:
            for order, ah in LINEAR_AH_NAMES_BY_ORDER.items():
                if want_op == "linear" and got == ah.get(key) and domain.horizontal_staggering != "Ah":
                    raise ValueError(f"{key} = {got} needs a domain created with horizontal_staggering='Ah'")
                if want_op == "linear" and got == ah.get(key) and domain.sbp_order != order:
                    raise ValueError(f"{key} = {got} needs a domain created with sbp_order={order}")
            for order, other in LINEAR_NAMES_BY_ORDER.items():
                if got == other.get(key):
                    raise ValueError(f"{key} = {got} needs a domain created with sbp_order={order}")
            raise ValueError(f"unsupported {key}: {got} (this build implements {want})")
    if domain.operator != want_op:
        raise ValueError(f"{kind} needs a domain created with operator='{want_op}' (got '{domain.operator}')")
    if abs(float(grav) - domain.grav) > 0.0:
        raise ValueError(f"grav {grav} differs from the domain's {domain.grav}")
    if want_op == "advective":
        op = OperatorSwmAdv(domain, grav)
        if orography_generator is not None:
            op.set_orography(orography_generator)
        return op
    if orography_generator is not None:
        raise ValueError("linear_swm_operator has no orography")
    return OperatorSwmLin(domain, config["h_mean"], grav)


class OperatorSwmAdv(OperatorSwmLin):
    """operator_adv_swm_t, covariant Ch branch: h is the full depth (no mean depth)."""

    def __init__(self, domain: Domain, grav: float):
        self.domain = domain
        self.h_mean = None
        self.grav = float(grav)

    def set_member_h_mean(self, member: int, h_mean: float):
        raise ValueError("the advective operator has no mean depth")

    def set_orography(self, orography):
        """h_surf of the operator (set_scalar_test_field(h_surf, orography_generator, mesh_p),
        operator_swm_factory_mod.f90:365-366): a generator with get_scalar_field(x, y, z)
        on the unit sphere (testcases.Ts5Orography), or an array packed like h; None
        removes it."""
        if orography is None:
            check(_lib.load().swe_set_orography(self.domain.ctx, None), self.domain.ctx, "orography")
            return
        if hasattr(orography, "get_scalar_field"):
            from .testcases import mesh_geometry
            r, _, _ = mesh_geometry(self.domain.N, "xy")
            hs = orography.get_scalar_field(r[..., 0], r[..., 1], r[..., 2])
        else:
            hs = orography
        hs = np.ascontiguousarray(hs, dtype=np.float64)
        if hs.shape != state_shapes(self.domain.N)[0]:
            raise ValueError(f"orography shape {hs.shape}, need {state_shapes(self.domain.N)[0]}")
        check(_lib.load().swe_set_orography(self.domain.ctx, dptr(hs)), self.domain.ctx, "orography")


# ---------------------------------------------------------------------------
# C staggering: the C-grid operators the reference runs (its linear operator on C aborts in
# coriolis_Cgrid_t%calc_coriolis, coriolis_Cgrid_mod.f90:28-37)
# ---------------------------------------------------------------------------
C_OPERATOR_NAMES = {"grad": "grad_c_sbp_sat_42", "div": "div_c_sbp_sat_42", "co2contra": "co2contra_c_sbp42_new"}


def _need_c(domain: Domain, name: str):
    if domain.horizontal_staggering != "C":
        raise ValueError(f"{name} needs a domain created with horizontal_staggering='C'")


class GradC:
    """grad_c_sbp_sat_42 (grad_factory_mod.f90:115-150, grad_sbp_sat_mod.f90:24-76)."""

    def __init__(self, domain: Domain):
        _need_c(domain, C_OPERATOR_NAMES["grad"])
        self.domain = domain

    def calc_grad(self, out: StvecSwm, src: StvecSwm):
        """out.u, out.v (x, y points) = gradient of src.h (cell centres)."""
        check(_lib.load().swe_c_grad(self.domain.ctx, out.handle, src.handle), self.domain.ctx, "grad_c")


class DivC:
    """div_c_sbp_sat_42 (div_factory_mod.f90:112-156, div_sbp_sat_mod.f90:29-80)."""

    def __init__(self, domain: Domain):
        _need_c(domain, C_OPERATOR_NAMES["div"])
        self.domain = domain

    def calc_div(self, out: StvecSwm, src: StvecSwm):
        """out.h (cell centres) = divergence of the contravariant (src.u, src.v)."""
        check(_lib.load().swe_c_div(self.domain.ctx, out.handle, src.handle), self.domain.ctx, "div_c")


class Co2ContraC:
    """co2contra_c_sbp42_new (co2contra_Cgrid_mod.f90, transform_co2contra_c_sbp_new)."""

    def __init__(self, domain: Domain):
        _need_c(domain, C_OPERATOR_NAMES["co2contra"])
        self.domain = domain

    def transform(self, out: StvecSwm, src: StvecSwm):
        """out.u, out.v = contravariant components of the covariant (src.u, src.v)."""
        check(_lib.load().swe_operator_contravariant(self.domain.ctx, out.handle, src.handle), self.domain.ctx,
              "co2contra_c")


def create_grad_operator(domain: Domain, name: str):
    if name != C_OPERATOR_NAMES["grad"]:
        raise ValueError(f"unknown C-grid gradient {name!r} (this build implements {C_OPERATOR_NAMES['grad']})")
    return GradC(domain)


def create_div_operator(domain: Domain, name: str):
    if name != C_OPERATOR_NAMES["div"]:
        raise ValueError(f"unknown C-grid divergence {name!r} (this build implements {C_OPERATOR_NAMES['div']})")
    return DivC(domain)


def create_co2contra_operator(domain: Domain, name: str):
    if name != C_OPERATOR_NAMES["co2contra"]:
        raise ValueError(f"unknown C-grid co2contra {name!r} (this build implements {C_OPERATOR_NAMES['co2contra']})")
    return Co2ContraC(domain)


class Rk4:
    """rk4_t: classic RK4 with k1..k4 fused into per-stage device kernels."""

    def step(self, v0: StvecSwm, operator: OperatorSwmLin, domain: Domain | None, dt: float):
        check(_lib.load().swe_rk4_step(operator.domain.ctx, v0.handle, float(dt)), operator.domain.ctx, "rk4 step")

    def steps(self, v0: StvecSwm, operator: OperatorSwmLin, domain: Domain | None, dt: float, nsteps: int):
        check(_lib.load().swe_rk4_steps(operator.domain.ctx, v0.handle, float(dt), int(nsteps)),
              operator.domain.ctx, "rk4 steps")

    def steps_members(self, v0: StvecSwm, operator: OperatorSwmLin, dt_per_member, nsteps: int):
        """nsteps steps with one dt per member; dt 0 freezes a member (continuous batching)."""
        dts = np.ascontiguousarray(dt_per_member, dtype=np.float64)
        if dts.shape != (operator.domain.n_members,):
            raise ValueError(f"need {operator.domain.n_members} time steps, got shape {dts.shape}")
        check(_lib.load().swe_rk4_steps_members(operator.domain.ctx, v0.handle, dptr(dts), int(nsteps)),
              operator.domain.ctx, "rk4 steps (members)")


class DomainGroup:
    """The RK4 steps of several domains (cube sizes and member counts of their own, one
    precision, the linear operator on Ch in SBP 4-2, one split kernel configuration)
    as one grid per kernel: twelve launches per step for the whole group, on the first
    domain's stream.  Each domain gets the bits its own Rk4.steps_members gives with
    the same configuration."""

    def __init__(self, domains):
        self.domains = list(domains)
        arr = (ctypes.c_void_p * len(self.domains))(*[d.ctx for d in self.domains])
        h = ctypes.c_void_p()
        check(_lib.load().swe_group_create(arr, len(self.domains), ctypes.byref(h)), self.domains[0].ctx,
              "group create")
        self.handle = h

    def _check(self, rc: int, what: str):
        if rc != _lib.SWE_OK:
            detail = _lib.load().swe_group_last_error(self.handle)
            raise SweError(f"{what}: {_lib.ERRORS.get(rc, rc)}: {detail.decode() if detail else ''}")

    def steps_members(self, states, dts, nsteps: int):
        """nsteps RK4 steps of states[k] (of domain k) with the per-member time steps
        dts[k]; a time step of 0 freezes a member."""
        if len(states) != len(self.domains) or len(dts) != len(self.domains):
            raise ValueError(f"need {len(self.domains)} states and time-step arrays")
        keep = [np.ascontiguousarray(x, dtype=np.float64) for x in dts]
        for d, x in zip(self.domains, keep):
            if x.shape != (d.n_members,):
                raise ValueError(f"need {d.n_members} time steps, got shape {x.shape}")
        sv = (ctypes.c_void_p * len(states))(*[st.handle for st in states])
        dv = (_lib._dp * len(keep))(*[dptr(x) for x in keep])
        self._check(_lib.load().swe_group_rk4_steps_members(self.handle, sv, dv, int(nsteps)), "group steps")

    def synchronize(self):
        self._check(_lib.load().swe_group_synchronize(self.handle), "group synchronize")

    @property
    def launches(self) -> int:
        return int(_lib.load().swe_group_launch_count(self.handle))

    def destroy(self):
        if self.handle:
            _lib.load().swe_group_destroy(self.handle)
            self.handle = None


def create_group(domains) -> DomainGroup:
    return DomainGroup(domains)


class OperatorSwmDiff:
    """operator_swm_diff_t (operator_swm_diff_mod.f90:27-49): hordiff_uv on (u, v) and hordiff
    on h, the narrow-Laplacian diffusion of the Ah staggering."""

    def __init__(self, domain: Domain, lap_order: int, uv_coeff: float, h_coeff: float):
        self.domain = domain
        self.lap_order = int(lap_order)
        self.uv_coeff = float(uv_coeff)
        self.h_coeff = float(h_coeff)

    def apply(self, vout: StvecSwm, vin: StvecSwm, domain: Domain | None = None):
        if not isinstance(vout, StvecSwm) or not isinstance(vin, StvecSwm):
            raise ValueError("swm operator failure: vin or vout of wrong type")
        check(_lib.load().swe_diffusion_apply(self.domain.ctx, vout.handle, vin.handle, self.lap_order,
                                              self.uv_coeff, self.h_coeff), self.domain.ctx, "diffusion apply")


def create_swm_diff_operator(config: dict, domain: Domain) -> OperatorSwmDiff:
    """operator_swm_diff_factory_mod.f90:11-36 with the hordiff names of the Ah staggering
    (hordiff_factory_mod.f90:33-44,61-68): hordiff_uv_name 'hordiff_vec_xyz_Ah_sbp_<o>_narrow'
    with uv_diff_coeff, hordiff_h_name 'hordiff_scalar_Ah_sbp_<o>_narrow' with h_diff_coeff,
    o = 21, 42 or 63, the same for both."""
    if domain.horizontal_staggering != "Ah":
        raise ValueError("the narrow-Laplacian diffusion operators need a domain created with "
                         "horizontal_staggering='Ah'")
    uv, h = config.get("hordiff_uv_name"), config.get("hordiff_h_name")
    orders = set()
    for name, prefix in ((uv, "hordiff_vec_xyz_Ah_sbp_"), (h, "hordiff_scalar_Ah_sbp_")):
        if not (isinstance(name, str) and name.startswith(prefix) and name.endswith("_narrow")):
            raise ValueError(f"unsupported hordiff operator: {name}")
        orders.add(name[len(prefix):-len("_narrow")])
    if orders not in ({"21"}, {"42"}, {"63"}):
        raise ValueError(f"hordiff operators {uv}, {h}: the _sbp_21_narrow, _sbp_42_narrow and _sbp_63_narrow "
                         "pairs are built (one order for both)")
    order = int(orders.pop())
    if order == 42 and domain.N < 11:
        raise ValueError("the _sbp_42_narrow diffusion needs N >= 11 (its closure blocks of six rows overlap below)")
    if order == 63 and domain.N < 17:
        raise ValueError("the _sbp_63_narrow diffusion needs N >= 17 (its closure blocks of nine rows overlap below)")
    return OperatorSwmDiff(domain, order, config.get("uv_diff_coeff", 0.0), config.get("h_diff_coeff", 0.0))


class ExplicitEul1:
    """explicit_Eul1_t (explicit_Eul1_mod.f90:20-28): v0 += dt operator(v0)."""

    def step(self, v0: StvecSwm, operator, domain: Domain | None, dt: float):
        if isinstance(operator, OperatorSwmDiff):
            check(_lib.load().swe_diffusion_step(operator.domain.ctx, v0.handle, float(dt), operator.lap_order,
                                                 operator.uv_coeff, operator.h_coeff), operator.domain.ctx,
                  "diffusion step")
            return
        tend = v0.create_similar()
        operator.apply(tend, v0, domain)
        v0.update(float(dt), tend)


def create_timescheme(state: StvecSwm, name: str):
    if name == "rk4":
        return Rk4()
    if name == "explicit_Eul1":
        return ExplicitEul1()
    raise ValueError(f"unknown timescheme_name: {name}")


def edge_links() -> np.ndarray:
    """Host-only connectivity table (6, 4, 5): nb, nside, rev, sn, st."""
    out = (ctypes.c_int * 120)()
    check(_lib.load().swe_edge_links(out))
    return np.frombuffer(out, dtype=np.int32).reshape(6, 4, 5).copy()

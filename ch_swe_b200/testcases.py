"""Initial conditions of the shallow-water test cases used on the hot path, in the
packed host layout of include/chswe.h (numpy, FP64).

* ``gaussian_hill``  ~ setup_Gaussian_hill_linear_test (src/models/shallow_water/testcases/
  gaussian_hill_linear_test_mod.f90:30-68) with generate_gaussian_hill_scalar_field
  (src/test_fields/test_fields_mod.f90:491-514): h = amp * exp(-(r/d0)^2), r the
  great-circle distance to (lam0, phi0); u = v = 0.
* ``williamson2``    ~ setup_Williamson_test2 (.../testcases/Williamson_test2_mod.f90:32-111):
  solid rotation about ``axis`` with speed u0 (test_fields_mod.f90:586-615) in covariant
  components and the balanced height (test_fields_mod.f90:857-894); ``linear_mode``
  drops the u0^2/2 term.
* ``williamson5``    ~ setup_Williamson_test5 (.../testcases/Williamson_test5_mod.f90:30-107):
  the test-2 height and solid rotation with h_mean 5960 m and u0 20 m/s, minus the
  orography of ``Ts5Orography`` (ts5_orography_generator_t, test_fields_mod.f90:211-219,
  1118-1136: a cone of 2000 m and radius pi/9 centred at (0, sqrt(3)/2, 1/2)).

Geometry: equiangular gnomonic panels (src/metric/metric_2d_ecs_mod.f90:126-411) in
the reference's panel frames (src/topology/cubed_sphere_topology_mod.f90:29-55).
"""
from __future__ import annotations

import numpy as np

from .swm import EARTH_GRAV, EARTH_OMEGA, EARTH_RADIUS

_EX = np.array([[-1, 0, 0], [0, 0, -1], [1, 0, 0], [0, 0, 1], [1, 0, 0], [1, 0, 0]], dtype=np.float64)
_EY = np.array([[0, 1, 0], [0, 1, 0], [0, 1, 0], [0, 1, 0], [0, 0, 1], [0, 0, -1]], dtype=np.float64)
_NN = np.array([[0, 0, 1], [-1, 0, 0], [0, 0, -1], [1, 0, 0], [0, 1, 0], [0, -1, 0]], dtype=np.float64)


def _angles(N: int, n: int, shift: float) -> np.ndarray:
    hx = (0.25 * np.pi - (-0.25 * np.pi)) / float(N)
    return -0.25 * np.pi + (np.arange(n) + shift) * hx


def _to_real(p: int, v: np.ndarray) -> np.ndarray:
    # proto-face vector components (x, y, z) -> sphere frame of panel p
    return v[..., 0, None] * _EX[p] + v[..., 1, None] * _EY[p] - v[..., 2, None] * _NN[p]


def mesh_geometry(N: int, mesh: str):
    """Unit position vectors r and tangent vectors a1, a2 of a mesh ('xy', 'y', 'x' or 'o',
    the cell centres), each (6, ny, nx, 3)."""
    si, sj = {"xy": (0.0, 0.0), "y": (0.5, 0.0), "x": (0.0, 0.5), "o": (0.5, 0.5)}[mesh]
    nx = N + 1 if si == 0.0 else N
    ny = N + 1 if sj == 0.0 else N
    ta = np.tan(_angles(N, nx, si))[None, :]
    tb = np.tan(_angles(N, ny, sj))[:, None]
    ta, tb = np.broadcast_arrays(ta, tb)
    sg = np.sqrt(1.0 + ta * ta + tb * tb)
    rp = np.stack([ta / sg, tb / sg, 1.0 / sg], axis=-1)
    s15 = (1.0 + ta ** 2 + tb ** 2) ** 1.5
    a1p = np.stack([(1 + ta ** 2) * (1 + tb ** 2) / s15, -ta * tb * (1 + ta ** 2) / s15, -ta * (1 + ta ** 2) / s15], -1)
    a2p = np.stack([-ta * tb * (1 + tb ** 2) / s15, (1 + ta ** 2) * (1 + tb ** 2) / s15, -tb * (1 + tb ** 2) / s15], -1)
    r = np.stack([_to_real(p, rp) for p in range(6)])
    a1 = np.stack([_to_real(p, a1p) for p in range(6)])
    a2 = np.stack([_to_real(p, a2p) for p in range(6)])
    return r, a1, a2


def gaussian_hill(N: int, lam0: float = np.pi, phi0: float = 0.0, d0: float = 0.25, amp: float = 1.0,
                  staggering: str = "Ch"):
    r, _, _ = mesh_geometry(N, "xy")
    x0, y0, z0 = np.cos(phi0) * np.cos(lam0), np.cos(phi0) * np.sin(lam0), np.sin(phi0)
    d = np.clip(r[..., 0] * x0 + r[..., 1] * y0 + r[..., 2] * z0, -1.0, 1.0)
    h = amp * np.exp(-(np.arccos(d) / d0) ** 2)
    if staggering == "Ah":
        return np.ascontiguousarray(h), np.zeros((6, N + 1, N + 1)), np.zeros((6, N + 1, N + 1))
    return np.ascontiguousarray(h), np.zeros((6, N + 1, N)), np.zeros((6, N, N + 1))


def gaussian_sum(N: int, centres, widths, amps):
    """Sum of Gaussian bumps (ensemble initial states)."""
    h = np.zeros((6, N + 1, N + 1))
    for (lam0, phi0), d0, a in zip(centres, widths, amps):
        h += gaussian_hill(N, lam0, phi0, d0, a)[0]
    return h, np.zeros((6, N + 1, N)), np.zeros((6, N, N + 1))


def williamson2(N: int, u0: float = np.pi * EARTH_RADIUS / 6.0 / (23 * 60 * 60 + 56 * 60 + 4),
                h_mean: float = 29400.0 / EARTH_GRAV, axis=(0.0, 0.0, 1.0), linear_mode: bool = False,
                radius: float = EARTH_RADIUS, omega: float = EARTH_OMEGA, grav: float = EARTH_GRAV,
                staggering: str = "Ch"):
    ax = np.asarray(axis, dtype=np.float64)
    ax = ax / np.sqrt(np.sum(ax ** 2))
    r, _, _ = mesh_geometry(N, "xy")
    rn = r / np.linalg.norm(r, axis=-1, keepdims=True)
    phi = np.arcsin(rn @ ax)
    mt = 0.0 if linear_mode else 1.0
    h = h_mean - (radius * omega * u0 + mt * 0.5 * u0 ** 2) / grav * np.sin(phi) ** 2
    out = [np.ascontiguousarray(h)]
    meshes = (("xy", 1), ("xy", 2)) if staggering == "Ah" else (("y", 1), ("x", 2))
    for mesh, comp in meshes:
        rm, a1, a2 = mesh_geometry(N, mesh)
        rn = rm / np.linalg.norm(rm, axis=-1, keepdims=True)
        vel = u0 * np.cross(ax, rn)
        b = a1 if comp == 1 else a2
        out.append(np.ascontiguousarray(np.sum(vel * b, axis=-1)))
    return tuple(out)


class Ts5Orography:
    """ts5_orography_generator_t (test_fields_mod.f90:211-219, 1118-1136): h_surf =
    h_mount * max(0, 1 - dist / r_mount), dist the great-circle distance (radians) to the
    point (x_mount, y_mount, z_mount) of the unit sphere."""

    def __init__(self, r_mount: float = np.pi / 9.0, h_mount: float = 2000.0, x_mount: float = 0.0,
                 y_mount: float = 0.5 * np.sqrt(3.0), z_mount: float = 0.5):
        self.r_mount, self.h_mount = float(r_mount), float(h_mount)
        self.c = (float(x_mount), float(y_mount), float(z_mount))

    def get_scalar_field(self, x, y, z):
        dot = np.clip(x * self.c[0] + y * self.c[1] + z * self.c[2], -1.0, 1.0)
        return self.h_mount * np.maximum(0.0, 1.0 - np.arccos(dot) / self.r_mount)


def williamson5(N: int, u0: float = 20.0, h_mean: float = 5960.0, r_mount: float = np.pi / 9.0,
                h_mount: float = 2000.0, axis=(0.0, 0.0, 1.0)):
    """setup_Williamson_test5: returns (h, u, v, h_surf), h the fluid depth (the balanced
    test-2 height minus the orography) and h_surf the orography on the xy mesh."""
    h, u, v = williamson2(N, u0=u0, h_mean=h_mean, axis=axis)
    r, _, _ = mesh_geometry(N, "xy")
    hs = Ts5Orography(r_mount=r_mount, h_mount=h_mount).get_scalar_field(r[..., 0], r[..., 1], r[..., 2])
    return np.ascontiguousarray(h - hs), u, v, np.ascontiguousarray(hs)

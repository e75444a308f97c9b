"""Seeded ensemble workloads: many members of one cube size advanced together.

The batched-ensemble configuration: M members of a C_N linear shallow-water
model, each with its own mean depth H ~ U[500, 2000] m and 1-4 Gaussian bumps
(centres uniform on the sphere, widths U[0.05, 0.3] rad, amplitudes U[-2, 2] m),
u = v = 0.  All members live in one context (one allocation, one set of
launches per stage); the reference runs them one after another
(src/models/shallow_water/testcases/gaussian_hill_linear_test_mod.f90:30-68 is
its single-member initial state).
"""
from __future__ import annotations

import numpy as np

from . import testcases


def member_params(n_members: int, seed: int):
    """Per member: (H, [(lam0, phi0), ...], [d0, ...], [amp, ...])."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_members):
        H = rng.uniform(500.0, 2000.0)
        nb = int(rng.integers(1, 5))
        z = rng.uniform(-1.0, 1.0, nb)
        lam = rng.uniform(0.0, 2.0 * np.pi, nb)
        centres = [(float(l), float(np.arcsin(zz))) for l, zz in zip(lam, z)]
        widths = [float(w) for w in rng.uniform(0.05, 0.3, nb)]
        amps = [float(a) for a in rng.uniform(-2.0, 2.0, nb)]
        out.append((float(H), centres, widths, amps))
    return out


def initial_states(N: int, params):
    """Stacked (M, ...) h, u, v initial states for member_params output."""
    hs, us, vs = [], [], []
    for _, centres, widths, amps in params:
        h, u, v = testcases.gaussian_sum(N, centres, widths, amps)
        hs.append(h)
        us.append(u)
        vs.append(v)
    return np.stack(hs), np.stack(us), np.stack(vs)


def create_ensemble(N: int, n_members: int, seed: int, precision: str = "fp32"):
    """Domain, operator, state (uploaded) and per-member parameters of one ensemble."""
    from .swm import create_domain, create_stvec_swm, create_swm_operator
    params = member_params(n_members, seed)
    dom = create_domain(N, precision=precision, n_members=n_members, h_mean=params[0][0])
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": params[0][0]}, dom)
    for k, (H, _, _, _) in enumerate(params):
        op.set_member_h_mean(k, H)
    st = create_stvec_swm(dom)
    h, u, v = initial_states(N, params)
    st.upload(h, u, v, member=None)
    return dom, op, st, params

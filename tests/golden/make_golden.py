"""Generates tests/golden/oracle_c8.npz: seeded C8 inputs with the oracle's apply and
3 RK4 steps.  These fixtures pin the oracle against accidental change; they are
not outputs of the reference (no Fortran toolchain exists to produce those)."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import Oracle  # noqa: E402

if __name__ == "__main__":
    N, H, dt, nsteps = 8, 800.0, 1800.0, 3
    rng = np.random.default_rng(20261203)
    o = Oracle(N, h_mean=H)
    h = rng.standard_normal((6, N + 1, N + 1))
    u = rng.standard_normal((6, N + 1, N))
    v = rng.standard_normal((6, N, N + 1))
    dh, du, dv = o.apply(h, u, v)
    h3, u3, v3 = o.rk4(h, u, v, dt, nsteps)
    np.savez_compressed(os.path.join(HERE, "oracle_c8.npz"), h=h, u=u, v=v, dh=dh, du=du, dv=dv,
                        h3=h3, u3=u3, v3=v3, h_mean=H, dt=dt, nsteps=nsteps)

"""ch_swe_b200 -- B200 (sm_100a) explicit shallow-water time step of ch_swe on the
Ch-staggered equiangular cubed sphere: SBP 4-2 gradient, divergence, Coriolis and
metric operators, the six-panel edge synchronisation and the RK4 update, behind
the C ABI in include/chswe.h.  See ``ch_swe_b200.swm`` for the reference-shaped API.
"""
from ._lib import SweError, load  # noqa: F401
from .swm import (Domain, OperatorSwmLin, Rk4, StvecSwm, create_domain, create_stvec_swm,  # noqa: F401
                  create_swm_diff_operator, create_swm_operator, create_timescheme, edge_links, state_shapes)

__all__ = ["SweError", "load", "Domain", "OperatorSwmLin", "Rk4", "StvecSwm", "create_domain",
           "create_stvec_swm", "create_swm_diff_operator", "create_swm_operator", "create_timescheme", "edge_links",
           "state_shapes"]

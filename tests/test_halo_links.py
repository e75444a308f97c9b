"""The device path's panel-edge connectivity (a geometric derivation from the
panel frames, swe_api.cu:compute_links) against the reference's exchange
machinery as restated literally in the oracle (transform_index, tile
intersections, pack order, signs).  CPU only: swe_edge_links needs no GPU."""
import numpy as np
import pytest

from oracle.oracle import Oracle

N = 12


@pytest.fixture(scope="module")
def links(lib_built, oracle_built):
    from ch_swe_b200 import edge_links
    return edge_links(), Oracle(N)


def side_vertex(s, a, depth):
    return [(1 + depth, a), (N + 1 - depth, a), (a, 1 + depth), (a, N + 1 - depth)][s]


def test_links_form_a_cube(links):
    L, _ = links
    for p in range(6):
        nbs = {int(L[p, s, 0]) for s in range(4)}
        assert len(nbs) == 4 and p not in nbs
        for s in range(4):
            nb, ns = int(L[p, s, 0]), int(L[p, s, 1])
            assert int(L[nb, ns, 0]) == p and int(L[nb, ns, 1]) == s   # symmetric


def test_scalar_xy_halo_full_width3(links):
    L, o = links
    rng = np.random.default_rng(0)
    h = rng.standard_normal((6, N + 1, N + 1))
    w = 3
    H = o.halo_probe(0, h, w=w)
    for t in range(6):
        for s in range(4):
            nb, ns, rev, _, _ = L[t, s]
            for a in range(1, N + 2):
                ap = N + 2 - a if rev else a
                for d in range(3):
                    i, j = [(0 - d, a), (N + 2 + d, a), (a, 0 - d), (a, N + 2 + d)][s]
                    k, l = side_vertex(ns, ap, d)
                    assert H[t, j + w - 1, i + w - 1] == h[nb, l - 1, k - 1]


def test_vector_xy_halo_cross_width1(links):
    L, o = links
    rng = np.random.default_rng(1)
    up, vp = rng.standard_normal((6, N + 1, N + 1)), rng.standard_normal((6, N + 1, N + 1))
    U, V = o.halo_probe(1, up, vp, w=1)
    for t in range(6):
        for s in range(4):
            nb, ns, rev, sn, st = L[t, s]
            for a in range(1, N + 2):
                ap = N + 2 - a if rev else a
                i, j = [(0, a), (N + 2, a), (a, 0), (a, N + 2)][s]
                k, l = side_vertex(ns, ap, 0)
                upn, vpn = up[nb, l - 1, k - 1], vp[nb, l - 1, k - 1]
                nrm, tan = (upn, vpn) if ns <= 1 else (vpn, upn)
                uh, vh = (sn * nrm, st * tan) if s <= 1 else (st * tan, sn * nrm)
                assert U[t, j, i] == uh and V[t, j, i] == vh


def test_ch_vector_halo_normal_component(links):
    L, o = links
    rng = np.random.default_rng(2)
    ut, vt = rng.standard_normal((6, N + 1, N)), rng.standard_normal((6, N, N + 1))
    A, B = o.halo_probe(2, ut, vt, w=3)
    for t in range(6):
        for s in range(4):
            nb, ns, rev, sn, _ = L[t, s]
            for a in range(1, N + 2):
                ap = N + 2 - a if rev else a
                for c in (1, 2, 3):
                    val = [ut[nb, ap - 1, c - 1], ut[nb, ap - 1, N - c], vt[nb, c - 1, ap - 1], vt[nb, N - c, ap - 1]][ns]
                    ref = [A[t, a + 2, 3 - c], A[t, a + 2, N + c + 2], B[t, 3 - c, a + 2], B[t, N + c + 2, a + 2]][s]
                    assert ref == sn * val


def test_ch_tendency_exchange_cross_width1(links):
    """The width-1 'cross' Ch exchange behind the advective tendency edge sync
    (vector_advection_Ch_mod.f90:56): the halo row/column next to a duplicated
    edge holds the neighbour's tangential component there, with the tangential
    sign (swe_advective.cuh:adv_edge_sync)."""
    L, o = links
    rng = np.random.default_rng(3)
    u, v = rng.standard_normal((6, N + 1, N)), rng.standard_normal((6, N, N + 1))
    w = 2
    U, V = o.halo_probe(4, u, v, w=w)
    for t in range(6):
        for s in range(4):
            nb, ns, rev, sn, st = L[t, s]
            for c in range(1, N + 1):
                cp = N + 1 - c if rev else c
                nbv = u[nb, 0 if ns == 2 else N, cp - 1] if ns >= 2 else v[nb, cp - 1, 0 if ns == 0 else N]
                if s >= 2:
                    got = U[t, (0 if s == 2 else N + 2) + w - 1, c + w - 1]
                else:
                    got = V[t, c + w - 1, (0 if s == 0 else N + 2) + w - 1]
                assert got == st * nbv


def test_c_grid_o_point_halo_width3(links):
    """The o-point exchange (create_o_points_halo_exchange): beyond side s at depth d, the
    neighbour's cell at depth d from its side, along index reversed by the link."""
    L, o = links
    rng = np.random.default_rng(5)
    h = rng.standard_normal((6, N, N))
    w = 3
    H = o.c_halo_probe(0, h, w=w)
    for t in range(6):
        for s in range(4):
            nb, ns, rev, _, _ = L[t, s]
            for a in range(1, N + 1):
                ap = N + 1 - a if rev else a
                for d in range(3):
                    i, j = [(0 - d, a), (N + 1 + d, a), (a, 0 - d), (a, N + 1 + d)][s]
                    k, l = [(d + 1, ap), (N - d, ap), (ap, d + 1), (ap, N - d)][ns]
                    assert H[t, j + w - 1, i + w - 1] == h[nb, l - 1, k - 1]


def test_c_grid_vector_halo_first_node(links):
    """The C vector exchange (create_symmetric_halo_vec_exchange_C): the first node beyond
    side s holds the neighbour's normal component at its own edge node, times the
    normal-component sign -- the value the C divergence SAT reads."""
    L, o = links
    rng = np.random.default_rng(6)
    u, v = rng.standard_normal((6, N, N + 1)), rng.standard_normal((6, N + 1, N))
    w = 4
    U, V = o.c_halo_probe(1, u, v, w=w)
    for t in range(6):
        for s in range(4):
            nb, ns, rev, sn, _ = L[t, s]
            for a in range(1, N + 1):
                ap = N + 1 - a if rev else a
                got = [U[t, a + w - 1, w - 1], U[t, a + w - 1, N + 2 + w - 1],
                       V[t, w - 1, a + w - 1], V[t, N + 2 + w - 1, a + w - 1]][s]
                nbv = [u[nb, ap - 1, 0], u[nb, ap - 1, N], v[nb, 0, ap - 1], v[nb, N, ap - 1]][ns]
                assert got == sn * nbv

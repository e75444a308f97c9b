// swe_cgrid.cuh -- the SBP 4-2 operators of the C staggering (domain_factory_mod.f90:281-295:
// h on the cell centres o, u on the x points, v on the y points):
//   k_c_grad       grad_c_sbp_sat_42: grad_sbp_sat_t with the centres->nodes difference and
//                  its SAT on the o-point halo of width 3 (grad_factory_mod.f90:115-150,
//                  grad_sbp_sat_mod.f90:24-76);
//   k_c_div        div_c_sbp_sat_42: div_sbp_SAT_t with the nodes->centres difference and its
//                  SAT on the C vector halo, no projection (div_factory_mod.f90:112-156,
//                  div_sbp_sat_mod.f90:29-80);
//   k_c_co2contra  co2contra_c_sbp42_new: u, v to the cell centres, times J Qi12 and swapped,
//                  back to the faces, ut = Qi11 u + (.)/J, vt = Qi22 v + (.)/J
//                  (co2contra_Cgrid_mod.f90, transform_co2contra_c_sbp_new).
// One thread per output point, reading its stencil straight from global memory; the
// panel-edge halos come from the neighbouring panels through the Link table:
//   o-point halo at depth d beyond side s: the neighbour's cell at depth d from its side,
//     along index reversed when the link says so (create_o_points_halo_exchange);
//   C vector halo at the first node beyond side s: the normal-component sign times the
//     neighbour's normal component at its own edge node (create_symmetric_halo_vec_exchange_C).
#pragma once

#include "swe_kernels.cuh"

namespace chswe {

template <class T>
struct CMetric {
    const T *iJao;    // o: 1 / (J a)
    const T *JQ12o;   // o: J Qi12
    const T *Q11x, *iJx, *Jx;   // x points: Qi11, 1/J, J
    const T *Q22y, *iJy, *Jy;   // y points: Qi22, 1/J, J
    T inv_hxa;        // 1 / (hx a)
    T inv_hx;         // 1 / hx
};

// The cell of panel t at depth dd (1 = next to the side) beyond side s, along centre a.
__device__ __forceinline__ void c_halo_cell(int N, int t, int s, int a, int dd, int &p, int &k, int &l)
{
    const Link L = c_link[t][s];
    const int ap = L.rev ? N + 1 - a : a;
    p = L.nb;
    switch (L.nside) {
    case SIDE_L: k = dd; l = ap; break;
    case SIDE_R: k = N + 1 - dd; l = ap; break;
    case SIDE_B: k = ap; l = dd; break;
    default: k = ap; l = N + 1 - dd; break;
    }
}

// gx on the x points (i = 1..N+1, j = 1..N) and gy on the y points of h on the cell centres.
template <class T>
__global__ void k_c_grad(const T *__restrict__ Y, T *__restrict__ G, Dims d, CMetric<T> m)
{
    using SB = SbpOrder<42>;
    const int N = d.N, n = N + 1;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int t = blockIdx.z % NPAN, mem = blockIdx.z / NPAN;
    if (i > n || j > n) return;
    const T *ym = Y + mem * d.ms, *h = ym + t * d.ps;
    T *g = G + mem * d.ms + t * d.ps;
    auto hv = [&](int k, int l) { return __ldg(h + box_off(d.P, k, l)); };
    // the neighbour's cell centre beyond side s at depth dd, along a
    auto halo = [&](int s, int a, int dd) {
        int p, k, l;
        c_halo_cell(N, t, s, a, dd, p, k, l);
        return __ldg(ym + p * d.ps + box_off(d.P, k, l));
    };
    if (j <= N) {
        // x points: the centres->nodes difference along i with its SAT on rows 1 and n
        auto f = [&](int c) { return hv(c, j); };
        T gx = SB::template dc2i<T>(i, n, f);
        if (i == 1) {
            T ssum = T(SB::r1(1)) * (f(1) - halo(SIDE_L, j, 1));
#pragma unroll
            for (int k = 2; k <= SB::NR; k++) ssum += T(SB::r1(k)) * (f(k) - halo(SIDE_L, j, k));
            gx += T(SB::SATC) * ssum;
        }
        if (i == n) {
            T ssum = T(SB::r1(1)) * (f(N) - halo(SIDE_R, j, 1));
#pragma unroll
            for (int k = 2; k <= SB::NR; k++) ssum += T(SB::r1(k)) * (f(n - k) - halo(SIDE_R, j, k));
            gx -= T(SB::SATC) * ssum;
        }
        g[d.fs + box_off(d.P, i, j)] = gx * m.inv_hxa;
    }
    if (i <= N) {
        auto f = [&](int c) { return hv(i, c); };
        T gy = SB::template dc2i<T>(j, n, f);
        if (j == 1) {
            T ssum = T(SB::r1(1)) * (f(1) - halo(SIDE_B, i, 1));
#pragma unroll
            for (int k = 2; k <= SB::NR; k++) ssum += T(SB::r1(k)) * (f(k) - halo(SIDE_B, i, k));
            gy += T(SB::SATC) * ssum;
        }
        if (j == n) {
            T ssum = T(SB::r1(1)) * (f(N) - halo(SIDE_T, i, 1));
#pragma unroll
            for (int k = 2; k <= SB::NR; k++) ssum += T(SB::r1(k)) * (f(n - k) - halo(SIDE_T, i, k));
            gy -= T(SB::SATC) * ssum;
        }
        g[2 * d.fs + box_off(d.P, i, j)] = gy * m.inv_hxa;
    }
}

// The divergence on the cell centres of (ut on the x points, vt on the y points).
template <class T>
__global__ void k_c_div(const T *__restrict__ W, T *__restrict__ D, Dims d, CMetric<T> m)
{
    using SB = SbpOrder<42>;
    const int N = d.N, n = N + 1;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int t = blockIdx.z % NPAN, mem = blockIdx.z / NPAN;
    if (i > N || j > N) return;
    const T *wm = W + mem * d.ms, *u = wm + d.fs + t * d.ps, *v = wm + 2 * d.fs + t * d.ps;
    auto Ju = [&](int k) { const int64_t o = box_off(d.P, k, j); return __ldg(m.Jx + o) * __ldg(u + o); };
    auto Jv = [&](int l) { const int64_t o = box_off(d.P, i, l); return __ldg(m.Jy + o) * __ldg(v + o); };
    // J times the neighbour's normal component at its edge node beyond side s, along a,
    // with the normal-component sign
    auto halo = [&](int s, int a) {
        const Link L = c_link[t][s];
        const int ap = L.rev ? N + 1 - a : a;
        const T *nb = wm + L.nb * d.ps;
        int k, l;
        const T *comp, *J;
        switch (L.nside) {
        case SIDE_L: k = 1; l = ap; comp = nb + d.fs; J = m.Jx; break;
        case SIDE_R: k = n; l = ap; comp = nb + d.fs; J = m.Jx; break;
        case SIDE_B: k = ap; l = 1; comp = nb + 2 * d.fs; J = m.Jy; break;
        default: k = ap; l = n; comp = nb + 2 * d.fs; J = m.Jy; break;
        }
        const int64_t o = box_off(d.P, k, l);
        return T(L.sn) * (__ldg(J + o) * __ldg(comp + o));
    };
    T dx = SB::template di2c<T>(i, N, Ju);
    if (i <= SB::NSAT) dx += T(SB::satw(i)) * (Ju(1) - halo(SIDE_L, j));
    if (i >= n - SB::NSAT) dx += T(SB::satw(n - i)) * (halo(SIDE_R, j) - Ju(n));
    T dy = SB::template di2c<T>(j, N, Jv);
    if (j <= SB::NSAT) dy += T(SB::satw(j)) * (Jv(1) - halo(SIDE_B, i));
    if (j >= n - SB::NSAT) dy += T(SB::satw(n - j)) * (halo(SIDE_T, i) - Jv(n));
    const int64_t o = box_off(d.P, i, j);
    D[mem * d.ms + t * d.ps + o] = (dx * m.inv_hx + dy * m.inv_hx) * __ldg(m.iJao + o);
}

// Contravariant (ut on the x points, vt on the y points) of the covariant (u, v).
template <class T>
__global__ void k_c_co2contra(const T *__restrict__ Y, T *__restrict__ W, Dims d, CMetric<T> m)
{
    using SB = SbpOrder<42>;
    const int N = d.N, n = N + 1;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int t = blockIdx.z % NPAN, mem = blockIdx.z / NPAN;
    if (i > n || j > n) return;
    const T *u = Y + mem * d.ms + d.fs + t * d.ps, *v = Y + mem * d.ms + 2 * d.fs + t * d.ps;
    T *w = W + mem * d.ms + t * d.ps;
    if (j <= N) {
        // ut at x point (i, j): the centres->nodes interpolation along i of
        // JQ12 I_nodes->centres,y(v) on the cell centres of row j
        auto vc = [&](int k) {
            auto col = [&](int l) { return __ldg(v + box_off(d.P, k, l)); };
            return __ldg(m.JQ12o + box_off(d.P, k, j)) * SB::template ii2c<T>(j, N, col);
        };
        const int64_t o = box_off(d.P, i, j);
        w[d.fs + o] = __ldg(m.Q11x + o) * __ldg(u + o) + SB::template ic2i<T>(i, n, vc) * __ldg(m.iJx + o);
    }
    if (i <= N) {
        auto uc = [&](int l) {
            auto row = [&](int k) { return __ldg(u + box_off(d.P, k, l)); };
            return __ldg(m.JQ12o + box_off(d.P, i, l)) * SB::template ii2c<T>(i, N, row);
        };
        const int64_t o = box_off(d.P, i, j);
        w[2 * d.fs + o] = __ldg(m.Q22y + o) * __ldg(v + o) + SB::template ic2i<T>(j, n, uc) * __ldg(m.iJy + o);
    }
}

}  // namespace chswe

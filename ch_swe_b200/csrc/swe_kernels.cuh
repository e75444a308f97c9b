// swe_kernels.cuh -- device building blocks of the linear shallow-water RK4 step
// on the Ch-staggered equiangular cubed sphere (SBP 4-2): global-memory panel
// views, the cube-edge halo reads that replace the reference's MPI exchanges,
// the edge synchronisations, and the elementwise kernels.  The per-stage
// kernels are in swe_tiled.cuh:
//   k_co2contra : (u, v) of the stage input -> contravariant (ut, vt)
//                 (co2contra_Ch_mod.f90:27-94)
//   k_stage     : gradient + SAT, Coriolis with the ECS vector edge sync,
//                 divergence + SAT with the Ah scalar edge sync, the linear
//                 tendency (operator_swm_lin_mod.f90:66-108) and the RK4 update
//                 (rk4_mod.f90:28-40) fused in one pass.
// Threads that own panel-boundary vertices read the neighbouring panel in the
// same allocation through the `Link` table and recompute the few neighbour
// edge values they need, instead of waiting for an exchange.
#pragma once

#include "swe_common.cuh"
#include "swe_sbp.cuh"

namespace chswe {

// Edge connectivity, filled once per device by the host.
__constant__ Link c_link[NPAN][4];

// Read-only view of one field of one panel: v(i, j) with the reference's 1-based indices.
template <class T>
struct GV {
    const T *p;
    int P;
    __device__ __forceinline__ T operator()(int i, int j) const { return __ldg(p + (j - 1 + MG) * P + (i - 1 + MG)); }
};

template <class T>
__device__ __forceinline__ GV<T> gview(const T *member_base, const Dims &d, int field, int panel)
{
    return GV<T>{member_base + field * d.fs + panel * d.ps, d.P};
}
template <class T>
__device__ __forceinline__ GV<T> mview(const T *p, const Dims &d)
{
    return GV<T>{p, d.P};
}

// Vertex of side s at along-edge index a (1..N+1), `depth` nodes inward.
__device__ __forceinline__ void side_vertex(int N, int s, int a, int depth, int &i, int &j)
{
    switch (s) {
    case SIDE_L: i = 1 + depth; j = a; break;
    case SIDE_R: i = N + 1 - depth; j = a; break;
    case SIDE_B: i = a; j = 1 + depth; break;
    default: i = a; j = N + 1 - depth; break;
    }
}

// Raw Coriolis vertex vector (coriolis_Ch_mod.f90:97-120) at xy point (k, l) of
// panel t: up = fJ2 I_c2i,y(vt), vp = -fJ2 I_c2i,x(ut).
template <class T>
__device__ __forceinline__ void cor_raw(const T *W, const Dims &d, const MetricView<T> &m, int t, int k, int l,
                                        T &up, T &vp)
{
    const int n = d.N + 1;
    const GV<T> U = gview(W, d, 1, t), V = gview(W, d, 2, t);
    T ur = ic2i<T>(k, n, [&](int c) { return U(c, l); });
    T vr = ic2i<T>(l, n, [&](int c) { return V(k, c); });
    T f = mview(m.fJ2 + t * d.ps, d)(k, l);
    up = f * vr;
    vp = -f * ur;
}

// Halo vector at side s, along-edge index a, as the reference's 'cross' vector
// exchange delivers it: the neighbour's raw vertex vector in this panel's frame.
template <class T>
__device__ __forceinline__ void cor_halo(const T *W, const Dims &d, const MetricView<T> &m, int t, int s, int a,
                                         T &uph, T &vph)
{
    const Link L = c_link[t][s];
    int ap = L.rev ? d.N + 2 - a : a;
    int k, l;
    side_vertex(d.N, L.nside, ap, 0, k, l);
    T upn, vpn;
    cor_raw(W, d, m, L.nb, k, l, upn, vpn);
    bool nlr = L.nside <= SIDE_R;
    T nrm = nlr ? upn : vpn, tan = nlr ? vpn : upn;
    if (s <= SIDE_R) { uph = T(L.sn) * nrm; vph = T(L.st) * tan; }
    else { vph = T(L.sn) * nrm; uph = T(L.st) * tan; }
}

// Covariant ECS Ah vector sync (ecs_Ah_vec_sync_mod.f90:62-125, called with
// (U, V) = (vp, up)) at a panel-boundary vertex (k, l): the synchronised up from
// the own raw up (V), and the synchronised vp from the own raw vp (U).
template <class T>
__device__ __forceinline__ T sync_up(const T *W, const Dims &d, const MetricView<T> &m, int t, int k, int l, T V)
{
    const int n = d.N + 1;
    const bool il = (k == 1), ir = (k == n), ib = (l == 1);
    T uh, vh;
    if (il || ir) {
        cor_halo(W, d, m, t, il ? SIDE_L : SIDE_R, l, uh, vh);
        const T qx = __ldg((il ? m.ql : m.qr) + l - 1);
        if (l == 1 || l == n) {
            T uh2, vh2;
            cor_halo(W, d, m, t, ib ? SIDE_B : SIDE_T, k, uh2, vh2);
            return (V + uh + uh2 + qx * vh) / T(3);
        }
        return T(0.5) * (V + uh + qx * vh);
    }
    cor_halo(W, d, m, t, ib ? SIDE_B : SIDE_T, k, uh, vh);
    return T(0.5) * (V + uh);
}

template <class T>
__device__ __forceinline__ T sync_vp(const T *W, const Dims &d, const MetricView<T> &m, int t, int k, int l, T U)
{
    const int n = d.N + 1;
    const bool il = (k == 1), ir = (k == n), ib = (l == 1), it = (l == n);
    T uh, vh;
    if (ib || it) {
        cor_halo(W, d, m, t, ib ? SIDE_B : SIDE_T, k, uh, vh);
        const T qy = __ldg((ib ? m.qb : m.qt) + k - 1);
        if (il || ir) {
            T uh1, vh1;
            cor_halo(W, d, m, t, il ? SIDE_L : SIDE_R, l, uh1, vh1);
            return (U + vh1 + vh + qy * uh) / T(3);
        }
        return T(0.5) * (U + vh + qy * uh);
    }
    cor_halo(W, d, m, t, il ? SIDE_L : SIDE_R, l, uh, vh);
    return T(0.5) * (U + vh);
}

// J * (normal contravariant component) of the neighbour across side s, at centre
// depth c = 1..3 and along-edge index a: the halo the Ch vector exchange
// (exchange_halo_Ch_mod.f90) delivers for the divergence SAT.
template <class T>
__device__ __forceinline__ T ju_halo(const T *W, const Dims &d, const MetricView<T> &m, int t, int s, int a, int c)
{
    const Link L = c_link[t][s];
    const int N = d.N;
    const int ap = L.rev ? N + 2 - a : a;
    const GV<T> Jy = mview(m.Jy, d), Jx = mview(m.Jx, d);
    const GV<T> U = gview(W, d, 1, L.nb), V = gview(W, d, 2, L.nb);
    T val;
    switch (L.nside) {
    case SIDE_L: val = Jy(c, ap) * U(c, ap); break;
    case SIDE_R: val = Jy(N + 1 - c, ap) * U(N + 1 - c, ap); break;
    case SIDE_B: val = Jx(ap, c) * V(ap, c); break;
    default: val = Jx(ap, N + 1 - c) * V(ap, N + 1 - c); break;
    }
    return T(L.sn) * val;
}

// Divergence at xy point (k, l) before the Ah projection (div_sbp_sat_mod.f90:54-80),
// SAT terms (sbp_diff_c2i_42_mod.f90:195-251) included.
template <class T>
__device__ __forceinline__ T div_raw(const T *W, const Dims &d, const MetricView<T> &m, int t, int k, int l)
{
    using namespace sbp;
    const int N = d.N, n = N + 1;
    const GV<T> U = gview(W, d, 1, t), V = gview(W, d, 2, t), Jy = mview(m.Jy, d), Jx = mview(m.Jx, d);
    auto ju = [&](int c) { return Jy(c, l) * U(c, l); };
    auto jv = [&](int c) { return Jx(k, c) * V(k, c); };
    T dx = dc2i<T>(k, n, ju);
    if (k == 1)
        dx += T(SATC) * (T(R11) * (ju(1) - ju_halo(W, d, m, t, SIDE_L, l, 1)) +
                         T(R12) * (ju(2) - ju_halo(W, d, m, t, SIDE_L, l, 2)) +
                         T(R13) * (ju(3) - ju_halo(W, d, m, t, SIDE_L, l, 3)));
    else if (k == n)
        dx -= T(SATC) * (T(R11) * (ju(N) - ju_halo(W, d, m, t, SIDE_R, l, 1)) +
                         T(R12) * (ju(N - 1) - ju_halo(W, d, m, t, SIDE_R, l, 2)) +
                         T(R13) * (ju(N - 2) - ju_halo(W, d, m, t, SIDE_R, l, 3)));
    T dy = dc2i<T>(l, n, jv);
    if (l == 1)
        dy += T(SATC) * (T(R11) * (jv(1) - ju_halo(W, d, m, t, SIDE_B, k, 1)) +
                         T(R12) * (jv(2) - ju_halo(W, d, m, t, SIDE_B, k, 2)) +
                         T(R13) * (jv(3) - ju_halo(W, d, m, t, SIDE_B, k, 3)));
    else if (l == n)
        dy -= T(SATC) * (T(R11) * (jv(N) - ju_halo(W, d, m, t, SIDE_T, k, 1)) +
                         T(R12) * (jv(N - 1) - ju_halo(W, d, m, t, SIDE_T, k, 2)) +
                         T(R13) * (jv(N - 2) - ju_halo(W, d, m, t, SIDE_T, k, 3)));
    return (dx * m.inv_hx + dy * m.inv_hx) * mview(m.iJa, d)(k, l);
}

template <class T>
__device__ __forceinline__ T div_halo(const T *W, const Dims &d, const MetricView<T> &m, int t, int s, int a)
{
    const Link L = c_link[t][s];
    int ap = L.rev ? d.N + 2 - a : a;
    int k, l;
    side_vertex(d.N, L.nside, ap, 0, k, l);
    return div_raw(W, d, m, L.nb, k, l);
}

// Divergence after the Ah scalar sync (halo_Ah_scalar_sync_mod.f90:43-98) at a
// panel-boundary vertex.
template <class T>
__device__ __forceinline__ T div_sync(const T *W, const Dims &d, const MetricView<T> &m, int t, int k, int l)
{
    const int n = d.N + 1;
    T f = div_raw(W, d, m, t, k, l);
    const bool il = (k == 1), ir = (k == n), ib = (l == 1), it = (l == n);
    if ((il || ir) && (ib || it)) {
        T fx = div_halo(W, d, m, t, il ? SIDE_L : SIDE_R, l);
        T fy = div_halo(W, d, m, t, ib ? SIDE_B : SIDE_T, k);
        return (f + fx + fy) / T(3);
    }
    if (il || ir) return T(0.5) * (f + div_halo(W, d, m, t, il ? SIDE_L : SIDE_R, l));
    return T(0.5) * (f + div_halo(W, d, m, t, ib ? SIDE_B : SIDE_T, k));
}

// h at the neighbour's copy of the shared vertex (xy halo index 0 / N+2).
template <class T>
__device__ __forceinline__ T h_halo(const T *Y, const Dims &d, int t, int s, int a)
{
    const Link L = c_link[t][s];
    int ap = L.rev ? d.N + 2 - a : a;
    int k, l;
    side_vertex(d.N, L.nside, ap, 0, k, l);
    return gview(Y, d, 0, L.nb)(k, l);
}

// Edge buffer: for every member, panel, side and along-edge vertex a = 1..N+1
// the synchronised (up, vp, div) of that panel-boundary vertex.
__device__ __forceinline__ int64_t edge_index(int N, int mem, int t, int s, int a)
{
    return ((((int64_t)mem * NPAN + t) * 4 + s) * (N + 1) + (a - 1)) * 3;
}

// The panel-boundary vertices' synchronised Coriolis vector (ECS Ah vector sync)
// and divergence (Ah scalar sync), computed once per stage: the work the
// reference does with its 'cross' and 'full' exchanges before the edge loops.
// grid: x over along-edge vertices, y over panel*4 + side, z over members.
template <class T>
__global__ void __launch_bounds__(128) k_edge(const T *__restrict__ Wc, T *__restrict__ E, Dims d, MetricView<T> m)
{
    const int N = d.N, n = N + 1;
    const int a = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (a > n) return;
    const int t = blockIdx.y / 4, s = blockIdx.y % 4, mem = blockIdx.z;
    const T *w = Wc + mem * d.ms;
    int k, l;
    side_vertex(N, s, a, 0, k, l);
    T up, vp;
    cor_raw(w, d, m, t, k, l, up, vp);
    T *e = E + edge_index(N, mem, t, s, a);
    e[0] = sync_up(w, d, m, t, k, l, up);
    e[1] = sync_vp(w, d, m, t, k, l, vp);
    e[2] = div_sync(w, d, m, t, k, l);
}

// Synchronised (up, vp, div) of panel-boundary vertex (k, l) from the edge buffer.
template <class T>
__device__ __forceinline__ const T *edge_entry(const T *E, int N, int mem, int t, int k, int l)
{
    const int n = N + 1;
    if (k == 1) return E + edge_index(N, mem, t, SIDE_L, l);
    if (k == n) return E + edge_index(N, mem, t, SIDE_R, l);
    if (l == 1) return E + edge_index(N, mem, t, SIDE_B, k);
    return E + edge_index(N, mem, t, SIDE_T, k);
}

// RK4 stage parameters.
struct StageArgs {
    int mode;          // 0: write the tendency A(y) to out; 1..4: RK4 stage
    double dt;
    const double *Hm;  // per-member mean depth
};

// Kahan-compensated state update for FP32 (s += inc with compensation c).
__device__ __forceinline__ void kahan_add(float &s, float &c, float inc)
{
    float yk = inc - c;
    float tk = s + yk;
    c = (tk - s) - yk;
    s = tk;
}

// y = s1*v1 + s2*v2 (v2 may be null) or y += s1*v1 + s2*v2 over the whole box.
template <class T>
__global__ void k_axpby(T *y, const T *v1, const T *v2, double s1, double s2, int accumulate, int64_t n)
{
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; k < n; k += stride) {
        T r = T(s1) * v1[k];
        if (v2) r = r + T(s2) * v2[k];
        y[k] = accumulate ? y[k] + r : r;
    }
}

}  // namespace chswe

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
//   k_edge      : the synchronised Coriolis vector and divergence of every
//                 panel-boundary vertex, once per stage, into the edge buffer.
// Neighbouring panels live in the same allocation: threads read across a cube
// edge through the `Link` table instead of waiting for an exchange.
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

// One raw quantity at boundary vertex (k, l) of panel t, before any edge sync:
//   q = 0: up = fJ2 I_c2i,y(vt)      q = 1: vp = -fJ2 I_c2i,x(ut)
//          (coriolis_Ch_mod.f90:97-120)
//   q = 2: c2i x-difference of J ut  q = 3: c2i y-difference of J vt
//          with the SAT terms of sbp_diff_c2i_42_mod.f90:195-251 on the panel edge
//          (div_sbp_sat_mod.f90:54-80 before the 1/(hx J) scaling).
template <class T>
__device__ __forceinline__ T edge_raw(const T *W, const Dims &d, const MetricView<T> &m, int t, int k, int l, int q)
{
    using namespace sbp;
    const int N = d.N, n = N + 1;
    const GV<T> U = gview(W, d, 1, t), V = gview(W, d, 2, t);
    if (q == 0) return mview(m.fJ2 + t * d.ps, d)(k, l) * ic2i<T>(l, n, [&](int c) { return V(k, c); });
    if (q == 1) return -mview(m.fJ2 + t * d.ps, d)(k, l) * ic2i<T>(k, n, [&](int c) { return U(c, l); });
    const GV<T> Jy = mview(m.Jy, d), Jx = mview(m.Jx, d);
    if (q == 2) {
        auto ju = [&](int c) { return Jy(c, l) * U(c, l); };
        T dx = dc2i<T>(k, n, ju);
        if (k == 1)
            dx += T(SATC) * (T(R11) * (ju(1) - ju_halo(W, d, m, t, SIDE_L, l, 1)) +
                             T(R12) * (ju(2) - ju_halo(W, d, m, t, SIDE_L, l, 2)) +
                             T(R13) * (ju(3) - ju_halo(W, d, m, t, SIDE_L, l, 3)));
        else if (k == n)
            dx -= T(SATC) * (T(R11) * (ju(N) - ju_halo(W, d, m, t, SIDE_R, l, 1)) +
                             T(R12) * (ju(N - 1) - ju_halo(W, d, m, t, SIDE_R, l, 2)) +
                             T(R13) * (ju(N - 2) - ju_halo(W, d, m, t, SIDE_R, l, 3)));
        return dx;
    }
    auto jv = [&](int c) { return Jx(k, c) * V(k, c); };
    T dy = dc2i<T>(l, n, jv);
    if (l == 1)
        dy += T(SATC) * (T(R11) * (jv(1) - ju_halo(W, d, m, t, SIDE_B, k, 1)) +
                         T(R12) * (jv(2) - ju_halo(W, d, m, t, SIDE_B, k, 2)) +
                         T(R13) * (jv(3) - ju_halo(W, d, m, t, SIDE_B, k, 3)));
    else if (l == n)
        dy -= T(SATC) * (T(R11) * (jv(N) - ju_halo(W, d, m, t, SIDE_T, k, 1)) +
                         T(R12) * (jv(N - 1) - ju_halo(W, d, m, t, SIDE_T, k, 2)) +
                         T(R13) * (jv(N - 2) - ju_halo(W, d, m, t, SIDE_T, k, 3)));
    return dy;
}

// The neighbour's copy (panel nb, vertex (kk, ll)) of boundary vertex (k, l) of
// panel t across side s.
__device__ __forceinline__ void nb_vertex(int N, int t, int s, int k, int l, int &nb, int &kk, int &ll)
{
    const Link L = c_link[t][s];
    const int a = s <= SIDE_R ? l : k;
    nb = L.nb;
    side_vertex(N, L.nside, L.rev ? N + 2 - a : a, 0, kk, ll);
}

// The neighbour's raw vertex vector (upn, vpn) in this panel's frame, as the
// reference's 'cross' vector exchange delivers it across side s.
template <class T>
__device__ __forceinline__ void halo_vec(int t, int s, T upn, T vpn, T &uh, T &vh)
{
    const Link L = c_link[t][s];
    const bool nlr = L.nside <= SIDE_R;
    const T nrm = nlr ? upn : vpn, tan = nlr ? vpn : upn;
    if (s <= SIDE_R) { uh = T(L.sn) * nrm; vh = T(L.st) * tan; }
    else { vh = T(L.sn) * nrm; uh = T(L.st) * tan; }
}

constexpr int EDGE_CHUNK = 32;    // along-edge vertices per block (balanced split, at most 32)
constexpr int EDGE_THREADS = 288; // 8 warps of raw stencils + 1 warp for the third panel at corners

// The panel-boundary vertices' synchronised Coriolis vector (ECS Ah covariant
// vector sync, ecs_Ah_vec_sync_mod.f90:62-125 with (U, V) = (vp, up)) and
// divergence (Ah scalar sync, halo_Ah_scalar_sync_mod.f90:43-98): the work the
// reference does with its 'cross' and 'full' exchanges before the edge loops.
// Block = (chunk of vertices along one side of one panel of one member).
// Phase 1: every raw quantity the chunk needs is one thread's stencil: warp w < 8
// takes quantity w % 4 for copy w / 4 (own vertex / neighbour across this side),
// warp 8 the copy of the third panel at the two cube corners.  Phase 2 combines
// the copies from shared memory.  Copies are stored by direction (x-neighbour
// across L/R, y-neighbour across B/T), so the two sides that meet at a corner
// compute bit-identical corner values.
template <class T>
__global__ void __launch_bounds__(EDGE_THREADS) k_edge(const T *__restrict__ Wc, T *__restrict__ E, Dims d,
                                                        MetricView<T> m)
{
    __shared__ T raw[3][4][EDGE_CHUNK];   // [own, x-neighbour, y-neighbour][quantity][vertex]
    const int N = d.N, n = N + 1;
    const int t = blockIdx.y >> 2, s = blockIdx.y & 3, mem = blockIdx.z;
    const int a0 = 1 + (blockIdx.x * n) / gridDim.x, a1 = 1 + ((blockIdx.x + 1) * n) / gridDim.x;
    const T *w = Wc + mem * d.ms;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool xs = s <= SIDE_R;
    if (warp < 8) {
        const int a = a0 + lane, q = warp & 3;
        if (a < a1) {
            int k, l;
            side_vertex(N, s, a, 0, k, l);
            if (warp < 4) {
                raw[0][q][lane] = edge_raw(w, d, m, t, k, l, q);
            } else {
                int nb, kk, ll;
                nb_vertex(N, t, s, k, l, nb, kk, ll);
                raw[xs ? 1 : 2][q][lane] = edge_raw(w, d, m, nb, kk, ll, q);
            }
        }
    } else if (lane < 8) {
        // the other neighbour of the corner vertices a = 1 and a = N+1
        const int a = lane < 4 ? 1 : n, q = lane & 3;
        if (a >= a0 && a < a1) {
            int k, l, nb, kk, ll;
            side_vertex(N, s, a, 0, k, l);
            const int s2 = xs ? (l == 1 ? SIDE_B : SIDE_T) : (k == 1 ? SIDE_L : SIDE_R);
            nb_vertex(N, t, s2, k, l, nb, kk, ll);
            raw[xs ? 2 : 1][q][a - a0] = edge_raw(w, d, m, nb, kk, ll, q);
        }
    }
    __syncthreads();
    if (threadIdx.x >= a1 - a0) return;
    const int v = threadIdx.x, a = a0 + v;
    int k, l;
    side_vertex(N, s, a, 0, k, l);
    const bool il = (k == 1), ir = (k == n), ib = (l == 1), it = (l == n);
    const bool cx = il || ir, cy = ib || it;
    const GV<T> iJa = mview(m.iJa, d);
    const T V = raw[0][0][v], U = raw[0][1][v];
    const T f = (raw[0][2][v] * m.inv_hx + raw[0][3][v] * m.inv_hx) * iJa(k, l);
    T uhx = 0, vhx = 0, fx = 0, uhy = 0, vhy = 0, fy = 0;
    if (cx) {
        const int sx = il ? SIDE_L : SIDE_R;
        int nb, kk, ll;
        nb_vertex(N, t, sx, k, l, nb, kk, ll);
        halo_vec(t, sx, raw[1][0][v], raw[1][1][v], uhx, vhx);
        fx = (raw[1][2][v] * m.inv_hx + raw[1][3][v] * m.inv_hx) * iJa(kk, ll);
    }
    if (cy) {
        const int sy = ib ? SIDE_B : SIDE_T;
        int nb, kk, ll;
        nb_vertex(N, t, sy, k, l, nb, kk, ll);
        halo_vec(t, sy, raw[2][0][v], raw[2][1][v], uhy, vhy);
        fy = (raw[2][2][v] * m.inv_hx + raw[2][3][v] * m.inv_hx) * iJa(kk, ll);
    }
    T sup, svp, sdiv;
    if (cx && cy) {
        const T qx = __ldg((il ? m.ql : m.qr) + l - 1), qy = __ldg((ib ? m.qb : m.qt) + k - 1);
        sup = (V + uhx + uhy + qx * vhx) / T(3);
        svp = (U + vhx + vhy + qy * uhy) / T(3);
        sdiv = (f + fx + fy) / T(3);
    } else if (cx) {
        const T qx = __ldg((il ? m.ql : m.qr) + l - 1);
        sup = T(0.5) * (V + uhx + qx * vhx);
        svp = T(0.5) * (U + vhx);
        sdiv = T(0.5) * (f + fx);
    } else {
        const T qy = __ldg((ib ? m.qb : m.qt) + k - 1);
        sup = T(0.5) * (V + uhy);
        svp = T(0.5) * (U + vhy + qy * uhy);
        sdiv = T(0.5) * (f + fy);
    }
    T *e = E + edge_index(N, mem, t, s, a);
    e[0] = sup;
    e[1] = svp;
    e[2] = sdiv;
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

// swe_kernels.cuh -- sm_100a kernels of the linear shallow-water RK4 step on the
// Ch-staggered equiangular cubed sphere (SBP 4-2), templated on the stencil type.
//
// This header holds the global-memory building blocks (stencil tables, edge
// links, the neighbour-panel values used at panel boundaries) and the small
// elementwise kernels; the per-stage kernels are in swe_tiled.cuh:
//   k_co2contra_t : (u, v) of the stage input -> contravariant (ut, vt)
//                   (co2contra_Ch_mod.f90:27-94)
//   k_stage_t     : gradient + SAT, Coriolis with the ECS vector edge sync,
//                   divergence + SAT with the Ah scalar edge sync, the linear
//                   tendency (operator_swm_lin_mod.f90:66-108) and the RK4 update
//                   (rk4_mod.f90:28-40) fused in one pass.
// The MPI halo exchange of the reference is replaced by index-mapped reads of
// the neighbouring panel in the same allocation (`Link` table): panel-edge
// threads recompute the neighbour's edge values they need instead of waiting
// for an exchange.
#pragma once

#include "swe_common.cuh"

namespace chswe {

// Tables filled once per device by the host (single translation unit).
__constant__ OpTab<double> c_op64[4];
__constant__ OpTab<float> c_op32[4];
__constant__ Link c_link[NPAN][4];
__constant__ double c_sat64[8];
__constant__ float c_sat32[8];

template <class T> __device__ __forceinline__ const OpTab<T> &optab(int op);
template <> __device__ __forceinline__ const OpTab<double> &optab<double>(int op) { return c_op64[op]; }
template <> __device__ __forceinline__ const OpTab<float> &optab<float>(int op) { return c_op32[op]; }
template <class T> __device__ __forceinline__ T satc(int k);
template <> __device__ __forceinline__ double satc<double>(int k) { return c_sat64[k]; }
template <> __device__ __forceinline__ float satc<float>(int k) { return c_sat32[k]; }
// SAT constants: [0..2] 0.5*R1r/hrr of the i2c difference, [3] 0.5/h11 of the
// c2i difference, [4..6] R11, R12, R13.

// Row k (1-based) of operator `op` with K outputs: returns the first input index
// and the five weights.
template <class T>
__device__ __forceinline__ int sten(int op, int k, int K, const T *&w)
{
    const OpTab<T> &o = optab<T>(op);
    if (k <= o.L) { w = o.lw[k - 1]; return o.lstart[k - 1]; }
    int r = K - k;
    if (r < o.L) { w = o.rw[r]; return K + o.rstart[r]; }
    w = o.iw;
    return k + o.ioff;
}

__device__ __forceinline__ int64_t ofs(const Dims &d, int i, int j) { return (int64_t)(j - 1) * d.P + (i - 1); }

// Field accessors inside one member's block (base = member start).
template <class T>
__device__ __forceinline__ T ld(const T *base, const Dims &d, int f, int t, int i, int j)
{
    return __ldg(base + f * d.fs + t * d.ps + ofs(d, i, j));
}

// Vertex of side `s` at along-edge index a (1..N+1), `depth` nodes inward.
__device__ __forceinline__ void side_vertex(int N, int s, int a, int depth, int &i, int &j)
{
    switch (s) {
    case SIDE_L: i = 1 + depth; j = a; break;
    case SIDE_R: i = N + 1 - depth; j = a; break;
    case SIDE_B: i = a; j = 1 + depth; break;
    default: i = a; j = N + 1 - depth; break;
    }
}

// ---------------------------------------------------------------------------
// building blocks reading global memory (used everywhere, and by panel-edge
// threads for the neighbour's values)
// ---------------------------------------------------------------------------

// Raw Coriolis vertex vector (coriolis_Ch_mod.f90:97-120) at xy point (k, l):
// up = fJ2 * I_c2i,y(vt), vp = -fJ2 * I_c2i,x(ut).
template <class T>
__device__ __forceinline__ void cor_raw(const T *W, const Dims &d, const MetricView<T> &m, int t, int k, int l,
                                        T &up, T &vp)
{
    const int N = d.N;
    const T *w;
    int s = sten<T>(OP_IC2I, k, N + 1, w);
    T ur = 0;
#pragma unroll
    for (int q = 0; q < 5; q++)
        if (w[q] != T(0)) ur += w[q] * ld(W, d, 1, t, s + q, l);
    s = sten<T>(OP_IC2I, l, N + 1, w);
    T vr = 0;
#pragma unroll
    for (int q = 0; q < 5; q++)
        if (w[q] != T(0)) vr += w[q] * ld(W, d, 2, t, k, s + q);
    T f = __ldg(m.fJ2 + t * d.ps + ofs(d, k, l));
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

// Synchronised Coriolis vertex vector: the covariant ECS Ah vector sync
// (ecs_Ah_vec_sync_mod.f90:62-125, called with (U, V) = (vp, up)).
template <class T>
__device__ __forceinline__ void cor_sync(const T *W, const Dims &d, const MetricView<T> &m, int t, int k, int l,
                                         T &ups, T &vps)
{
    const int n = d.N + 1;
    T V, U;
    cor_raw(W, d, m, t, k, l, V, U);   // V = up, U = vp
    bool il = (k == 1), ir = (k == n), ib = (l == 1), it = (l == n);
    if (!(il || ir || ib || it)) { ups = V; vps = U; return; }
    const T half = T(0.5);
    T uh, vh, Uh1, Vh1, Uh2, Vh2;
    if ((il || ir) && (ib || it)) {
        // cube corner: own value + the two neighbours' copies
        int sx = il ? SIDE_L : SIDE_R, sy = ib ? SIDE_B : SIDE_T;
        cor_halo(W, d, m, t, sx, l, uh, vh); Uh1 = vh; Vh1 = uh;   // x-side halo (U, V)
        cor_halo(W, d, m, t, sy, k, uh, vh); Uh2 = vh; Vh2 = uh;   // y-side halo
        T qx = il ? __ldg(m.ql + l - 1) : __ldg(m.qr + l - 1);
        T qy = ib ? __ldg(m.qb + k - 1) : __ldg(m.qt + k - 1);
        T Un = (U + Uh1 + Uh2 + qy * Vh2) / T(3);
        T Vn = (V + Vh1 + Vh2 + qx * Uh1) / T(3);
        ups = Vn; vps = Un;
        return;
    }
    if (il || ir) {
        cor_halo(W, d, m, t, il ? SIDE_L : SIDE_R, l, uh, vh);
        T q = il ? __ldg(m.ql + l - 1) : __ldg(m.qr + l - 1);
        T Un = half * (U + vh);
        T Vn = half * (V + uh + q * vh);
        ups = Vn; vps = Un;
        return;
    }
    // bottom / top side: V <- (V + V_h)/2, U <- (U + U_h + q V_h)/2
    cor_halo(W, d, m, t, ib ? SIDE_B : SIDE_T, k, uh, vh);
    T q = ib ? __ldg(m.qb + k - 1) : __ldg(m.qt + k - 1);
    T Vn = half * (V + uh);
    T Un = half * (U + vh + q * uh);
    ups = Vn; vps = Un;
}

// J * (normal contravariant component) of the neighbour across side s, at
// centre depth c = 1..3 and along-edge index a: the halo the Ch vector
// exchange (exchange_halo_Ch_mod.f90) delivers for the divergence SAT.
template <class T>
__device__ __forceinline__ T ju_halo(const T *W, const Dims &d, const MetricView<T> &m, int t, int s, int a, int c)
{
    const Link L = c_link[t][s];
    const int N = d.N;
    int ap = L.rev ? N + 2 - a : a;
    T val;
    switch (L.nside) {
    case SIDE_L: val = __ldg(m.Jy + ofs(d, c, ap)) * ld(W, d, 1, L.nb, c, ap); break;
    case SIDE_R: val = __ldg(m.Jy + ofs(d, N + 1 - c, ap)) * ld(W, d, 1, L.nb, N + 1 - c, ap); break;
    case SIDE_B: val = __ldg(m.Jx + ofs(d, ap, c)) * ld(W, d, 2, L.nb, ap, c); break;
    default: val = __ldg(m.Jx + ofs(d, ap, N + 1 - c)) * ld(W, d, 2, L.nb, ap, N + 1 - c); break;
    }
    return T(L.sn) * val;
}

// Divergence at xy point (k, l) before the Ah projection (div_sbp_sat_mod.f90:54-80).
template <class T>
__device__ __forceinline__ T div_raw(const T *W, const Dims &d, const MetricView<T> &m, int t, int k, int l)
{
    const int N = d.N, n = N + 1;
    const T *w;
    int s = sten<T>(OP_DC2I, k, n, w);
    T dx = 0;
#pragma unroll
    for (int q = 0; q < 5; q++) {
        int i = s + q;
        if (w[q] != T(0)) dx += w[q] * (__ldg(m.Jy + ofs(d, i, l)) * ld(W, d, 1, t, i, l));
    }
    const T c0 = satc<T>(3), R11 = satc<T>(4), R12 = satc<T>(5), R13 = satc<T>(6);
    if (k == 1) {
        T j1 = __ldg(m.Jy + ofs(d, 1, l)) * ld(W, d, 1, t, 1, l);
        T j2 = __ldg(m.Jy + ofs(d, 2, l)) * ld(W, d, 1, t, 2, l);
        T j3 = __ldg(m.Jy + ofs(d, 3, l)) * ld(W, d, 1, t, 3, l);
        dx += c0 * (R11 * (j1 - ju_halo(W, d, m, t, SIDE_L, l, 1)) + R12 * (j2 - ju_halo(W, d, m, t, SIDE_L, l, 2)) +
                    R13 * (j3 - ju_halo(W, d, m, t, SIDE_L, l, 3)));
    } else if (k == n) {
        T j1 = __ldg(m.Jy + ofs(d, N, l)) * ld(W, d, 1, t, N, l);
        T j2 = __ldg(m.Jy + ofs(d, N - 1, l)) * ld(W, d, 1, t, N - 1, l);
        T j3 = __ldg(m.Jy + ofs(d, N - 2, l)) * ld(W, d, 1, t, N - 2, l);
        dx -= c0 * (R11 * (j1 - ju_halo(W, d, m, t, SIDE_R, l, 1)) + R12 * (j2 - ju_halo(W, d, m, t, SIDE_R, l, 2)) +
                    R13 * (j3 - ju_halo(W, d, m, t, SIDE_R, l, 3)));
    }
    s = sten<T>(OP_DC2I, l, n, w);
    T dy = 0;
#pragma unroll
    for (int q = 0; q < 5; q++) {
        int j = s + q;
        if (w[q] != T(0)) dy += w[q] * (__ldg(m.Jx + ofs(d, k, j)) * ld(W, d, 2, t, k, j));
    }
    if (l == 1) {
        T j1 = __ldg(m.Jx + ofs(d, k, 1)) * ld(W, d, 2, t, k, 1);
        T j2 = __ldg(m.Jx + ofs(d, k, 2)) * ld(W, d, 2, t, k, 2);
        T j3 = __ldg(m.Jx + ofs(d, k, 3)) * ld(W, d, 2, t, k, 3);
        dy += c0 * (R11 * (j1 - ju_halo(W, d, m, t, SIDE_B, k, 1)) + R12 * (j2 - ju_halo(W, d, m, t, SIDE_B, k, 2)) +
                    R13 * (j3 - ju_halo(W, d, m, t, SIDE_B, k, 3)));
    } else if (l == n) {
        T j1 = __ldg(m.Jx + ofs(d, k, N)) * ld(W, d, 2, t, k, N);
        T j2 = __ldg(m.Jx + ofs(d, k, N - 1)) * ld(W, d, 2, t, k, N - 1);
        T j3 = __ldg(m.Jx + ofs(d, k, N - 2)) * ld(W, d, 2, t, k, N - 2);
        dy -= c0 * (R11 * (j1 - ju_halo(W, d, m, t, SIDE_T, k, 1)) + R12 * (j2 - ju_halo(W, d, m, t, SIDE_T, k, 2)) +
                    R13 * (j3 - ju_halo(W, d, m, t, SIDE_T, k, 3)));
    }
    return (dx * m.inv_hx + dy * m.inv_hx) * __ldg(m.iJa + ofs(d, k, l));
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

// Divergence after the Ah scalar sync (halo_Ah_scalar_sync_mod.f90:43-98).
template <class T>
__device__ __forceinline__ T div_sync(const T *W, const Dims &d, const MetricView<T> &m, int t, int k, int l)
{
    const int n = d.N + 1;
    T f = div_raw(W, d, m, t, k, l);
    bool il = (k == 1), ir = (k == n), ib = (l == 1), it = (l == n);
    if (!(il || ir || ib || it)) return f;
    if ((il || ir) && (ib || it)) {
        T fx = div_halo(W, d, m, t, il ? SIDE_L : SIDE_R, l);
        T fy = div_halo(W, d, m, t, ib ? SIDE_B : SIDE_T, k);
        return (f + fx + fy) / T(3);
    }
    if (il) return T(0.5) * (div_halo(W, d, m, t, SIDE_L, l) + f);
    if (ir) return T(0.5) * (f + div_halo(W, d, m, t, SIDE_R, l));
    if (ib) return T(0.5) * (f + div_halo(W, d, m, t, SIDE_B, k));
    return T(0.5) * (f + div_halo(W, d, m, t, SIDE_T, k));
}

// h at the neighbour's copy of the shared vertex (xy halo index 0 / N+2).
template <class T>
__device__ __forceinline__ T h_halo(const T *Y, const Dims &d, int t, int s, int a)
{
    const Link L = c_link[t][s];
    int ap = L.rev ? d.N + 2 - a : a;
    int k, l;
    side_vertex(d.N, L.nside, ap, 0, k, l);
    return ld(Y, d, 0, L.nb, k, l);
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

// RK4 stage parameters.
struct StageArgs {
    int mode;          // 0: write the tendency A(y) to out; 1..4: RK4 stage
    double dt;
    const double *Hm;  // per-member mean depth
};

// Kahan-compensated state update for FP32 (v0 += inc with compensation c).
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

// swe_diff.cuh -- horizontal diffusion on the Ah staggering, the operator the reference
// applies after each step of the dynamics (shallow_water_mod.f90:95-100,117-118;
// operator_swm_diff_mod.f90:27-49) in its _sbp_21_narrow form
// (hordiff_factory_mod.f90:33-34,61-62):
//   h:     hordiff_scalar_Ah_sbp_21_narrow   tend = -(c a hx)^4 L(L(h))
//   u, v:  hordiff_vec_xyz_Ah_sbp_21_narrow  the covariant wind to Cartesian components
//          with the contravariant basis, the same scalar diffusion of each component,
//          back with the same basis (as cart2cube_vec does for covariant components,
//          vec_math_mod.f90:196-219), then the covariant ECS Ah vector sync
//          (hordiff_colocated_mod.f90:42-58)
// L is laplace_Ah_sbp21_narrow (laplace_Ah_sbp21_narrow_mod.f90:25-239): narrow second
// differences with the variable coefficients Qi11 J, Qi22 J, the mixed terms
// D1(Qi12 J D1 f), boundary penalties, / (hx a)^2 / J, and the Ah scalar sync.
//
// The four scalar fields of a member (h and the three Cartesian wind components) are
// diffused together: scratch sets hold [member][field 0..3][panel][box], and every
// Laplacian is three launches over all of them (first differences; the Laplacian's raw
// values, kept for the sync on the panel edges and final inside; the sync).  A step is
// nine launches: k_dif_prep, two Laplacians, k_dif_vraw (the Cartesian tendencies
// projected back), k_dif_update (the vector sync and the Euler update or the tendency).
#pragma once

#include "swe_ah.cuh"

namespace chswe {

constexpr int DIF_FIELDS = 4;   // h, and the wind's x, y, z components

// One scalar field of the scratch sets: field q of member mem.
__device__ __forceinline__ int64_t dif_base(const Dims &d, int mem, int q)
{
    return ((int64_t)mem * DIF_FIELDS + q) * NPAN * d.ps;
}

// The contravariant basis b1, b2 (Cartesian, unit sphere) of every vertex: [panel][6][box].
template <class T>
struct DifView {
    const T *b;
    double h2;   // (hx a)^2
};

// (h, b1 u + b2 v) of the state -> the four scalar fields of each member.
template <class T>
__global__ void __launch_bounds__(256) k_dif_prep(const T *__restrict__ Y, T *__restrict__ X, Dims d, DifView<T> v)
{
    const int n = d.N + 1;
    const int mem = blockIdx.z / NPAN, t = blockIdx.z % NPAN;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    pdl_trigger();
    pdl_wait();
    if (i > n || j > n) return;
    const int64_t o = box_off(d.P, i, j), po = mem * d.ms + t * d.ps + o;
    const T h = Y[po], u = Y[po + d.fs], w = Y[po + 2 * d.fs];
    const T *b = v.b + (int64_t)t * 6 * d.ps + o;
    X[dif_base(d, mem, 0) + t * d.ps + o] = h;
#pragma unroll
    for (int k = 0; k < 3; k++)
        X[dif_base(d, mem, 1 + k) + t * d.ps + o] = b[k * d.ps] * u + b[(3 + k) * d.ps] * w;
}

// calc_tile_d1x_d1y: d1x = D1x(f) J Qi12, d1y = D1y(f) J Qi12 (sbp_diff_21 node differences).
// Grid z: panel + NPAN * (field + 4 member).
template <class T>
__global__ void __launch_bounds__(256) k_dif_d1(const T *__restrict__ F, T *__restrict__ D1X, T *__restrict__ D1Y, Dims d,
                                                AhView<T> a)
{
    const int n = d.N + 1;
    const int t = blockIdx.z % NPAN;
    const int64_t base = (int64_t)(blockIdx.z / NPAN) * NPAN * d.ps + t * d.ps;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    pdl_trigger();
    pdl_wait();
    if (i > n || j > n) return;
    const GV<T> f{F + base, d.P};
    const int64_t o = box_off(d.P, i, j);
    const T J = __ldg(a.J + o), Q2 = __ldg(a.Q2 + o);
    D1X[base + o] = dn2n21<T>(i, n, [&](int k) { return f(k, j); }) * J * Q2;
    D1Y[base + o] = dn2n21<T>(j, n, [&](int l) { return f(i, l); }) * J * Q2;
}

// calc_laplace_tile and divide_by_J_self: the panel-local Laplacian of every vertex; the
// panel-boundary vertices' values go to R (for the sync), the others to OUT.
template <class T>
__global__ void __launch_bounds__(256) k_dif_lap(const T *__restrict__ F, const T *__restrict__ D1X,
                                                 const T *__restrict__ D1Y, T *__restrict__ R, T *__restrict__ OUT, Dims d,
                                                 AhView<T> a, DifView<T> v)
{
    const int n = d.N + 1;
    const int t = blockIdx.z % NPAN;
    const int64_t base = (int64_t)(blockIdx.z / NPAN) * NPAN * d.ps + t * d.ps;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    pdl_trigger();
    pdl_wait();
    if (i > n || j > n) return;
    const GV<T> f{F + base, d.P}, dx1{D1X + base, d.P}, dy1{D1Y + base, d.P};
    const GV<T> J{a.J, d.P}, Q1{a.Q1, d.P}, Q3{a.Q3, d.P};
    auto bx = [&](int k) { return Q1(k, j) * J(k, j); };
    auto by = [&](int l) { return Q3(i, l) * J(i, l); };
    T d2x, d2y;
    if (i == 1) {
        const T bc = bx(1), bp = bx(2);
        d2x = (-(bc + bp) * f(1, j) + (bc + bp) * f(2, j));
    } else if (i == n) {
        const T bc = bx(n), bm = bx(n - 1);
        d2x = (bc + bm) * f(n - 1, j) + (-(bc + bm)) * f(n, j);
    } else {
        const T bm = bx(i - 1), bc = bx(i), bp = bx(i + 1);
        const T cm = (bm + bc) / T(2), cc = -(bm + T(2) * bc + bp) / T(2), cp = (bp + bc) / T(2);
        d2x = (cp * f(i + 1, j) + cc * f(i, j) + cm * f(i - 1, j));
    }
    if (j == 1) {
        const T bc = by(1), bp = by(2);
        d2y = -(bc + bp) * f(i, 1) + (bc + bp) * f(i, 2);
    } else if (j == n) {
        const T bc = by(n), bm = by(n - 1);
        d2y = (bc + bm) * f(i, n - 1) + (-(bc + bm)) * f(i, n);
    } else {
        const T bm = by(j - 1), bc = by(j), bp = by(j + 1);
        const T cm = (bm + bc) / T(2), cc = -(bm + T(2) * bc + bp) / T(2), cp = (bp + bc) / T(2);
        d2y = (cp * f(i, j + 1) + cc * f(i, j) + cm * f(i, j - 1));
    }
    // the boundary penalties, all on d2f_x and in the reference's order
    if (i == 1) d2x = d2x - T(0.5) * (T(2) * (T(-2) * dy1(1, j)));
    if (i == n) d2x = d2x - T(0.5) * (T(2) * (T(2) * dy1(n, j)));
    if (j == 1) d2x = d2x - T(0.5) * (T(2) * (T(-2) * dx1(i, 1)));
    if (j == n) d2x = d2x - T(0.5) * (T(2) * (T(2) * dx1(i, n)));
    const T dyx = dn2n21<T>(j, n, [&](int l) { return dx1(i, l); });
    const T dxy = dn2n21<T>(i, n, [&](int k) { return dy1(k, j); });
    T r = d2x + d2y;
    r = r + dxy + dyx;
    r = r / T(v.h2);
    r = r / J(i, j);
    const int64_t o = box_off(d.P, i, j);
    if (i == 1 || i == n || j == 1 || j == n) R[base + o] = r;
    else OUT[base + o] = r;
}

// The Ah scalar sync of the panel-boundary vertices (halo_Ah_scalar_sync_mod.f90:43-98):
// the mean of the copies, in the reference's order.  Thread e of 4N takes boundary vertex
// e of its panel (bottom i = 1..N, right j = 1..N, top i = 2..N+1, left j = 2..N+1).
template <class T>
__global__ void __launch_bounds__(256) k_dif_sync(const T *__restrict__ R, T *__restrict__ OUT, Dims d)
{
    const int N = d.N, n = N + 1;
    const int t = blockIdx.z % NPAN;
    const int64_t fb = (int64_t)(blockIdx.z / NPAN) * NPAN * d.ps;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    pdl_trigger();
    pdl_wait();
    if (e >= 4 * N) return;
    const int s = e / N, a = e % N;
    int i, j;
    switch (s) {
    case 0: i = 1 + a; j = 1; break;
    case 1: i = n; j = 1 + a; break;
    case 2: i = 2 + a; j = n; break;
    default: i = 1; j = 2 + a; break;
    }
    auto val = [&](int p, int k, int l) { return R[fb + p * d.ps + box_off(d.P, k, l)]; };
    auto copy = [&](int side) {
        const Link L = c_link[t][side];
        int kk, ll;
        side_vertex(N, L.nside, nb_along(L, n, along(side, i, j)), 0, kk, ll);
        return val(L.nb, kk, ll);
    };
    const T own = val(t, i, j);
    const bool il = i == 1, ir = i == n, jb = j == 1, jt = j == n;
    T r;
    if ((il || ir) && (jb || jt)) r = (own + copy(il ? SIDE_L : SIDE_R) + copy(jb ? SIDE_B : SIDE_T)) / T(3);
    else if (il) r = T(0.5) * (copy(SIDE_L) + own);
    else if (ir) r = T(0.5) * (own + copy(SIDE_R));
    else if (jb) r = T(0.5) * (own + copy(SIDE_B));
    else r = T(0.5) * (own + copy(SIDE_T));
    OUT[fb + t * d.ps + box_off(d.P, i, j)] = r;
}

// The wind's Cartesian tendencies c_uv L(L(.)) projected on b1, b2 (before the vector sync).
template <class T>
__global__ void __launch_bounds__(256) k_dif_vraw(const T *__restrict__ B, T *__restrict__ UR, T *__restrict__ VR, Dims d,
                                                  DifView<T> v, T kuv)
{
    const int n = d.N + 1;
    const int mem = blockIdx.z / NPAN, t = blockIdx.z % NPAN;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    pdl_trigger();
    pdl_wait();
    if (i > n || j > n) return;
    const int64_t o = box_off(d.P, i, j), to = t * d.ps + o;
    const T tx = kuv * B[dif_base(d, mem, 1) + to], ty = kuv * B[dif_base(d, mem, 2) + to],
            tz = kuv * B[dif_base(d, mem, 3) + to];
    const T *b = v.b + (int64_t)t * 6 * d.ps + o;
    const int64_t mo = (int64_t)mem * NPAN * d.ps + to;
    UR[mo] = tx * b[0] + ty * b[d.ps] + tz * b[2 * d.ps];
    VR[mo] = tx * b[3 * d.ps] + ty * b[4 * d.ps] + tz * b[5 * d.ps];
}

// The covariant ECS Ah vector sync of (u, v) tendencies (syncronize_grad_on_edges with
// (U, V) = (v, u), ecs_Ah_vec_sync_mod.f90:34-125), h's tendency c_h L(L(h)), then
// APPLY: the tendency into OUT; otherwise the Euler update Y += dt tend (explicit_Eul1).
template <class T, bool APPLY>
__global__ void __launch_bounds__(256) k_dif_update(T *Y, T *__restrict__ OUT, const T *__restrict__ B,
                                                    const T *__restrict__ UR, const T *__restrict__ VR, Dims d,
                                                    MetricView<T> m, T kh, T dt)
{
    const int N = d.N, n = N + 1;
    const int mem = blockIdx.z / NPAN, t = blockIdx.z % NPAN;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    pdl_trigger();
    pdl_wait();
    if (i > n || j > n) return;
    const int64_t o = box_off(d.P, i, j), mb = (int64_t)mem * NPAN * d.ps;
    const T th = kh * B[dif_base(d, mem, 0) + t * d.ps + o];
    T gx = UR[mb + t * d.ps + o], gy = VR[mb + t * d.ps + o];
    const bool il = i == 1, ir = i == n, jb = j == 1, jt = j == n;
    const bool cx = il || ir, cy = jb || jt;
    if (cx || cy) {
        auto nb = [&](int s, int a, T &un, T &vn) {
            const Link L = c_link[t][s];
            int kk, ll;
            side_vertex(N, L.nside, nb_along(L, n, a), 0, kk, ll);
            const int64_t q = mb + L.nb * d.ps + box_off(d.P, kk, ll);
            halo_vec(t, s, UR[q], VR[q], un, vn);
        };
        T uhx = 0, vhx = 0, uhy = 0, vhy = 0, qx = 0, qy = 0;
        if (cx) {
            nb(il ? SIDE_L : SIDE_R, j, uhx, vhx);
            qx = (il ? m.ql : m.qr)[j - 1];
        }
        if (cy) {
            nb(jb ? SIDE_B : SIDE_T, i, uhy, vhy);
            qy = (jb ? m.qb : m.qt)[i - 1];
        }
        if (cx && cy) {
            const T sx = (gx + uhx + uhy + qx * vhx) / T(3);
            gy = (gy + vhx + vhy + qy * uhy) / T(3);
            gx = sx;
        } else if (cx) {
            gx = T(0.5) * (gx + uhx + qx * vhx);
            gy = T(0.5) * (gy + vhx);
        } else {
            gx = T(0.5) * (gx + uhy);
            gy = T(0.5) * (gy + vhy + qy * uhy);
        }
    }
    const int64_t po = mem * d.ms + t * d.ps + o;
    if constexpr (APPLY) {
        OUT[po] = th;
        OUT[po + d.fs] = gx;
        OUT[po + 2 * d.fs] = gy;
    } else {
        Y[po] = Y[po] + dt * th;
        Y[po + d.fs] = Y[po + d.fs] + dt * gx;
        Y[po + 2 * d.fs] = Y[po + 2 * d.fs] + dt * gy;
    }
}

}  // namespace chswe

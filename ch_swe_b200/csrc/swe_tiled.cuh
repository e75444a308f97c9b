// swe_tiled.cuh -- the per-stage stencil kernels, shared-memory tiled.
//
// A block of 32 x 8 threads owns a tile [i0, i1) x [j0, j1) of the (N+1) x (N+1)
// box of one panel of one member.  Tiles are balanced: gridDim.x tiles split the
// N+1 columns into widths floor/ceil((N+1)/gridDim.x) <= TILE_XM, likewise rows
// (<= TILE_YM), so N+1 = 32k+1 gives no one-column slivers.  The block copies the
// windows it needs (tile plus stencil footprint) from the zero-margined panel
// boxes into shared memory without bounds checks, then evaluates the SBP
// stencils there.  Warps run along rows, so closure branches of y-direction
// stencils are warp-uniform; x-direction closures diverge only in the warps
// that touch a panel's left or right edge.  Panel-boundary vertices take their
// synchronised values from the edge buffer written by k_edge.
//
// Footprints: a nodes->centres stencil for outputs [a, b) reads inputs
// [a-2, b+3); a centres->nodes stencil reads [a-3, b+2) (closure rows included).
#pragma once

#include "swe_kernels.cuh"

namespace chswe {

constexpr int TILE_XN = 32;     // nominal tile width (tiles = ceil(N / TILE_XN))
constexpr int TILE_YN = 16;     // nominal tile height
constexpr int TILE_XM = 33;     // maximal tile width  (balanced split of N+1 columns)
constexpr int TILE_YM = 17;     // maximal tile height
constexpr int TB_X = 32, TB_Y = 8;   // threads per block
constexpr int STAGE_THREADS = TB_X * TB_Y;
constexpr int WX = TILE_XM + 5, WY = TILE_YM + 5;   // window extents with stencil footprint

__device__ __forceinline__ void tile_range(int n, int &i0, int &i1, int &j0, int &j1)
{
    i0 = 1 + (blockIdx.x * n) / gridDim.x;
    i1 = 1 + ((blockIdx.x + 1) * n) / gridDim.x;
    j0 = 1 + (blockIdx.y * n) / gridDim.y;
    j1 = 1 + ((blockIdx.y + 1) * n) / gridDim.y;
}

// Shared-memory window of NX x NY points with origin (x0, y0) (1-based indices).
template <class T, int NX, int NY>
struct Win {
    T a[NX * NY];
    __device__ __forceinline__ T &at(int x0, int y0, int i, int j) { return a[(j - y0) * NX + (i - x0)]; }
    __device__ __forceinline__ Line<T> row(int x0, int y0, int j) const { return Line<T>{a + (j - y0) * NX - x0, 1}; }
    __device__ __forceinline__ Line<T> col(int x0, int y0, int i) const { return Line<T>{a + (i - x0) - y0 * NX, NX}; }
};

// Copy the window [x0, x0+NX) x [y0, y0+NY) of a zero-margined panel box.
template <class T, int NX, int NY>
__device__ __forceinline__ void stage(Win<T, NX, NY> &w, const T *panel, int P, int x0, int y0)
{
    const T *g = panel + box_off(P, x0, y0);
    for (int r = threadIdx.y; r < NY; r += TB_Y)
        for (int c = threadIdx.x; c < NX; c += TB_X) w.a[r * NX + c] = __ldg(g + r * P + c);
}

// Interior rows of the four operators (the closure rows go through the general
// functions of swe_sbp.cuh).
template <class T> __device__ __forceinline__ T ic2i_in(int k, const Line<T> &f)
{
    return (T(9) * (f(k) + f(k - 1)) - (f(k + 1) + f(k - 2))) * T(0.0625);
}
template <class T> __device__ __forceinline__ T ii2c_in(int k, const Line<T> &f)
{
    return (T(9) * (f(k + 1) + f(k)) - (f(k + 2) + f(k - 1))) * T(0.0625);
}
template <class T> __device__ __forceinline__ T dc2i_in(int k, const Line<T> &f)
{
    return (T(27) * (f(k) - f(k - 1)) - (f(k + 1) - f(k - 2))) * T(1.0 / 24.0);
}
template <class T> __device__ __forceinline__ T di2c_in(int k, const Line<T> &f)
{
    return (T(27) * (f(k + 1) - f(k)) - (f(k + 2) - f(k - 1))) * T(1.0 / 24.0);
}
template <class T> __device__ __forceinline__ T ic2i_x(int k, int nx, const Line<T> &f)
{
    return (k >= 5 && k <= nx - 4) ? ic2i_in<T>(k, f) : ic2i<T>(k, nx, f);
}
template <class T> __device__ __forceinline__ T ii2c_x(int k, int n, const Line<T> &f)
{
    return (k >= 4 && k <= n - 3) ? ii2c_in<T>(k, f) : ii2c<T>(k, n, f);
}
template <class T> __device__ __forceinline__ T dc2i_x(int k, int nx, const Line<T> &f)
{
    return (k >= 5 && k <= nx - 4) ? dc2i_in<T>(k, f) : dc2i<T>(k, nx, f);
}
template <class T> __device__ __forceinline__ T di2c_x(int k, int n, const Line<T> &f)
{
    return (k >= 4 && k <= n - 3) ? di2c_in<T>(k, f) : di2c<T>(k, n, f);
}

// ---------------------------------------------------------------------------
// contravariant components (co2contra_Ch_mod.f90:27-94)
//   ut = Qi11 u + J^-1 I_i2c,x( J Qi12 I_c2i,y(v) ),  vt = Qi22 v + J^-1 I_i2c,y( J Qi12 I_c2i,x(u) )
// ---------------------------------------------------------------------------
template <class T>
struct Co2Smem {
    Win<T, WX, WY> v;              // origin (i0-2, j0-3)
    Win<T, WX, WY> u;              // origin (i0-3, j0-2)
    Win<T, WX, TILE_YM> vq;        // J Qi12 I_c2i,y(v) at xy, origin (i0-2, j0)
    Win<T, TILE_XM, WY> uq;        // J Qi12 I_c2i,x(u) at xy, origin (i0, j0-2)
};

template <class T>
__global__ void __launch_bounds__(STAGE_THREADS) k_co2contra(const T *__restrict__ Y, T *__restrict__ W, Dims d,
                                                              MetricView<T> m)
{
    __shared__ Co2Smem<T> sm;
    const int N = d.N, n = N + 1, P = d.P;
    int i0, i1, j0, j1;
    tile_range(n, i0, i1, j0, j1);
    const int tw = i1 - i0, th = j1 - j0;
    const int t = blockIdx.z % NPAN, mem = blockIdx.z / NPAN;
    const T *y = Y + mem * d.ms + t * d.ps;
    T *w = W + mem * d.ms + t * d.ps;
    const int vx0 = i0 - 2, vy0 = j0 - 3, ux0 = i0 - 3, uy0 = j0 - 2;

    stage(sm.v, y + 2 * d.fs, P, vx0, vy0);
    stage(sm.u, y + 1 * d.fs, P, ux0, uy0);
    __syncthreads();
    for (int r = threadIdx.y; r < th; r += TB_Y) {
        const int l = j0 + r;
        const bool inner = (l >= 5 && l <= n - 4);   // warp-uniform
        for (int c = threadIdx.x; c < tw + 5; c += TB_X) {
            const int k = vx0 + c;
            const Line<T> f = sm.v.col(vx0, vy0, k);
            const T q = inner ? ic2i_in<T>(l, f) : ic2i<T>(l, n, f);
            sm.vq.a[r * WX + c] = q * __ldg(m.JQ12 + box_off(P, k, l));
        }
    }
    for (int r = threadIdx.y; r < th + 5; r += TB_Y) {
        const int l = uy0 + r;
        const Line<T> f = sm.u.row(ux0, uy0, l);
        for (int c = threadIdx.x; c < tw; c += TB_X) {
            const int k = i0 + c;
            sm.uq.a[r * TILE_XM + c] = ic2i_x<T>(k, n, f) * __ldg(m.JQ12 + box_off(P, k, l));
        }
    }
    __syncthreads();
    for (int r = threadIdx.y; r < th; r += TB_Y) {
        const int j = j0 + r;
        const bool jin = (j >= 4 && j <= N - 3);   // warp-uniform
        const Line<T> fq = sm.vq.row(vx0, j0, j);
        for (int c = threadIdx.x; c < tw; c += TB_X) {
            const int i = i0 + c;
            const int64_t o = box_off(P, i, j);
            if (i <= N)
                w[d.fs + o] = __ldg(m.Q11y + o) * sm.u.at(ux0, uy0, i, j) + ii2c_x<T>(i, N, fq) * __ldg(m.iJy + o);
            if (j <= N) {
                const Line<T> g = sm.uq.col(i0, uy0, i);
                const T acc = jin ? ii2c_in<T>(j, g) : ii2c<T>(j, N, g);
                w[2 * d.fs + o] = __ldg(m.Q22x + o) * sm.v.at(vx0, vy0, i, j) + acc * __ldg(m.iJx + o);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// fused stage: tendency of the linear operator + RK4 update
// ---------------------------------------------------------------------------
template <class T>
struct StageSmem {
    Win<T, WX, WY> h;              // origin (i0-2, j0-2)
    Win<T, WX, WY> ut;             // origin (i0-3, j0-2)
    Win<T, WX, WY> vt;             // origin (i0-2, j0-3)
    Win<T, WX, TILE_YM> ju;        // J ut on the tile rows, origin (i0-3, j0)
    Win<T, TILE_XM, WY> jv;        // J vt on the tile columns, origin (i0, j0-3)
    Win<T, WX, TILE_YM> up;        // synchronised up, origin (i0-2, j0)
    Win<T, TILE_XM, WY> vp;        // synchronised vp, origin (i0, j0-2)
    Win<T, TILE_XM, TILE_YM> dv;   // synchronised divergence, origin (i0, j0)
};

//   mode 0: out = A(y)
//   mode 1: Y1 = V0 + dt/2 k,  ACC = dt/6 k
//   mode 2: Y1 = V0 + dt/2 k,  ACC += dt/3 k
//   mode 3: Y1 = V0 + dt   k,  ACC += dt/3 k
//   mode 4: V0 += ACC + dt/6 k          (FP32: Kahan with compensation CMP)
template <class T>
__global__ void __launch_bounds__(STAGE_THREADS) k_stage(const T *__restrict__ Yin, const T *__restrict__ Wc,
                                                          const T *__restrict__ E, T *V0, T *Y1, T *ACC, T *CMP,
                                                          Dims d, MetricView<T> m, StageArgs a)
{
    using namespace sbp;
    __shared__ StageSmem<T> sm;
    const int N = d.N, n = N + 1, P = d.P;
    int i0, i1, j0, j1;
    tile_range(n, i0, i1, j0, j1);
    const int tw = i1 - i0, th = j1 - j0;
    const int t = blockIdx.z % NPAN, mem = blockIdx.z / NPAN;
    const int64_t mo = mem * d.ms;
    const T *y = Yin + mo;                 // member base (h_halo needs the other panels)
    const T *w = Wc + mo;
    const T *yp = y + t * d.ps, *wp = w + t * d.ps;
    const int hx0 = i0 - 2, hy0 = j0 - 2, ux0 = i0 - 3, uy0 = j0 - 2, vx0 = i0 - 2, vy0 = j0 - 3;

    // ---- stage h, ut, vt and the J-weighted copies the divergence reads
    stage(sm.h, yp, P, hx0, hy0);
    {
        const T *g = wp + d.fs + box_off(P, ux0, uy0), *gj = m.Jy + box_off(P, ux0, uy0);
        for (int r = threadIdx.y; r < WY; r += TB_Y)
            for (int c = threadIdx.x; c < WX; c += TB_X) {
                const T v = __ldg(g + r * P + c);
                sm.ut.a[r * WX + c] = v;
                if (r >= 2 && r < TILE_YM + 2) sm.ju.a[(r - 2) * WX + c] = __ldg(gj + r * P + c) * v;
            }
    }
    {
        const T *g = wp + 2 * d.fs + box_off(P, vx0, vy0), *gj = m.Jx + box_off(P, vx0, vy0);
        for (int r = threadIdx.y; r < WY; r += TB_Y)
            for (int c = threadIdx.x; c < WX; c += TB_X) {
                const T v = __ldg(g + r * P + c);
                sm.vt.a[r * WX + c] = v;
                if (c >= 2 && c < TILE_XM + 2) sm.jv.a[r * TILE_XM + (c - 2)] = __ldg(gj + r * P + c) * v;
            }
    }
    __syncthreads();

    // ---- Coriolis vertex vectors and divergence; panel-boundary vertices from the edge buffer
    const T *fJ2 = m.fJ2 + t * d.ps;
    for (int r = threadIdx.y; r < th; r += TB_Y) {
        const int l = j0 + r;
        const bool inner = (l >= 5 && l <= n - 4);      // warp-uniform
        const bool brow = (l == 1 || l == n);           // warp-uniform
        for (int c = threadIdx.x; c < tw + 5; c += TB_X) {
            const int k = vx0 + c;
            T val;
            if (brow || k == 1 || k == n) {
                val = (k >= 1 && k <= n) ? edge_entry(E, N, mem, t, k, l)[0] : T(0);
            } else {
                const Line<T> f = sm.vt.col(vx0, vy0, k);
                val = __ldg(fJ2 + box_off(P, k, l)) * (inner ? ic2i_in<T>(l, f) : ic2i<T>(l, n, f));
            }
            sm.up.a[r * WX + c] = val;
        }
    }
    for (int r = threadIdx.y; r < th + 5; r += TB_Y) {
        const int l = uy0 + r;
        const bool lin = (l >= 1 && l <= n), brow = (l == 1 || l == n);
        const Line<T> f = sm.ut.row(ux0, uy0, l);
        for (int c = threadIdx.x; c < tw; c += TB_X) {
            const int k = i0 + c;
            T val;
            if (lin && (brow || k == 1 || k == n))
                val = edge_entry(E, N, mem, t, k, l)[1];
            else
                val = -__ldg(fJ2 + box_off(P, k, l)) * ic2i_x<T>(k, n, f);
            sm.vp.a[r * TILE_XM + c] = val;
        }
    }
    for (int r = threadIdx.y; r < th; r += TB_Y) {
        const int l = j0 + r;
        const bool inner = (l >= 5 && l <= n - 4), brow = (l == 1 || l == n);
        const Line<T> fx = sm.ju.row(ux0, j0, l);
        for (int c = threadIdx.x; c < tw; c += TB_X) {
            const int k = i0 + c;
            T val;
            if (brow || k == 1 || k == n) {
                val = edge_entry(E, N, mem, t, k, l)[2];
            } else {
                const Line<T> fy = sm.jv.col(i0, vy0, k);
                const T dx = dc2i_x<T>(k, n, fx);
                const T dy = inner ? dc2i_in<T>(l, fy) : dc2i<T>(l, n, fy);
                val = (dx * m.inv_hx + dy * m.inv_hx) * __ldg(m.iJa + box_off(P, k, l));
            }
            sm.dv.a[r * TILE_XM + c] = val;
        }
    }
    __syncthreads();

    // ---- tendencies and the RK4 update
    const T H = T(a.Hm[mem]);
    const T dt = T(a.dt);
    T *v0 = V0 + mo + t * d.ps, *y1 = Y1 + mo + t * d.ps, *acc = ACC + mo + t * d.ps;
    T *cmp = CMP ? CMP + mo + t * d.ps : nullptr;
    const int64_t fs = d.fs;
    for (int r = threadIdx.y; r < th; r += TB_Y) {
        const int j = j0 + r;
        const bool jin = (j >= 4 && j <= N - 3);   // warp-uniform
        const Line<T> hrow = sm.h.row(hx0, hy0, j), uprow = sm.up.row(vx0, j0, j);
        for (int c = threadIdx.x; c < tw; c += TB_X) {
            const int i = i0 + c;
            const int64_t o = box_off(P, i, j);
            const T kh = -H * sm.dv.a[r * TILE_XM + c];
            T ku = 0, kv = 0;
            if (i <= N) {
                T gx = di2c_x<T>(i, N, hrow);
                if (i <= 3) {
                    const T sat = i == 1 ? T(SATI1) : (i == 2 ? T(SATI2) : T(SATI3));
                    gx += sat * (hrow(1) - h_halo(y, d, t, SIDE_L, j));
                }
                if (i >= N - 2) {
                    const T sat = i == N ? T(SATI1) : (i == N - 1 ? T(SATI2) : T(SATI3));
                    gx += sat * (h_halo(y, d, t, SIDE_R, j) - hrow(n));
                }
                gx = gx * m.inv_hxa;
                ku = -m.grav * gx + ii2c_x<T>(i, N, uprow) * __ldg(m.iJy + o);
            }
            if (j <= N) {
                const Line<T> hcol = sm.h.col(hx0, hy0, i), vpcol = sm.vp.col(i0, uy0, i);
                T gy = jin ? di2c_in<T>(j, hcol) : di2c<T>(j, N, hcol);
                if (j <= 3) {
                    const T sat = j == 1 ? T(SATI1) : (j == 2 ? T(SATI2) : T(SATI3));
                    gy += sat * (hcol(1) - h_halo(y, d, t, SIDE_B, i));
                }
                if (j >= N - 2) {
                    const T sat = j == N ? T(SATI1) : (j == N - 1 ? T(SATI2) : T(SATI3));
                    gy += sat * (h_halo(y, d, t, SIDE_T, i) - hcol(n));
                }
                gy = gy * m.inv_hxa;
                const T cv = jin ? ii2c_in<T>(j, vpcol) : ii2c<T>(j, N, vpcol);
                kv = -m.grav * gy + cv * __ldg(m.iJx + o);
            }

            const int64_t oh = o, ou = o + fs, ov = o + 2 * fs;
            const bool hu = (i <= N), hv = (j <= N);
            if (a.mode == 0) {
                y1[oh] = kh;
                if (hu) y1[ou] = ku;
                if (hv) y1[ov] = kv;
                continue;
            }
            if (a.mode <= 3) {
                const T ca = (a.mode == 3) ? dt : T(0.5) * dt;
                const T cb = (a.mode == 1) ? dt / T(6) : dt / T(3);
                y1[oh] = v0[oh] + ca * kh;
                if (hu) y1[ou] = v0[ou] + ca * ku;
                if (hv) y1[ov] = v0[ov] + ca * kv;
                if (a.mode == 1) {
                    acc[oh] = cb * kh;
                    if (hu) acc[ou] = cb * ku;
                    if (hv) acc[ov] = cb * kv;
                } else {
                    acc[oh] += cb * kh;
                    if (hu) acc[ou] += cb * ku;
                    if (hv) acc[ov] += cb * kv;
                }
                continue;
            }
            const T cb = dt / T(6);
            if constexpr (sizeof(T) == 4) {
                float s0 = v0[oh], c0 = cmp[oh];
                kahan_add(s0, c0, acc[oh] + cb * kh);
                v0[oh] = s0; cmp[oh] = c0;
                if (hu) { float s1 = v0[ou], c1 = cmp[ou]; kahan_add(s1, c1, acc[ou] + cb * ku); v0[ou] = s1; cmp[ou] = c1; }
                if (hv) { float s2 = v0[ov], c2 = cmp[ov]; kahan_add(s2, c2, acc[ov] + cb * kv); v0[ov] = s2; cmp[ov] = c2; }
            } else {
                v0[oh] = v0[oh] + (acc[oh] + cb * kh);
                if (hu) v0[ou] = v0[ou] + (acc[ou] + cb * ku);
                if (hv) v0[ov] = v0[ov] + (acc[ov] + cb * kv);
            }
        }
    }
}

}  // namespace chswe

// swe_tiled.cuh -- the two per-stage kernels, shared-memory tiled.
//
// A block owns a tile [i0, i1) x [j0, j1) of the (N+1) x (N+1) box of one panel
// of one member.  Tiles are balanced: gridDim.x tiles split the N+1 columns into
// widths of floor/ceil((N+1)/gridDim.x) (at most TXM), likewise rows (at most TYM),
// so N+1 = 32k+1 gives no one-column slivers.  A block stages the inputs it
// needs (tile plus stencil footprint, clipped to the panel, zero outside) in
// shared memory with coalesced row loads and evaluates the SBP stencils there;
// panel-boundary vertices take their synchronised values from the edge buffer
// written by k_edge (swe_kernels.cuh).
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
constexpr int STAGE_THREADS = 256;

__device__ __forceinline__ void tile_range(int n, int &i0, int &i1, int &j0, int &j1)
{
    i0 = 1 + (int)(((long long)blockIdx.x * n) / gridDim.x);
    i1 = 1 + (int)(((long long)(blockIdx.x + 1) * n) / gridDim.x);
    j0 = 1 + (int)(((long long)blockIdx.y * n) / gridDim.y);
    j1 = 1 + (int)(((long long)(blockIdx.y + 1) * n) / gridDim.y);
}

// Shared-memory window [x0, x0+NX) x [y0, y0+NY), row-major.
template <class T, int NX, int NY>
struct Win {
    T a[NX * NY];
    __device__ __forceinline__ T &at(int x0, int y0, int i, int j) { return a[(j - y0) * NX + (i - x0)]; }
};

// Stage window [x0, x0+NX) x [y0, y0+NY) of a panel field; zero outside [1,vx] x [1,vy].
template <class T, int NX, int NY>
__device__ __forceinline__ void stage(Win<T, NX, NY> &w, const GV<T> &g, int x0, int y0, int vx, int vy)
{
    // batches of four independent loads per thread before the shared-memory stores
    constexpr int TOT = NX * NY, B = 4;
    for (int q0 = threadIdx.x; q0 < TOT; q0 += B * STAGE_THREADS) {
        T v[B];
#pragma unroll
        for (int b = 0; b < B; b++) {
            const int q = q0 + b * STAGE_THREADS;
            const int ci = q % NX, cj = q / NX;
            const int i = x0 + ci, j = y0 + cj;
            v[b] = (q < TOT && i >= 1 && i <= vx && j >= 1 && j <= vy) ? g(i, j) : T(0);
        }
#pragma unroll
        for (int b = 0; b < B; b++) {
            const int q = q0 + b * STAGE_THREADS;
            if (q < TOT) w.a[q] = v[b];
        }
    }
}

// ---------------------------------------------------------------------------
// contravariant components (co2contra_Ch_mod.f90:27-94)
//   ut = Qi11 u + J^-1 I_i2c,x( J Qi12 I_c2i,y(v) ),  vt = Qi22 v + J^-1 I_i2c,y( J Qi12 I_c2i,x(u) )
// ---------------------------------------------------------------------------
template <class T>
struct Co2Smem {
    static constexpr int XM = TILE_XM, YM = TILE_YM;
    Win<T, XM + 5, YM + 5> v;    // cols [i0-2, ...), rows [j0-3, ...)
    Win<T, XM + 5, YM + 5> u;    // cols [i0-3, ...), rows [j0-2, ...)
    Win<T, XM + 5, YM> vq;       // J Qi12 I_c2i,y(v) at xy: cols [i0-2, ...), rows [j0, ...)
    Win<T, XM, YM + 5> uq;       // J Qi12 I_c2i,x(u) at xy: cols [i0, ...),   rows [j0-2, ...)
};

template <class T>
__global__ void __launch_bounds__(STAGE_THREADS) k_co2contra(const T *__restrict__ Y, T *__restrict__ W, Dims d,
                                                              MetricView<T> m)
{
    __shared__ Co2Smem<T> sm;
    constexpr int XM = TILE_XM, YM = TILE_YM;
    const int N = d.N, n = N + 1;
    int i0, i1, j0, j1;
    tile_range(n, i0, i1, j0, j1);
    const int t = blockIdx.z % NPAN, mem = blockIdx.z / NPAN;
    const T *y = Y + mem * d.ms;
    T *w = W + mem * d.ms;
    const int vx0 = i0 - 2, vy0 = j0 - 3, ux0 = i0 - 3, uy0 = j0 - 2;

    stage(sm.v, gview(y, d, 2, t), vx0, vy0, n, N);
    stage(sm.u, gview(y, d, 1, t), ux0, uy0, N, n);
    __syncthreads();
    const GV<T> JQ = mview(m.JQ12, d);
    for (int q = threadIdx.x; q < (XM + 5) * YM; q += STAGE_THREADS) {
        const int k = vx0 + q % (XM + 5), l = j0 + q / (XM + 5);
        T r = 0;
        if (k >= 1 && k <= n && l < j1)
            r = ic2i<T>(l, n, [&](int c) { return sm.v.at(vx0, vy0, k, c); }) * JQ(k, l);
        sm.vq.a[q] = r;
    }
    for (int q = threadIdx.x; q < XM * (YM + 5); q += STAGE_THREADS) {
        const int k = i0 + q % XM, l = uy0 + q / XM;
        T r = 0;
        if (k < i1 && l >= 1 && l <= n)
            r = ic2i<T>(k, n, [&](int c) { return sm.u.at(ux0, uy0, c, l); }) * JQ(k, l);
        sm.uq.a[q] = r;
    }
    __syncthreads();
    const int tw = i1 - i0, npts = tw * (j1 - j0);
    const GV<T> Q11 = mview(m.Q11y, d), iJy = mview(m.iJy, d), Q22 = mview(m.Q22x, d), iJx = mview(m.iJx, d);
    T *wu = w + 1 * d.fs + t * d.ps, *wv = w + 2 * d.fs + t * d.ps;
    for (int q = threadIdx.x; q < npts; q += STAGE_THREADS) {
        const int i = i0 + q % tw, j = j0 + q / tw;
        const int o = (j - 1) * d.P + (i - 1);
        if (i <= N) {
            T acc = ii2c<T>(i, N, [&](int c) { return sm.vq.at(vx0, j0, c, j); });
            wu[o] = Q11(i, j) * sm.u.at(ux0, uy0, i, j) + acc * iJy(i, j);
        }
        if (j <= N) {
            T acc = ii2c<T>(j, N, [&](int c) { return sm.uq.at(i0, uy0, i, c); });
            wv[o] = Q22(i, j) * sm.v.at(vx0, vy0, i, j) + acc * iJx(i, j);
        }
    }
}

// ---------------------------------------------------------------------------
// fused stage: tendency of the linear operator + RK4 update
// ---------------------------------------------------------------------------
template <class T>
struct StageSmem {
    static constexpr int XM = TILE_XM, YM = TILE_YM;
    Win<T, XM + 5, YM + 5> h;    // cols [i0-2, ...), rows [j0-2, ...)
    Win<T, XM + 5, YM + 5> ut;   // cols [i0-3, ...), rows [j0-2, ...)
    Win<T, XM + 5, YM + 5> vt;   // cols [i0-2, ...), rows [j0-3, ...)
    Win<T, XM + 5, YM> ju;       // J ut on the tile rows:    cols [i0-3, ...), rows [j0, ...)
    Win<T, XM, YM + 5> jv;       // J vt on the tile columns: cols [i0, ...),   rows [j0-3, ...)
    Win<T, XM + 5, YM> up;       // synchronised up: cols [i0-2, ...), rows [j0, ...)
    Win<T, XM, YM + 5> vp;       // synchronised vp: cols [i0, ...),   rows [j0-2, ...)
    Win<T, XM, YM> dv;           // synchronised divergence on the tile
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
    constexpr int XM = TILE_XM, YM = TILE_YM, NX5 = TILE_XM + 5;
    const int N = d.N, n = N + 1;
    int i0, i1, j0, j1;
    tile_range(n, i0, i1, j0, j1);
    const int t = blockIdx.z % NPAN, mem = blockIdx.z / NPAN;
    const int64_t mo = mem * d.ms;
    const T *y = Yin + mo;
    const T *w = Wc + mo;
    const int hx0 = i0 - 2, hy0 = j0 - 2, ux0 = i0 - 3, uy0 = j0 - 2, vx0 = i0 - 2, vy0 = j0 - 3;

    // ---- stage h, ut, vt (and J ut, J vt where the divergence needs them)
    stage(sm.h, gview(y, d, 0, t), hx0, hy0, n, n);
    {
        const GV<T> U = gview(w, d, 1, t), Jy = mview(m.Jy, d);
        constexpr int TOT = NX5 * (YM + 5), B = 4;
        for (int q0 = threadIdx.x; q0 < TOT; q0 += B * STAGE_THREADS) {
            T v[B], jj[B];
#pragma unroll
            for (int b = 0; b < B; b++) {
                const int q = q0 + b * STAGE_THREADS;
                const int ci = q % NX5, cj = q / NX5;
                const int i = ux0 + ci, j = uy0 + cj;
                const bool ok = (q < TOT && i >= 1 && i <= N && j >= 1 && j <= n);
                v[b] = ok ? U(i, j) : T(0);
                jj[b] = (ok && cj >= 2 && cj < YM + 2) ? Jy(i, j) : T(0);
            }
#pragma unroll
            for (int b = 0; b < B; b++) {
                const int q = q0 + b * STAGE_THREADS;
                if (q >= TOT) continue;
                const int ci = q % NX5, cj = q / NX5;
                sm.ut.a[q] = v[b];
                if (cj >= 2 && cj < YM + 2) sm.ju.a[(cj - 2) * NX5 + ci] = jj[b] * v[b];
            }
        }
    }
    {
        const GV<T> V = gview(w, d, 2, t), Jx = mview(m.Jx, d);
        constexpr int TOT = NX5 * (YM + 5), B = 4;
        for (int q0 = threadIdx.x; q0 < TOT; q0 += B * STAGE_THREADS) {
            T v[B], jj[B];
#pragma unroll
            for (int b = 0; b < B; b++) {
                const int q = q0 + b * STAGE_THREADS;
                const int ci = q % NX5, cj = q / NX5;
                const int i = vx0 + ci, j = vy0 + cj;
                const bool ok = (q < TOT && i >= 1 && i <= n && j >= 1 && j <= N);
                v[b] = ok ? V(i, j) : T(0);
                jj[b] = (ok && ci >= 2 && ci < XM + 2) ? Jx(i, j) : T(0);
            }
#pragma unroll
            for (int b = 0; b < B; b++) {
                const int q = q0 + b * STAGE_THREADS;
                if (q >= TOT) continue;
                const int ci = q % NX5, cj = q / NX5;
                sm.vt.a[q] = v[b];
                if (ci >= 2 && ci < XM + 2) sm.jv.a[cj * XM + (ci - 2)] = jj[b] * v[b];
            }
        }
    }
    __syncthreads();

    // ---- Coriolis vertex vectors and divergence; panel-boundary vertices synchronised
    const GV<T> fJ2 = mview(m.fJ2 + t * d.ps, d);
    for (int q = threadIdx.x; q < NX5 * YM; q += STAGE_THREADS) {
        const int k = vx0 + q % NX5, l = j0 + q / NX5;
        T r = 0;
        if (k >= 1 && k <= n && l < j1) {
            if (k == 1 || k == n || l == 1 || l == n)
                r = edge_entry(E, N, mem, t, k, l)[0];
            else
                r = fJ2(k, l) * ic2i<T>(l, n, [&](int c) { return sm.vt.at(vx0, vy0, k, c); });
        }
        sm.up.a[q] = r;
    }
    for (int q = threadIdx.x; q < XM * (YM + 5); q += STAGE_THREADS) {
        const int k = i0 + q % XM, l = uy0 + q / XM;
        T r = 0;
        if (k < i1 && l >= 1 && l <= n) {
            if (k == 1 || k == n || l == 1 || l == n)
                r = edge_entry(E, N, mem, t, k, l)[1];
            else
                r = -fJ2(k, l) * ic2i<T>(k, n, [&](int c) { return sm.ut.at(ux0, uy0, c, l); });
        }
        sm.vp.a[q] = r;
    }
    const int tw = i1 - i0, npts = tw * (j1 - j0);
    const GV<T> iJa = mview(m.iJa, d);
    for (int q = threadIdx.x; q < npts; q += STAGE_THREADS) {
        const int k = i0 + q % tw, l = j0 + q / tw;
        T r;
        if (k == 1 || k == n || l == 1 || l == n) {
            r = edge_entry(E, N, mem, t, k, l)[2];
        } else {
            T dx = dc2i<T>(k, n, [&](int c) { return sm.ju.at(ux0, j0, c, l); });
            T dy = dc2i<T>(l, n, [&](int c) { return sm.jv.at(i0, vy0, k, c); });
            r = (dx * m.inv_hx + dy * m.inv_hx) * iJa(k, l);
        }
        sm.dv.at(i0, j0, k, l) = r;
    }
    __syncthreads();

    // ---- tendencies and the RK4 update
    const T H = T(a.Hm[mem]);
    const GV<T> iJy = mview(m.iJy, d), iJx = mview(m.iJx, d);
    const T dt = T(a.dt);
    T *v0 = V0 + mo + t * d.ps, *y1 = Y1 + mo + t * d.ps, *acc = ACC + mo + t * d.ps;
    T *cmp = CMP ? CMP + mo + t * d.ps : nullptr;
    for (int q = threadIdx.x; q < npts; q += STAGE_THREADS) {
        const int i = i0 + q % tw, j = j0 + q / tw;
        const T kh = -H * sm.dv.at(i0, j0, i, j);
        T ku = 0, kv = 0;
        if (i <= N) {
            T gx = di2c<T>(i, N, [&](int c) { return sm.h.at(hx0, hy0, c, j); });
            if (i <= 3) {
                const T sat = i == 1 ? T(SATI1) : (i == 2 ? T(SATI2) : T(SATI3));
                gx += sat * (sm.h.at(hx0, hy0, 1, j) - h_halo(y, d, t, SIDE_L, j));
            }
            if (i >= N - 2) {
                const T sat = i == N ? T(SATI1) : (i == N - 1 ? T(SATI2) : T(SATI3));
                gx += sat * (h_halo(y, d, t, SIDE_R, j) - sm.h.at(hx0, hy0, n, j));
            }
            gx = gx * m.inv_hxa;
            const T cu = ii2c<T>(i, N, [&](int c) { return sm.up.at(vx0, j0, c, j); }) * iJy(i, j);
            ku = -m.grav * gx + cu;
        }
        if (j <= N) {
            T gy = di2c<T>(j, N, [&](int c) { return sm.h.at(hx0, hy0, i, c); });
            if (j <= 3) {
                const T sat = j == 1 ? T(SATI1) : (j == 2 ? T(SATI2) : T(SATI3));
                gy += sat * (sm.h.at(hx0, hy0, i, 1) - h_halo(y, d, t, SIDE_B, i));
            }
            if (j >= N - 2) {
                const T sat = j == N ? T(SATI1) : (j == N - 1 ? T(SATI2) : T(SATI3));
                gy += sat * (h_halo(y, d, t, SIDE_T, i) - sm.h.at(hx0, hy0, i, n));
            }
            gy = gy * m.inv_hxa;
            const T cv = ii2c<T>(j, N, [&](int c) { return sm.vp.at(i0, uy0, i, c); }) * iJx(i, j);
            kv = -m.grav * gy + cv;
        }

        const int o = (j - 1) * d.P + (i - 1);
        const int oh = o, ou = o + (int)d.fs, ov = o + 2 * (int)d.fs;
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

}  // namespace chswe

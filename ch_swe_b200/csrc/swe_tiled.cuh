// swe_tiled.cuh -- shared-memory tiled versions of the two per-stage kernels.
//
// A block owns a TX x TY tile of the (N+1) x (N+1) box of one panel of one
// member.  It stages the inputs it needs (tile plus stencil halo, clipped to
// the panel) in shared memory with coalesced row loads, evaluates the SBP
// stencils from there, and only the threads that own panel-boundary vertices
// read the neighbouring panel (through the global-memory building blocks of
// swe_kernels.cuh) for the edge synchronisation and SAT terms.
#pragma once

#include "swe_kernels.cuh"

namespace chswe {

// sum_q w_q s[(start + q - origin) * stride]; taps with zero weight are skipped
// (closure rows may point outside the staged tile there).
template <class T>
__device__ __forceinline__ T sten_smem(int op, int k, int K, const T *s, int origin, int stride)
{
    const T *w;
    int st = sten<T>(op, k, K, w) - origin;
    T acc = 0;
#pragma unroll
    for (int q = 0; q < 5; q++)
        if (w[q] != T(0)) acc += w[q] * s[(st + q) * stride];
    return acc;
}

// Stage a rectangular window [x0, x0+nx) x [y0, y0+ny) of field f of panel t
// into shared memory (row-major, row length nx); points outside the valid
// range [1, vx] x [1, vy] are set to zero.
template <class T>
__device__ __forceinline__ void stage_window(T *s, const T *base, const Dims &d, int f, int t, int x0, int nx, int y0,
                                             int ny, int vx, int vy, int tid, int nthr)
{
    const T *src = base + f * d.fs + t * d.ps;
    for (int q = tid; q < nx * ny; q += nthr) {
        int ci = q % nx, cj = q / nx;
        int i = x0 + ci, j = y0 + cj;
        s[q] = (i >= 1 && i <= vx && j >= 1 && j <= vy) ? __ldg(src + ofs(d, i, j)) : T(0);
    }
}

// ---------------------------------------------------------------------------
// contravariant components
// ---------------------------------------------------------------------------
template <class T, int TX, int TY>
struct Co2Smem {
    // Footprints: a nodes->centres stencil for outputs [a, b) reads inputs [a-2, b+3),
    // a centres->nodes stencil reads [a-3, b+2) (closure rows included).
    static constexpr int VNX = TX + 5, VNY = TY + 5;   // v  : cols [i0-2, i0+TX+3), rows [j0-3, j0+TY+2)
    static constexpr int UNX = TX + 5, UNY = TY + 5;   // u  : cols [i0-3, i0+TX+2), rows [j0-2, j0+TY+3)
    static constexpr int QNX = TX + 5, QNY = TY;       // J Qi12 I_c2i,y(v) : cols [i0-2, i0+TX+3), rows [j0, j0+TY)
    static constexpr int RNX = TX, RNY = TY + 5;       // J Qi12 I_c2i,x(u) : cols [i0, i0+TX), rows [j0-2, j0+TY+3)
    T v[VNX * VNY];
    T u[UNX * UNY];
    T vq[QNX * QNY];
    T uq[RNX * RNY];
};

template <class T, int TX, int TY>
__global__ void __launch_bounds__(TX *TY) k_co2contra_t(const T *__restrict__ Y, T *__restrict__ W, Dims d,
                                                         MetricView<T> m)
{
    using S = Co2Smem<T, TX, TY>;
    __shared__ S sm;
    const int N = d.N;
    const int i0 = blockIdx.x * TX + 1, j0 = blockIdx.y * TY + 1;
    const int t = blockIdx.z % NPAN, mem = blockIdx.z / NPAN;
    const int tid = threadIdx.y * TX + threadIdx.x, nthr = TX * TY;
    const T *y = Y + mem * d.ms;
    T *w = W + mem * d.ms;
    const int vx0 = i0 - 2, vy0 = j0 - 3, ux0 = i0 - 3, uy0 = j0 - 2;

    stage_window(sm.v, y, d, 2, t, vx0, S::VNX, vy0, S::VNY, N + 1, N, tid, nthr);
    stage_window(sm.u, y, d, 1, t, ux0, S::UNX, uy0, S::UNY, N, N + 1, tid, nthr);
    __syncthreads();
    // J Qi12 * I_c2i,y(v) at xy nodes (k, l)
    for (int q = tid; q < S::QNX * S::QNY; q += nthr) {
        int k = vx0 + q % S::QNX, l = j0 + q / S::QNX;
        T r = 0;
        if (k >= 1 && k <= N + 1 && l >= 1 && l <= N + 1)
            r = sten_smem<T>(OP_IC2I, l, N + 1, sm.v + (k - vx0), vy0, S::VNX) * __ldg(m.JQ12 + ofs(d, k, l));
        sm.vq[q] = r;
    }
    // J Qi12 * I_c2i,x(u) at xy nodes (k, l)
    for (int q = tid; q < S::RNX * S::RNY; q += nthr) {
        int k = i0 + q % S::RNX, l = uy0 + q / S::RNX;
        T r = 0;
        if (k >= 1 && k <= N + 1 && l >= 1 && l <= N + 1)
            r = sten_smem<T>(OP_IC2I, k, N + 1, sm.u + (l - uy0) * S::UNX, ux0, 1) * __ldg(m.JQ12 + ofs(d, k, l));
        sm.uq[q] = r;
    }
    __syncthreads();
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
    if (i <= N && j <= N + 1) {
        T acc = sten_smem<T>(OP_II2C, i, N, sm.vq + (j - j0) * S::QNX, vx0, 1);
        T uij = sm.u[(j - uy0) * S::UNX + (i - ux0)];
        w[1 * d.fs + t * d.ps + ofs(d, i, j)] = __ldg(m.Q11y + ofs(d, i, j)) * uij + acc * __ldg(m.iJy + ofs(d, i, j));
    }
    if (i <= N + 1 && j <= N) {
        T acc = sten_smem<T>(OP_II2C, j, N, sm.uq + (i - i0), uy0, S::RNX);
        T vij = sm.v[(j - vy0) * S::VNX + (i - vx0)];
        w[2 * d.fs + t * d.ps + ofs(d, i, j)] = __ldg(m.Q22x + ofs(d, i, j)) * vij + acc * __ldg(m.iJx + ofs(d, i, j));
    }
}

// ---------------------------------------------------------------------------
// fused stage: tendency + RK4 update
// ---------------------------------------------------------------------------
template <class T, int TX, int TY>
struct StageSmem {
    static constexpr int HNX = TX + 5, HNY = TY + 5;   // h  : cols [i0-2, i0+TX+3), rows [j0-2, j0+TY+3)
    static constexpr int UNX = TX + 5, UNY = TY + 5;   // ut : cols [i0-3, i0+TX+2), rows [j0-2, j0+TY+3)
    static constexpr int VNX = TX + 5, VNY = TY + 5;   // vt : cols [i0-2, i0+TX+3), rows [j0-3, j0+TY+2)
    static constexpr int PNX = TX + 5, PNY = TY;       // synced up : cols [i0-2, i0+TX+3), rows [j0, j0+TY)
    static constexpr int QNX = TX, QNY = TY + 5;       // synced vp : cols [i0, i0+TX), rows [j0-2, j0+TY+3)
    T h[HNX * HNY];
    T ut[UNX * UNY];
    T vt[VNX * VNY];
    T up[PNX * PNY];
    T vp[QNX * QNY];
};

template <class T, int TX, int TY>
__global__ void __launch_bounds__(TX *TY) k_stage_t(const T *__restrict__ Yin, const T *__restrict__ Wc, T *V0, T *Y1,
                                                     T *ACC, T *CMP, Dims d, MetricView<T> m, StageArgs a)
{
    using S = StageSmem<T, TX, TY>;
    __shared__ S sm;
    const int N = d.N, n = N + 1;
    const int i0 = blockIdx.x * TX + 1, j0 = blockIdx.y * TY + 1;
    const int t = blockIdx.z % NPAN, mem = blockIdx.z / NPAN;
    const int tid = threadIdx.y * TX + threadIdx.x, nthr = TX * TY;
    const int64_t mo = mem * d.ms;
    const T *y = Yin + mo;
    const T *w = Wc + mo;
    const int hx0 = i0 - 2, hy0 = j0 - 2, ux0 = i0 - 3, uy0 = j0 - 2, vx0 = i0 - 2, vy0 = j0 - 3;

    stage_window(sm.h, y, d, 0, t, hx0, S::HNX, hy0, S::HNY, n, n, tid, nthr);
    stage_window(sm.ut, w, d, 1, t, ux0, S::UNX, uy0, S::UNY, N, n, tid, nthr);
    stage_window(sm.vt, w, d, 2, t, vx0, S::VNX, vy0, S::VNY, n, N, tid, nthr);
    __syncthreads();

    // Coriolis vertex vectors: up = fJ2 I_c2i,y(vt) on the up window, vp = -fJ2 I_c2i,x(ut)
    // on the vp window; panel-boundary vertices take the synchronised value.
    const T *fJ2 = m.fJ2 + t * d.ps;
    for (int q = tid; q < S::PNX * S::PNY; q += nthr) {
        int k = vx0 + q % S::PNX, l = j0 + q / S::PNX;
        T r = 0;
        if (k >= 1 && k <= n && l >= 1 && l <= n) {
            if (k == 1 || k == n || l == 1 || l == n) {
                T vps;
                cor_sync(w, d, m, t, k, l, r, vps);
            } else {
                r = __ldg(fJ2 + ofs(d, k, l)) * sten_smem<T>(OP_IC2I, l, n, sm.vt + (k - vx0), vy0, S::VNX);
            }
        }
        sm.up[q] = r;
    }
    for (int q = tid; q < S::QNX * S::QNY; q += nthr) {
        int k = i0 + q % S::QNX, l = uy0 + q / S::QNX;
        T r = 0;
        if (k >= 1 && k <= n && l >= 1 && l <= n) {
            if (k == 1 || k == n || l == 1 || l == n) {
                T ups;
                cor_sync(w, d, m, t, k, l, ups, r);
            } else {
                r = -__ldg(fJ2 + ofs(d, k, l)) * sten_smem<T>(OP_IC2I, k, n, sm.ut + (l - uy0) * S::UNX, ux0, 1);
            }
        }
        sm.vp[q] = r;
    }

    // divergence at the own xy point (Ah-synchronised on the panel boundary)
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
    const bool own = (i <= n && j <= n);
    T dvg = 0;
    if (own) {
        if (i == 1 || i == n || j == 1 || j == n) {
            dvg = div_sync(w, d, m, t, i, j);
        } else {
            // interior: c2i differences of J ut along x and J vt along y (no SAT)
            const T *wx;
            int s = sten<T>(OP_DC2I, i, n, wx);
            T dx = 0;
#pragma unroll
            for (int q = 0; q < 5; q++) {
                int ii = s + q;
                if (wx[q] != T(0))
                    dx += wx[q] * (__ldg(m.Jy + ofs(d, ii, j)) * sm.ut[(j - uy0) * S::UNX + (ii - ux0)]);
            }
            s = sten<T>(OP_DC2I, j, n, wx);
            T dy = 0;
#pragma unroll
            for (int q = 0; q < 5; q++) {
                int jj = s + q;
                if (wx[q] != T(0))
                    dy += wx[q] * (__ldg(m.Jx + ofs(d, i, jj)) * sm.vt[(jj - vy0) * S::VNX + (i - vx0)]);
            }
            dvg = (dx * m.inv_hx + dy * m.inv_hx) * __ldg(m.iJa + ofs(d, i, j));
        }
    }
    __syncthreads();
    if (!own) return;

    const T H = T(a.Hm[mem]);
    T kh = -H * dvg, ku = 0, kv = 0;
    const T *hrow = sm.h + (j - hy0) * S::HNX;   // row j of h, origin hx0
    if (i <= N) {
        T gx = sten_smem<T>(OP_DI2C, i, N, hrow, hx0, 1);
        if (i <= 3) gx += satc<T>(i - 1) * (hrow[1 - hx0] - h_halo(y, d, t, SIDE_L, j));
        if (i >= N - 2) gx += satc<T>(N - i) * (h_halo(y, d, t, SIDE_R, j) - hrow[n - hx0]);
        gx = gx * m.inv_hxa;
        T cu = sten_smem<T>(OP_II2C, i, N, sm.up + (j - j0) * S::PNX, vx0, 1) * __ldg(m.iJy + ofs(d, i, j));
        ku = -m.grav * gx + cu;
    }
    if (j <= N) {
        const T *hcol = sm.h + (i - hx0);   // column i of h, origin hy0, stride HNX
        T gy = sten_smem<T>(OP_DI2C, j, N, hcol, hy0, S::HNX);
        if (j <= 3) gy += satc<T>(j - 1) * (hcol[(1 - hy0) * S::HNX] - h_halo(y, d, t, SIDE_B, i));
        if (j >= N - 2) gy += satc<T>(N - j) * (h_halo(y, d, t, SIDE_T, i) - hcol[(n - hy0) * S::HNX]);
        gy = gy * m.inv_hxa;
        T cv = sten_smem<T>(OP_II2C, j, N, sm.vp + (i - i0), uy0, S::QNX) * __ldg(m.iJx + ofs(d, i, j));
        kv = -m.grav * gy + cv;
    }

    const int64_t base = mo + t * d.ps + ofs(d, i, j);
    const int64_t ih = base, iu = base + d.fs, iv = base + 2 * d.fs;
    const bool hu = (i <= N), hv = (j <= N);
    if (a.mode == 0) {
        Y1[ih] = kh;
        if (hu) Y1[iu] = ku;
        if (hv) Y1[iv] = kv;
        return;
    }
    const T dt = T(a.dt);
    if (a.mode <= 3) {
        const T ca = (a.mode == 3) ? dt : T(0.5) * dt;
        const T cb = (a.mode == 1) ? dt / T(6) : dt / T(3);
        Y1[ih] = V0[ih] + ca * kh;
        if (hu) Y1[iu] = V0[iu] + ca * ku;
        if (hv) Y1[iv] = V0[iv] + ca * kv;
        if (a.mode == 1) {
            ACC[ih] = cb * kh;
            if (hu) ACC[iu] = cb * ku;
            if (hv) ACC[iv] = cb * kv;
        } else {
            ACC[ih] += cb * kh;
            if (hu) ACC[iu] += cb * ku;
            if (hv) ACC[iv] += cb * kv;
        }
        return;
    }
    const T cb = dt / T(6);
    if constexpr (sizeof(T) == 4) {
        float s0 = V0[ih], c0 = CMP[ih];
        kahan_add(s0, c0, ACC[ih] + cb * kh);
        V0[ih] = s0; CMP[ih] = c0;
        if (hu) { float s1 = V0[iu], c1 = CMP[iu]; kahan_add(s1, c1, ACC[iu] + cb * ku); V0[iu] = s1; CMP[iu] = c1; }
        if (hv) { float s2 = V0[iv], c2 = CMP[iv]; kahan_add(s2, c2, ACC[iv] + cb * kv); V0[iv] = s2; CMP[iv] = c2; }
    } else {
        V0[ih] = V0[ih] + (ACC[ih] + cb * kh);
        if (hu) V0[iu] = V0[iu] + (ACC[iu] + cb * ku);
        if (hv) V0[iv] = V0[iv] + (ACC[iv] + cb * kv);
    }
}

}  // namespace chswe

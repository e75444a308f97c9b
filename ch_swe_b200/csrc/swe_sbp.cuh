// swe_sbp.cuh -- the one-dimensional SBP 4-2 operators of the Ch grid as
// device stencils over an accessor f(index) (1-based input index).
//
// Coefficients (src/differential_operators/sbp_operators/):
//   difference nodes -> centres   sbp_diff_i2c_42_mod.f90:12-20,  stencil :29-160, SAT :162-274
//   difference centres -> nodes   sbp_diff_c2i_42_mod.f90:12-22,  stencil :32-193, SAT :195-251
//   interpolation nodes -> centres sbp_interp_i2c_42_mod.f90:18-35
//   interpolation centres -> nodes sbp_interp_c2i_42_mod.f90:13-27
// Interior rows use compile-time coefficients; closure rows (three or four at
// each end) are selected by a branch that is warp-uniform away from panel edges.
#pragma once

#include "sbp63.h"

namespace chswe {
namespace sbp {

// difference, nodes -> centres
constexpr double DI11 = -79.0 / 78.0, DI12 = 27.0 / 26.0, DI13 = -1.0 / 26.0, DI14 = 1.0 / 78.0;
constexpr double DI21 = 2.0 / 21.0, DI22 = -9.0 / 7.0, DI23 = 9.0 / 7.0, DI24 = -2.0 / 21.0;
constexpr double DI31 = 1.0 / 75.0, DI33 = -27.0 / 25.0, DI34 = 83.0 / 75.0, DI35 = -1.0 / 25.0;
// boundary projection and SAT weights 0.5 R1r / h_rr of the nodes -> centres difference
constexpr double R11 = 15.0 / 8.0, R12 = -5.0 / 4.0, R13 = 3.0 / 8.0;
constexpr double SATI1 = 0.5 * R11 / (13.0 / 12.0), SATI2 = 0.5 * R12 / (7.0 / 8.0), SATI3 = 0.5 * R13 / (25.0 / 24.0);
// difference, centres -> nodes
constexpr double DC11 = -2.0, DC12 = 3.0, DC13 = -1.0, DC21 = -1.0, DC22 = 1.0;
constexpr double DC31 = 1.0 / 24.0, DC32 = -9.0 / 8.0, DC33 = 9.0 / 8.0, DC34 = -1.0 / 24.0;
constexpr double DC41 = -1.0 / 71.0, DC42 = 6.0 / 71.0, DC43 = -83.0 / 71.0, DC44 = 81.0 / 71.0, DC45 = -3.0 / 71.0;
constexpr double SATC = 0.5 / (7.0 / 18.0);
// interpolation free parameters
constexpr double C13 = 0.1264926207034815, C14 = -0.029892648949074313;
// interpolation, nodes -> centres
constexpr double II11 = 1.0 / 2.0 + C13 + 2.0 * C14, II12 = 1.0 / 2.0 - 2.0 * C13 - 3.0 * C14, II13 = C13, II14 = C14;
constexpr double II21 = -8.0 / 63.0 - 52.0 / 21.0 * C13 - 104.0 / 21.0 * C14;
constexpr double II22 = 29.0 / 42.0 + 104.0 / 21.0 * C13 + 52.0 / 7.0 * C14;
constexpr double II23 = -52.0 / 21.0 * C13 + 1.0 / 2.0, II24 = -52.0 / 21.0 * C14 - 4.0 / 63.0;
constexpr double II31 = 26.0 / 25.0 * C13 + 52.0 / 25.0 * C14 - 1.0 / 25.0;
constexpr double II32 = -1.0 / 50.0 - 52.0 / 25.0 * C13 - 78.0 / 25.0 * C14;
constexpr double II33 = 3.0 / 5.0 + 26.0 / 25.0 * C13, II34 = 13.0 / 25.0 + 26.0 / 25.0 * C14, II35 = -3.0 / 50.0;
// interpolation, centres -> nodes
constexpr double IC11 = 39.0 / 28.0 + 39.0 / 14.0 * C13 + 39.0 / 7.0 * C14;
constexpr double IC12 = -2.0 / 7.0 - 39.0 / 7.0 * C13 - 78.0 / 7.0 * C14;
constexpr double IC13 = 39.0 / 14.0 * C13 + 39.0 / 7.0 * C14 - 3.0 / 28.0;
constexpr double IC21 = 13.0 / 27.0 - 52.0 / 27.0 * C13 - 26.0 / 9.0 * C14;
constexpr double IC22 = 29.0 / 54.0 + 104.0 / 27.0 * C13 + 52.0 / 9.0 * C14;
constexpr double IC23 = -1.0 / 54.0 - 52.0 / 27.0 * C13 - 26.0 / 9.0 * C14;
constexpr double IC31 = 13.0 / 12.0 * C13, IC32 = -13.0 / 6.0 * C13 + 7.0 / 16.0, IC33 = 5.0 / 8.0 + 13.0 / 12.0 * C13,
                 IC34 = -1.0 / 16.0;
constexpr double IC41 = 78.0 / 71.0 * C14, IC42 = -156.0 / 71.0 * C14 - 4.0 / 71.0, IC43 = 39.0 / 71.0 + 78.0 / 71.0 * C14,
                 IC44 = 81.0 / 142.0, IC45 = -9.0 / 142.0;

}  // namespace sbp

// Difference nodes -> centres at centre k of n (inputs nodes 1..n+1).
template <class T, class F>
__device__ __forceinline__ T di2c(int k, int n, const F &f)
{
    using namespace sbp;
    if (k >= 4 && k <= n - 3) return (T(27) * (f(k + 1) - f(k)) - (f(k + 2) - f(k - 1))) * T(1.0 / 24.0);
    if (k == 1) return T(DI11) * f(1) + T(DI12) * f(2) + T(DI13) * f(3) + T(DI14) * f(4);
    if (k == 2) return T(DI21) * f(1) + T(DI22) * f(2) + T(DI23) * f(3) + T(DI24) * f(4);
    if (k == 3) return T(DI31) * f(1) + T(DI33) * f(3) + T(DI34) * f(4) + T(DI35) * f(5);
    if (k == n - 2) return -T(DI31) * f(n + 1) - T(DI33) * f(n - 1) - T(DI34) * f(n - 2) - T(DI35) * f(n - 3);
    if (k == n - 1) return -T(DI21) * f(n + 1) - T(DI22) * f(n) - T(DI23) * f(n - 1) - T(DI24) * f(n - 2);
    return -T(DI11) * f(n + 1) - T(DI12) * f(n) - T(DI13) * f(n - 1) - T(DI14) * f(n - 2);
}

// Difference centres -> nodes at node k of nx (inputs centres 1..nx-1).
template <class T, class F>
__device__ __forceinline__ T dc2i(int k, int nx, const F &f)
{
    using namespace sbp;
    if (k >= 5 && k <= nx - 4) return (T(27) * (f(k) - f(k - 1)) - (f(k + 1) - f(k - 2))) * T(1.0 / 24.0);
    if (k == 1) return T(DC11) * f(1) + T(DC12) * f(2) + T(DC13) * f(3);
    if (k == 2) return T(DC21) * f(1) + T(DC22) * f(2);
    if (k == 3) return T(DC31) * f(1) + T(DC32) * f(2) + T(DC33) * f(3) + T(DC34) * f(4);
    if (k == 4) return T(DC41) * f(1) + T(DC42) * f(2) + T(DC43) * f(3) + T(DC44) * f(4) + T(DC45) * f(5);
    if (k == nx - 3)
        return -T(DC41) * f(nx - 1) - T(DC42) * f(nx - 2) - T(DC43) * f(nx - 3) - T(DC44) * f(nx - 4) -
               T(DC45) * f(nx - 5);
    if (k == nx - 2) return -T(DC31) * f(nx - 1) - T(DC32) * f(nx - 2) - T(DC33) * f(nx - 3) - T(DC34) * f(nx - 4);
    if (k == nx - 1) return -T(DC21) * f(nx - 1) - T(DC22) * f(nx - 2);
    return -T(DC11) * f(nx - 1) - T(DC12) * f(nx - 2) - T(DC13) * f(nx - 3);
}

// Interpolation nodes -> centres at centre k of n.
template <class T, class F>
__device__ __forceinline__ T ii2c(int k, int n, const F &f)
{
    using namespace sbp;
    if (k >= 4 && k <= n - 3) return (T(9) * (f(k + 1) + f(k)) - (f(k + 2) + f(k - 1))) * T(0.0625);
    if (k == 1) return T(II11) * f(1) + T(II12) * f(2) + T(II13) * f(3) + T(II14) * f(4);
    if (k == 2) return T(II21) * f(1) + T(II22) * f(2) + T(II23) * f(3) + T(II24) * f(4);
    if (k == 3) return T(II31) * f(1) + T(II32) * f(2) + T(II33) * f(3) + T(II34) * f(4) + T(II35) * f(5);
    if (k == n - 2)
        return T(II31) * f(n + 1) + T(II32) * f(n) + T(II33) * f(n - 1) + T(II34) * f(n - 2) + T(II35) * f(n - 3);
    if (k == n - 1) return T(II21) * f(n + 1) + T(II22) * f(n) + T(II23) * f(n - 1) + T(II24) * f(n - 2);
    return T(II11) * f(n + 1) + T(II12) * f(n) + T(II13) * f(n - 1) + T(II14) * f(n - 2);
}

// Interpolation centres -> nodes at node k of nx.
template <class T, class F>
__device__ __forceinline__ T ic2i(int k, int nx, const F &f)
{
    using namespace sbp;
    if (k >= 5 && k <= nx - 4) return (T(9) * (f(k) + f(k - 1)) - (f(k + 1) + f(k - 2))) * T(0.0625);
    if (k == 1) return T(IC11) * f(1) + T(IC12) * f(2) + T(IC13) * f(3);
    if (k == 2) return T(IC21) * f(1) + T(IC22) * f(2) + T(IC23) * f(3);
    if (k == 3) return T(IC31) * f(1) + T(IC32) * f(2) + T(IC33) * f(3) + T(IC34) * f(4);
    if (k == 4) return T(IC41) * f(1) + T(IC42) * f(2) + T(IC43) * f(3) + T(IC44) * f(4) + T(IC45) * f(5);
    if (k == nx - 3)
        return T(IC41) * f(nx - 1) + T(IC42) * f(nx - 2) + T(IC43) * f(nx - 3) + T(IC44) * f(nx - 4) +
               T(IC45) * f(nx - 5);
    if (k == nx - 2) return T(IC31) * f(nx - 1) + T(IC32) * f(nx - 2) + T(IC33) * f(nx - 3) + T(IC34) * f(nx - 4);
    if (k == nx - 1) return T(IC21) * f(nx - 1) + T(IC22) * f(nx - 2) + T(IC23) * f(nx - 3);
    return T(IC11) * f(nx - 1) + T(IC12) * f(nx - 2) + T(IC13) * f(nx - 3);
}

// SBP 2-1 operators (sbp_diff_i2c_21_mod.f90:33-41, sbp_diff_c2i_21_mod.f90:32-42,
// sbp_interp_i2c_21_mod.f90:25-31, sbp_interp_c2i_21_mod.f90:25-35): two-point
// interior rows, one-sided first and last rows of the centres->nodes operators.
template <class T, class F>
__device__ __forceinline__ T di2c21(int k, int, const F &f) { return f(k + 1) - f(k); }
template <class T, class F>
__device__ __forceinline__ T dc2i21(int k, int nx, const F &f)
{
    if (k == 1) return f(2) - f(1);
    if (k == nx) return f(nx - 1) - f(nx - 2);
    return f(k) - f(k - 1);
}
template <class T, class F>
__device__ __forceinline__ T ii2c21(int k, int, const F &f) { return T(0.5) * (f(k + 1) + f(k)); }
template <class T, class F>
__device__ __forceinline__ T ic2i21(int k, int nx, const F &f)
{
    if (k == 1) return f(1);
    if (k == nx) return f(nx - 1);
    return T(0.5) * (f(k) + f(k - 1));
}

// SBP 6-3 operators (sbp_diff_i2c_63_mod.f90:84-134, sbp_diff_c2i_63_mod.f90:82-124,
// sbp_interp_i2c_63_mod.f90:82-130, sbp_interp_c2i_63_mod.f90:70-112): six-point
// interior rows, table-driven closure rows (sbp63.h), mirrored at the far end.
template <class T, class F>
__device__ __forceinline__ T di2c63(int k, int n, const F &f)
{
    const double *C = D_SBP63_DI_C;
    if (k >= 7 && k <= n - 6)
        return T(C[0]) * (f(k + 1) - f(k)) + T(C[1]) * (f(k + 2) - f(k - 1)) + T(C[2]) * (f(k + 3) - f(k - 2));
    const int w[6] = {5, 5, 6, 7, 8, 9};
    const bool lo = k <= 6;
    const int r = lo ? k : n + 1 - k;
    T a = T(0);
    for (int j = 0; j < w[r - 1]; j++) a += T(D_SBP63_DI_Q[r - 1][j]) * (lo ? f(j + 1) : f(n + 1 - j));
    return lo ? a : -a;
}
template <class T, class F>
__device__ __forceinline__ T dc2i63(int k, int nx, const F &f)
{
    const double *C = D_SBP63_DC_C;
    if (k >= 6 && k <= nx - 5)
        return T(C[0]) * (f(k) - f(k - 1)) + T(C[1]) * (f(k + 1) - f(k - 2)) + T(C[2]) * (f(k + 2) - f(k - 3));
    const int w[5] = {6, 6, 6, 6, 7};
    const bool lo = k <= 5;
    const int r = lo ? k : nx + 1 - k;
    T a = T(0);
    for (int j = 0; j < w[r - 1]; j++) a += T(D_SBP63_DC_Q[r - 1][j]) * (lo ? f(j + 1) : f(nx - 1 - j));
    return lo ? a : -a;
}
template <class T, class F>
__device__ __forceinline__ T ii2c63(int k, int n, const F &f)
{
    const double *C = D_SBP63_II_C;
    if (k >= 7 && k <= n - 6)
        return T(C[0]) * (f(k + 1) + f(k)) + T(C[1]) * (f(k + 2) + f(k - 1)) + T(C[2]) * (f(k + 3) + f(k - 2));
    const int w[6] = {5, 5, 6, 7, 8, 9};
    const bool lo = k <= 6;
    const int r = lo ? k : n + 1 - k;
    T a = T(0);
    for (int j = 0; j < w[r - 1]; j++) a += T(D_SBP63_II_Q[r - 1][j]) * (lo ? f(j + 1) : f(n + 1 - j));
    return a;
}
template <class T, class F>
__device__ __forceinline__ T ic2i63(int k, int nx, const F &f)
{
    const double *C = D_SBP63_IC_C;
    if (k >= 6 && k <= nx - 5)
        return T(C[0]) * (f(k) + f(k - 1)) + T(C[1]) * (f(k + 1) + f(k - 2)) + T(C[2]) * (f(k + 2) + f(k - 3));
    const int w[5] = {6, 6, 6, 6, 7};
    const bool lo = k <= 5;
    const int r = lo ? k : nx + 1 - k;
    T a = T(0);
    for (int j = 0; j < w[r - 1]; j++) a += T(D_SBP63_IC_Q[r - 1][j]) * (lo ? f(j + 1) : f(nx - 1 - j));
    return a;
}

// The order-dependent parts of the Ch operators, by SBP order (42, 21 or 63):
//   C2I_LO/HI: nodes k in [C2I_LO, nx - C2I_HI] use the interior c2i rows;
//   I2C_LO/HI: centres k in [I2C_LO, n - I2C_HI] use the interior i2c rows;
//   GRAD_LO/HI: centres with the interior i2c difference and no gradient SAT;
//   U_LO/HI: u-point columns [U_LO, N - U_HI] clear of both (the grad_x + I_i2c,x pass);
//   V_LO/HI: rows [V_LO, N - V_HI] clear of the c2i and i2c closures, the gradient SAT
//            and the panel-boundary rows (the final pass);
//   RUN_OK: the interior rows read four consecutive inputs (the stencil runs);
//   NSAT, satw(r): gradient SAT weights 0.5 R1r / h_rr of rows r = 1..NSAT (mirrored);
//   NDEP: inputs of the first c2i rows; the edge strips hold NDEP normal lines;
//   ic1(d), dc1(d): first c2i interpolation / difference row, input d = 1..NDEP;
//   NR, r1(d), SATC: divergence SAT 0.5 / h11 * sum_d R1d (f(d) - f(1 - d)), d <= NR.
template <int ORD>
struct SbpOrder;

template <>
struct SbpOrder<42> {
    static constexpr int C2I_LO = 5, C2I_HI = 4, I2C_LO = 4, I2C_HI = 3, GRAD_LO = 4, GRAD_HI = 3;
    static constexpr int U_LO = 4, U_HI = 3, V_LO = 5, V_HI = 3;
    static constexpr bool RUN_OK = true;
    static constexpr int NSAT = 3, NDEP = 3, NR = 3;
    static constexpr double SATC = sbp::SATC;
    static __device__ __forceinline__ double satw(int r) { return r == 1 ? sbp::SATI1 : (r == 2 ? sbp::SATI2 : sbp::SATI3); }
    static __device__ __forceinline__ double ic1(int d) { return d == 1 ? sbp::IC11 : (d == 2 ? sbp::IC12 : sbp::IC13); }
    static __device__ __forceinline__ double dc1(int d) { return d == 1 ? sbp::DC11 : (d == 2 ? sbp::DC12 : sbp::DC13); }
    static __device__ __forceinline__ double r1(int d) { return d == 1 ? sbp::R11 : (d == 2 ? sbp::R12 : sbp::R13); }
    template <class T, class F> static __device__ __forceinline__ T di2c(int k, int n, const F &f) { return chswe::di2c<T>(k, n, f); }
    template <class T, class F> static __device__ __forceinline__ T dc2i(int k, int nx, const F &f) { return chswe::dc2i<T>(k, nx, f); }
    template <class T, class F> static __device__ __forceinline__ T ii2c(int k, int n, const F &f) { return chswe::ii2c<T>(k, n, f); }
    template <class T, class F> static __device__ __forceinline__ T ic2i(int k, int nx, const F &f) { return chswe::ic2i<T>(k, nx, f); }
    // interior rows on four consecutive inputs: c2i rows take v0..v3 = f(k-2..k+1),
    // i2c rows v0..v3 = f(k-1..k+2)
    template <class T> static __device__ __forceinline__ T interp4(T v0, T v1, T v2, T v3)
    {
        return (T(9) * (v2 + v1) - (v3 + v0)) * T(0.0625);
    }
    template <class T> static __device__ __forceinline__ T diff4(T v0, T v1, T v2, T v3)
    {
        return (T(27) * (v2 - v1) - (v3 - v0)) * T(1.0 / 24.0);
    }
    template <class T, class F> static __device__ __forceinline__ T ic2i_in(int k, const F &f) { return interp4<T>(f(k - 2), f(k - 1), f(k), f(k + 1)); }
    template <class T, class F> static __device__ __forceinline__ T dc2i_in(int k, const F &f) { return diff4<T>(f(k - 2), f(k - 1), f(k), f(k + 1)); }
    template <class T, class F> static __device__ __forceinline__ T ii2c_in(int k, const F &f) { return interp4<T>(f(k - 1), f(k), f(k + 1), f(k + 2)); }
    template <class T, class F> static __device__ __forceinline__ T di2c_in(int k, const F &f) { return diff4<T>(f(k - 1), f(k), f(k + 1), f(k + 2)); }
};

template <>
struct SbpOrder<21> {
    static constexpr int C2I_LO = 2, C2I_HI = 1, I2C_LO = 1, I2C_HI = 0, GRAD_LO = 3, GRAD_HI = 2;
    static constexpr int U_LO = 3, U_HI = 2, V_LO = 3, V_HI = 2;
    static constexpr bool RUN_OK = true;
    // h11 = h22 = 1 (i2c), h11 = 1/2 (c2i), R11 = 3/2, R12 = -1/2
    static constexpr int NSAT = 2, NDEP = 3, NR = 2;
    static constexpr double SATC = 0.5 / 0.5;
    static __device__ __forceinline__ double satw(int r) { return r == 1 ? 0.5 * 1.5 : 0.5 * -0.5; }
    static __device__ __forceinline__ double ic1(int d) { return d == 1 ? 1.0 : 0.0; }
    static __device__ __forceinline__ double dc1(int d) { return d == 1 ? -1.0 : (d == 2 ? 1.0 : 0.0); }
    static __device__ __forceinline__ double r1(int d) { return d == 1 ? 1.5 : -0.5; }
    template <class T, class F> static __device__ __forceinline__ T di2c(int k, int n, const F &f) { return di2c21<T>(k, n, f); }
    template <class T, class F> static __device__ __forceinline__ T dc2i(int k, int nx, const F &f) { return dc2i21<T>(k, nx, f); }
    template <class T, class F> static __device__ __forceinline__ T ii2c(int k, int n, const F &f) { return ii2c21<T>(k, n, f); }
    template <class T, class F> static __device__ __forceinline__ T ic2i(int k, int nx, const F &f) { return ic2i21<T>(k, nx, f); }
    template <class T> static __device__ __forceinline__ T interp4(T, T v1, T v2, T) { return T(0.5) * (v2 + v1); }
    template <class T> static __device__ __forceinline__ T diff4(T, T v1, T v2, T) { return v2 - v1; }
    template <class T, class F> static __device__ __forceinline__ T ic2i_in(int k, const F &f) { return T(0.5) * (f(k) + f(k - 1)); }
    template <class T, class F> static __device__ __forceinline__ T dc2i_in(int k, const F &f) { return f(k) - f(k - 1); }
    template <class T, class F> static __device__ __forceinline__ T ii2c_in(int k, const F &f) { return T(0.5) * (f(k + 1) + f(k)); }
    template <class T, class F> static __device__ __forceinline__ T di2c_in(int k, const F &f) { return f(k + 1) - f(k); }
};

template <>
struct SbpOrder<63> {
    static constexpr int C2I_LO = 6, C2I_HI = 5, I2C_LO = 7, I2C_HI = 6, GRAD_LO = 7, GRAD_HI = 6;
    static constexpr int U_LO = 7, U_HI = 6, V_LO = 7, V_HI = 6;
    static constexpr bool RUN_OK = false;   // six-point interior rows: evaluated per output
    static constexpr int NSAT = 4, NDEP = 6, NR = 4;
    static constexpr double SATC = 0.5 / (95.0 / 288.0);   // 0.5 / h11 of sbp_diff_c2i_63_mod.f90:12
    static __device__ __forceinline__ double satw(int r) { return 0.5 * D_SBP63_R[r - 1] / D_SBP63_H_C[r - 1]; }
    static __device__ __forceinline__ double ic1(int d) { return D_SBP63_IC_Q[0][d - 1]; }
    static __device__ __forceinline__ double dc1(int d) { return D_SBP63_DC_Q[0][d - 1]; }
    static __device__ __forceinline__ double r1(int d) { return D_SBP63_R[d - 1]; }
    template <class T, class F> static __device__ __forceinline__ T di2c(int k, int n, const F &f) { return di2c63<T>(k, n, f); }
    template <class T, class F> static __device__ __forceinline__ T dc2i(int k, int nx, const F &f) { return dc2i63<T>(k, nx, f); }
    template <class T, class F> static __device__ __forceinline__ T ii2c(int k, int n, const F &f) { return ii2c63<T>(k, n, f); }
    template <class T, class F> static __device__ __forceinline__ T ic2i(int k, int nx, const F &f) { return ic2i63<T>(k, nx, f); }
    // the stencil runs are not built for 6-3 (RUN_OK): placeholders
    template <class T> static __device__ __forceinline__ T interp4(T, T, T, T) { return T(0); }
    template <class T> static __device__ __forceinline__ T diff4(T, T, T, T) { return T(0); }
    template <class T, class F> static __device__ __forceinline__ T ic2i_in(int k, const F &f)
    {
        const double *C = D_SBP63_IC_C;
        return T(C[0]) * (f(k) + f(k - 1)) + T(C[1]) * (f(k + 1) + f(k - 2)) + T(C[2]) * (f(k + 2) + f(k - 3));
    }
    template <class T, class F> static __device__ __forceinline__ T dc2i_in(int k, const F &f)
    {
        const double *C = D_SBP63_DC_C;
        return T(C[0]) * (f(k) - f(k - 1)) + T(C[1]) * (f(k + 1) - f(k - 2)) + T(C[2]) * (f(k + 2) - f(k - 3));
    }
    template <class T, class F> static __device__ __forceinline__ T ii2c_in(int k, const F &f)
    {
        const double *C = D_SBP63_II_C;
        return T(C[0]) * (f(k + 1) + f(k)) + T(C[1]) * (f(k + 2) + f(k - 1)) + T(C[2]) * (f(k + 3) + f(k - 2));
    }
    template <class T, class F> static __device__ __forceinline__ T di2c_in(int k, const F &f)
    {
        const double *C = D_SBP63_DI_C;
        return T(C[0]) * (f(k + 1) - f(k)) + T(C[1]) * (f(k + 2) - f(k - 1)) + T(C[2]) * (f(k + 3) - f(k - 2));
    }
};

}  // namespace chswe

namespace chswe {

// Strided view of a line of inputs in shared memory: f(c) = p[c * s] (p points at
// input index 0).  The *_s variants evaluate interior rows inline and send the
// few closure rows to out-of-line copies, so interior points execute only the
// four-tap formula.
template <class T>
struct Line {
    const T *p;
    int s;
    __device__ __forceinline__ T operator()(int c) const { return p[c * s]; }
};

template <class T> __device__ __noinline__ T di2c_cl(int k, int n, Line<T> f) { return di2c<T>(k, n, f); }
template <class T> __device__ __noinline__ T dc2i_cl(int k, int nx, Line<T> f) { return dc2i<T>(k, nx, f); }
template <class T> __device__ __noinline__ T ii2c_cl(int k, int n, Line<T> f) { return ii2c<T>(k, n, f); }
template <class T> __device__ __noinline__ T ic2i_cl(int k, int nx, Line<T> f) { return ic2i<T>(k, nx, f); }

template <class T>
__device__ __forceinline__ T di2c_s(int k, int n, Line<T> f)
{
    if (__builtin_expect(k >= 4 && k <= n - 3, 1))
        return (T(27) * (f(k + 1) - f(k)) - (f(k + 2) - f(k - 1))) * T(1.0 / 24.0);
    return di2c_cl<T>(k, n, f);
}
template <class T>
__device__ __forceinline__ T dc2i_s(int k, int nx, Line<T> f)
{
    if (__builtin_expect(k >= 5 && k <= nx - 4, 1))
        return (T(27) * (f(k) - f(k - 1)) - (f(k + 1) - f(k - 2))) * T(1.0 / 24.0);
    return dc2i_cl<T>(k, nx, f);
}
template <class T>
__device__ __forceinline__ T ii2c_s(int k, int n, Line<T> f)
{
    if (__builtin_expect(k >= 4 && k <= n - 3, 1)) return (T(9) * (f(k + 1) + f(k)) - (f(k + 2) + f(k - 1))) * T(0.0625);
    return ii2c_cl<T>(k, n, f);
}
template <class T>
__device__ __forceinline__ T ic2i_s(int k, int nx, Line<T> f)
{
    if (__builtin_expect(k >= 5 && k <= nx - 4, 1)) return (T(9) * (f(k) + f(k - 1)) - (f(k + 1) + f(k - 2))) * T(0.0625);
    return ic2i_cl<T>(k, nx, f);
}

}  // namespace chswe

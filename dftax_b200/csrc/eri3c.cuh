// 3-center (ab|c) kernel for one (LA, LB, LC) class, LA >= LB.
//
// One thread computes one (shell pair, auxiliary shell) triple:
//   (ab|c)[i][m] = pref * sum_h Esph[i][h] W_m[h],
//   W_m[h = (t,u,v)] = sum_{c in cart(LC)} T[c][m] R^0_{t+cx, u+cy, v+cz}(P - C)
// with pref = K_ab c_a c_b c_c 2 pi^{5/2} / (g_ab g_c sqrt(g_ab + g_c)) * (-1/(2 g_c))^LC.
// Esph (the bra pair's E tables already in spherical components) comes from
// the primitive-pair setup; the aux side uses only the top-degree Hermite
// terms of a solid harmonic (Hobson's theorem), which is exact for harmonic
// transformation blocks (checked when the plan is made).
// This is the 3-center integral of dftax/integrals/eri3c_bucketed.py:376-426
// followed by its per-block cart->sph (:835-844).
#pragma once

#include "md_device.cuh"

namespace dfjk {

template <int LA, int LB, int LC>
__global__ void __launch_bounds__(128) eri3c_kernel(Eri3cArgs a) {
  constexpr int NA = 2 * LA + 1, NB = 2 * LB + 1, NC = 2 * LC + 1, NCC = nc_(LC);
  constexpr int LAB = LA + LB, M = LAB + LC, NH = hcount(LAB), NR = hcount(M), NAB = NA * NB;
  __shared__ double sT[NCC * NC];
  for (int q = threadIdx.x; q < NCC * NC; q += blockDim.x) sT[q] = a.c2s_aux[q];
  __syncthreads();
  const int slot = blockIdx.y * blockDim.x + threadIdx.x;
  if (slot >= a.aux_count) return;
  const int64_t pr = a.pair_begin + blockIdx.x;
  const int kc = a.aux_sorted[a.aux_begin + slot];
  const double C0 = a.aux.cen[3 * kc], C1 = a.aux.cen[3 * kc + 1], C2 = a.aux.cen[3 * kc + 2];
  const int cp0 = a.aux.prim0[kc], cnp = a.aux.nprim[kc];

  const int64_t pp0 = a.pair_pp0[pr];
  const int npp = a.pair_npp[pr];
  const int64_t row0 = a.pair_row0[pr] - a.row_base;
  const int col = a.col_base + slot * NC;

  if (npp == 1 && cnp == 1) {
    // One primitive triple (uncontracted shells): every (i, m) is final as
    // soon as it is formed, so it goes straight to the output and no
    // accumulator array is kept (that array lives in local memory).
    const double P0 = a.pp_P[3 * pp0], P1 = a.pp_P[3 * pp0 + 1], P2 = a.pp_P[3 * pp0 + 2];
    const double g = a.pp_g[pp0];
    const double* E = a.esph + (pp0 - a.esph_pp0) * (NAB * NH);
    const double gc = a.aux.pexp[cp0], cc = a.aux.pcoef[cp0];
    const double rho = g * gc / (g + gc);
    const double X = P0 - C0, Y = P1 - C1, Z = P2 - C2;
    double F[M + 1];
    boys_operator<M>(rho * (X * X + Y * Y + Z * Z), rho, a.omega, a.boys, a.boys_asym, F);
    double R[NR];
    hermite_r<M>(rho, X, Y, Z, F, R);
    double hob = 1.0;
    const double i2gc = -0.5 / gc;
#pragma unroll
    for (int k = 0; k < LC; ++k) hob *= i2gc;
    const double pref = a.pp_pref[pp0] * cc * kTwoPi25 / (g * gc * sqrt(g + gc)) * hob;
#pragma unroll 1
    for (int m = 0; m < NC; ++m) {
      double w[NH];
#pragma unroll
      for (int t = 0; t <= LAB; ++t)
#pragma unroll
        for (int u = 0; u <= LAB - t; ++u)
#pragma unroll
          for (int v = 0; v <= LAB - t - u; ++v) {
            double s = 0.0;
#pragma unroll
            for (int c = 0; c < NCC; ++c)
              s += sT[c * NC + m] * R[hidx(t + comp_x(LC, c), u + comp_y(LC, c), v + comp_z(LC, c))];
            w[hidx(t, u, v)] = s * pref;
          }
#pragma unroll 1
      for (int i = 0; i < NAB; ++i) {
        const double* Ei = E + i * NH;
        double s = 0.0;
#pragma unroll
        for (int h = 0; h < NH; ++h) s += __ldg(Ei + h) * w[h];
        const int64_t o = (row0 + i) * a.ld + col + m;
        if (a.out_f32) static_cast<float*>(a.out)[o] = (float)s;
        else static_cast<double*>(a.out)[o] = s;
      }
    }
    return;
  }

  double acc[NAB * NC];
#pragma unroll 1
  for (int q = 0; q < NAB * NC; ++q) acc[q] = 0.0;
#pragma unroll 1
  for (int q = 0; q < npp; ++q) {
    const int64_t pp = pp0 + q;
    const double P0 = a.pp_P[3 * pp], P1 = a.pp_P[3 * pp + 1], P2 = a.pp_P[3 * pp + 2];
    const double g = a.pp_g[pp];
    const double pab = a.pp_pref[pp];
    const double* E = a.esph + (pp - a.esph_pp0) * (NAB * NH);
#pragma unroll 1
    for (int ic = 0; ic < cnp; ++ic) {
      const double gc = a.aux.pexp[cp0 + ic];
      const double cc = a.aux.pcoef[cp0 + ic];
      const double rho = g * gc / (g + gc);
      const double X = P0 - C0, Y = P1 - C1, Z = P2 - C2;
      double F[M + 1];
      boys_operator<M>(rho * (X * X + Y * Y + Z * Z), rho, a.omega, a.boys, a.boys_asym, F);
      double R[NR];
      hermite_r<M>(rho, X, Y, Z, F, R);
      double hob = 1.0;
      const double i2gc = -0.5 / gc;
#pragma unroll
      for (int k = 0; k < LC; ++k) hob *= i2gc;
      const double pref = pab * cc * kTwoPi25 / (g * gc * sqrt(g + gc)) * hob;
#pragma unroll 1
      for (int m = 0; m < NC; ++m) {
        double w[NH];
#pragma unroll
        for (int t = 0; t <= LAB; ++t)
#pragma unroll
          for (int u = 0; u <= LAB - t; ++u)
#pragma unroll
            for (int v = 0; v <= LAB - t - u; ++v) {
              double s = 0.0;
#pragma unroll
              for (int c = 0; c < NCC; ++c)
                s += sT[c * NC + m] * R[hidx(t + comp_x(LC, c), u + comp_y(LC, c), v + comp_z(LC, c))];
              w[hidx(t, u, v)] = s * pref;
            }
#pragma unroll 1
        for (int i = 0; i < NAB; ++i) {
          const double* Ei = E + i * NH;
          double s = 0.0;
#pragma unroll
          for (int h = 0; h < NH; ++h) s += __ldg(Ei + h) * w[h];
          acc[i * NC + m] += s;
        }
      }
    }
  }
  if (a.out_f32) {
    float* out = static_cast<float*>(a.out);
#pragma unroll 1
    for (int i = 0; i < NAB; ++i)
#pragma unroll
      for (int m = 0; m < NC; ++m) out[(row0 + i) * a.ld + col + m] = (float)acc[i * NC + m];
  } else {
    double* out = static_cast<double*>(a.out);
#pragma unroll 1
    for (int i = 0; i < NAB; ++i)
#pragma unroll
      for (int m = 0; m < NC; ++m) out[(row0 + i) * a.ld + col + m] = acc[i * NC + m];
  }
}

template <int LA, int LB>
inline bool launch_lc(int lc, dim3 grid, cudaStream_t s, const Eri3cArgs& a) {
  switch (lc) {
    case 0: eri3c_kernel<LA, LB, 0><<<grid, 128, 0, s>>>(a); return true;
    case 1: eri3c_kernel<LA, LB, 1><<<grid, 128, 0, s>>>(a); return true;
    case 2: eri3c_kernel<LA, LB, 2><<<grid, 128, 0, s>>>(a); return true;
    case 3: eri3c_kernel<LA, LB, 3><<<grid, 128, 0, s>>>(a); return true;
    case 4: eri3c_kernel<LA, LB, 4><<<grid, 128, 0, s>>>(a); return true;
    default: return false;
  }
}

bool launch_eri3c_00(int lc, dim3 grid, cudaStream_t s, const Eri3cArgs& a);
bool launch_eri3c_10(int lc, dim3 grid, cudaStream_t s, const Eri3cArgs& a);
bool launch_eri3c_11(int lc, dim3 grid, cudaStream_t s, const Eri3cArgs& a);
bool launch_eri3c_20(int lc, dim3 grid, cudaStream_t s, const Eri3cArgs& a);
bool launch_eri3c_21(int lc, dim3 grid, cudaStream_t s, const Eri3cArgs& a);
bool launch_eri3c_22(int lc, dim3 grid, cudaStream_t s, const Eri3cArgs& a);
bool launch_eri3c_30(int lc, dim3 grid, cudaStream_t s, const Eri3cArgs& a);
bool launch_eri3c_31(int lc, dim3 grid, cudaStream_t s, const Eri3cArgs& a);
bool launch_eri3c_32(int lc, dim3 grid, cudaStream_t s, const Eri3cArgs& a);
bool launch_eri3c_33(int lc, dim3 grid, cudaStream_t s, const Eri3cArgs& a);

inline bool launch_eri3c(int l1, int l2, int lc, dim3 grid, cudaStream_t s, const Eri3cArgs& a) {
  switch (l1 * 4 + l2) {
    case 0: return launch_eri3c_00(lc, grid, s, a);
    case 4: return launch_eri3c_10(lc, grid, s, a);
    case 5: return launch_eri3c_11(lc, grid, s, a);
    case 8: return launch_eri3c_20(lc, grid, s, a);
    case 9: return launch_eri3c_21(lc, grid, s, a);
    case 10: return launch_eri3c_22(lc, grid, s, a);
    case 12: return launch_eri3c_30(lc, grid, s, a);
    case 13: return launch_eri3c_31(lc, grid, s, a);
    case 14: return launch_eri3c_32(lc, grid, s, a);
    case 15: return launch_eri3c_33(lc, grid, s, a);
    default: return false;
  }
}

}  // namespace dfjk

// Device helpers shared by the McMurchie-Davidson kernels: Hermite index
// packing, cartesian component tables, Boys function, Hermite R ladder and
// two-center E tables. Formulas follow dftax/integrals/eri3c_bucketed.py
// (:290-369) and dftax/energy/boys.py (:130-176).
#pragma once

#include "common.h"

#include <type_traits>
#include <utility>

namespace dfjk {

// Hermite triples (t, u, v) with t + u + v <= L, packed by total order, then
// u + v, then v.
__host__ __device__ constexpr int hcount(int L) { return L < 0 ? 0 : (L + 1) * (L + 2) * (L + 3) / 6; }
__host__ __device__ constexpr int hidx(int t, int u, int v) {
  return hcount(t + u + v - 1) + (u + v) * (u + v + 1) / 2 + v;
}
__host__ __device__ constexpr int nc_(int l) { return (l + 1) * (l + 2) / 2; }
// cartesian component k of shell l in dftax order (lx descending, then ly)
__host__ __device__ constexpr int comp_x(int l, int k) {
  int lx = l, kk = k;
  while (kk > l - lx) { kk -= (l - lx + 1); --lx; }
  return lx;
}
__host__ __device__ constexpr int comp_y(int l, int k) {
  int lx = l, kk = k;
  while (kk > l - lx) { kk -= (l - lx + 1); --lx; }
  return (l - lx) - kk;
}
__host__ __device__ constexpr int comp_z(int l, int k) { return l - comp_x(l, k) - comp_y(l, k); }

constexpr double kTwoPi25 = 34.98683665524972;   // 2 pi^{5/2}

// (t, u, v) of the packed Hermite index h, at compile time (inverse of hidx)
__host__ __device__ constexpr int horder(int h) {
  int k = 0;
  while (hcount(k) <= h) ++k;
  return k;
}
__host__ __device__ constexpr int hsum_uv(int h) {
  const int r = h - hcount(horder(h) - 1);
  int q = 0;
  while ((q + 1) * (q + 2) / 2 <= r) ++q;
  return q;
}
__host__ __device__ constexpr int hv(int h) {
  return h - hcount(horder(h) - 1) - hsum_uv(h) * (hsum_uv(h) + 1) / 2;
}
__host__ __device__ constexpr int hu(int h) { return hsum_uv(h) - hv(h); }
__host__ __device__ constexpr int ht(int h) { return horder(h) - hsum_uv(h); }

// f(std::integral_constant<int, i>) for i = 0 .. N-1 (or N-1 .. 0): every index
// derived from i is a constant expression, so arrays indexed by it stay in
// registers
template <class F, int... I>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void static_for(F&& f) {
  static_for_impl(f, std::make_integer_sequence<int, N>{});
}
template <int N, class F, int... I>
__device__ __forceinline__ void static_for_desc_impl(F&& f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, N - 1 - I>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void static_for_desc(F&& f) {
  static_for_desc_impl<N>(f, std::make_integer_sequence<int, N>{});
}

// Boys F_0..F_M at t: nearest table node + degree-6 Taylor for t < 40,
// asymptotic 0.5 Gamma(n+1/2) t^{-n-1/2} beyond (dftax/energy/boys.py:130-176).
template <int M>
__device__ __forceinline__ void boys_eval(double t, const double* __restrict__ tbl,
                                          const double* __restrict__ asym, double (&F)[M + 1]) {
  if (t < kBoysTmax) {
    int j = (int)rint(t / kBoysDt);
    j = j < 0 ? 0 : (j > kBoysNgrid - 1 ? kBoysNgrid - 1 : j);
    const double dx = (double)j * kBoysDt - t;
    const double* row = tbl + j * (kBoysNmax + 1);
    double c[M + kBoysOrder + 1];
#pragma unroll
    for (int q = 0; q <= M + kBoysOrder; ++q) c[q] = __ldg(row + q);
#pragma unroll
    for (int n = 0; n <= M; ++n) {
      double a = c[n + kBoysOrder];
#pragma unroll
      for (int k = kBoysOrder - 1; k >= 0; --k) a = c[n + k] + a * dx * (1.0 / (k + 1));
      F[n] = a;
    }
  } else {
    const double s = 1.0 / t;
    double f = __ldg(asym) * sqrt(s);
    F[0] = f;
#pragma unroll
    for (int n = 1; n <= M; ++n) {
      f = f * (n - 0.5) * s;
      F[n] = f;
    }
  }
}

// Boys values of the Hermite base for the Coulomb operator (omega == 0) or
// the long-range erf(omega r)/r operator (omega > 0): with
// s = omega^2 / (omega^2 + rho), F_m(t) becomes s^(m+1/2) F_m(s t)
// (dftax/integrals/eri3c_bucketed.py:342-346).
template <int M>
__device__ __forceinline__ void boys_operator(double t, double rho, double omega,
                                              const double* __restrict__ tbl,
                                              const double* __restrict__ asym, double (&F)[M + 1]) {
  if (omega > 0.0) {
    const double s = omega * omega / (omega * omega + rho);
    boys_eval<M>(s * t, tbl, asym, F);
    double f = sqrt(s);
#pragma unroll
    for (int n = 0; n <= M; ++n) {
      F[n] *= f;
      f *= s;
    }
  } else {
    boys_eval<M>(t, tbl, asym, F);
  }
}

// Hermite R^0_{tuv}, t+u+v <= M, packed by hidx, in place over the levels
// m = M..0 from R^m_000 = (-2 rho)^m F_m. At level m the entries of total
// order k are updated in descending k, so the orders k-1 and k-2 they read
// still hold level m+1.
template <int M>
__device__ __forceinline__ void hermite_r(double rho, double X, double Y, double Z,
                                          const double (&F)[M + 1], double (&R)[hcount(M)]) {
  double b[M + 1];
  const double m2r = -2.0 * rho;
  double pw = 1.0;
#pragma unroll
  for (int n = 0; n <= M; ++n) {
    b[n] = pw * F[n];
    pw *= m2r;
  }
  R[0] = b[M];
#pragma unroll
  for (int n = M - 1; n >= 0; --n) {
#pragma unroll
    for (int k = M - n; k >= 1; --k) {
#pragma unroll
      for (int t = k; t >= 0; --t) {
#pragma unroll
        for (int v = 0; v <= k - t; ++v) {
          const int u = k - t - v;
          double val;
          if (v > 0) {
            val = Z * R[hidx(t, u, v - 1)];
            if (v > 1) val += (v - 1) * R[hidx(t, u, v - 2)];
          } else if (u > 0) {
            val = Y * R[hidx(t, u - 1, 0)];
            if (u > 1) val += (u - 1) * R[hidx(t, u - 2, 0)];
          } else {
            val = X * R[hidx(t - 1, 0, 0)];
            if (t > 1) val += (t - 1) * R[hidx(t - 2, 0, 0)];
          }
          R[hidx(t, u, v)] = val;
        }
      }
    }
    R[0] = b[n];
  }
}

// hermite_r with every index a compile-time constant (for small M): the same
// in-place ladder, entries visited in descending packed index (descending
// order), so the orders k-1 and k-2 read still hold level m+1.
template <int M>
__device__ __forceinline__ void hermite_r_ct(double rho, double X, double Y, double Z,
                                             const double (&F)[M + 1], double (&R)[hcount(M)]) {
  double b[M + 1];
  const double m2r = -2.0 * rho;
  double pw = 1.0;
#pragma unroll
  for (int n = 0; n <= M; ++n) {
    b[n] = pw * F[n];
    pw *= m2r;
  }
  R[0] = b[M];
  static_for<M>([&](auto L) {
    constexpr int n = M - 1 - decltype(L)::value;
    static_for_desc<hcount(M)>([&](auto H) {
      constexpr int h = decltype(H)::value;
      constexpr int k = horder(h), t = ht(h), u = hu(h), v = hv(h);
      if constexpr (k >= 1 && k <= M - n) {
        double val;
        if constexpr (v > 0) {
          val = Z * R[hidx(t, u, v - 1)];
          if constexpr (v > 1) val += (v - 1) * R[hidx(t, u, v - 2)];
        } else if constexpr (u > 0) {
          val = Y * R[hidx(t, u - 1, 0)];
          if constexpr (u > 1) val += (u - 1) * R[hidx(t, u - 2, 0)];
        } else {
          val = X * R[hidx(t - 1, 0, 0)];
          if constexpr (t > 1) val += (t - 1) * R[hidx(t - 2, 0, 0)];
        }
        R[h] = val;
      }
    });
    R[0] = b[n];
  });
}

// Two-center E[i][j][t] for one axis, i <= LA, j <= LB, t <= i + j
// (MD recursion, eri3c_bucketed.py:290-313).
template <int LA, int LB>
__device__ __forceinline__ void e_axis(double a, double b, double xab,
                                       double (&E)[LA + 1][LB + 1][LA + LB + 1]) {
  constexpr int T = LA + LB + 1;
  const double g = a + b, i2g = 0.5 / g;
  const double xpa = -b * xab / g, xpb = a * xab / g;
#pragma unroll
  for (int i = 0; i <= LA; ++i)
#pragma unroll
    for (int j = 0; j <= LB; ++j)
#pragma unroll
      for (int t = 0; t < T; ++t) E[i][j][t] = 0.0;
  E[0][0][0] = 1.0;
#pragma unroll
  for (int i = 0; i < LA; ++i)
#pragma unroll
    for (int t = 0; t <= i + 1; ++t) {
      double v = (t <= i) ? xpa * E[i][0][t] : 0.0;
      if (t > 0) v += i2g * E[i][0][t - 1];
      if (t + 1 <= i) v += (t + 1) * E[i][0][t + 1];
      E[i + 1][0][t] = v;
    }
#pragma unroll
  for (int j = 0; j < LB; ++j)
#pragma unroll
    for (int i = 0; i <= LA; ++i)
#pragma unroll
      for (int t = 0; t <= i + j + 1; ++t) {
        double v = (t <= i + j) ? xpb * E[i][j][t] : 0.0;
        if (t > 0) v += i2g * E[i][j][t - 1];
        if (t + 1 <= i + j) v += (t + 1) * E[i][j][t + 1];
        E[i][j + 1][t] = v;
      }
}

struct Eri3cArgs {
  const int64_t* pair_row0;
  const int64_t* pair_pp0;
  const int* pair_npp;
  const double* pp_P;
  const double* pp_g;
  const double* pp_pref;
  const double* esph;        // class block base: [pp - esph_pp0][na*nb][nherm]
  int64_t esph_pp0;
  const int* aux_sorted;     // sorted position -> aux shell
  ShellView aux;
  const double* c2s_aux;     // (ncart x 2lc+1) block of the LC group
  const double* boys;
  const double* boys_asym;
  int64_t pair_begin;        // global pair index of blockIdx.x == 0
  int aux_begin;             // sorted position of the first LC shell
  int aux_count;
  int col_base;              // first column of the LC group
  int64_t row_base;          // global row of out[0]
  int64_t ld;
  void* out;
  int out_f32;               // 1: float output, 0: double
  double omega;              // > 0: erf(omega r)/r operator
  int uncontracted;          // 1: every orbital and aux shell has one primitive
};


}  // namespace dfjk

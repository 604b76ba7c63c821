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

// classes up to this total angular momentum form R and W with compile-time
// indices (hermite_r_ct, static_for): their arrays then stay in registers
constexpr int kStaticM = 6;

// One block of the per-thread kernel: shell pair a.pair_begin + bx, auxiliary
// slots by * blockDim.x + threadIdx.x (the grid position of a plain launch,
// or a work-queue entry of a batched one).
template <int LA, int LB, int LC>
__device__ __forceinline__ void eri3c_block(const Eri3cArgs a, const int64_t bx, const int by) {
  constexpr int NA = 2 * LA + 1, NB = 2 * LB + 1, NC = 2 * LC + 1, NCC = nc_(LC);
  constexpr int LAB = LA + LB, M = LAB + LC, NH = hcount(LAB), NR = hcount(M), NAB = NA * NB;
  __shared__ double sT[NCC * NC];
  for (int q = threadIdx.x; q < NCC * NC; q += blockDim.x) sT[q] = a.c2s_aux[q];
  __syncthreads();
  const int slot = by * blockDim.x + threadIdx.x;
  if (slot >= a.aux_count) return;
  const int64_t pr = a.pair_begin + bx;
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
    if constexpr (M <= kStaticM) hermite_r_ct<M>(rho, X, Y, Z, F, R);
    else hermite_r<M>(rho, X, Y, Z, F, R);
    double hob = 1.0;
    const double i2gc = -0.5 / gc;
#pragma unroll
    for (int k = 0; k < LC; ++k) hob *= i2gc;
    const double pref = a.pp_pref[pp0] * cc * kTwoPi25 / (g * gc * sqrt(g + gc)) * hob;
#pragma unroll 1
    for (int m = 0; m < NC; ++m) {
      double w[NH];
      if constexpr (M <= kStaticM) {
        // every R index a constant expression: R and w stay in registers
        static_for<NH>([&](auto H) {
          constexpr int h = decltype(H)::value, t = ht(h), u = hu(h), v = hv(h);
          double s = 0.0;
          static_for<NCC>([&](auto Cc) {
            constexpr int c = decltype(Cc)::value;
            constexpr int r = hidx(t + comp_x(LC, c), u + comp_y(LC, c), v + comp_z(LC, c));
            s += sT[c * NC + m] * R[r];
          });
          w[h] = s * pref;
        });
      } else {
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

// ---------------------------------------------------------------------------
// Heavy classes (LA + LB + LC >= kCoopM) of uncontracted shells: one warp per
// (shell pair, aux shell) triple, four warps per block sharing the pair's
// spherical bra E table in shared memory (rows padded to an odd stride). Per
// triple the warp forms
//   * the Boys values, one order per lane (per-order Taylor from the table);
//   * the Hermite R ladder, level by level, in two shared buffers, each lane
//     updating its fixed set of (t, u, v) entries;
//   * W_m[h] = pref sum_c T[c][m] R[h + c], one h per lane;
//   * (ab|c)[i][m] = sum_h E[i][h] W_m[h], lanes over i with all 2LC+1
//     components of m in registers (one E load and 2LC+1 broadcast W loads
//     per 2(2LC+1) FMAs).
// The per-thread kernel above keeps each triple in one thread, whose R table
// (up to 286 doubles) and accumulators then live in local memory.
// ---------------------------------------------------------------------------
constexpr int kCoopM = 7;

template <int LA, int LB, int LC>
struct CoopShape {
  static constexpr int NA = 2 * LA + 1, NB = 2 * LB + 1, NC = 2 * LC + 1, NCC = nc_(LC);
  static constexpr int LAB = LA + LB, M = LAB + LC, NH = hcount(LAB), NR = hcount(M);
  static constexpr int NAB = NA * NB, NHP = NH | 1;
  static constexpr int WARP_DOUBLES = 2 * NR + NC * NH + (M + 1);
  static constexpr size_t smem = (size_t)(NAB * NHP + NCC * NC + 4 * WARP_DOUBLES) * sizeof(double);
};

// (t, u, v) of the packed Hermite index h (inverse of hidx)
__device__ __forceinline__ void hdecode(int h, int& t, int& u, int& v) {
  int k = 0;
  while (hcount(k) <= h) ++k;
  const int r = h - hcount(k - 1);
  int q = 0;
  while ((q + 1) * (q + 2) / 2 <= r) ++q;
  v = r - q * (q + 1) / 2;
  u = q - v;
  t = k - q;
}

// F_n(t) alone, by the same table scheme as boys_eval
__device__ __forceinline__ double boys_order(int n, double t, const double* __restrict__ tbl,
                                             const double* __restrict__ asym) {
  if (t < kBoysTmax) {
    int j = (int)rint(t / kBoysDt);
    j = j < 0 ? 0 : (j > kBoysNgrid - 1 ? kBoysNgrid - 1 : j);
    const double dx = (double)j * kBoysDt - t;
    const double* row = tbl + j * (kBoysNmax + 1);
    double acc = __ldg(row + n + kBoysOrder);
#pragma unroll
    for (int k = kBoysOrder - 1; k >= 0; --k) acc = __ldg(row + n + k) + acc * dx * (1.0 / (k + 1));
    return acc;
  }
  const double s = 1.0 / t;
  double f = __ldg(asym) * sqrt(s);
  for (int k = 1; k <= n; ++k) f = f * (k - 0.5) * s;
  return f;
}

// One block of the cooperative kernel: shell pair a.pair_begin + bx, its
// warps taking auxiliary slots by * 4 + warp, then every gy * 4 further.
template <int LA, int LB, int LC>
__device__ __forceinline__ void eri3c_coop_block(const Eri3cArgs a, const int64_t bx,
                                                 const int by, const int gy) {
  using S = CoopShape<LA, LB, LC>;
  constexpr int NC = S::NC, NCC = S::NCC, M = S::M, NH = S::NH, NR = S::NR;
  constexpr int NAB = S::NAB, NHP = S::NHP;
  constexpr int RJ = (NR + 31) / 32, HJ = (NH + 31) / 32;
  static_assert(NAB <= 64, "two bra rows per lane");
  extern __shared__ double sm[];
  double* sE = sm;
  double* sT = sE + NAB * NHP;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* sRa = sT + NCC * NC + warp * S::WARP_DOUBLES;
  double* sRb = sRa + NR;
  double* sW = sRb + NR;
  double* sB = sW + NC * NH;

  const int64_t pr = a.pair_begin + bx;
  const int64_t pp0 = a.pair_pp0[pr];
  {
    const double* E = a.esph + (pp0 - a.esph_pp0) * (NAB * NH);
    for (int q = threadIdx.x; q < NAB * NH; q += blockDim.x) sE[(q / NH) * NHP + q % NH] = E[q];
    for (int q = threadIdx.x; q < NCC * NC; q += blockDim.x) sT[q] = a.c2s_aux[q];
  }
  __syncthreads();
  const double P0 = a.pp_P[3 * pp0], P1 = a.pp_P[3 * pp0 + 1], P2 = a.pp_P[3 * pp0 + 2];
  const double g = a.pp_g[pp0], pab = a.pp_pref[pp0];
  const int64_t row0 = a.pair_row0[pr] - a.row_base;

  // the R entries this lane updates: h = lane + 32 j, with the entries it reads
  int r_ord[RJ], r_s1[RJ], r_s2[RJ], r_ax[RJ];
  double r_mul[RJ];
#pragma unroll
  for (int j = 0; j < RJ; ++j) {
    const int h = lane + 32 * j;
    r_ord[j] = M + 1;
    r_s1[j] = r_s2[j] = -1;
    r_ax[j] = 0;
    r_mul[j] = 0.0;
    if (h < NR) {
      int t, u, v;
      hdecode(h, t, u, v);
      r_ord[j] = t + u + v;
      if (v > 0) {
        r_ax[j] = 2; r_s1[j] = hidx(t, u, v - 1);
        if (v > 1) { r_s2[j] = hidx(t, u, v - 2); r_mul[j] = v - 1; }
      } else if (u > 0) {
        r_ax[j] = 1; r_s1[j] = hidx(t, u - 1, 0);
        if (u > 1) { r_s2[j] = hidx(t, u - 2, 0); r_mul[j] = u - 1; }
      } else if (t > 0) {
        r_ax[j] = 0; r_s1[j] = hidx(t - 1, 0, 0);
        if (t > 1) { r_s2[j] = hidx(t - 2, 0, 0); r_mul[j] = t - 1; }
      }
    }
  }
  // the bra Hermite entries h this lane forms W for
  int w_t[HJ], w_u[HJ], w_v[HJ];
#pragma unroll
  for (int j = 0; j < HJ; ++j) {
    w_t[j] = w_u[j] = w_v[j] = -1;
    if (lane + 32 * j < NH) hdecode(lane + 32 * j, w_t[j], w_u[j], w_v[j]);
  }
  const int i0 = lane, i1 = lane + 32;

  for (int slot = by * 4 + warp; slot < a.aux_count; slot += gy * 4) {
    const int kc = a.aux_sorted[a.aux_begin + slot];
    const int cp0 = a.aux.prim0[kc];
    const double gc = a.aux.pexp[cp0], cc = a.aux.pcoef[cp0];
    const double X = P0 - a.aux.cen[3 * kc], Y = P1 - a.aux.cen[3 * kc + 1],
                 Z = P2 - a.aux.cen[3 * kc + 2];
    const double rho = g * gc / (g + gc);
    const double T = rho * (X * X + Y * Y + Z * Z);
    // R^(n)_000 = (-2 rho)^n F_n, with the erf(omega r)/r scaling when omega > 0
    if (lane <= M) {
      double sat = 1.0, tt = T;
      if (a.omega > 0.0) {
        sat = a.omega * a.omega / (a.omega * a.omega + rho);
        tt = sat * T;
      }
      double f = boys_order(lane, tt, a.boys, a.boys_asym);
      if (a.omega > 0.0) {
        double sp = sqrt(sat);
        for (int k = 0; k < lane; ++k) sp *= sat;
        f *= sp;
      }
      double pw = 1.0;
      for (int k = 0; k < lane; ++k) pw *= -2.0 * rho;
      sB[lane] = pw * f;
    }
    __syncwarp();
    // ladder m = M .. 0, ping-pong between the two buffers
    double* src = sRa;
    double* dst = sRb;
    if (lane == 0) src[0] = sB[M];
    __syncwarp();
    for (int n = M - 1; n >= 0; --n) {
      const int lim = M - n;
#pragma unroll
      for (int j = 0; j < RJ; ++j) {
        if (r_ord[j] > lim) continue;
        const int h = lane + 32 * j;
        double val;
        if (r_ord[j] == 0) {
          val = sB[n];
        } else {
          const double c = r_ax[j] == 0 ? X : (r_ax[j] == 1 ? Y : Z);
          val = c * src[r_s1[j]];
          if (r_s2[j] >= 0) val += r_mul[j] * src[r_s2[j]];
        }
        dst[h] = val;
      }
      __syncwarp();
      double* tmp = src;
      src = dst;
      dst = tmp;
    }
    const double* R = src;   // level 0
    double hob = 1.0;
    const double i2gc = -0.5 / gc;
#pragma unroll
    for (int k = 0; k < LC; ++k) hob *= i2gc;
    const double pref = pab * cc * kTwoPi25 / (g * gc * sqrt(g + gc)) * hob;
    // W_m[h] for this lane's h
#pragma unroll
    for (int j = 0; j < HJ; ++j) {
      if (w_t[j] < 0) continue;
      const int h = lane + 32 * j;
      double r[NCC];
#pragma unroll
      for (int c = 0; c < NCC; ++c)
        r[c] = R[hidx(w_t[j] + comp_x(LC, c), w_u[j] + comp_y(LC, c), w_v[j] + comp_z(LC, c))];
#pragma unroll
      for (int m = 0; m < NC; ++m) {
        double sacc = 0.0;
#pragma unroll
        for (int c = 0; c < NCC; ++c) sacc += sT[c * NC + m] * r[c];
        sW[m * NH + h] = sacc * pref;
      }
    }
    __syncwarp();
    // (ab|c)[i][m] for the lane's bra rows
    double acc0[NC], acc1[NC];
#pragma unroll
    for (int m = 0; m < NC; ++m) acc0[m] = acc1[m] = 0.0;
    const bool has0 = i0 < NAB, has1 = i1 < NAB;
    const double* e0 = sE + (has0 ? i0 : 0) * NHP;
    const double* e1 = sE + (has1 ? i1 : 0) * NHP;
#pragma unroll 4
    for (int h = 0; h < NH; ++h) {
      const double x0 = e0[h], x1 = e1[h];
#pragma unroll
      for (int m = 0; m < NC; ++m) {
        const double w = sW[m * NH + h];
        acc0[m] += x0 * w;
        acc1[m] += x1 * w;
      }
    }
    const int col = a.col_base + slot * NC;
    if (a.out_f32) {
      float* out = static_cast<float*>(a.out);
#pragma unroll
      for (int m = 0; m < NC; ++m) {
        if (has0) out[(row0 + i0) * a.ld + col + m] = (float)acc0[m];
        if (has1) out[(row0 + i1) * a.ld + col + m] = (float)acc1[m];
      }
    } else {
      double* out = static_cast<double*>(a.out);
#pragma unroll
      for (int m = 0; m < NC; ++m) {
        if (has0) out[(row0 + i0) * a.ld + col + m] = acc0[m];
        if (has1) out[(row0 + i1) * a.ld + col + m] = acc1[m];
      }
    }
    __syncwarp();
  }
}

template <int LA, int LB, int LC>
__global__ void __launch_bounds__(128) eri3c_kernel(Eri3cArgs a) {
  eri3c_block<LA, LB, LC>(a, blockIdx.x, blockIdx.y);
}

template <int LA, int LB, int LC>
__global__ void __launch_bounds__(128) eri3c_coop_kernel(Eri3cArgs a) {
  eri3c_coop_block<LA, LB, LC>(a, blockIdx.x, blockIdx.y, gridDim.y);
}

// Several plans' rows of one (LA, LB | LC) class in one launch: a work queue
// of segments (one plan's run of shell pairs of the class with its
// arguments), flattened to blocks; block q finds its segment by bisection and
// computes exactly what the plain launch's block of that segment computes.
// (A persistent loop over the queue made the compiler's work on these large
// bodies grow sevenfold, so each queue entry is a block.)
struct Eri3cBatch {
  const Eri3cArgs* seg;      // per segment (device)
  const int64_t* blk0;       // first queue entry of each segment, [nseg + 1]
  const int* ydim;           // y extent of each segment's plain grid
  int nseg;
  int64_t total;             // queue entries = blocks of the launch
};

__device__ __forceinline__ int batch_segment(const Eri3cBatch& b, int64_t q) {
  int lo = 0, hi = b.nseg;
  while (hi - lo > 1) {
    const int mid = (lo + hi) / 2;
    if (b.blk0[mid] <= q) lo = mid;
    else hi = mid;
  }
  return lo;
}

template <int LA, int LB, int LC>
__global__ void __launch_bounds__(128) eri3c_batch_kernel(Eri3cBatch b) {
  const int64_t q = blockIdx.x;
  const int sg = batch_segment(b, q);
  const int64_t local = q - b.blk0[sg];
  const int y = b.ydim[sg];
  eri3c_block<LA, LB, LC>(b.seg[sg], local / y, (int)(local % y));
}

// the classes whose rows are batched: those below the cooperative kernel's
// size (heavier classes keep one launch per plan; duplicating their large
// bodies would double the library's build time)
template <int LA, int LB, int LC>
inline bool launch_one_batch(unsigned blocks, cudaStream_t s, const Eri3cBatch& b) {
  if constexpr (LA + LB + LC < kCoopM) {
    eri3c_batch_kernel<LA, LB, LC><<<blocks, 128, 0, s>>>(b);
    return true;
  } else {
    return false;
  }
}

template <int LA, int LB>
inline bool launch_lc_batch(int lc, unsigned blocks, cudaStream_t s, const Eri3cBatch& b) {
  switch (lc) {
    case 0: return launch_one_batch<LA, LB, 0>(blocks, s, b);
    case 1: return launch_one_batch<LA, LB, 1>(blocks, s, b);
    case 2: return launch_one_batch<LA, LB, 2>(blocks, s, b);
    case 3: return launch_one_batch<LA, LB, 3>(blocks, s, b);
    case 4: return launch_one_batch<LA, LB, 4>(blocks, s, b);
    default: return false;
  }
}

template <int LA, int LB, int LC>
inline void launch_one(dim3 grid, cudaStream_t s, const Eri3cArgs& a) {
  if constexpr (LA + LB + LC >= kCoopM) {
    if (a.uncontracted) {
      constexpr size_t smem = CoopShape<LA, LB, LC>::smem;
      cudaFuncSetAttribute(eri3c_coop_kernel<LA, LB, LC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
      dim3 g2(grid.x, (unsigned)((a.aux_count + 15) / 16));
      eri3c_coop_kernel<LA, LB, LC><<<g2, 128, smem, s>>>(a);
      return;
    }
  }
  eri3c_kernel<LA, LB, LC><<<grid, 128, 0, s>>>(a);
}

template <int LA, int LB>
inline bool launch_lc(int lc, dim3 grid, cudaStream_t s, const Eri3cArgs& a) {
  switch (lc) {
    case 0: launch_one<LA, LB, 0>(grid, s, a); return true;
    case 1: launch_one<LA, LB, 1>(grid, s, a); return true;
    case 2: launch_one<LA, LB, 2>(grid, s, a); return true;
    case 3: launch_one<LA, LB, 3>(grid, s, a); return true;
    case 4: launch_one<LA, LB, 4>(grid, s, a); return true;
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

#define DFJK_ERI3C_BATCH_DECL(A, B) \
  bool launch_eri3c_batch_##A##B(int lc, unsigned blocks, cudaStream_t s, const Eri3cBatch& b);
DFJK_ERI3C_BATCH_DECL(0, 0)
DFJK_ERI3C_BATCH_DECL(1, 0)
DFJK_ERI3C_BATCH_DECL(1, 1)
DFJK_ERI3C_BATCH_DECL(2, 0)
DFJK_ERI3C_BATCH_DECL(2, 1)
DFJK_ERI3C_BATCH_DECL(2, 2)
DFJK_ERI3C_BATCH_DECL(3, 0)
DFJK_ERI3C_BATCH_DECL(3, 1)
DFJK_ERI3C_BATCH_DECL(3, 2)
DFJK_ERI3C_BATCH_DECL(3, 3)
#undef DFJK_ERI3C_BATCH_DECL

inline bool launch_eri3c_batch(int l1, int l2, int lc, unsigned blocks, cudaStream_t s,
                               const Eri3cBatch& b) {
  switch (l1 * 4 + l2) {
    case 0: return launch_eri3c_batch_00(lc, blocks, s, b);
    case 4: return launch_eri3c_batch_10(lc, blocks, s, b);
    case 5: return launch_eri3c_batch_11(lc, blocks, s, b);
    case 8: return launch_eri3c_batch_20(lc, blocks, s, b);
    case 9: return launch_eri3c_batch_21(lc, blocks, s, b);
    case 10: return launch_eri3c_batch_22(lc, blocks, s, b);
    case 12: return launch_eri3c_batch_30(lc, blocks, s, b);
    case 13: return launch_eri3c_batch_31(lc, blocks, s, b);
    case 14: return launch_eri3c_batch_32(lc, blocks, s, b);
    case 15: return launch_eri3c_batch_33(lc, blocks, s, b);
    default: return false;
  }
}

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

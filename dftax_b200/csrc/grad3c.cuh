// Geometry derivative of the 3-center integrals (ab|c), contracted on the fly
// with a weight G of the 3-center row layout (rows = bra function pairs of
// the kept shell pairs, columns = auxiliary functions in sorted order).
//
// For one kept shell pair (a, b) (a has the larger l, center A; b center B)
// and one auxiliary shell c (center C) a thread forms
//   fA = sum_{i,m} G[i][m] d(ab|c)[i][m]/dA,  fC = sum_{i,m} G[i][m] d(ab|c)[i][m]/dC,
// and fB = -fA - fC (the integral is unchanged when all three centers move
// together). In the McMurchie-Davidson form of eri3c.cuh,
//   (ab|c)[i][m] = pref sum_h Esph[i][h] W_m[h],  W_m[h] = sum_c T[c][m] R_{h+c}(P - C),
// only R depends on C: dR_{tuv}/dC_x = -R_{t+1,u,v}. d/dA acts on the bra
// Gaussian, d/dA_x x_A^k e^{-a x_A^2} = 2a x_A^{k+1} e^{..} - k x_A^{k-1} e^{..},
// so its Hermite expansion uses D^x = 2a E^{k+1,j} - k E^{k-1,j} (one order
// higher in t + u + v; pair_deriv_kernel, in spherical components).
// dftax obtains the same derivatives by differentiating its integral build
// (dftax/ks/forces.py:245-270 through dftax/integrals/eri3c_bucketed.py:376-426).
#pragma once

#include "md_device.cuh"

namespace dfjk {

struct PairDerivArgs {
  const int* pp_pair;
  const int* pp_pa;
  const int* pp_pb;
  const int* pair_s1;
  const int* pair_s2;
  ShellView orb;
  const double* c2s;
  int off1, off2;
  int64_t pp_begin, pp_count;
  double* dsph;         // [pp - pp_begin][3][na*nb][hcount(l1 + l2 + 1)]
};

// One thread per (primitive pair, spherical function pair, direction).
template <int L1, int L2>
__global__ void __launch_bounds__(128) pair_deriv_kernel(PairDerivArgs a) {
  constexpr int NA = 2 * L1 + 1, NB = 2 * L2 + 1, NAB = NA * NB, NH1 = hcount(L1 + L2 + 1);
  constexpr int CA = nc_(L1), CB = nc_(L2), T1 = L1 + L2 + 2;
  const int64_t gid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t local = gid / (3 * NAB);
  if (local >= a.pp_count) return;
  const int rem = (int)(gid % (3 * NAB));
  const int dir = rem / NAB, ab = rem % NAB;
  const int ia = ab / NB, ib = ab % NB;
  const int64_t pp = a.pp_begin + local;
  const int pr = a.pp_pair[pp];
  const int s1 = a.pair_s1[pr], s2 = a.pair_s2[pr];
  const int p1 = a.orb.prim0[s1] + a.pp_pa[pp], p2 = a.orb.prim0[s2] + a.pp_pb[pp];
  const double al = a.orb.pexp[p1], be = a.orb.pexp[p2];
  double E[3][L1 + 2][L2 + 1][T1];
#pragma unroll 1
  for (int x = 0; x < 3; ++x) e_axis<L1 + 1, L2>(al, be, a.orb.cen[3 * s1 + x] - a.orb.cen[3 * s2 + x], E[x]);
  // coefficient of Hermite order t on axis x for exponents (li, mi): the plain
  // table, or on the derivative axis 2 al E[li+1] - li E[li-1]
  auto coef = [&](int x, int li, int mi, int t) -> double {
    if (x != dir) return t <= li + mi ? E[x][li][mi][t] : 0.0;
    double v = 2.0 * al * E[x][li + 1][mi][t];
    if (li > 0 && t <= li - 1 + mi) v -= li * E[x][li - 1][mi][t];
    return v;
  };
  double out[NH1];
#pragma unroll
  for (int h = 0; h < NH1; ++h) out[h] = 0.0;
  const double* TA = a.c2s + a.off1;
  const double* TB = a.c2s + a.off2;
#pragma unroll 1
  for (int ca = 0; ca < CA; ++ca) {
    const double ta = TA[ca * NA + ia];
    if (ta == 0.0) continue;
    const int la[3] = {comp_x(L1, ca), comp_y(L1, ca), comp_z(L1, ca)};
#pragma unroll 1
    for (int cb = 0; cb < CB; ++cb) {
      const double tab = ta * TB[cb * NB + ib];
      if (tab == 0.0) continue;
      const int lb[3] = {comp_x(L2, cb), comp_y(L2, cb), comp_z(L2, cb)};
      const int tx = la[0] + lb[0] + (dir == 0), ty = la[1] + lb[1] + (dir == 1),
                tz = la[2] + lb[2] + (dir == 2);
#pragma unroll 1
      for (int t = 0; t <= tx; ++t) {
        const double ct = tab * coef(0, la[0], lb[0], t);
        if (ct == 0.0) continue;
#pragma unroll 1
        for (int u = 0; u <= ty; ++u) {
          const double cu = ct * coef(1, la[1], lb[1], u);
          if (cu == 0.0) continue;
#pragma unroll 1
          for (int v = 0; v <= tz; ++v) out[hidx(t, u, v)] += cu * coef(2, la[2], lb[2], v);
        }
      }
    }
  }
  double* dst = a.dsph + ((local * 3 + dir) * NAB + ab) * NH1;
#pragma unroll 1
  for (int h = 0; h < NH1; ++h) dst[h] = out[h];
}

struct Grad3cArgs {
  const int64_t* pair_row0;
  const int64_t* pair_pp0;
  const int* pair_npp;
  const int* pair_s1;
  const int* pair_s2;
  const double* pp_P;
  const double* pp_g;
  const double* pp_pref;
  const double* esph;        // class block base: [pp - esph_pp0][na*nb][nh]
  int64_t esph_pp0;
  const double* dsph;        // [pp - dsph_pp0][3][na*nb][nh1]
  int64_t dsph_pp0;
  const int* aux_sorted;
  ShellView aux;
  const double* c2s_aux;     // (ncart x 2lc+1) block of the LC group
  const double* boys;
  const double* boys_asym;
  int64_t pair_begin;        // global pair index of blockIdx.x == 0
  int aux_begin, aux_count, col_base;
  int64_t row_base;          // global row of G[0]
  int64_t ld;
  const double* G;
  double omega;
  double* grad_orb;          // [orbital shell][3]
  double* grad_aux;          // [aux shell][3]
};

// Hermite R^0_{tuv} for t+u+v <= M (packed by hidx) with runtime loops: the
// same in-place ladder as hermite_r, kept rolled so the high orders of the
// derivative classes compile to a small kernel (R lives in local memory).
// F holds F_n(t) on entry and (-2 rho)^n F_n(t) on return.
__device__ __forceinline__ void hermite_r_rolled(int M, double rho, double X, double Y, double Z,
                                                 double* F, double* R) {
  const double m2r = -2.0 * rho;
  double pw = 1.0;
  for (int n = 0; n <= M; ++n) {
    F[n] *= pw;
    pw *= m2r;
  }
  R[0] = F[M];
#pragma unroll 1
  for (int n = M - 1; n >= 0; --n) {
#pragma unroll 1
    for (int k = M - n; k >= 1; --k) {
#pragma unroll 1
      for (int t = k; t >= 0; --t) {
#pragma unroll 1
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
    R[0] = F[n];
  }
}

template <int LA, int LB, int LC>
__global__ void __launch_bounds__(128) grad3c_kernel(Grad3cArgs a) {
  constexpr int NA = 2 * LA + 1, NB = 2 * LB + 1, NC = 2 * LC + 1, NCC = nc_(LC);
  constexpr int LAB = LA + LB, NH = hcount(LAB), NH1 = hcount(LAB + 1), NAB = NA * NB;
  constexpr int M1 = LAB + LC + 1, NR = hcount(M1);
  __shared__ double sT[NCC * NC];
  __shared__ int sC[NCC][3];
  __shared__ double red[4][6];
  for (int q = threadIdx.x; q < NCC * NC; q += blockDim.x) sT[q] = a.c2s_aux[q];
  for (int q = threadIdx.x; q < NCC; q += blockDim.x) {
    sC[q][0] = comp_x(LC, q);
    sC[q][1] = comp_y(LC, q);
    sC[q][2] = comp_z(LC, q);
  }
  __syncthreads();
  const int slot = blockIdx.y * blockDim.x + threadIdx.x;
  const int64_t pr = a.pair_begin + blockIdx.x;
  const int s1 = a.pair_s1[pr], s2 = a.pair_s2[pr];
  const bool same = s1 == s2;   // fA + fB = -fC lands on one shell: no d/dA needed
  double fA[3] = {0.0, 0.0, 0.0}, fC[3] = {0.0, 0.0, 0.0};
  if (slot < a.aux_count) {
    const int kc = a.aux_sorted[a.aux_begin + slot];
    const double C0 = a.aux.cen[3 * kc], C1 = a.aux.cen[3 * kc + 1], C2 = a.aux.cen[3 * kc + 2];
    const int cp0 = a.aux.prim0[kc], cnp = a.aux.nprim[kc];
    const int64_t pp0 = a.pair_pp0[pr];
    const int npp = a.pair_npp[pr];
    const double* Grow = a.G + (a.pair_row0[pr] - a.row_base) * a.ld + a.col_base + slot * NC;
    double R[NR], w[NH1], gh[NH], dh[3 * NH1];
#pragma unroll 1
    for (int q = 0; q < npp; ++q) {
      const int64_t pp = pp0 + q;
      const double P0 = a.pp_P[3 * pp], P1 = a.pp_P[3 * pp + 1], P2 = a.pp_P[3 * pp + 2];
      const double g = a.pp_g[pp];
      const double pab = a.pp_pref[pp];
      const double* E = a.esph + (pp - a.esph_pp0) * (NAB * NH);
      const double* D = a.dsph + (pp - a.dsph_pp0) * (3 * NAB * NH1);
#pragma unroll 1
      for (int ic = 0; ic < cnp; ++ic) {
        const double gc = a.aux.pexp[cp0 + ic], cc = a.aux.pcoef[cp0 + ic];
        const double rho = g * gc / (g + gc);
        const double X = P0 - C0, Y = P1 - C1, Z = P2 - C2;
        double F[M1 + 1];
        boys_operator<M1>(rho * (X * X + Y * Y + Z * Z), rho, a.omega, a.boys, a.boys_asym, F);
        hermite_r_rolled(M1, rho, X, Y, Z, F, R);
        double hob = 1.0;
        for (int k = 0; k < LC; ++k) hob *= -0.5 / gc;
        const double pref = pab * cc * kTwoPi25 / (g * gc * sqrt(g + gc)) * hob;
#pragma unroll 1
        for (int m = 0; m < NC; ++m) {
          // W_m[h] = pref sum_c T[c][m] R_{h + c}, h of order <= LAB + 1
#pragma unroll 1
          for (int t = 0; t <= LAB + 1; ++t)
#pragma unroll 1
            for (int u = 0; u <= LAB + 1 - t; ++u)
#pragma unroll 1
              for (int v = 0; v <= LAB + 1 - t - u; ++v) {
                double sum = 0.0;
#pragma unroll 1
                for (int c = 0; c < NCC; ++c)
                  sum += sT[c * NC + m] * R[hidx(t + sC[c][0], u + sC[c][1], v + sC[c][2])];
                w[hidx(t, u, v)] = sum * pref;
              }
          // G-weighted Hermite coefficients of the bra: plain and d/dA
#pragma unroll 1
          for (int h = 0; h < NH; ++h) gh[h] = 0.0;
#pragma unroll 1
          for (int h = 0; h < 3 * NH1; ++h) dh[h] = 0.0;
#pragma unroll 1
          for (int i = 0; i < NAB; ++i) {
            const double gi = Grow[(int64_t)i * a.ld + m];
            if (gi == 0.0) continue;
            const double* Ei = E + i * NH;
#pragma unroll 4
            for (int h = 0; h < NH; ++h) gh[h] += gi * __ldg(Ei + h);
            if (!same) {
#pragma unroll 1
              for (int d = 0; d < 3; ++d) {
                const double* Di = D + (d * NAB + i) * NH1;
#pragma unroll 4
                for (int h = 0; h < NH1; ++h) dh[d * NH1 + h] += gi * __ldg(Di + h);
              }
            }
          }
#pragma unroll 1
          for (int t = 0; t <= LAB; ++t)
#pragma unroll 1
            for (int u = 0; u <= LAB - t; ++u)
#pragma unroll 1
              for (int v = 0; v <= LAB - t - u; ++v) {
                const double e = gh[hidx(t, u, v)];
                fC[0] -= e * w[hidx(t + 1, u, v)];
                fC[1] -= e * w[hidx(t, u + 1, v)];
                fC[2] -= e * w[hidx(t, u, v + 1)];
              }
          if (!same) {
#pragma unroll 1
            for (int d = 0; d < 3; ++d) {
              double sum = 0.0;
#pragma unroll 4
              for (int h = 0; h < NH1; ++h) sum += dh[d * NH1 + h] * w[h];
              fA[d] += sum;
            }
          }
        }
      }
    }
    // the auxiliary shells of the block differ: one atomic add each
    for (int d = 0; d < 3; ++d) atomicAdd(a.grad_aux + 3 * kc + d, fC[d]);
  }
  // fA and fB = -fA - fC summed over the block (one shell pair)
  double v[6] = {fA[0], fA[1], fA[2], -fA[0] - fC[0], -fA[1] - fC[1], -fA[2] - fC[2]};
#pragma unroll
  for (int k = 0; k < 6; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < 6; ++k) red[warp][k] = v[k];
  __syncthreads();
  if (threadIdx.x < 6) {
    double sum = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) sum += red[q][threadIdx.x];
    const int sh = threadIdx.x < 3 ? s1 : s2;
    atomicAdd(a.grad_orb + 3 * sh + threadIdx.x % 3, sum);
  }
}

template <int LA, int LB>
inline bool launch_grad3c_lc(int lc, dim3 grid, cudaStream_t s, const Grad3cArgs& a) {
  switch (lc) {
    case 0: grad3c_kernel<LA, LB, 0><<<grid, 128, 0, s>>>(a); return true;
    case 1: grad3c_kernel<LA, LB, 1><<<grid, 128, 0, s>>>(a); return true;
    case 2: grad3c_kernel<LA, LB, 2><<<grid, 128, 0, s>>>(a); return true;
    case 3: grad3c_kernel<LA, LB, 3><<<grid, 128, 0, s>>>(a); return true;
    case 4: grad3c_kernel<LA, LB, 4><<<grid, 128, 0, s>>>(a); return true;
    default: return false;
  }
}

template <int LA, int LB>
inline void launch_pair_deriv_t(unsigned blocks, cudaStream_t s, const PairDerivArgs& a) {
  pair_deriv_kernel<LA, LB><<<blocks, 128, 0, s>>>(a);
}

#define DFJK_GRAD3C_DECL(A, B)                                                              \
  bool launch_grad3c_##A##B(int lc, dim3 grid, cudaStream_t s, const Grad3cArgs& a);       \
  void launch_pair_deriv_##A##B(unsigned blocks, cudaStream_t s, const PairDerivArgs& a);
DFJK_GRAD3C_DECL(0, 0)
DFJK_GRAD3C_DECL(1, 0)
DFJK_GRAD3C_DECL(1, 1)
DFJK_GRAD3C_DECL(2, 0)
DFJK_GRAD3C_DECL(2, 1)
DFJK_GRAD3C_DECL(2, 2)
DFJK_GRAD3C_DECL(3, 0)
DFJK_GRAD3C_DECL(3, 1)
DFJK_GRAD3C_DECL(3, 2)
DFJK_GRAD3C_DECL(3, 3)
#undef DFJK_GRAD3C_DECL

}  // namespace dfjk

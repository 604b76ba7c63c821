// Boys table and kernel, primitive-pair setup, 2-center metric and Schwarz
// kernels, and the launchers of all integral kernels (float64 arithmetic).
//
// Formulas follow dftax/integrals/eri3c_bucketed.py (E tables :290-323,
// Hermite R :326-369, 3-center :376-426, 2-center :697-734) and
// dftax/energy/boys.py (:81-176). Design decisions, not a translation of the
// reference's vmapped einsums:
//   * the bra pair's E tables are transformed to spherical components once per
//     primitive pair ("Esph", [na*nb][nherm]) by pair_setup_kernel;
//   * a spherical auxiliary shell is a solid harmonic whose single-center
//     Hermite expansion keeps only its top-degree terms (Hobson's theorem):
//     S_lm(r) e^{-g r^2} = (2g)^{-l} sum_c T[c][m] Lambda_c;
//   * aux columns are sorted by l, so a warp of the 3-center kernel writes
//     contiguous column runs of one row.
#include "eri3c.cuh"
#include "md_device.cuh"
#include "internal.h"

#include <cmath>
#include <map>
#include <tuple>

namespace dfjk {

// ---------------------------------------------------------------------------
// Boys table (dftax/energy/boys.py:81-123): ascending series at a high order,
// then the downward recursion F_{n-1} = (2t F_n + e^{-t}) / (2n-1).
// ---------------------------------------------------------------------------

void boys_table_host(std::vector<double>& tbl, std::vector<double>& asym) {
  const int ng = kBoysNgrid, nc = kBoysNmax + 1;
  tbl.assign((size_t)ng * nc, 0.0);
  const int top = (kBoysNmax > (int)kBoysTmax ? kBoysNmax : (int)kBoysTmax) + 20;
  std::vector<double> t(ng), term(ng), acc(ng), f(ng), emt(ng);
  for (int j = 0; j < ng; ++j) {
    t[j] = j * kBoysDt;
    emt[j] = std::exp(-t[j]);
    term[j] = 1.0 / (2 * top + 1);
    acc[j] = term[j];
  }
  for (int k = 1; k < 500; ++k) {
    double tmax = 0.0, amin = 1e300;
    for (int j = 0; j < ng; ++j) {
      term[j] = term[j] * (2.0 * t[j]) / (2 * top + 2 * k + 1);
      acc[j] += term[j];
      tmax = term[j] > tmax ? term[j] : tmax;
      amin = acc[j] < amin ? acc[j] : amin;
    }
    if (tmax <= 1e-18 * amin) break;
  }
  for (int j = 0; j < ng; ++j) f[j] = emt[j] * acc[j];
  for (int n = top; n > 0; --n) {
    for (int j = 0; j < ng; ++j) {
      if (n <= kBoysNmax) tbl[(size_t)j * nc + n] = f[j];
      f[j] = (2.0 * t[j] * f[j] + emt[j]) / (2 * n - 1);
    }
  }
  for (int j = 0; j < ng; ++j) tbl[(size_t)j * nc] = f[j];
  asym.resize(nc);
  for (int n = 0; n < nc; ++n) asym[n] = 0.5 * std::exp(std::lgamma(n + 0.5));
}

__global__ void boys_kernel(const double* __restrict__ t, int64_t n, int nmax,
                            const double* __restrict__ tbl, const double* __restrict__ asym,
                            double* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double F[19];
  boys_eval<18>(t[i], tbl, asym, F);
  for (int k = 0; k <= nmax; ++k) out[i * (nmax + 1) + k] = F[k];
}

void launch_boys(const Context& c, const double* t, int64_t n, int nmax, double* out,
                 cudaStream_t s) {
  if (n <= 0) return;
  int64_t blocks = (n + 255) / 256;
  boys_kernel<<<(unsigned)blocks, 256, 0, s>>>(t, n, nmax, c.boys.as<double>(),
                                               c.boys_asym.as<double>(), out);
  DFJK_LAUNCHED();
}

// runtime versions of the packing helpers
__device__ __forceinline__ int hidx_rt(int t, int u, int v) {
  const int n = t + u + v;
  return n * (n + 1) * (n + 2) / 6 + (u + v) * (u + v + 1) / 2 + v;
}
__device__ __forceinline__ void comp_rt(int l, int k, int& x, int& y, int& z) {
  int lx = l, kk = k;
  while (kk > l - lx) { kk -= (l - lx + 1); --lx; }
  x = lx;
  y = (l - lx) - kk;
  z = l - x - y;
}

// ---------------------------------------------------------------------------
// Primitive-pair setup: P, g_ab, K_ab c_a c_b and Esph[i][h]
// ---------------------------------------------------------------------------

struct PairArgs {
  const int* pp_pair;   // primitive pair -> shell pair
  const int* pp_pa;     // primitive index within s1
  const int* pp_pb;
  const int* pair_s1;
  const int* pair_s2;
  ShellView orb;
  const double* c2s;    // packed blocks
  int off1, off2;       // block offsets for l1, l2
  int64_t pp_begin, pp_count;
  double* pp_P;         // 3 per pp
  double* pp_g;
  double* pp_pref;
  double* esph;         // class block base: [pp][na*nb][nh]
};

template <int L1, int L2>
__global__ void __launch_bounds__(128) pair_setup_kernel(PairArgs a) {
  constexpr int NA = 2 * L1 + 1, NB = 2 * L2 + 1, NH = hcount(L1 + L2);
  constexpr int CA = nc_(L1), CB = nc_(L2);
  const int64_t gid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t local = gid / (NA * NB);
  if (local >= a.pp_count) return;
  const int ab = (int)(gid % (NA * NB));
  const int ia = ab / NB, ib = ab % NB;
  const int64_t pp = a.pp_begin + local;
  const int pr = a.pp_pair[pp];
  const int s1 = a.pair_s1[pr], s2 = a.pair_s2[pr];
  const int p1 = a.orb.prim0[s1] + a.pp_pa[pp], p2 = a.orb.prim0[s2] + a.pp_pb[pp];
  const double al = a.orb.pexp[p1], be = a.orb.pexp[p2];
  const double A[3] = {a.orb.cen[3 * s1], a.orb.cen[3 * s1 + 1], a.orb.cen[3 * s1 + 2]};
  const double B[3] = {a.orb.cen[3 * s2], a.orb.cen[3 * s2 + 1], a.orb.cen[3 * s2 + 2]};
  const double g = al + be;
  double Ex[L1 + 1][L2 + 1][L1 + L2 + 1], Ey[L1 + 1][L2 + 1][L1 + L2 + 1],
      Ez[L1 + 1][L2 + 1][L1 + L2 + 1];
  e_axis<L1, L2>(al, be, A[0] - B[0], Ex);
  e_axis<L1, L2>(al, be, A[1] - B[1], Ey);
  e_axis<L1, L2>(al, be, A[2] - B[2], Ez);
  double out[NH];
#pragma unroll 1
  for (int h = 0; h < NH; ++h) out[h] = 0.0;
  const double* TA = a.c2s + a.off1;
  const double* TB = a.c2s + a.off2;
#pragma unroll 1
  for (int ca = 0; ca < CA; ++ca) {
    const double ta = TA[ca * NA + ia];
    if (ta == 0.0) continue;
    int ax, ay, az;
    comp_rt(L1, ca, ax, ay, az);
#pragma unroll 1
    for (int cb = 0; cb < CB; ++cb) {
      const double tab = ta * TB[cb * NB + ib];
      if (tab == 0.0) continue;
      int bx, by, bz;
      comp_rt(L2, cb, bx, by, bz);
#pragma unroll 1
      for (int t = 0; t <= ax + bx; ++t) {
        const double et = tab * Ex[ax][bx][t];
#pragma unroll 1
        for (int u = 0; u <= ay + by; ++u) {
          const double eu = et * Ey[ay][by][u];
#pragma unroll 1
          for (int v = 0; v <= az + bz; ++v) out[hidx_rt(t, u, v)] += eu * Ez[az][bz][v];
        }
      }
    }
  }
  double* dst = a.esph + (local * (NA * NB) + ab) * NH;
#pragma unroll 1
  for (int h = 0; h < NH; ++h) dst[h] = out[h];
  if (ab == 0) {
    const double ab2 = (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) +
                       (A[2] - B[2]) * (A[2] - B[2]);
    a.pp_P[3 * pp + 0] = (al * A[0] + be * B[0]) / g;
    a.pp_P[3 * pp + 1] = (al * A[1] + be * B[1]) / g;
    a.pp_P[3 * pp + 2] = (al * A[2] + be * B[2]) / g;
    a.pp_g[pp] = g;
    a.pp_pref[pp] = exp(-al * be / g * ab2) * a.orb.pcoef[p1] * a.orb.pcoef[p2];
  }
}

// ---------------------------------------------------------------------------
// 2-center (P|Q), spherical, aux columns in sorted order:
// (P|Q)[p][q] = 2 pi^{5/2} c_a c_b / (a b sqrt(a+b)) (2a)^{-LP} (-2b)^{-LQ}
//               * sum_{c1, c2} T_P[c1][p] T_Q[c2][q] R_{c1 + c2}(rho, A - B)
// ---------------------------------------------------------------------------

struct Eri2cArgs {
  const int* aux_sorted;
  ShellView aux;
  const double* c2s;
  int offP, offQ;
  const double* boys;
  const double* boys_asym;
  int beginP, countP, beginQ, countQ;   // sorted positions
  int colP, colQ;                       // first columns of the groups
  int64_t ld;
  double* out;
  double omega;                         // > 0: erf(omega r)/r operator
};

template <int LP, int LQ>
__global__ void __launch_bounds__(128) eri2c_kernel(Eri2cArgs a) {
  constexpr int NP = 2 * LP + 1, NQ = 2 * LQ + 1, CP = nc_(LP), CQ = nc_(LQ);
  constexpr int M = LP + LQ, NR = hcount(M);
  const int64_t gid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (gid >= (int64_t)a.countP * a.countQ) return;
  const int ip = (int)(gid / a.countQ), iq = (int)(gid % a.countQ);
  if (LP == LQ && ip > iq) return;   // same group: each unordered pair once
  const int sp = a.aux_sorted[a.beginP + ip], sq = a.aux_sorted[a.beginQ + iq];
  const double X = a.aux.cen[3 * sp] - a.aux.cen[3 * sq];
  const double Y = a.aux.cen[3 * sp + 1] - a.aux.cen[3 * sq + 1];
  const double Z = a.aux.cen[3 * sp + 2] - a.aux.cen[3 * sq + 2];
  double acc[NP * NQ];
#pragma unroll 1
  for (int q = 0; q < NP * NQ; ++q) acc[q] = 0.0;
  const double* TP = a.c2s + a.offP;
  const double* TQ = a.c2s + a.offQ;
#pragma unroll 1
  for (int i = 0; i < a.aux.nprim[sp]; ++i) {
    const double al = a.aux.pexp[a.aux.prim0[sp] + i], ca = a.aux.pcoef[a.aux.prim0[sp] + i];
#pragma unroll 1
    for (int j = 0; j < a.aux.nprim[sq]; ++j) {
      const double be = a.aux.pexp[a.aux.prim0[sq] + j], cb = a.aux.pcoef[a.aux.prim0[sq] + j];
      const double rho = al * be / (al + be);
      double F[M + 1];
      boys_operator<M>(rho * (X * X + Y * Y + Z * Z), rho, a.omega, a.boys, a.boys_asym, F);
      double R[NR];
      hermite_r<M>(rho, X, Y, Z, F, R);
      double hob = kTwoPi25 * ca * cb / (al * be * sqrt(al + be));
#pragma unroll
      for (int k = 0; k < LP; ++k) hob *= 0.5 / al;
#pragma unroll
      for (int k = 0; k < LQ; ++k) hob *= -0.5 / be;
#pragma unroll 1
      for (int c1 = 0; c1 < CP; ++c1) {
        int x1, y1, z1;
        comp_rt(LP, c1, x1, y1, z1);
#pragma unroll 1
        for (int c2 = 0; c2 < CQ; ++c2) {
          int x2, y2, z2;
          comp_rt(LQ, c2, x2, y2, z2);
          const double r = hob * R[hidx_rt(x1 + x2, y1 + y2, z1 + z2)];
#pragma unroll 1
          for (int p = 0; p < NP; ++p) {
            const double tp = __ldg(TP + c1 * NP + p) * r;
            if (tp == 0.0) continue;
#pragma unroll 1
            for (int q = 0; q < NQ; ++q) acc[p * NQ + q] += tp * __ldg(TQ + c2 * NQ + q);
          }
        }
      }
    }
  }
  const int r0 = a.colP + ip * NP, c0 = a.colQ + iq * NQ;
#pragma unroll 1
  for (int p = 0; p < NP; ++p)
#pragma unroll 1
    for (int q = 0; q < NQ; ++q) {
      a.out[(int64_t)(r0 + p) * a.ld + c0 + q] = acc[p * NQ + q];
      a.out[(int64_t)(c0 + q) * a.ld + r0 + p] = acc[p * NQ + q];
    }
}

// ---------------------------------------------------------------------------
// Schwarz diagonal: max over cartesian component pairs of sqrt((ab|ab))
// (the 4-center diagonal of dftax/integrals/eri4c.py:206-220, maxed per shell
// pair as in eri3c_bucketed.py:140-169)
// ---------------------------------------------------------------------------

struct SchwarzArgs {
  const int* pa;
  const int* pb;
  int64_t count;
  ShellView orb;
  const double* boys;
  const double* boys_asym;
  double* qmax;
};

template <int LA, int LB>
__global__ void __launch_bounds__(64) schwarz_kernel(SchwarzArgs a) {
  constexpr int CA = nc_(LA), CB = nc_(LB), LAB = LA + LB, M = 2 * LAB, NR = hcount(M);
  const int64_t gid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (gid >= a.count) return;
  const int s1 = a.pa[gid], s2 = a.pb[gid];
  const double A[3] = {a.orb.cen[3 * s1], a.orb.cen[3 * s1 + 1], a.orb.cen[3 * s1 + 2]};
  const double B[3] = {a.orb.cen[3 * s2], a.orb.cen[3 * s2 + 1], a.orb.cen[3 * s2 + 2]};
  const double ab2 = (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) +
                     (A[2] - B[2]) * (A[2] - B[2]);
  double diag[CA * CB];
#pragma unroll 1
  for (int i = 0; i < CA * CB; ++i) diag[i] = 0.0;
  const int n1 = a.orb.nprim[s1], n2 = a.orb.nprim[s2];
#pragma unroll 1
  for (int i1 = 0; i1 < n1; ++i1)
#pragma unroll 1
    for (int j1 = 0; j1 < n2; ++j1) {
      const double al = a.orb.pexp[a.orb.prim0[s1] + i1], be = a.orb.pexp[a.orb.prim0[s2] + j1];
      const double c1 = a.orb.pcoef[a.orb.prim0[s1] + i1] * a.orb.pcoef[a.orb.prim0[s2] + j1];
      const double p = al + be;
      double Ex[LA + 1][LB + 1][LAB + 1], Ey[LA + 1][LB + 1][LAB + 1], Ez[LA + 1][LB + 1][LAB + 1];
      e_axis<LA, LB>(al, be, A[0] - B[0], Ex);
      e_axis<LA, LB>(al, be, A[1] - B[1], Ey);
      e_axis<LA, LB>(al, be, A[2] - B[2], Ez);
      const double P[3] = {(al * A[0] + be * B[0]) / p, (al * A[1] + be * B[1]) / p,
                           (al * A[2] + be * B[2]) / p};
      const double K1 = exp(-al * be / p * ab2) * c1;
#pragma unroll 1
      for (int i2 = 0; i2 < n1; ++i2)
#pragma unroll 1
        for (int j2 = 0; j2 < n2; ++j2) {
          const double ga = a.orb.pexp[a.orb.prim0[s1] + i2], gb = a.orb.pexp[a.orb.prim0[s2] + j2];
          const double c2 = a.orb.pcoef[a.orb.prim0[s1] + i2] * a.orb.pcoef[a.orb.prim0[s2] + j2];
          const double q = ga + gb;
          double Fx[LA + 1][LB + 1][LAB + 1], Fy[LA + 1][LB + 1][LAB + 1], Fz[LA + 1][LB + 1][LAB + 1];
          e_axis<LA, LB>(ga, gb, A[0] - B[0], Fx);
          e_axis<LA, LB>(ga, gb, A[1] - B[1], Fy);
          e_axis<LA, LB>(ga, gb, A[2] - B[2], Fz);
          const double Q[3] = {(ga * A[0] + gb * B[0]) / q, (ga * A[1] + gb * B[1]) / q,
                               (ga * A[2] + gb * B[2]) / q};
          const double K2 = exp(-ga * gb / q * ab2) * c2;
          const double rho = p * q / (p + q);
          const double X = P[0] - Q[0], Y = P[1] - Q[1], Z = P[2] - Q[2];
          double F[M + 1];
          boys_eval<M>(rho * (X * X + Y * Y + Z * Z), a.boys, a.boys_asym, F);
          double R[NR];
          hermite_r<M>(rho, X, Y, Z, F, R);
          const double pref = K1 * K2 * kTwoPi25 / (p * q * sqrt(p + q));
#pragma unroll 1
          for (int ia = 0; ia < CA; ++ia)
#pragma unroll 1
            for (int ib = 0; ib < CB; ++ib) {
              int ax, ay, az, bx, by, bz;
              comp_rt(LA, ia, ax, ay, az);
              comp_rt(LB, ib, bx, by, bz);
              double s = 0.0;
#pragma unroll 1
              for (int t1 = 0; t1 <= ax + bx; ++t1)
#pragma unroll 1
                for (int u1 = 0; u1 <= ay + by; ++u1)
#pragma unroll 1
                  for (int v1 = 0; v1 <= az + bz; ++v1) {
                    const double e1 = Ex[ax][bx][t1] * Ey[ay][by][u1] * Ez[az][bz][v1];
#pragma unroll 1
                    for (int t2 = 0; t2 <= ax + bx; ++t2)
#pragma unroll 1
                      for (int u2 = 0; u2 <= ay + by; ++u2)
#pragma unroll 1
                        for (int v2 = 0; v2 <= az + bz; ++v2) {
                          const double e2 = Fx[ax][bx][t2] * Fy[ay][by][u2] * Fz[az][bz][v2];
                          const double sg = ((t2 + u2 + v2) & 1) ? -1.0 : 1.0;
                          s += e1 * e2 * sg * R[hidx_rt(t1 + t2, u1 + u2, v1 + v2)];
                        }
                  }
              diag[ia * CB + ib] += pref * s;
            }
        }
    }
  double m = 0.0;
#pragma unroll 1
  for (int i = 0; i < CA * CB; ++i) m = fmax(m, sqrt(fmax(diag[i], 0.0)));
  a.qmax[gid] = m;
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------

static ShellView view(const Shells& s) {
  return ShellView{s.d_l.as<int>(), s.d_nprim.as<int>(), s.d_prim0.as<int>(),
                   s.d_cen.as<double>(), s.d_pexp.as<double>(), s.d_pcoef.as<double>()};
}

#define DFJK_L1L2_CASES(X) \
  X(0, 0) X(1, 0) X(1, 1) X(2, 0) X(2, 1) X(2, 2) X(3, 0) X(3, 1) X(3, 2) X(3, 3)

void launch_pair_setup(Plan& p, cudaStream_t s) {
  for (const ClassRange& cr : p.classes) {
    if (cr.pp_count == 0) continue;
    PairArgs a;
    a.pp_pair = p.d_pp_pair.as<int>();
    a.pp_pa = p.d_pp_pa.as<int>();
    a.pp_pb = p.d_pp_pb.as<int>();
    a.pair_s1 = p.d_pair_s1.as<int>();
    a.pair_s2 = p.d_pair_s2.as<int>();
    a.orb = view(p.orb);
    a.c2s = p.c2s_orb.dev.as<double>();
    a.off1 = p.c2s_orb.off[cr.l1];
    a.off2 = p.c2s_orb.off[cr.l2];
    a.pp_begin = cr.pp_begin;
    a.pp_count = cr.pp_count;
    a.pp_P = p.d_pp_P.as<double>();
    a.pp_g = p.d_pp_g.as<double>();
    a.pp_pref = p.d_pp_pref.as<double>();
    a.esph = p.d_esph.as<double>() + cr.esph_off;
    const int nab = (2 * cr.l1 + 1) * (2 * cr.l2 + 1);
    const int64_t threads = cr.pp_count * nab;
    const unsigned blocks = (unsigned)((threads + 127) / 128);
    bool done = false;
#define X(A, B)                                                        \
  if (cr.l1 == A && cr.l2 == B) {                                      \
    pair_setup_kernel<A, B><<<blocks, 128, 0, s>>>(a);                 \
    done = true;                                                       \
  }
    DFJK_L1L2_CASES(X)
#undef X
    if (!done) fail(DFJK_ERR_UNSUPPORTED, "pair class (%d,%d) not compiled", cr.l1, cr.l2);
    DFJK_LAUNCHED();
  }
}

void launch_eri3c_rows(Plan& p, int64_t pair_begin, int64_t pair_end, int64_t row_base,
                       void* out, int64_t ld, bool f32, cudaStream_t s) {
  const Context& c = *p.ctx;
  auto single = [](const std::vector<int>& np) {
    for (int n : np)
      if (n != 1) return false;
    return true;
  };
  const int uncontracted = single(p.orb.nprim) && single(p.aux.nprim) ? 1 : 0;
  for (const ClassRange& cr : p.classes) {
    const int64_t b = pair_begin > cr.begin ? pair_begin : cr.begin;
    const int64_t e = pair_end < cr.begin + cr.count ? pair_end : cr.begin + cr.count;
    if (b >= e) continue;
    for (int lc = 0; lc <= p.aux.lmax; ++lc) {
      if (p.aux_lcount[lc] == 0) continue;
      Eri3cArgs a;
      a.pair_row0 = p.d_pair_row0.as<int64_t>();
      a.pair_pp0 = p.d_pair_pp0.as<int64_t>();
      a.pair_npp = p.d_pair_npp.as<int>();
      a.pp_P = p.d_pp_P.as<double>();
      a.pp_g = p.d_pp_g.as<double>();
      a.pp_pref = p.d_pp_pref.as<double>();
      a.esph = p.d_esph.as<double>() + cr.esph_off;
      a.esph_pp0 = cr.pp_begin;
      a.aux_sorted = p.d_aux_sorted.as<int>();
      a.aux = view(p.aux);
      a.c2s_aux = p.c2s_aux.dev.as<double>() + p.c2s_aux.off[lc];
      a.boys = c.boys.as<double>();
      a.boys_asym = c.boys_asym.as<double>();
      a.aux_begin = p.aux_lbegin[lc];
      a.aux_count = p.aux_lcount[lc];
      a.col_base = p.aux_col0[p.aux_order[p.aux_lbegin[lc]]];
      a.row_base = row_base;
      a.ld = ld;
      a.out = out;
      a.out_f32 = f32 ? 1 : 0;
      a.omega = p.atten;
      a.uncontracted = uncontracted;
      const int ychunks = (a.aux_count + 127) / 128;
      for (int64_t q = b; q < e; q += (int64_t)1 << 30) {
        const int64_t n = (e - q) < ((int64_t)1 << 30) ? (e - q) : ((int64_t)1 << 30);
        a.pair_begin = q;
        dim3 grid((unsigned)n, (unsigned)ychunks);
        const bool ok = launch_eri3c(cr.l1, cr.l2, lc, grid, s, a);
        if (!ok) fail(DFJK_ERR_UNSUPPORTED, "3-center class (%d,%d|%d) not compiled", cr.l1, cr.l2, lc);
        DFJK_LAUNCHED();
      }
    }
  }
}

void launch_eri3c_rows_batch(const std::vector<Plan*>& ps, cudaStream_t s) {
  if (ps.empty()) return;
  const Context& c = *ps[0]->ctx;
  auto single = [](const std::vector<int>& np) {
    for (int n : np)
      if (n != 1) return false;
    return true;
  };
  // segments per light (l1, l2 | lc) class, in plan order
  struct Group {
    std::vector<Eri3cArgs> seg;
    std::vector<int64_t> blk0{0};
    std::vector<int> ydim;
  };
  std::map<std::tuple<int, int, int>, Group> groups;
  for (Plan* pp : ps) {
    Plan& p = *pp;
    const int uncontracted = single(p.orb.nprim) && single(p.aux.nprim) ? 1 : 0;
    for (const ClassRange& cr : p.classes) {
      if (cr.count == 0) continue;
      for (int lc = 0; lc <= p.aux.lmax; ++lc) {
        if (p.aux_lcount[lc] == 0) continue;
        Eri3cArgs a;
        a.pair_row0 = p.d_pair_row0.as<int64_t>();
        a.pair_pp0 = p.d_pair_pp0.as<int64_t>();
        a.pair_npp = p.d_pair_npp.as<int>();
        a.pp_P = p.d_pp_P.as<double>();
        a.pp_g = p.d_pp_g.as<double>();
        a.pp_pref = p.d_pp_pref.as<double>();
        a.esph = p.d_esph.as<double>() + cr.esph_off;
        a.esph_pp0 = cr.pp_begin;
        a.aux_sorted = p.d_aux_sorted.as<int>();
        a.aux = view(p.aux);
        a.c2s_aux = p.c2s_aux.dev.as<double>() + p.c2s_aux.off[lc];
        a.boys = c.boys.as<double>();
        a.boys_asym = c.boys_asym.as<double>();
        a.aux_begin = p.aux_lbegin[lc];
        a.aux_count = p.aux_lcount[lc];
        a.col_base = p.aux_col0[p.aux_order[p.aux_lbegin[lc]]];
        a.row_base = 0;
        a.ld = p.naux;
        a.out = p.ws_raw.p;
        a.out_f32 = 0;
        a.omega = p.atten;
        a.uncontracted = uncontracted;
        a.pair_begin = cr.begin;
        const int y = (a.aux_count + 127) / 128;
        if (cr.l1 + cr.l2 + lc >= kCoopM) {
          // heavy classes keep the plain launch of this plan (launch_one picks
          // the cooperative kernel for uncontracted shells)
          if (!launch_eri3c(cr.l1, cr.l2, lc, dim3((unsigned)cr.count, (unsigned)y), s, a))
            fail(DFJK_ERR_UNSUPPORTED, "3-center class (%d,%d|%d) not compiled", cr.l1, cr.l2, lc);
          DFJK_LAUNCHED();
          continue;
        }
        Group& g = groups[{cr.l1, cr.l2, lc}];
        g.seg.push_back(a);
        g.ydim.push_back(y);
        g.blk0.push_back(g.blk0.back() + cr.count * (int64_t)y);
      }
    }
  }
  // the queue tables: one set of buffers per group, freed into the device
  // cache (whose reuse waits for the device) when this function returns; the
  // pageable host tables are staged by the time each copy returns
  std::vector<DevBuf> keep(groups.size() * 3);
  size_t k = 0;
  for (auto& kv : groups) {
    const int l1 = std::get<0>(kv.first), l2 = std::get<1>(kv.first), lc = std::get<2>(kv.first);
    Group& g = kv.second;
    DevBuf& dseg = keep[k++];
    DevBuf& dblk = keep[k++];
    DevBuf& dy = keep[k++];
    dseg.alloc(g.seg.size() * sizeof(Eri3cArgs));
    DFJK_CUDA(cudaMemcpyAsync(dseg.p, g.seg.data(), g.seg.size() * sizeof(Eri3cArgs),
                              cudaMemcpyHostToDevice, s));
    dblk.alloc(g.blk0.size() * sizeof(int64_t));
    DFJK_CUDA(cudaMemcpyAsync(dblk.p, g.blk0.data(), g.blk0.size() * sizeof(int64_t),
                              cudaMemcpyHostToDevice, s));
    dy.alloc(g.ydim.size() * sizeof(int));
    DFJK_CUDA(cudaMemcpyAsync(dy.p, g.ydim.data(), g.ydim.size() * sizeof(int),
                              cudaMemcpyHostToDevice, s));
    Eri3cBatch b;
    b.seg = dseg.as<Eri3cArgs>();
    b.blk0 = dblk.as<int64_t>();
    b.ydim = dy.as<int>();
    b.nseg = (int)g.seg.size();
    b.total = g.blk0.back();
    const unsigned blocks = (unsigned)b.total;   // one block per queue entry
    if (blocks == 0) continue;
    if (!launch_eri3c_batch(l1, l2, lc, blocks, s, b))
      fail(DFJK_ERR_UNSUPPORTED, "3-center class (%d,%d|%d) not compiled", l1, l2, lc);
    DFJK_LAUNCHED();
  }
}

#define DFJK_LPLQ_CASES(X)                                                    \
  X(0, 0) X(1, 0) X(1, 1) X(2, 0) X(2, 1) X(2, 2) X(3, 0) X(3, 1) X(3, 2) X(3, 3) \
  X(4, 0) X(4, 1) X(4, 2) X(4, 3) X(4, 4)

void launch_eri2c(Plan& p, double* out, int64_t ld, cudaStream_t s) {
  const Context& c = *p.ctx;
  for (int lp = 0; lp <= p.aux.lmax; ++lp) {
    if (!p.aux_lcount[lp]) continue;
    for (int lq = 0; lq <= lp; ++lq) {
      if (!p.aux_lcount[lq]) continue;
      Eri2cArgs a;
      a.aux_sorted = p.d_aux_sorted.as<int>();
      a.aux = view(p.aux);
      a.c2s = p.c2s_aux.dev.as<double>();
      a.offP = p.c2s_aux.off[lp];
      a.offQ = p.c2s_aux.off[lq];
      a.boys = c.boys.as<double>();
      a.omega = p.atten;
      a.boys_asym = c.boys_asym.as<double>();
      a.beginP = p.aux_lbegin[lp];
      a.countP = p.aux_lcount[lp];
      a.beginQ = p.aux_lbegin[lq];
      a.countQ = p.aux_lcount[lq];
      a.colP = p.aux_col0[p.aux_order[a.beginP]];
      a.colQ = p.aux_col0[p.aux_order[a.beginQ]];
      a.ld = ld;
      a.out = out;
      const int64_t n = (int64_t)a.countP * a.countQ;
      const unsigned blocks = (unsigned)((n + 127) / 128);
      bool done = false;
#define X(A, B)                                              \
  if (lp == A && lq == B) {                                  \
    eri2c_kernel<A, B><<<blocks, 128, 0, s>>>(a);            \
    done = true;                                             \
  }
      DFJK_LPLQ_CASES(X)
#undef X
      if (!done) fail(DFJK_ERR_UNSUPPORTED, "aux class (%d,%d) not compiled", lp, lq);
      DFJK_LAUNCHED();
    }
  }
}

void launch_schwarz(const Context& c, Shells& sh, const std::vector<int>& pa,
                    const std::vector<int>& pb, std::vector<double>& qmax) {
  const int64_t n = (int64_t)pa.size();
  qmax.assign(n, 0.0);
  std::vector<std::vector<int64_t>> groups(16);
  for (int64_t i = 0; i < n; ++i) {
    int l1 = sh.l[pa[i]], l2 = sh.l[pb[i]];
    if (l1 < l2) std::swap(l1, l2);
    groups[l1 * 4 + l2].push_back(i);
  }
  for (int l1 = 0; l1 <= 3; ++l1)
    for (int l2 = 0; l2 <= l1; ++l2) {
      auto& g = groups[l1 * 4 + l2];
      if (g.empty()) continue;
      std::vector<int> ga(g.size()), gb(g.size());
      for (size_t i = 0; i < g.size(); ++i) {
        int x = pa[g[i]], y = pb[g[i]];
        if (sh.l[x] < sh.l[y]) std::swap(x, y);
        ga[i] = x;
        gb[i] = y;
      }
      DevBuf da, db, dq;
      upload(da, ga);
      upload(db, gb);
      dq.alloc(g.size() * sizeof(double));
      SchwarzArgs a{da.as<int>(), db.as<int>(), (int64_t)g.size(), view(sh),
                    c.boys.as<double>(), c.boys_asym.as<double>(), dq.as<double>()};
      const unsigned blocks = (unsigned)((g.size() + 63) / 64);
      bool done = false;
#define X(A, B)                                     \
  if (l1 == A && l2 == B) {                         \
    schwarz_kernel<A, B><<<blocks, 64>>>(a);        \
    done = true;                                    \
  }
      DFJK_L1L2_CASES(X)
#undef X
      if (!done) fail(DFJK_ERR_UNSUPPORTED, "schwarz class (%d,%d) not compiled", l1, l2);
      DFJK_LAUNCHED();
      std::vector<double> q(g.size());
      DFJK_CUDA(cudaMemcpy(q.data(), dq.p, g.size() * sizeof(double), cudaMemcpyDeviceToHost));
      for (size_t i = 0; i < g.size(); ++i) qmax[g[i]] = q[i];
    }
}

}  // namespace dfjk

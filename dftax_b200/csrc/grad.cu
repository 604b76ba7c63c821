// Nuclear gradient of the DF energy at a fixed density.
//
// dftax's forces() differentiate the energy through the integral build
// (dftax/ks/forces.py:245-270), with the metric pseudo-inverse differentiated
// by d(V+) = -V+ dV V+ (_metric_pinv_jvp, dftax/ks/terms.py:196-204). For
// E = 1/2 c^T V+ c + sum_s k_s sum_PQ V+_PQ tr(P_s T_P P_s T_Q) (c_P =
// tr(P_tot T_P), T_P = (..|P), k_s = -a_x/4 closed shell, -a_x/2 per spin)
// that derivative is
//   dE = sum_{mn,P} G[mn][P] d(mn|P) - 1/2 sum_PQ W[P][Q] d(P|Q),
// and in terms of the plan's B = T L (V+ = L L^T) and g = B^T vec(P_tot):
//   H[r][x] = w_r (g_x P_tot[r] + sum_s 2 k_s (P_s B_x P_s)[r])   (w_r = 2 for
//             off-diagonal bra pairs: they stand for (m,n) and (n,m)),
//   M = H^T B = g g^T + sum_s 2 k_s tr(P_s B_x P_s B_y),  E = 1/2 tr(M),
//   G = H L^T (3-center row layout),  W = L M L^T.
// G and W are contracted with the integral derivatives on the fly
// (grad3c.cuh; grad2c_kernel below); nothing of size rows x naux beyond one
// chunk of G is kept.
#include "grad3c.cuh"
#include "internal.h"

#include <algorithm>

namespace dfjk {

namespace {

ShellView view(const Shells& s) {
  return ShellView{s.d_l.as<int>(), s.d_nprim.as<int>(), s.d_prim0.as<int>(),
                   s.d_cen.as<double>(), s.d_pexp.as<double>(), s.d_pcoef.as<double>()};
}

bool launch_grad3c(int l1, int l2, int lc, dim3 grid, cudaStream_t s, const Grad3cArgs& a) {
  switch (l1 * 4 + l2) {
    case 0: return launch_grad3c_00(lc, grid, s, a);
    case 4: return launch_grad3c_10(lc, grid, s, a);
    case 5: return launch_grad3c_11(lc, grid, s, a);
    case 8: return launch_grad3c_20(lc, grid, s, a);
    case 9: return launch_grad3c_21(lc, grid, s, a);
    case 10: return launch_grad3c_22(lc, grid, s, a);
    case 12: return launch_grad3c_30(lc, grid, s, a);
    case 13: return launch_grad3c_31(lc, grid, s, a);
    case 14: return launch_grad3c_32(lc, grid, s, a);
    case 15: return launch_grad3c_33(lc, grid, s, a);
    default: return false;
  }
}

bool launch_pair_deriv(int l1, int l2, unsigned blocks, cudaStream_t s, const PairDerivArgs& a) {
  switch (l1 * 4 + l2) {
    case 0: launch_pair_deriv_00(blocks, s, a); return true;
    case 4: launch_pair_deriv_10(blocks, s, a); return true;
    case 5: launch_pair_deriv_11(blocks, s, a); return true;
    case 8: launch_pair_deriv_20(blocks, s, a); return true;
    case 9: launch_pair_deriv_21(blocks, s, a); return true;
    case 10: launch_pair_deriv_22(blocks, s, a); return true;
    case 12: launch_pair_deriv_30(blocks, s, a); return true;
    case 13: launch_pair_deriv_31(blocks, s, a); return true;
    case 14: launch_pair_deriv_32(blocks, s, a); return true;
    case 15: launch_pair_deriv_33(blocks, s, a); return true;
    default: return false;
  }
}

// H[r][x] = w_r g[x] Ptot[m][n]   (x < ldb; g is zero past the kept directions)
__global__ void h_init_kernel(const double* __restrict__ g, const double* __restrict__ Ptot,
                              int64_t nao, const int* __restrict__ rm, const int* __restrict__ rn,
                              const int8_t* __restrict__ kind, int64_t nrows, int64_t ldb,
                              double* __restrict__ H) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nrows * ldb) return;
  const int64_t r = i / ldb, x = i % ldb;
  const double wr = kind[r] == 2 ? 2.0 : 1.0;
  H[i] = wr * g[x] * Ptot[(int64_t)rm[r] * nao + rn[r]];
}

// Bd[x][m][n] = B[r][x0 + x] for every row r = (m, n); off-diagonal rows also
// fill [n][m] (the rows of a diagonal shell pair hold both orders already)
__global__ void unpack_b_kernel(const double* __restrict__ B, int64_t ldb, int64_t nrows,
                                const int* __restrict__ rm, const int* __restrict__ rn,
                                const int8_t* __restrict__ kind, int64_t nao, int64_t x0,
                                int64_t nx, double* __restrict__ Bd) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nrows * nx) return;
  const int64_t r = i / nx, x = i % nx;
  const double v = B[r * ldb + x0 + x];
  const int m = rm[r], n = rn[r];
  double* plane = Bd + x * nao * nao;
  plane[(int64_t)m * nao + n] = v;
  if (kind[r] == 2) plane[(int64_t)n * nao + m] = v;
}

// H[r][x0 + x] += w_r a T[x][m][n]
__global__ void h_add_kernel(const double* __restrict__ T, int64_t nao, const int* __restrict__ rm,
                             const int* __restrict__ rn, const int8_t* __restrict__ kind,
                             int64_t nrows, int64_t ldb, int64_t x0, int64_t nx, double a,
                             double* __restrict__ H) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nrows * nx) return;
  const int64_t r = i / nx, x = i % nx;
  const double wr = kind[r] == 2 ? 2.0 : 1.0;
  H[r * ldb + x0 + x] += wr * a * T[x * nao * nao + (int64_t)rm[r] * nao + rn[r]];
}

__global__ void add2_kernel(const double* __restrict__ a, const double* __restrict__ b, int64_t n,
                            double* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] + b[i];
}

// out[0] = sum_i M[i][i] (one block, fixed order)
__global__ void trace_kernel(const double* __restrict__ M, int64_t n, int64_t ld,
                             double* __restrict__ out) {
  __shared__ double part[256];
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += M[i * ld + i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = part[0];
}

// ---------------------------------------------------------------------------
// 2-center derivative: (P|Q) depends on A - B only, so
//   d(P|Q)/dA_x = hob sum_{c1,c2} T_P[c1][p] T_Q[c2][q] R_{c1 + c2 + e_x}(A - B) = -d/dB_x.
// One thread per unordered pair of shells of the (LP, LQ) groups; the
// contribution -1/2 sum_{p,q} W[p][q] d(p|q) counts both orders of a pair.
// ---------------------------------------------------------------------------

struct Grad2cArgs {
  const int* aux_sorted;
  ShellView aux;
  const double* c2s;
  int offP, offQ;
  const double* boys;
  const double* boys_asym;
  int beginP, countP, beginQ, countQ;
  int colP, colQ;
  int64_t ld;
  const double* W;       // naux x naux, sorted columns (symmetric)
  double omega;
  double* grad_aux;      // [aux shell][3]
};

template <int LP, int LQ>
__global__ void __launch_bounds__(128) grad2c_kernel(Grad2cArgs a) {
  constexpr int NP = 2 * LP + 1, NQ = 2 * LQ + 1, CP = nc_(LP), CQ = nc_(LQ);
  constexpr int M1 = LP + LQ + 1, NR = hcount(M1);
  const int64_t gid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (gid >= (int64_t)a.countP * a.countQ) return;
  const int ip = (int)(gid / a.countQ), iq = (int)(gid % a.countQ);
  if (LP == LQ && ip >= iq) return;   // same group: each unordered pair once; a shell with itself has no derivative
  const int sp = a.aux_sorted[a.beginP + ip], sq = a.aux_sorted[a.beginQ + iq];
  const double X = a.aux.cen[3 * sp] - a.aux.cen[3 * sq];
  const double Y = a.aux.cen[3 * sp + 1] - a.aux.cen[3 * sq + 1];
  const double Z = a.aux.cen[3 * sp + 2] - a.aux.cen[3 * sq + 2];
  const double* TP = a.c2s + a.offP;
  const double* TQ = a.c2s + a.offQ;
  // W projected on the cartesian components: Wc[c1][c2] = sum_{p,q} T_P W T_Q
  double Wc[CP * CQ];
  const int r0 = a.colP + ip * NP, c0 = a.colQ + iq * NQ;
#pragma unroll 1
  for (int c1 = 0; c1 < CP; ++c1)
#pragma unroll 1
    for (int c2 = 0; c2 < CQ; ++c2) {
      double s = 0.0;
#pragma unroll 1
      for (int p = 0; p < NP; ++p) {
        const double tp = __ldg(TP + c1 * NP + p);
        if (tp == 0.0) continue;
#pragma unroll 1
        for (int q = 0; q < NQ; ++q) s += tp * __ldg(TQ + c2 * NQ + q) * a.W[(int64_t)(r0 + p) * a.ld + c0 + q];
      }
      Wc[c1 * CQ + c2] = s;
    }
  double f[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
  for (int i = 0; i < a.aux.nprim[sp]; ++i) {
    const double al = a.aux.pexp[a.aux.prim0[sp] + i], ca = a.aux.pcoef[a.aux.prim0[sp] + i];
#pragma unroll 1
    for (int j = 0; j < a.aux.nprim[sq]; ++j) {
      const double be = a.aux.pexp[a.aux.prim0[sq] + j], cb = a.aux.pcoef[a.aux.prim0[sq] + j];
      const double rho = al * be / (al + be);
      double F[M1 + 1];
      boys_operator<M1>(rho * (X * X + Y * Y + Z * Z), rho, a.omega, a.boys, a.boys_asym, F);
      double R[NR];
      hermite_r<M1>(rho, X, Y, Z, F, R);
      double hob = kTwoPi25 * ca * cb / (al * be * sqrt(al + be));
#pragma unroll
      for (int k = 0; k < LP; ++k) hob *= 0.5 / al;
#pragma unroll
      for (int k = 0; k < LQ; ++k) hob *= -0.5 / be;
#pragma unroll 1
      for (int c1 = 0; c1 < CP; ++c1) {
        const int x1 = comp_x(LP, c1), y1 = comp_y(LP, c1), z1 = comp_z(LP, c1);
#pragma unroll 1
        for (int c2 = 0; c2 < CQ; ++c2) {
          const double wc = hob * Wc[c1 * CQ + c2];
          if (wc == 0.0) continue;
          const int x = x1 + comp_x(LQ, c2), y = y1 + comp_y(LQ, c2), z = z1 + comp_z(LQ, c2);
          f[0] += wc * R[hidx(x + 1, y, z)];
          f[1] += wc * R[hidx(x, y + 1, z)];
          f[2] += wc * R[hidx(x, y, z + 1)];
        }
      }
    }
  }
  // -1/2 (W_pq + W_qp) d(p|q)/dA = -f on P's center, +f on Q's (dB = -dA)
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    atomicAdd(a.grad_aux + 3 * sp + d, -f[d]);
    atomicAdd(a.grad_aux + 3 * sq + d, f[d]);
  }
}

#define DFJK_G2_CASES(X)                                                      \
  X(0, 0) X(1, 0) X(1, 1) X(2, 0) X(2, 1) X(2, 2) X(3, 0) X(3, 1) X(3, 2) X(3, 3) \
  X(4, 0) X(4, 1) X(4, 2) X(4, 3) X(4, 4)

void launch_grad2c(Plan& p, const double* W, double* grad_aux, cudaStream_t s) {
  const Context& c = *p.ctx;
  for (int lp = 0; lp <= p.aux.lmax; ++lp) {
    if (!p.aux_lcount[lp]) continue;
    for (int lq = 0; lq <= lp; ++lq) {
      if (!p.aux_lcount[lq]) continue;
      Grad2cArgs a;
      a.aux_sorted = p.d_aux_sorted.as<int>();
      a.aux = view(p.aux);
      a.c2s = p.c2s_aux.dev.as<double>();
      a.offP = p.c2s_aux.off[lp];
      a.offQ = p.c2s_aux.off[lq];
      a.boys = c.boys.as<double>();
      a.boys_asym = c.boys_asym.as<double>();
      a.beginP = p.aux_lbegin[lp];
      a.countP = p.aux_lcount[lp];
      a.beginQ = p.aux_lbegin[lq];
      a.countQ = p.aux_lcount[lq];
      a.colP = p.aux_col0[p.aux_order[a.beginP]];
      a.colQ = p.aux_col0[p.aux_order[a.beginQ]];
      a.ld = p.naux;
      a.W = W;
      a.omega = p.atten;
      a.grad_aux = grad_aux;
      const int64_t n = (int64_t)a.countP * a.countQ;
      const unsigned blocks = (unsigned)((n + 127) / 128);
      bool done = false;
#define X(A, B)                                              \
  if (lp == A && lq == B) {                                  \
    grad2c_kernel<A, B><<<blocks, 128, 0, s>>>(a);           \
    done = true;                                             \
  }
      DFJK_G2_CASES(X)
#undef X
      if (!done) fail(DFJK_ERR_UNSUPPORTED, "aux derivative class (%d,%d) not compiled", lp, lq);
      DFJK_LAUNCHED();
    }
  }
}

// derivative tables of the pairs [b, e) of class cr into dsph, then the
// 3-center derivative contraction of those pairs with G (rows from row_base)
void launch_grad3c_pairs(Plan& p, const ClassRange& cr, int64_t b, int64_t e, double* dsph,
                         const double* G, int64_t row_base, double* grad_orb, double* grad_aux,
                         cudaStream_t s) {
  const Context& c = *p.ctx;
  const int64_t pp_b = p.pair_pp0[b];
  const int64_t pp_e = p.pair_pp0[e - 1] + p.pair_npp[e - 1];
  const int nab = (2 * cr.l1 + 1) * (2 * cr.l2 + 1);
  {
    PairDerivArgs a;
    a.pp_pair = p.d_pp_pair.as<int>();
    a.pp_pa = p.d_pp_pa.as<int>();
    a.pp_pb = p.d_pp_pb.as<int>();
    a.pair_s1 = p.d_pair_s1.as<int>();
    a.pair_s2 = p.d_pair_s2.as<int>();
    a.orb = view(p.orb);
    a.c2s = p.c2s_orb.dev.as<double>();
    a.off1 = p.c2s_orb.off[cr.l1];
    a.off2 = p.c2s_orb.off[cr.l2];
    a.pp_begin = pp_b;
    a.pp_count = pp_e - pp_b;
    a.dsph = dsph;
    const int64_t threads = a.pp_count * 3 * nab;
    if (!launch_pair_deriv(cr.l1, cr.l2, (unsigned)((threads + 127) / 128), s, a))
      fail(DFJK_ERR_UNSUPPORTED, "pair derivative class (%d,%d) not compiled", cr.l1, cr.l2);
    DFJK_LAUNCHED();
  }
  for (int lc = 0; lc <= p.aux.lmax; ++lc) {
    if (p.aux_lcount[lc] == 0) continue;
    Grad3cArgs a;
    a.pair_row0 = p.d_pair_row0.as<int64_t>();
    a.pair_pp0 = p.d_pair_pp0.as<int64_t>();
    a.pair_npp = p.d_pair_npp.as<int>();
    a.pair_s1 = p.d_pair_s1.as<int>();
    a.pair_s2 = p.d_pair_s2.as<int>();
    a.pp_P = p.d_pp_P.as<double>();
    a.pp_g = p.d_pp_g.as<double>();
    a.pp_pref = p.d_pp_pref.as<double>();
    a.esph = p.d_esph.as<double>() + cr.esph_off;
    a.esph_pp0 = cr.pp_begin;
    a.dsph = dsph;
    a.dsph_pp0 = pp_b;
    a.aux_sorted = p.d_aux_sorted.as<int>();
    a.aux = view(p.aux);
    a.c2s_aux = p.c2s_aux.dev.as<double>() + p.c2s_aux.off[lc];
    a.boys = c.boys.as<double>();
    a.boys_asym = c.boys_asym.as<double>();
    a.pair_begin = b;
    a.aux_begin = p.aux_lbegin[lc];
    a.aux_count = p.aux_lcount[lc];
    a.col_base = p.aux_col0[p.aux_order[p.aux_lbegin[lc]]];
    a.row_base = row_base;
    a.ld = p.naux;
    a.G = G;
    a.omega = p.atten;
    a.grad_orb = grad_orb;
    a.grad_aux = grad_aux;
    dim3 grid((unsigned)(e - b), (unsigned)((a.aux_count + 127) / 128));
    if (!launch_grad3c(cr.l1, cr.l2, lc, grid, s, a))
      fail(DFJK_ERR_UNSUPPORTED, "3-center derivative class (%d,%d|%d) not compiled", cr.l1, cr.l2, lc);
    DFJK_LAUNCHED();
  }
}

}  // namespace

double energy_gradient(Plan& p, const double* P, int nspin, double hf, double* grad_orb,
                       double* grad_aux, cudaStream_t s) {
  Context& c = *p.ctx;
  const int64_t n = p.nao, nn = n * n, ldb = p.ldb, naux = p.naux, rows = p.nrows;
  check_finite(p, P, nn * nspin, s, "the density");
  DFJK_CUDA(cudaMemsetAsync(grad_orb, 0, (size_t)p.orb.n * 3 * sizeof(double), s));
  DFJK_CUDA(cudaMemsetAsync(grad_aux, 0, (size_t)p.aux.n * 3 * sizeof(double), s));
  DevBuf Ptot_b, g, H, M, T, W;
  const double* Ptot = P;
  if (nspin == 2) {
    Ptot_b.alloc(nn * sizeof(double));
    add2_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(P, P + nn, nn, Ptot_b.as<double>());
    DFJK_LAUNCHED();
    Ptot = Ptot_b.as<double>();
  }
  g.alloc(ldb * sizeof(double));
  gamma_from_density(p, Ptot, g.as<double>(), s);
  // H = w (g P_tot + sum_s 2 k_s P_s B_x P_s)
  H.alloc((size_t)std::max<int64_t>(rows, 1) * ldb * sizeof(double));
  if (rows > 0) {
    h_init_kernel<<<(unsigned)((rows * ldb + 255) / 256), 256, 0, s>>>(
        g.as<double>(), Ptot, n, p.d_row_m.as<int>(), p.d_row_n.as<int>(), p.d_row_w.as<int8_t>(),
        rows, ldb, H.as<double>());
    DFJK_LAUNCHED();
  }
  DFJK_CUBLAS(cublasSetStream(c.cublas, s));
  if (hf != 0.0 && rows > 0) {
    const double k = (nspin == 1 ? -0.25 : -0.5) * hf;
    const int64_t xc = std::max<int64_t>(1, std::min<int64_t>(p.nfit, ((int64_t)1 << 30) / (16 * nn)));
    DevBuf Bd, T1;
    Bd.alloc((size_t)xc * nn * sizeof(double));
    T1.alloc((size_t)xc * nn * sizeof(double));
    const double one = 1.0, zero = 0.0;
    for (int sp = 0; sp < nspin; ++sp) {
      const double* Ps = P + sp * nn;
      for (int64_t x0 = 0; x0 < p.nfit; x0 += xc) {
        const int64_t nx = std::min(xc, p.nfit - x0);
        DFJK_CUDA(cudaMemsetAsync(Bd.p, 0, (size_t)nx * nn * sizeof(double), s));
        unpack_b_kernel<<<(unsigned)((rows * nx + 255) / 256), 256, 0, s>>>(
            p.d_B.as<double>(), ldb, rows, p.d_row_m.as<int>(), p.d_row_n.as<int>(),
            p.d_row_w.as<int8_t>(), n, x0, nx, Bd.as<double>());
        DFJK_LAUNCHED();
        // T1_x = B_x P_s, Bd_x = P_s T1_x (all symmetric but T1)
        DFJK_CUBLAS(cublasDgemmStridedBatched(c.cublas, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, (int)n,
                                              (int)n, &one, Bd.as<double>(), (int)n, nn, Ps, (int)n,
                                              0, &zero, T1.as<double>(), (int)n, nn, (int)nx));
        DFJK_CUBLAS(cublasDgemmStridedBatched(c.cublas, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, (int)n,
                                              (int)n, &one, Ps, (int)n, 0, T1.as<double>(), (int)n,
                                              nn, &zero, Bd.as<double>(), (int)n, nn, (int)nx));
        h_add_kernel<<<(unsigned)((rows * nx + 255) / 256), 256, 0, s>>>(
            Bd.as<double>(), n, p.d_row_m.as<int>(), p.d_row_n.as<int>(), p.d_row_w.as<int8_t>(),
            rows, ldb, x0, nx, 2.0 * k, H.as<double>());
        DFJK_LAUNCHED();
      }
    }
  }
  // M = H^T B (ldb x ldb); E = 1/2 tr(M)
  const double one = 1.0, zero = 0.0;
  M.alloc((size_t)ldb * ldb * sizeof(double));
  if (rows > 0) {
    DFJK_CUBLAS(cublasDgemm(c.cublas, CUBLAS_OP_N, CUBLAS_OP_T, (int)ldb, (int)ldb, (int)rows, &one,
                            H.as<double>(), (int)ldb, p.d_B.as<double>(), (int)ldb, &zero,
                            M.as<double>(), (int)ldb));
  } else {
    DFJK_CUDA(cudaMemsetAsync(M.p, 0, (size_t)ldb * ldb * sizeof(double), s));
  }
  DevBuf tr;
  tr.alloc(sizeof(double));
  trace_kernel<<<1, 256, 0, s>>>(M.as<double>(), ldb, ldb, tr.as<double>());
  DFJK_LAUNCHED();
  // W = L M L^T
  T.alloc((size_t)naux * ldb * sizeof(double));
  W.alloc((size_t)naux * naux * sizeof(double));
  DFJK_CUBLAS(cublasDgemm(c.cublas, CUBLAS_OP_N, CUBLAS_OP_N, (int)naux, (int)ldb, (int)ldb, &one,
                          p.d_L.as<double>(), (int)naux, M.as<double>(), (int)ldb, &zero,
                          T.as<double>(), (int)naux));
  DFJK_CUBLAS(cublasDgemm(c.cublas, CUBLAS_OP_N, CUBLAS_OP_T, (int)naux, (int)naux, (int)ldb,
                          &one, T.as<double>(), (int)naux, p.d_L.as<double>(), (int)naux,
                          &zero, W.as<double>(), (int)naux));
  M.free();
  T.free();
  launch_grad2c(p, W.as<double>(), grad_aux, s);
  // G = H L^T chunk by chunk, contracted with the 3-center derivatives
  if (rows > 0) {
    auto chunks = pair_chunks(p, naux, chunk_budget(p));
    int64_t maxrows = 1;
    for (auto& ch : chunks) maxrows = std::max(maxrows, rows_of(p, ch.first, ch.second));
    DevBuf G, dsph;
    G.alloc((size_t)maxrows * naux * sizeof(double));
    const int64_t dsph_budget = (int64_t)512 << 20;   // bytes of derivative tables per launch
    dsph.alloc((size_t)dsph_budget);
    for (auto& ch : chunks) {
      const int64_t r0 = p.pair_row0[ch.first], nr = rows_of(p, ch.first, ch.second);
      DFJK_CUBLAS(cublasDgemm(c.cublas, CUBLAS_OP_N, CUBLAS_OP_N, (int)naux, (int)nr, (int)ldb, &one,
                              p.d_L.as<double>(), (int)naux, H.as<double>() + r0 * ldb, (int)ldb,
                              &zero, G.as<double>(), (int)naux));
      for (const ClassRange& cr : p.classes) {
        const int64_t b = std::max(ch.first, cr.begin), e = std::min(ch.second, cr.begin + cr.count);
        if (b >= e) continue;
        const int nab = (2 * cr.l1 + 1) * (2 * cr.l2 + 1);
        const int64_t per_pp = 3 * (int64_t)nab * hcount(cr.l1 + cr.l2 + 1) * (int64_t)sizeof(double);
        // sub-runs whose primitive pairs' derivative tables fit in dsph
        int64_t q = b;
        while (q < e) {
          int64_t qe = q, npp = 0;
          while (qe < e && (qe == q || (npp + p.pair_npp[qe]) * per_pp <= dsph_budget)) npp += p.pair_npp[qe++];
          if (npp * per_pp > dsph_budget)
            fail(DFJK_ERR_MEMORY, "derivative tables of one shell pair exceed %lld bytes",
                 (long long)dsph_budget);
          launch_grad3c_pairs(p, cr, q, qe, dsph.as<double>(), G.as<double>(), r0, grad_orb,
                              grad_aux, s);
          q = qe;
        }
      }
    }
  }
  double e = 0.0;
  DFJK_CUDA(cudaMemcpyAsync(&e, tr.p, sizeof(double), cudaMemcpyDeviceToHost, s));
  DFJK_CUDA(cudaStreamSynchronize(s));
  return 0.5 * e;
}

}  // namespace dfjk

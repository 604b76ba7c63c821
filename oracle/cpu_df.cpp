// Compiled, multithreaded CPU restatement of dftax's density-fitting integrals.
//
// TEST INFRASTRUCTURE ONLY: the timed CPU baseline and a second checker beside
// the numpy oracle (oracle/md.py, which it is tested against). The product
// library never links or calls it.
//
// Follows dftax/integrals/eri3c_bucketed.py, the same steps as oracle/md.py:
//   * two-center Hermite E tables by the McMurchie-Davidson recursion
//     E^{i+1,j}_t = X_PA E_t + 1/(2p) E_{t-1} + (t+1) E_{t+1} and likewise in j
//     with X_PB (_bump/_E_table, :290-313); single-center auxiliary tables with
//     X_PA = 0 (_Ec_table, :316-323), signed by (-1)^tau (:409);
//   * R^0_{tuv} by the descending m-ladder from R^m_000 = (-2 rho)^m
//     F_m(rho |PC|^2) (_hermite_table, :326-369);
//   * (ab|c) = K_AB 2 pi^{5/2} / (p g_c sqrt(p + g_c))
//       * sum_{t,u,v} E^{ab}_{tuv} sum_{tau,ups,phi} (-1)^{tau+ups+phi}
//         E^c_{tau ups phi} R_{t+tau, u+ups, v+phi}
//     contracted over primitives (_make_class_kernel, :376-426);
//   * cart -> sph with each shell's own block of the basis's cart2sph, written
//     to the (ab) block and its (ba) mirror of the dense (nao, nao, naux)
//     tensor (eri3c_matrix_bucketed, :782-854);
//   * (P|Q) with single-center tables on both sides (_make_eri2c_kernel,
//     :697-734; eri2c_matrix_bucketed, :746-779);
//   * the Boys function by dftax's table scheme (dftax/energy/boys.py:130-176):
//     the nearest node of the 0.1-spaced table and a degree-6 Taylor series,
//     the asymptotic form from t = 40. The table is passed in (oracle/boys.py
//     builds it).
//
// Work is split over shell pairs (3-center) or auxiliary shell rows (2-center)
// with an atomic counter; every pair writes its own output blocks.
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr int kLmax = 4;                  // auxiliary shells up to g, orbitals up to f
constexpr int kMt = 3 + 3 + kLmax + 2;    // Hermite orders + 1 (la + lb + lc + 1, padded)
constexpr int kOrder = 6;
constexpr double kDt = 0.1;
constexpr double kTmax = 40.0;
constexpr int kTblCols = 25;
constexpr double kTwoPi25 = 34.98683665524972;   // 2 pi^{5/2}

struct Basis {
  int nsh;
  const int* l;
  const double* cen;     // 3 per shell
  const int* nprim;
  const int* prim0;
  const double* pexp;    // per primitive
  const double* pcoef;   // per primitive (uniform over a shell's cartesian rows)
  const int* ang;        // per shell: ncart(l) x 3 (lx, ly, lz) in the basis's row order
  const int* ang0;       // offset of a shell's components in ang (in rows)
  const double* c2s;     // per shell: ncart x nsph block, row-major
  const int64_t* c2s0;   // offset of a shell's block in c2s
  const int* nsph;       // spherical functions of a shell
  const int64_t* sph0;   // first spherical index of a shell
};

struct Boys {
  const double* tbl;     // NGRID x 25
  int ngrid;
  double eval(int n, double t) const {
    if (t < kTmax) {
      int j = (int)std::nearbyint(t / kDt);
      if (j < 0) j = 0;
      if (j > ngrid - 1) j = ngrid - 1;
      const double dx = j * kDt - t;
      const double* row = tbl + (int64_t)j * kTblCols;
      double acc = row[n + kOrder];
      for (int k = kOrder - 1; k >= 0; --k) acc = row[n + k] + acc * dx / (k + 1);
      return acc;
    }
    const double a = n + 0.5;
    return 0.5 * std::exp(std::lgamma(a)) * std::pow(t, -a);
  }
};

inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// E[i][j][t] for one axis: i <= la, j <= lb, t <= la + lb
void e_axis(int la, int lb, double a, double b, double xab, double (*E)[kLmax + 1][kMt]) {
  const double p = a + b, i2g = 0.5 / p;
  const double xpa = -b * xab / p, xpb = a * xab / p;
  const int mt = la + lb + 1;
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j <= lb; ++j)
      for (int t = 0; t < mt + 1; ++t) E[i][j][t] = 0.0;
  E[0][0][0] = 1.0;
  for (int i = 0; i < la; ++i)
    for (int t = 0; t <= i + 1; ++t)
      E[i + 1][0][t] = xpa * E[i][0][t] + (t > 0 ? i2g * E[i][0][t - 1] : 0.0) +
                       (t + 1) * E[i][0][t + 1];
  for (int j = 0; j < lb; ++j)
    for (int i = 0; i <= la; ++i)
      for (int t = 0; t <= i + j + 1; ++t)
        E[i][j + 1][t] = xpb * E[i][j][t] + (t > 0 ? i2g * E[i][j][t - 1] : 0.0) +
                         (t + 1) * E[i][j][t + 1];
}

// single-center table (X_PA = 0), signed by (-1)^tau: Ec[k][tau]
void ec_axis(int lc, double g, double (*Ec)[kMt]) {
  const double i2g = 0.5 / g;
  for (int k = 0; k <= lc; ++k)
    for (int t = 0; t <= lc + 1; ++t) Ec[k][t] = 0.0;
  Ec[0][0] = 1.0;
  for (int k = 0; k < lc; ++k)
    for (int t = 0; t <= k + 1; ++t)
      Ec[k + 1][t] = (t > 0 ? i2g * Ec[k][t - 1] : 0.0) + (t + 1) * Ec[k][t + 1];
  for (int k = 0; k <= lc; ++k)
    for (int t = 1; t <= lc; t += 2) Ec[k][t] = -Ec[k][t];
}

// R^0_{tuv}, t + u + v < mt, stored R[t][u][v]
struct RTable {
  double v[kMt][kMt][kMt];
};

// the ladder alternates between the two tables; returns the one holding R^0
const RTable* hermite_r(double rho, double X, double Y, double Z, int mt, const Boys& boys,
                        RTable& R, RTable& tmp) {
  const double targ = rho * (X * X + Y * Y + Z * Z);
  double base[kMt];
  double m2r = 1.0;
  for (int m = 0; m < mt; ++m) {
    base[m] = m2r * boys.eval(m, targ);
    m2r *= -2.0 * rho;
  }
  // level m holds R^m_{tuv} for t + u + v <= mt - 1 - m
  RTable* cur = &R;
  RTable* nxt = &tmp;
  cur->v[0][0][0] = base[mt - 1];
  for (int m = mt - 2; m >= 0; --m) {
    const int top = mt - 1 - m;
    for (int t = 0; t <= top; ++t)
      for (int u = 0; u <= top - t; ++u)
        for (int w = 0; w <= top - t - u; ++w) {
          double r;
          if (t == 0 && u == 0 && w == 0) r = base[m];
          else if (t > 0) r = X * cur->v[t - 1][u][w] + (t > 1 ? (t - 1) * cur->v[t - 2][u][w] : 0.0);
          else if (u > 0) r = Y * cur->v[t][u - 1][w] + (u > 1 ? (u - 1) * cur->v[t][u - 2][w] : 0.0);
          else r = Z * cur->v[t][u][w - 1] + (w > 1 ? (w - 1) * cur->v[t][u][w - 2] : 0.0);
          nxt->v[t][u][w] = r;
        }
    RTable* s = cur;
    cur = nxt;
    nxt = s;
  }
  return cur;
}

struct PairPrim {
  double p, P[3], K;
  double E[3][kLmax + 1][kLmax + 1][kMt];
};

// cartesian (ab|c) block [nca][ncb][ncc] of one triple, accumulated over primitives
void triple_cart(const Basis& ob, int a, int b, const std::vector<PairPrim>& pp,
                 const double* cab, const Basis& xb, int c, const Boys& boys, double* out,
                 RTable& R, RTable& tmp, std::vector<double>& W) {
  const int la = ob.l[a], lb = ob.l[b], lc = xb.l[c];
  const int nca = ncart(la), ncb = ncart(lb), ncc = ncart(lc);
  const int lab = la + lb, mt = lab + lc + 1;
  const int* anga = ob.ang + 3 * ob.ang0[a];
  const int* angb = ob.ang + 3 * ob.ang0[b];
  const int* angc = xb.ang + 3 * xb.ang0[c];
  const double* C = xb.cen + 3 * c;
  std::memset(out, 0, sizeof(double) * nca * ncb * ncc);
  const int nh = (lab + 1) * (lab + 1) * (lab + 1);
  W.resize((size_t)ncc * nh);
  for (size_t q = 0; q < pp.size(); ++q) {
    const PairPrim& e = pp[q];
    for (int k = 0; k < xb.nprim[c]; ++k) {
      const double gc = xb.pexp[xb.prim0[c] + k];
      const double cc = xb.pcoef[xb.prim0[c] + k];
      const double rho = e.p * gc / (e.p + gc);
      const double pref = e.K * kTwoPi25 / (e.p * gc * std::sqrt(e.p + gc)) * cab[q] * cc;
      const RTable& Rt = *hermite_r(rho, e.P[0] - C[0], e.P[1] - C[1], e.P[2] - C[2], mt, boys,
                                    R, tmp);
      double Ec[kLmax + 1][kMt];
      ec_axis(lc, gc, Ec);
      // W_k[t][u][v] = sum over the aux component's Hermite terms
      for (int kc = 0; kc < ncc; ++kc) {
        const int kx = angc[3 * kc], ky = angc[3 * kc + 1], kz = angc[3 * kc + 2];
        double* Wk = W.data() + (size_t)kc * nh;
        for (int t = 0; t <= lab; ++t)
          for (int u = 0; u <= lab - t; ++u)
            for (int v = 0; v <= lab - t - u; ++v) {
              double s = 0.0;
              for (int tx = kx & 1; tx <= kx; tx += 2)
                for (int ty = ky & 1; ty <= ky; ty += 2) {
                  const double exy = Ec[kx][tx] * Ec[ky][ty];
                  for (int tz = kz & 1; tz <= kz; tz += 2)
                    s += exy * Ec[kz][tz] * Rt.v[t + tx][u + ty][v + tz];
                }
              Wk[(t * (lab + 1) + u) * (lab + 1) + v] = s;
            }
      }
      for (int ia = 0; ia < nca; ++ia) {
        const int ax = anga[3 * ia], ay = anga[3 * ia + 1], az = anga[3 * ia + 2];
        for (int ib = 0; ib < ncb; ++ib) {
          const int bx = angb[3 * ib], by = angb[3 * ib + 1], bz = angb[3 * ib + 2];
          const double* Ex = e.E[0][ax][bx];
          const double* Ey = e.E[1][ay][by];
          const double* Ez = e.E[2][az][bz];
          double* o = out + ((size_t)ia * ncb + ib) * ncc;
          for (int kc = 0; kc < ncc; ++kc) {
            const double* Wk = W.data() + (size_t)kc * nh;
            double s = 0.0;
            for (int t = 0; t <= ax + bx; ++t)
              for (int u = 0; u <= ay + by; ++u) {
                const double exy = Ex[t] * Ey[u];
                const double* wr = Wk + (t * (lab + 1) + u) * (lab + 1);
                for (int v = 0; v <= az + bz; ++v) s += exy * Ez[v] * wr[v];
              }
            o[kc] += pref * s;
          }
        }
      }
    }
  }
}

void pair_prims(const Basis& ob, int a, int b, std::vector<PairPrim>& pp, std::vector<double>& cab) {
  const double* A = ob.cen + 3 * a;
  const double* B = ob.cen + 3 * b;
  const double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
  const double ab2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
  pp.clear();
  cab.clear();
  for (int i = 0; i < ob.nprim[a]; ++i)
    for (int j = 0; j < ob.nprim[b]; ++j) {
      const double al = ob.pexp[ob.prim0[a] + i], be = ob.pexp[ob.prim0[b] + j];
      PairPrim e;
      e.p = al + be;
      for (int x = 0; x < 3; ++x) e.P[x] = (al * A[x] + be * B[x]) / e.p;
      e.K = std::exp(-al * be / e.p * ab2);
      for (int x = 0; x < 3; ++x) e_axis(ob.l[a], ob.l[b], al, be, AB[x], e.E[x]);
      pp.push_back(e);
      cab.push_back(ob.pcoef[ob.prim0[a] + i] * ob.pcoef[ob.prim0[b] + j]);
    }
}

template <class Fn>
void parallel_for(int64_t n, int threads, Fn&& fn) {
  std::atomic<int64_t> next{0};
  auto work = [&]() {
    for (int64_t i; (i = next.fetch_add(1)) < n;) fn(i);
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < threads; ++t) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {

// Dense (nao, nao, naux) spherical 3-center tensor, both bra triangles, over
// the shell pairs a <= b listed in pa/pb (npair of them).
int cpu_eri3c_dense(
    int onsh, const int* ol, const double* ocen, const int* onprim, const int* oprim0,
    const double* opexp, const double* opcoef, const int* oang, const int* oang0,
    const double* oc2s, const int64_t* oc2s0, const int* onsph, const int64_t* osph0,
    int xnsh, const int* xl, const double* xcen, const int* xnprim, const int* xprim0,
    const double* xpexp, const double* xpcoef, const int* xang, const int* xang0,
    const double* xc2s, const int64_t* xc2s0, const int* xnsph, const int64_t* xsph0,
    int64_t npair, const int* pa, const int* pb, const double* boys_tbl, int ngrid,
    int64_t nao, int64_t naux, int threads, double* out) {
  Basis ob{onsh, ol, ocen, onprim, oprim0, opexp, opcoef, oang, oang0, oc2s, oc2s0, onsph, osph0};
  Basis xb{xnsh, xl, xcen, xnprim, xprim0, xpexp, xpcoef, xang, xang0, xc2s, xc2s0, xnsph, xsph0};
  for (int s = 0; s < onsh; ++s)
    if (ol[s] > 3) return 2;
  for (int s = 0; s < xnsh; ++s)
    if (xl[s] > kLmax) return 2;
  Boys boys{boys_tbl, ngrid};
  parallel_for(npair, threads < 1 ? 1 : threads, [&](int64_t q) {
    thread_local std::vector<PairPrim> pp;
    thread_local std::vector<double> cab, W, cart, half, sph;
    thread_local RTable R, tmp;
    const int a = pa[q], b = pb[q];
    pair_prims(ob, a, b, pp, cab);
    const int la = ob.l[a], lb = ob.l[b];
    const int nca = ncart(la), ncb = ncart(lb), na = ob.nsph[a], nb = ob.nsph[b];
    const double* Ta = ob.c2s + ob.c2s0[a];
    const double* Tb = ob.c2s + ob.c2s0[b];
    for (int c = 0; c < xnsh; ++c) {
      const int ncc = ncart(xb.l[c]), nc = xb.nsph[c];
      const double* Tc = xb.c2s + xb.c2s0[c];
      cart.resize((size_t)nca * ncb * ncc);
      triple_cart(ob, a, b, pp, cab.data(), xb, c, boys, cart.data(), R, tmp, W);
      // cart -> sph: first the aux index, then b, then a
      half.assign((size_t)nca * ncb * nc, 0.0);
      for (int i = 0; i < nca * ncb; ++i)
        for (int k = 0; k < ncc; ++k) {
          const double v = cart[(size_t)i * ncc + k];
          if (v == 0.0) continue;
          for (int mc = 0; mc < nc; ++mc) half[(size_t)i * nc + mc] += v * Tc[k * nc + mc];
        }
      sph.assign((size_t)na * nb * nc, 0.0);
      for (int ia = 0; ia < nca; ++ia)
        for (int ib = 0; ib < ncb; ++ib) {
          const double* h = half.data() + ((size_t)ia * ncb + ib) * nc;
          for (int ma = 0; ma < na; ++ma) {
            const double ta = Ta[ia * na + ma];
            if (ta == 0.0) continue;
            for (int mb = 0; mb < nb; ++mb) {
              const double w = ta * Tb[ib * nb + mb];
              if (w == 0.0) continue;
              double* o = sph.data() + ((size_t)ma * nb + mb) * nc;
              for (int mc = 0; mc < nc; ++mc) o[mc] += w * h[mc];
            }
          }
        }
      const int64_t r0 = ob.sph0[a], s0 = ob.sph0[b], c0 = xb.sph0[c];
      for (int ma = 0; ma < na; ++ma)
        for (int mb = 0; mb < nb; ++mb) {
          const double* v = sph.data() + ((size_t)ma * nb + mb) * nc;
          double* o1 = out + ((r0 + ma) * nao + (s0 + mb)) * naux + c0;
          double* o2 = out + ((s0 + mb) * nao + (r0 + ma)) * naux + c0;
          for (int mc = 0; mc < nc; ++mc) {
            o1[mc] = v[mc];
            o2[mc] = v[mc];
          }
        }
    }
  });
  return 0;
}

// (naux, naux) spherical metric (P|Q).
int cpu_eri2c(int xnsh, const int* xl, const double* xcen, const int* xnprim, const int* xprim0,
              const double* xpexp, const double* xpcoef, const int* xang, const int* xang0,
              const double* xc2s, const int64_t* xc2s0, const int* xnsph, const int64_t* xsph0,
              const double* boys_tbl, int ngrid, int64_t naux, int threads, double* out) {
  Basis xb{xnsh, xl, xcen, xnprim, xprim0, xpexp, xpcoef, xang, xang0, xc2s, xc2s0, xnsph, xsph0};
  for (int s = 0; s < xnsh; ++s)
    if (xl[s] > kLmax) return 2;
  Boys boys{boys_tbl, ngrid};
  parallel_for(xnsh, threads < 1 ? 1 : threads, [&](int64_t pidx) {
    thread_local RTable R, tmp;
    thread_local std::vector<double> cart, half, sph;
    const int p = (int)pidx;
    const int lp = xb.l[p], ncp = ncart(lp), np_ = xb.nsph[p];
    const int* angp = xb.ang + 3 * xb.ang0[p];
    const double* Tp = xb.c2s + xb.c2s0[p];
    const double* A = xb.cen + 3 * p;
    for (int q = 0; q <= p; ++q) {
      const int lq = xb.l[q], ncq = ncart(lq), nq = xb.nsph[q];
      const int* angq = xb.ang + 3 * xb.ang0[q];
      const double* Tq = xb.c2s + xb.c2s0[q];
      const double* B = xb.cen + 3 * q;
      const int mt = lp + lq + 1;
      cart.assign((size_t)ncp * ncq, 0.0);
      for (int i = 0; i < xb.nprim[p]; ++i)
        for (int j = 0; j < xb.nprim[q]; ++j) {
          const double a = xb.pexp[xb.prim0[p] + i], b = xb.pexp[xb.prim0[q] + j];
          const double rho = a * b / (a + b);
          const double pref = kTwoPi25 / (a * b * std::sqrt(a + b)) *
                              xb.pcoef[xb.prim0[p] + i] * xb.pcoef[xb.prim0[q] + j];
          const RTable& Rt = *hermite_r(rho, A[0] - B[0], A[1] - B[1], A[2] - B[2], mt, boys, R,
                                        tmp);
          double Ea[kLmax + 1][kMt], Eb[kLmax + 1][kMt];
          ec_axis(lp, a, Ea);
          ec_axis(lq, b, Eb);
          // the bra side is unsigned: undo the (-1)^t of ec_axis on it
          for (int k = 0; k <= lp; ++k)
            for (int t = 1; t <= lp; t += 2) Ea[k][t] = -Ea[k][t];
          for (int ip = 0; ip < ncp; ++ip) {
            const int ax = angp[3 * ip], ay = angp[3 * ip + 1], az = angp[3 * ip + 2];
            for (int iq = 0; iq < ncq; ++iq) {
              const int bx = angq[3 * iq], by = angq[3 * iq + 1], bz = angq[3 * iq + 2];
              double s = 0.0;
              for (int t = ax & 1; t <= ax; t += 2)
                for (int tx = bx & 1; tx <= bx; tx += 2)
                  for (int u = ay & 1; u <= ay; u += 2)
                    for (int ty = by & 1; ty <= by; ty += 2) {
                      const double exy = Ea[ax][t] * Eb[bx][tx] * Ea[ay][u] * Eb[by][ty];
                      for (int v = az & 1; v <= az; v += 2)
                        for (int tz = bz & 1; tz <= bz; tz += 2)
                          s += exy * Ea[az][v] * Eb[bz][tz] * Rt.v[t + tx][u + ty][v + tz];
                    }
              cart[(size_t)ip * ncq + iq] += pref * s;
            }
          }
        }
      half.assign((size_t)ncp * nq, 0.0);
      for (int ip = 0; ip < ncp; ++ip)
        for (int iq = 0; iq < ncq; ++iq)
          for (int mq = 0; mq < nq; ++mq) half[(size_t)ip * nq + mq] += cart[(size_t)ip * ncq + iq] * Tq[iq * nq + mq];
      sph.assign((size_t)np_ * nq, 0.0);
      for (int ip = 0; ip < ncp; ++ip)
        for (int mp = 0; mp < np_; ++mp)
          for (int mq = 0; mq < nq; ++mq) sph[(size_t)mp * nq + mq] += Tp[ip * np_ + mp] * half[(size_t)ip * nq + mq];
      const int64_t r0 = xb.sph0[p], s0 = xb.sph0[q];
      for (int mp = 0; mp < np_; ++mp)
        for (int mq = 0; mq < nq; ++mq) {
          out[(r0 + mp) * naux + s0 + mq] = sph[(size_t)mp * nq + mq];
          out[(s0 + mq) * naux + r0 + mp] = sph[(size_t)mp * nq + mq];
        }
    }
  });
  return 0;
}

}  // extern "C"

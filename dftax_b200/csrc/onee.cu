// One-electron integrals: overlap S, kinetic T and nuclear attraction V.
//
// One thread per orbital shell pair (first shell of the larger l), per class
// (LA, LB). Per primitive pair the McMurchie-Davidson E tables of each axis
// (eri3c_bucketed.py:290-313) are formed up to j = LB + 2, which gives
//   S_ij = K_AB (pi/p)^{3/2} E^x_{ij,0} E^y E^z,
//   T_ij = b (2 L_b + 3) S_ij - 2 b^2 sum_x S(i, j + 2_x)
//          - 1/2 sum_x j_x (j_x - 1) S(i, j - 2_x)       (eri3c_bucketed.py:611-623),
//   V_ij = -sum_C Z_C K_AB 2 pi / p sum_tuv E_t E_u E_v R_tuv(p, P - C)
//                                                      (eri3c_bucketed.py:486-518),
// with R summed over the nuclei before the contraction. The cartesian blocks
// go to spherical form with the basis's own blocks and are written at (a, b)
// and, transposed, at (b, a).
#include "md_device.cuh"
#include "scf.h"

namespace dfjk {
namespace {

struct OneeArgs {
  OrbView ov;
  const int* pa;
  const int* pb;
  int npair;
  int natom;
  const double* atom_xyz;
  const double* atom_z;
  const double* boys;
  const double* boys_asym;
  double* S;
  double* T;
  double* V;
};

template <int LA, int LB>
__global__ void __launch_bounds__(64) onee_kernel(OneeArgs a) {
  constexpr int NCA = nc_(LA), NCB = nc_(LB), M = LA + LB, NR = hcount(M);
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.npair) return;
  const ShellView& sh = a.ov.sh;
  const int s1 = a.pa[q], s2 = a.pb[q];
  const double A0 = sh.cen[3 * s1], A1 = sh.cen[3 * s1 + 1], A2 = sh.cen[3 * s1 + 2];
  const double B0 = sh.cen[3 * s2], B1 = sh.cen[3 * s2 + 1], B2 = sh.cen[3 * s2 + 2];
  const double AB[3] = {A0 - B0, A1 - B1, A2 - B2};
  const double ab2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
  double Sc[NCA][NCB], Tc[NCA][NCB], Vc[NCA][NCB];
  for (int i = 0; i < NCA; ++i)
    for (int j = 0; j < NCB; ++j) Sc[i][j] = Tc[i][j] = Vc[i][j] = 0.0;
  for (int ia = 0; ia < sh.nprim[s1]; ++ia) {
    for (int ib = 0; ib < sh.nprim[s2]; ++ib) {
      const double al = sh.pexp[sh.prim0[s1] + ia], be = sh.pexp[sh.prim0[s2] + ib];
      const double cc = sh.pcoef[sh.prim0[s1] + ia] * sh.pcoef[sh.prim0[s2] + ib];
      const double p = al + be;
      const double P0 = (al * A0 + be * B0) / p, P1 = (al * A1 + be * B1) / p,
                   P2 = (al * A2 + be * B2) / p;
      const double K = exp(-al * be / p * ab2);
      double Ex[LA + 1][LB + 3][LA + LB + 3], Ey[LA + 1][LB + 3][LA + LB + 3],
          Ez[LA + 1][LB + 3][LA + LB + 3];
      e_axis<LA, LB + 2>(al, be, AB[0], Ex);
      e_axis<LA, LB + 2>(al, be, AB[1], Ey);
      e_axis<LA, LB + 2>(al, be, AB[2], Ez);
      double Rs[NR];
#pragma unroll
      for (int h = 0; h < NR; ++h) Rs[h] = 0.0;
      for (int c = 0; c < a.natom; ++c) {
        const double X = P0 - a.atom_xyz[3 * c], Y = P1 - a.atom_xyz[3 * c + 1],
                     Z = P2 - a.atom_xyz[3 * c + 2];
        double F[M + 1], R[NR];
        boys_eval<M>(p * (X * X + Y * Y + Z * Z), a.boys, a.boys_asym, F);
        hermite_r<M>(p, X, Y, Z, F, R);
        const double z = a.atom_z[c];
#pragma unroll
        for (int h = 0; h < NR; ++h) Rs[h] -= z * R[h];
      }
      const double pref = cc * K * pow(3.141592653589793 / p, 1.5);
      const double vpref = cc * K * 2.0 * 3.141592653589793 / p;
#pragma unroll
      for (int i = 0; i < NCA; ++i) {
        const int ix = comp_x(LA, i), iy = comp_y(LA, i), iz = comp_z(LA, i);
#pragma unroll
        for (int j = 0; j < NCB; ++j) {
          const int jx = comp_x(LB, j), jy = comp_y(LB, j), jz = comp_z(LB, j);
          const double sx = Ex[ix][jx][0], sy = Ey[iy][jy][0], sz = Ez[iz][jz][0];
          const double s = sx * sy * sz;
          const double up = Ex[ix][jx + 2][0] * sy * sz + sx * Ey[iy][jy + 2][0] * sz +
                            sx * sy * Ez[iz][jz + 2][0];
          double dn = 0.0;
          if (jx >= 2) dn += jx * (jx - 1) * Ex[ix][jx - 2][0] * sy * sz;
          if (jy >= 2) dn += jy * (jy - 1) * sx * Ey[iy][jy - 2][0] * sz;
          if (jz >= 2) dn += jz * (jz - 1) * sx * sy * Ez[iz][jz - 2][0];
          Sc[i][j] += pref * s;
          Tc[i][j] += pref * (be * (2 * LB + 3) * s - 2.0 * be * be * up - 0.5 * dn);
          double v = 0.0;
          for (int t = 0; t <= ix + jx; ++t)
            for (int u = 0; u <= iy + jy; ++u) {
              const double exy = Ex[ix][jx][t] * Ey[iy][jy][u];
              for (int w = 0; w <= iz + jz; ++w) v += exy * Ez[iz][jz][w] * Rs[hidx(t, u, w)];
            }
          Vc[i][j] += vpref * v;
        }
      }
    }
  }
  // cart -> sph with the basis's blocks, written at (a, b) and (b, a)
  const int na = a.ov.nout[LA], nb = a.ov.nout[LB];
  const double* Ta = a.ov.c2s + a.ov.c2s_off[LA];
  const double* Tb = a.ov.c2s + a.ov.c2s_off[LB];
  const int64_t r0 = a.ov.out0[s1], c0 = a.ov.out0[s2], n = a.ov.nao;
  double* outs[3] = {a.S, a.T, a.V};
  for (int k = 0; k < 3; ++k) {
    if (!outs[k]) continue;
    const double(*B)[NCB] = k == 0 ? Sc : (k == 1 ? Tc : Vc);
    double* O = outs[k];
    for (int ma = 0; ma < na; ++ma)
      for (int mb = 0; mb < nb; ++mb) {
        double acc = 0.0;
        for (int i = 0; i < NCA; ++i) {
          const double ta = Ta[i * na + ma];
          if (ta == 0.0) continue;
          double r = 0.0;
          for (int j = 0; j < NCB; ++j) r += B[i][j] * Tb[j * nb + mb];
          acc += ta * r;
        }
        O[(r0 + ma) * n + c0 + mb] = acc;
        O[(c0 + mb) * n + r0 + ma] = acc;
      }
  }
}

template <int LA, int LB>
void launch_class(const OneeArgs& a, cudaStream_t s) {
  onee_kernel<LA, LB><<<(a.npair + 63) / 64, 64, 0, s>>>(a);
  DFJK_LAUNCHED();
}

void launch_any(int la, int lb, const OneeArgs& a, cudaStream_t s) {
  switch (la * 4 + lb) {
    case 0: return launch_class<0, 0>(a, s);
    case 4: return launch_class<1, 0>(a, s);
    case 5: return launch_class<1, 1>(a, s);
    case 8: return launch_class<2, 0>(a, s);
    case 9: return launch_class<2, 1>(a, s);
    case 10: return launch_class<2, 2>(a, s);
    case 12: return launch_class<3, 0>(a, s);
    case 13: return launch_class<3, 1>(a, s);
    case 14: return launch_class<3, 2>(a, s);
    case 15: return launch_class<3, 3>(a, s);
  }
  fail(DFJK_ERR_UNSUPPORTED, "one-electron integrals: class (%d, %d) not compiled", la, lb);
}

}  // namespace

void launch_one_electron(const Context& c, const OrbView& ov, int nshell, const std::vector<int>& l,
                         int natom, const double* atom_xyz, const double* atom_z, double* S,
                         double* T, double* V, cudaStream_t s) {
  // shell pairs by class, the shell of larger l first
  std::vector<int> pa[4][4], pb[4][4];
  for (int i = 0; i < nshell; ++i)
    for (int j = i; j < nshell; ++j) {
      int a = i, b = j;
      if (l[a] < l[b]) std::swap(a, b);
      if (l[a] > 3) fail(DFJK_ERR_UNSUPPORTED, "one-electron integrals support l <= 3");
      pa[l[a]][l[b]].push_back(a);
      pb[l[a]][l[b]].push_back(b);
    }
  std::vector<int> all_a, all_b;
  std::vector<std::pair<int, int>> cls;
  std::vector<int64_t> off;
  for (int la = 0; la < 4; ++la)
    for (int lb = 0; lb <= la; ++lb) {
      if (pa[la][lb].empty()) continue;
      cls.push_back({la, lb});
      off.push_back((int64_t)all_a.size());
      all_a.insert(all_a.end(), pa[la][lb].begin(), pa[la][lb].end());
      all_b.insert(all_b.end(), pb[la][lb].begin(), pb[la][lb].end());
    }
  DevBuf da, db;
  upload(da, all_a);
  upload(db, all_b);
  for (size_t k = 0; k < cls.size(); ++k) {
    OneeArgs a{};
    a.ov = ov;
    a.pa = da.as<int>() + off[k];
    a.pb = db.as<int>() + off[k];
    a.npair = (int)pa[cls[k].first][cls[k].second].size();
    a.natom = natom;
    a.atom_xyz = atom_xyz;
    a.atom_z = atom_z;
    a.boys = c.boys.as<double>();
    a.boys_asym = c.boys_asym.as<double>();
    a.S = S;
    a.T = T;
    a.V = V;
    launch_any(cls[k].first, cls[k].second, a, s);
  }
  // the pair lists are freed on return
  DFJK_CUDA(cudaStreamSynchronize(s));
}

}  // namespace dfjk

// Exchange-correlation energy and Fock matrix of a closed-shell density on a
// point grid, and the Becke partition of an atom-centered grid.
//
// Per chunk of G points (dftax/ks/terms.py:776-828, GridXC; energy/grid.py:10-45):
//   Phi[mu][g], dPhi[x][mu][g]   AO values and gradients (ao_kernel: one thread
//                                per point and shell, points fastest, so the
//                                stores of a warp are contiguous), as
//                                dftax/energy/gto.py:371-412 evaluates them;
//   X = Phi P                    cuBLAS DGEMM;
//   rho_g = sum_mu X Phi, grad rho_g = 2 sum_mu X dPhi        (rho_kernel);
//   e_g = w rho eps_xc(rho, grad rho) and its derivatives v_rho, v_grad by
//   forward-mode dual numbers over the same expression as dftax's PBE
//   (xc.py:87-252, PBE0 :584-601; points with rho <= 1e-10 contribute nothing,
//   as the double-where of grid.py:31-44 makes them);
//   W = v_rho/2 Phi + v_grad . dPhi, V += Phi^T W               (cuBLAS DGEMM);
// and at the end Vxc = V + V^T, the symmetrized P-gradient of E_xc
// (scf.py:42-46). The chunks run on kXcBranches concurrent streams (chunk k
// on branch k % kXcBranches, one V accumulator each, summed in branch order
// at the end); the energy is summed per block in a fixed order and then over
// blocks on the host, so the result is reproducible. The SCF calls this with
// the same buffers every iteration: the second call captures its launches
// (about eight per chunk, the branches forked and joined by events) in a
// CUDA graph and later calls replay it.
#include "md_device.cuh"
#include "scf.h"

#include <algorithm>
#include <cmath>
#include <thread>
#include <utility>

namespace dfjk {
namespace {

constexpr int kAoThreads = 128;
constexpr size_t kXcBlasWorkspace = (size_t)8 << 20;   // per XC branch cuBLAS handle
constexpr int kPtThreads = 256;

// ---------------------------------------------------------------------------
// Becke partition
// ---------------------------------------------------------------------------

// one thread per point; the point's distances to the atoms in shared memory
__global__ void becke_kernel(const double* __restrict__ pts, const int* __restrict__ owner,
                             const double* __restrict__ raw, int64_t n,
                             const double* __restrict__ xyz, const double* __restrict__ inv_rab,
                             const double* __restrict__ aab, int natom, double* __restrict__ w) {
  extern __shared__ double sr[];   // [natom][blockDim.x]
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int lt = threadIdx.x, nt = blockDim.x;
  if (i >= n) return;
  const double px = pts[3 * i], py = pts[3 * i + 1], pz = pts[3 * i + 2];
  for (int a = 0; a < natom; ++a) {
    const double dx = px - xyz[3 * a], dy = py - xyz[3 * a + 1], dz = pz - xyz[3 * a + 2];
    sr[a * nt + lt] = sqrt(dx * dx + dy * dy + dz * dz + 1e-30);
  }
  const int own = owner[i];
  double total = 0.0, mine = 0.0;
  for (int a = 0; a < natom; ++a) {
    const double ra = sr[a * nt + lt];
    double cell = 1.0;
    for (int b = 0; b < natom; ++b) {
      if (b == a) continue;
      const double mu = (ra - sr[b * nt + lt]) * inv_rab[a * natom + b];
      double f = mu + aab[a * natom + b] * (1.0 - mu * mu);
      f = 1.5 * f - 0.5 * f * f * f;
      f = 1.5 * f - 0.5 * f * f * f;
      f = 1.5 * f - 0.5 * f * f * f;
      cell *= 0.5 * (1.0 - f);
    }
    total += cell;
    if (a == own) mine = cell;
  }
  w[i] = raw[i] * mine / total;
}

// ---------------------------------------------------------------------------
// AO values and gradients
// ---------------------------------------------------------------------------

// p[n] for 0 <= n <= L (p[0] for n < 0) by selects, so p stays in registers
// whether or not n folds to a constant
template <int L>
__device__ __forceinline__ double pick(const double (&p)[L + 1], int n) {
  double r = p[0];
#pragma unroll
  for (int i = 1; i <= L; ++i) r = n == i ? p[i] : r;
  return r;
}

// values and gradients of one shell's NC cartesian components at (dx, dy,
// dz), in dftax's order (lx descending, then ly), transformed by the shell's
// block T (NC x nout) and stored at o, o + plane, ...; L is a template
// parameter so the component arrays stay in registers
template <int L>
__device__ __forceinline__ void ao_shell(const OrbView& ov, int s, double dx, double dy,
                                         double dz, bool live, int64_t o, int64_t G,
                                         int64_t plane, double* __restrict__ phi,
                                         double* __restrict__ dphi) {
  constexpr int NC = (L + 1) * (L + 2) / 2;
  const ShellView& sh = ov.sh;
  const int nout = ov.nout[L];                 // constant index: no local copy of ov
  const double* __restrict__ T = ov.c2s + ov.c2s_off[L];
  double val[NC], gx[NC], gy[NC], gz[NC];
#pragma unroll
  for (int k = 0; k < NC; ++k) val[k] = gx[k] = gy[k] = gz[k] = 0.0;
  if (live) {
    const double r2 = dx * dx + dy * dy + dz * dz;
    double rad = 0.0, drad = 0.0;
    for (int k = 0; k < sh.nprim[s]; ++k) {
      const double a = sh.pexp[sh.prim0[s] + k], c = sh.pcoef[sh.prim0[s] + k];
      const double e = c * exp(-a * r2);
      rad += e;
      drad += -2.0 * a * e;
    }
    double px[L + 1], py[L + 1], pz[L + 1];
    px[0] = py[0] = pz[0] = 1.0;
#pragma unroll
    for (int k = 1; k <= L; ++k) {
      px[k] = px[k - 1] * dx;
      py[k] = py[k - 1] * dy;
      pz[k] = pz[k - 1] * dz;
    }
#pragma unroll
    for (int k = 0; k < NC; ++k) {
      const int lx = comp_x(L, k), ly = comp_y(L, k), lz = L - lx - ly;
      const double xl = pick<L>(px, lx), yl = pick<L>(py, ly), zl = pick<L>(pz, lz);
      const double ang = xl * yl * zl;
      val[k] = ang * rad;
      const double dpx = lx * pick<L>(px, lx - 1);
      const double dpy = ly * pick<L>(py, ly - 1);
      const double dpz = lz * pick<L>(pz, lz - 1);
      gx[k] = dpx * yl * zl * rad + ang * drad * dx;
      gy[k] = xl * dpy * zl * rad + ang * drad * dy;
      gz[k] = xl * yl * dpz * rad + ang * drad * dz;
    }
  }
  for (int m = 0; m < nout; ++m) {
    double v = 0.0, a = 0.0, b = 0.0, c = 0.0;
#pragma unroll
    for (int q = 0; q < NC; ++q) {
      const double t = T[q * nout + m];
      v += val[q] * t;
      a += gx[q] * t;
      b += gy[q] * t;
      c += gz[q] * t;
    }
    const int64_t om = o + (int64_t)m * G;
    phi[om] = v;
    dphi[om] = a;
    dphi[plane + om] = b;
    dphi[2 * plane + om] = c;
  }
}

// Phi[k][g] (ld G), dPhi[x][k][g] for the chunk's shells of angular momentum
// L: shell j of the list is orbital shell shl[j] with compact AOs k =
// out0c[j] .. ; grid (ceil(G / 128), shells of the list). One instance per L,
// so the s and p shells, most of the work, do not carry the registers of the
// d and f cases.
template <int L>
__global__ void __launch_bounds__(kAoThreads) ao_kernel(OrbView ov, const int* __restrict__ shl,
                                                        const int* __restrict__ out0c,
                                                        const double* __restrict__ pts,
                                                        int64_t g0, int64_t ng, int64_t G, int nsig,
                                                        double* __restrict__ phi,
                                                        double* __restrict__ dphi) {
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int s = shl[blockIdx.y];
  if (g >= G) return;
  const ShellView& sh = ov.sh;
  const int64_t o = (int64_t)out0c[blockIdx.y] * G + g;
  const int64_t plane = (int64_t)nsig * G;
  const bool live = g < ng;
  double dx = 0.0, dy = 0.0, dz = 0.0;
  if (live) {
    const double* p = pts + 3 * (g0 + g);
    dx = p[0] - sh.cen[3 * s];
    dy = p[1] - sh.cen[3 * s + 1];
    dz = p[2] - sh.cen[3 * s + 2];
  }
  ao_shell<L>(ov, s, dx, dy, dz, live, o, G, plane, phi, dphi);
}

// Pc[k1][k2] = P[map[k1]][map[k2]]
__global__ void gather_p_kernel(const double* __restrict__ P, int nao, const int* __restrict__ map,
                                int nsig, double* __restrict__ Pc) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= (int64_t)nsig * nsig) return;
  const int64_t a = i / nsig, b = i % nsig;
  Pc[i] = P[(int64_t)map[a] * nao + map[b]];
}

// V[map[k1]][map[k2]] += Vc[k1][k2] (column-major Vc; the map is one-to-one)
__global__ void scatter_v_kernel(const double* __restrict__ Vc, int nsig, const int* __restrict__ map,
                                 int nao, double* __restrict__ V) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= (int64_t)nsig * nsig) return;
  const int64_t a = i % nsig, b = i / nsig;
  V[(int64_t)map[b] * nao + map[a]] += Vc[i];
}

// rho[g] = sum_mu X Phi, grad[x][g] = 2 sum_mu X dPhi_x. A block takes 16
// points with 16 lanes of mu each (mu = lane, lane + 16, ...: a warp reads 16
// consecutive points of two mu rows), so an 8192-point chunk fills 512
// blocks; the 16 partial sums are added in a fixed order, so the result does
// not depend on the launch.
// rho and grad rho of 2 kRhoPairs points per block: each thread takes two
// neighbouring points (16-byte loads; G is a multiple of 256, so the pair
// stays inside the chunk, and the padding points hold zeros) and every
// kRhoLanes-th function from ml, two functions per step; the kRhoLanes
// partial sums are added in a fixed order
constexpr int kRhoPairs = 16, kRhoLanes = 16;
__global__ void __launch_bounds__(kRhoPairs * kRhoLanes) rho_kernel(
    const double* __restrict__ X, const double* __restrict__ phi, const double* __restrict__ dphi,
    int nao, int64_t G, int64_t ng, double* __restrict__ rho, double* __restrict__ grad) {
  __shared__ double2 red[4][kRhoLanes][kRhoPairs];
  const int gi = threadIdx.x % kRhoPairs, ml = threadIdx.x / kRhoPairs;
  const int64_t g = 2 * (blockIdx.x * (int64_t)kRhoPairs + gi);
  const int64_t plane = (int64_t)nao * G;
  double2 r = {0.0, 0.0}, a = {0.0, 0.0}, b = {0.0, 0.0}, c = {0.0, 0.0};
  auto ld2 = [](const double* p) { return *reinterpret_cast<const double2*>(p); };
  auto acc = [&](int64_t o) {
    const double2 x = ld2(X + o), f = ld2(phi + o), dx = ld2(dphi + o),
                  dy = ld2(dphi + plane + o), dz = ld2(dphi + 2 * plane + o);
    r.x += x.x * f.x;
    r.y += x.y * f.y;
    a.x += x.x * dx.x;
    a.y += x.y * dx.y;
    b.x += x.x * dy.x;
    b.y += x.y * dy.y;
    c.x += x.x * dz.x;
    c.y += x.y * dz.y;
  };
  if (g < ng) {
    int mu = ml;
    for (; mu + kRhoLanes < nao; mu += 2 * kRhoLanes) {
      acc((int64_t)mu * G + g);
      acc((int64_t)(mu + kRhoLanes) * G + g);
    }
    if (mu < nao) acc((int64_t)mu * G + g);
  }
  red[0][ml][gi] = r;
  red[1][ml][gi] = a;
  red[2][ml][gi] = b;
  red[3][ml][gi] = c;
  __syncthreads();
  if (ml < 4 && g < ng) {
    double2 t = {0.0, 0.0};
#pragma unroll
    for (int q = 0; q < kRhoLanes; ++q) {
      t.x += red[ml][q][gi].x;
      t.y += red[ml][q][gi].y;
    }
    const double f = ml == 0 ? 1.0 : 2.0;
    double* out = ml == 0 ? rho : grad + (ml - 1) * G;
    out[g] = f * t.x;
    if (g + 1 < ng) out[g + 1] = f * t.y;
  }
}

// ---------------------------------------------------------------------------
// PBE by forward-mode dual numbers: value and d/d(rho, gx, gy, gz)
// ---------------------------------------------------------------------------

struct D4 {
  double v, d[4];
};
__device__ __forceinline__ D4 dc(double c) { return {c, {0.0, 0.0, 0.0, 0.0}}; }
__device__ __forceinline__ D4 operator+(D4 a, D4 b) {
  return {a.v + b.v, {a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2], a.d[3] + b.d[3]}};
}
__device__ __forceinline__ D4 operator*(D4 a, D4 b) {
  D4 r;
  r.v = a.v * b.v;
#pragma unroll
  for (int k = 0; k < 4; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
// quotient rule as (a' - (a/b) b') / b: one division
__device__ __forceinline__ D4 operator/(D4 a, D4 b) {
  D4 r;
  const double ib = 1.0 / b.v;
  r.v = a.v * ib;
#pragma unroll
  for (int k = 0; k < 4; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
  return r;
}
__device__ __forceinline__ D4 operator+(D4 a, double c) { a.v += c; return a; }
__device__ __forceinline__ D4 operator+(double c, D4 a) { a.v += c; return a; }
__device__ __forceinline__ D4 operator-(double c, D4 a) {
  return {c - a.v, {-a.d[0], -a.d[1], -a.d[2], -a.d[3]}};
}
__device__ __forceinline__ D4 operator*(D4 a, double c) {
  return {a.v * c, {a.d[0] * c, a.d[1] * c, a.d[2] * c, a.d[3] * c}};
}
__device__ __forceinline__ D4 operator*(double c, D4 a) { return a * c; }
__device__ __forceinline__ D4 operator/(D4 a, double c) { return a * (1.0 / c); }
__device__ __forceinline__ D4 operator/(double c, D4 a) { return dc(c) / a; }
__device__ __forceinline__ D4 dscale(D4 a, double f) {   // chain rule with df/dx = f
  D4 r;
#pragma unroll
  for (int k = 0; k < 4; ++k) r.d[k] = a.d[k] * f;
  return r;
}
__device__ __forceinline__ D4 dsqrt(D4 a) {
  const double q = sqrt(a.v);
  D4 r = dscale(a, 0.5 / q);
  r.v = q;
  return r;
}
// a^(1/3) for a > 0, with d/da = a^(1/3) / (3 a)
__device__ __forceinline__ D4 dcbrt(D4 a) {
  const double q = cbrt(a.v);
  D4 r = dscale(a, q / (3.0 * a.v));
  r.v = q;
  return r;
}
__device__ __forceinline__ D4 dlog1p(D4 a) {
  D4 r = dscale(a, 1.0 / (1.0 + a.v));
  r.v = log1p(a.v);
  return r;
}
__device__ __forceinline__ D4 dexpm1(D4 a) {
  const double q = expm1(a.v);
  D4 r = dscale(a, a.v > -0.5 ? q + 1.0 : exp(a.v));   // e^a = expm1(a) + 1 without cancellation
  r.v = q;
  return r;
}
// jnp.clip(x, lo): the bound itself (derivative 0) below lo
__device__ __forceinline__ D4 dclip(D4 a, double lo) { return a.v < lo ? dc(lo) : a; }

// eps_xc per particle of x_scale PBE exchange + c_scale PBE correlation,
// unpolarized (xc.py: PBEExchange._unpolarized, PBECorrelation with zeta = 0)
__device__ D4 pbe_eps(D4 rho, D4 gx, D4 gy, D4 gz, double xs, double cs) {
  constexpr double pi = 3.141592653589793;
  // exchange
  const D4 ax = gx + 1e-30, ay = gy + 1e-30, az = gz + 1e-30;
  const D4 gnorm = dsqrt(ax * ax + ay * ay + az * az);
  const D4 kF = dcbrt(3 * pi * pi * rho + 1e-30);
  const D4 s = gnorm / dclip(2 * kF * rho, 1e-30);
  const double kappa = 0.804, mu = 0.2195149727645171;
  const D4 ex_unif = -3 * kF / (4 * pi);
  const D4 fx = 1 + kappa - kappa / (1 + mu * s * s / kappa);
  const D4 ex = ex_unif * fx;
  // correlation: PW92 paramagnetic channel + PBE H with phi = 1
  const double gamma = (1.0 - 0.6931471805599453) / (pi * pi);
  const double beta = 0.06672455060314922;
  const double A = 0.0310907, a1 = 0.21370, b1 = 7.5957, b2 = 3.5876, b3 = 1.6382, b4 = 0.49294;
  const D4 rt = dclip(rho, 1e-20);
  const D4 rs = dcbrt(3 / (4 * pi * rt) + 1e-20);
  const D4 rss = dsqrt(rs);
  const D4 den = 2.0 * A * (b1 * rss + b2 * rs + b3 * rs * rss + b4 * rs * rs);
  const D4 eps_pw = -2.0 * A * (1.0 + a1 * rs) * dlog1p(1.0 / dclip(den, 1e-20));
  const D4 kf = dcbrt(3 * pi * pi * rt + 1e-20);
  const D4 ks = dsqrt(4 * kf / pi);
  const D4 gn = dsqrt(gx * gx + gy * gy + gz * gz + 1e-30);
  const D4 t = gn / dclip(2 * ks * rt, 1e-20);
  const D4 dA = gamma * dexpm1(-1.0 * eps_pw / gamma);
  const D4 Ac = beta / dclip(dA, 1e-20);
  const D4 t2 = t * t;
  const D4 f1 = t2 + Ac * (t2 * t2);
  const D4 frac = beta * f1 / dclip(gamma * (1.0 + Ac * f1), 1e-20);
  const D4 H = gamma * dlog1p(frac);
  return xs * ex + cs * (eps_pw + H);
}

// per point: rho, grad in, v_rho, v_grad out (in place); e per block
__global__ void __launch_bounds__(kPtThreads) pbe_kernel(double* __restrict__ rho,
                                                         double* __restrict__ grad,
                                                         const double* __restrict__ w, int64_t G,
                                                         int64_t ng, double xs, double cs,
                                                         double thresh, double* __restrict__ ered) {
  __shared__ double red[kPtThreads];
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double e = 0.0;
  if (g < ng) {
    const double r = rho[g];
    double vr = 0.0, v0 = 0.0, v1 = 0.0, v2 = 0.0;
    if (r > thresh) {
      const double wg = w[g];
      const D4 R = {r, {1.0, 0.0, 0.0, 0.0}};
      const D4 X = {grad[g], {0.0, 1.0, 0.0, 0.0}};
      const D4 Y = {grad[G + g], {0.0, 0.0, 1.0, 0.0}};
      const D4 Z = {grad[2 * G + g], {0.0, 0.0, 0.0, 1.0}};
      const D4 f = R * pbe_eps(R, X, Y, Z, xs, cs);
      e = wg * f.v;
      vr = wg * f.d[0];
      v0 = wg * f.d[1];
      v1 = wg * f.d[2];
      v2 = wg * f.d[3];
    }
    rho[g] = vr;
    grad[g] = v0;
    grad[G + g] = v1;
    grad[2 * G + g] = v2;
  }
  red[threadIdx.x] = e;
  __syncthreads();
  for (int o = kPtThreads / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) ered[blockIdx.x] = red[0];
}

// W[mu][g] = v_rho/2 Phi + v_grad . dPhi (zero past ng)
__global__ void w_kernel(const double* __restrict__ phi, const double* __restrict__ dphi,
                         const double* __restrict__ vr, const double* __restrict__ vg, int nao,
                         int64_t G, int64_t ng, double* __restrict__ W) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t plane = (int64_t)nao * G;
  if (i >= plane) return;
  const int64_t g = i % G;
  double v = 0.0;
  if (g < ng)
    v = 0.5 * vr[g] * phi[i] + vg[g] * dphi[i] + vg[G + g] * dphi[plane + i] +
        vg[2 * G + g] * dphi[2 * plane + i];
  W[i] = v;
}

// out = sum over the nb branch accumulators V_b (n x n, stride n*n) of
// V_b + V_b^T, in branch order
__global__ void symmetrize_sum_kernel(const double* __restrict__ V, int nb, int n,
                                      double* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t nn = (int64_t)n * n;
  if (i >= nn) return;
  const int64_t r = i / n, c = i % n;
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s += V[b * nn + i] + V[b * nn + c * n + r];
  out[i] = s;
}

}  // namespace

void launch_becke_partition(const double* pts, const int* owner, const double* raw, int64_t n,
                            const double* atom_xyz, const double* bragg, int natom, double* w,
                            cudaStream_t s) {
  if (n <= 0) return;
  // pair tables: 1 / R_AB and the size adjustment a_AB (becke.py: becke_partition)
  std::vector<double> inv((size_t)natom * natom, 0.0), aab((size_t)natom * natom, 0.0);
  for (int a = 0; a < natom; ++a)
    for (int b = 0; b < natom; ++b) {
      if (a == b) continue;
      const double dx = atom_xyz[3 * a] - atom_xyz[3 * b], dy = atom_xyz[3 * a + 1] - atom_xyz[3 * b + 1],
                   dz = atom_xyz[3 * a + 2] - atom_xyz[3 * b + 2];
      inv[(size_t)a * natom + b] = 1.0 / std::sqrt(dx * dx + dy * dy + dz * dz);
      const double chi = bragg[a] / bragg[b];
      const double u = (chi - 1.0) / (chi + 1.0);
      aab[(size_t)a * natom + b] = std::min(0.45, std::max(-0.45, u / (u * u - 1.0)));
    }
  std::vector<double> xyz(atom_xyz, atom_xyz + 3 * natom);
  DevBuf dxyz, dinv, daab;
  upload(dxyz, xyz);
  upload(dinv, inv);
  upload(daab, aab);
  int threads = 64;
  const size_t smem = (size_t)natom * threads * sizeof(double);
  if (smem > 200 * 1024) fail(DFJK_ERR_UNSUPPORTED, "Becke partition supports at most 400 atoms");
  DFJK_CUDA(cudaFuncSetAttribute(becke_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)std::max<size_t>(smem, 1)));
  becke_kernel<<<(unsigned)((n + threads - 1) / threads), threads, smem, s>>>(
      pts, owner, raw, n, dxyz.as<double>(), dinv.as<double>(), daab.as<double>(), natom, w);
  DFJK_LAUNCHED();
  DFJK_CUDA(cudaStreamSynchronize(s));   // the pair tables are freed on return
}

// interleaves the low 21 bits of x, y, z (Morton order)
static uint64_t morton3(uint64_t x, uint64_t y, uint64_t z) {
  auto spread = [](uint64_t v) {
    v &= 0x1fffffULL;
    v = (v | v << 32) & 0x1f00000000ffffULL;
    v = (v | v << 16) & 0x1f0000ff0000ffULL;
    v = (v | v << 8) & 0x100f00f00f00f00fULL;
    v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
    v = (v | v << 2) & 0x1249249249249249ULL;
    return v;
  };
  return spread(x) | spread(y) << 1 | spread(z) << 2;
}

void xc_sort(std::vector<double>& pts, std::vector<double>& w) {
  const int64_t n = (int64_t)w.size();
  if (n == 0) return;
  // contiguous index ranges, one per host thread (one thread below 64 k points)
  const int T = n < ((int64_t)1 << 16)
                    ? 1
                    : (int)std::min<unsigned>(16, std::max(1u, std::thread::hardware_concurrency()));
  auto lo_of = [&](int t) { return n * t / T; };
  // Morton order of 1-Bohr cells
  std::vector<double> los((size_t)3 * T, INFINITY);
  run_on_threads(T, [&](int t) {
    for (int64_t i = lo_of(t); i < lo_of(t + 1); ++i)
      for (int d = 0; d < 3; ++d) los[3 * t + d] = std::min(los[3 * t + d], pts[3 * i + d]);
  });
  double lo[3] = {INFINITY, INFINITY, INFINITY};
  for (int t = 0; t < T; ++t)
    for (int d = 0; d < 3; ++d) lo[d] = std::min(lo[d], los[3 * t + d]);
  std::vector<uint64_t> code(n), ktmp(n), cmaxs(T, 0);
  std::vector<int64_t> order(n), otmp(n);
  run_on_threads(T, [&](int t) {
    for (int64_t i = lo_of(t); i < lo_of(t + 1); ++i) {
      uint64_t c[3];
      for (int d = 0; d < 3; ++d) c[d] = (uint64_t)std::floor(pts[3 * i + d] - lo[d]);
      code[i] = morton3(c[0], c[1], c[2]);
      cmaxs[t] = std::max(cmaxs[t], code[i]);
      order[i] = i;
    }
  });
  const uint64_t cmax = *std::max_element(cmaxs.begin(), cmaxs.end());
  // order by (code, index): a stable LSD radix sort of the codes, 11 bits a
  // pass over the bits cmax needs. Per pass each thread counts its range;
  // the offsets run bucket by bucket and, within a bucket, thread by thread,
  // so every thread's elements land after those of lower indices (stable)
  int bits = 0;
  while (bits < 64 && (cmax >> bits) != 0) ++bits;
  constexpr int kRadixBits = 11;
  constexpr uint64_t kBuckets = (uint64_t)1 << kRadixBits, kMask = kBuckets - 1;
  std::vector<int64_t> hist((size_t)T * kBuckets);
  for (int shift = 0; shift < bits; shift += kRadixBits) {
    run_on_threads(T, [&](int t) {
      int64_t* h = hist.data() + (size_t)t * kBuckets;
      std::fill(h, h + kBuckets, 0);
      for (int64_t i = lo_of(t); i < lo_of(t + 1); ++i) h[(code[i] >> shift) & kMask]++;
    });
    int64_t run = 0;
    for (uint64_t b = 0; b < kBuckets; ++b)
      for (int t = 0; t < T; ++t) {
        int64_t& h = hist[(size_t)t * kBuckets + b];
        const int64_t c = h;
        h = run;
        run += c;
      }
    run_on_threads(T, [&](int t) {
      int64_t* h = hist.data() + (size_t)t * kBuckets;
      for (int64_t i = lo_of(t); i < lo_of(t + 1); ++i) {
        const int64_t dst = h[(code[i] >> shift) & kMask]++;
        ktmp[dst] = code[i];
        otmp[dst] = order[i];
      }
    });
    code.swap(ktmp);
    order.swap(otmp);
  }
  std::vector<double> p2(3 * n), w2(n);
  run_on_threads(T, [&](int t) {
    for (int64_t i = lo_of(t); i < lo_of(t + 1); ++i) {
      const int64_t j = order[i];
      for (int d = 0; d < 3; ++d) p2[3 * i + d] = pts[3 * j + d];
      w2[i] = w[j];
    }
  });
  pts.swap(p2);
  w.swap(w2);
}

void xc_chunk(const Shells& sh, const int (&nout)[8], const std::vector<double>& pts, int64_t G,
              double thresh, XcWork& ws) {
  XcChunks& out = ws.ch;
  const int64_t n = (int64_t)pts.size() / 3;
  out.g0.clear();
  out.ng.clear();
  out.sh_off.clear();
  out.sh_cnt.clear();
  out.ao_off.clear();
  out.ao_cnt.clear();
  out.max_ao = 0;
  out.total_ao = 0;
  out.gemm_flop = 0.0;
  out.G = G;
  if (ws.exec) cudaGraphExecDestroy(ws.exec);
  ws.exec = nullptr;
  for (auto& a : ws.g_args) a = nullptr;
  ws.calls = 0;
  if (n == 0) return;
  // per shell: |phi| + |grad phi| <= sum_k |c_k| (1 + r^l + l r^(l-1) + 2 a_k r^(l+1)) e^(-a_k r^2)
  // for r beyond the distance d from the shell to a box, the polynomial taken
  // at max(d, its peak) (it decreases past sqrt((l+1)/(2 a_k))) and the
  // Gaussian at d
  auto bound = [&](int s, double d) {
    const int l = sh.l[s];
    double b = 0.0;
    for (int k = 0; k < sh.nprim[s]; ++k) {
      const double a = sh.pexp[sh.prim0[s] + k], c = std::fabs(sh.pcoef[sh.prim0[s] + k]);
      const double r = std::max(d, std::sqrt((l + 1) / (2.0 * a)));
      const double rl = std::pow(r, l);
      b += c * (1.0 + rl + (l > 0 ? l * rl / r : 0.0) + 2.0 * a * rl * r) * std::exp(-a * d * d);
    }
    return b;
  };
  std::vector<int> shl, out0c, aomap;
  out.sh_lcnt.clear();
  for (int64_t g0 = 0; g0 < n; g0 += G) {
    const int64_t ng = std::min(G, n - g0);
    double bl[3] = {INFINITY, INFINITY, INFINITY}, bh[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = g0; i < g0 + ng; ++i)
      for (int d = 0; d < 3; ++d) {
        bl[d] = std::min(bl[d], pts[3 * i + d]);
        bh[d] = std::max(bh[d], pts[3 * i + d]);
      }
    out.g0.push_back(g0);
    out.ng.push_back(ng);
    out.sh_off.push_back((int)shl.size());
    out.ao_off.push_back((int64_t)aomap.size());
    int nao_c = 0;
    for (int s = 0; s < sh.n; ++s) {
      double d2 = 0.0;
      for (int d = 0; d < 3; ++d) {
        const double c = sh.cen[3 * s + d];
        const double e = c < bl[d] ? bl[d] - c : (c > bh[d] ? c - bh[d] : 0.0);
        d2 += e * e;
      }
      if (bound(s, std::sqrt(d2)) <= thresh) continue;
      shl.push_back(s);
      out0c.push_back(nao_c);
      const int no = nout[sh.l[s]];
      for (int m = 0; m < no; ++m) aomap.push_back(sh.out0[s] + m);
      nao_c += no;
    }
    out.sh_cnt.push_back((int)shl.size() - out.sh_off.back());
    // this chunk's shells grouped by l (stable), each keeping its compact
    // AOs: only the launch order changes, not the layout of Phi
    {
      const int j0 = out.sh_off.back(), j1 = (int)shl.size();
      std::vector<std::pair<int, int>> seg;
      int cnt[kXcMaxL + 1] = {};
      for (int j = j0; j < j1; ++j) {
        const int l = std::min<int>(sh.l[shl[j]], kXcMaxL);
        seg.push_back({shl[j], out0c[j]});
        ++cnt[l];
      }
      int pos = j0;
      for (int l = 0; l <= kXcMaxL; ++l) {
        for (const auto& e : seg)
          if (std::min<int>(sh.l[e.first], kXcMaxL) == l) {
            shl[pos] = e.first;
            out0c[pos] = e.second;
            ++pos;
          }
        out.sh_lcnt.push_back(cnt[l]);
      }
    }
    out.ao_cnt.push_back(nao_c);
    out.max_ao = std::max(out.max_ao, nao_c);
    out.total_ao += nao_c;
    out.gemm_flop += 4.0 * (double)G * nao_c * nao_c;   // X = Phi P and Phi^T W
  }
  upload(out.d_sh, shl);
  upload(out.d_sh_out0, out0c);
  upload(out.d_ao_map, aomap);
}

// enqueues one evaluation's device work on s (buffers already sized)
static void xc_enqueue(const Context& c, const OrbView& ov, const double* pts, const double* w,
                       const double* P, double* Vxc, const XcParams& xp, XcWork& ws,
                       cudaStream_t s) {
  const int nao = ov.nao;
  const int64_t nn = (int64_t)nao * nao;
  const XcChunks& ch = ws.ch;
  const int64_t G = ch.G;
  const int64_t nchunk = (int64_t)ch.g0.size();
  const int64_t nblk = (G + kPtThreads - 1) / kPtThreads;
  const double one = 1.0, zero = 0.0;
  const int nb = std::min(std::max(ws.nbr, 1), kXcBranches);
  // fork: every branch starts after the caller's prior work on s
  DFJK_CUDA(cudaEventRecord(c.xc_fork, s));
  for (int q = 0; q < nb; ++q) {
    DFJK_CUDA(cudaStreamWaitEvent(c.xc_stream[q], c.xc_fork, 0));
    DFJK_CUBLAS(cublasSetStream(c.xc_blas[q], c.xc_stream[q]));
    // (setting the stream resets the workspace: give it back each time)
    DFJK_CUBLAS(cublasSetWorkspace(c.xc_blas[q], c.xc_ws[q].p, kXcBlasWorkspace));
  }
  if (Vxc)
    for (int q = 0; q < nb; ++q)
      DFJK_CUDA(cudaMemsetAsync(ws.Vacc.as<double>() + q * nn, 0, nn * sizeof(double),
                                c.xc_stream[q]));
  for (int64_t k = 0; k < nchunk; ++k) {
    XcBranch& b = ws.br[k % nb];
    cudaStream_t bs = c.xc_stream[k % nb];
    cublasHandle_t blas = c.xc_blas[k % nb];
    double* Vacc = ws.Vacc.as<double>() + (k % nb) * nn;
    const int64_t g0 = ch.g0[k], ng = ch.ng[k];
    const int nsig = ch.ao_cnt[k], nsh = ch.sh_cnt[k];
    const int* map = ch.d_ao_map.as<int>() + ch.ao_off[k];
    if (nsig == 0) {
      DFJK_CUDA(cudaMemsetAsync(ws.ered.as<double>() + k * nblk, 0, nblk * sizeof(double), bs));
      continue;
    }
    const int64_t plane = (int64_t)nsig * G;
    // the chunk's shells are grouped by l: one launch per l present
    int j0 = ch.sh_off[k];
    for (int l = 0; l < kXcMaxL + 1; ++l) {
      const int cnt = ch.sh_lcnt[(size_t)k * (kXcMaxL + 1) + l];
      if (cnt == 0) continue;
      const dim3 grid((unsigned)((G + kAoThreads - 1) / kAoThreads), (unsigned)cnt);
      const int* shl = ch.d_sh.as<int>() + j0;
      const int* o0 = ch.d_sh_out0.as<int>() + j0;
      double* ph = b.phi.as<double>();
      double* dph = b.dphi.as<double>();
      switch (l) {
        case 0: ao_kernel<0><<<grid, kAoThreads, 0, bs>>>(ov, shl, o0, pts, g0, ng, G, nsig, ph, dph); break;
        case 1: ao_kernel<1><<<grid, kAoThreads, 0, bs>>>(ov, shl, o0, pts, g0, ng, G, nsig, ph, dph); break;
        case 2: ao_kernel<2><<<grid, kAoThreads, 0, bs>>>(ov, shl, o0, pts, g0, ng, G, nsig, ph, dph); break;
        default: ao_kernel<3><<<grid, kAoThreads, 0, bs>>>(ov, shl, o0, pts, g0, ng, G, nsig, ph, dph); break;
      }
      DFJK_LAUNCHED();
      j0 += cnt;
    }
    (void)nsh;
    gather_p_kernel<<<(unsigned)(((int64_t)nsig * nsig + 255) / 256), 256, 0, bs>>>(
        P, nao, map, nsig, b.Pc.as<double>());
    DFJK_LAUNCHED();
    // X (G x nsig, column-major: [k][g]) = Phi Pc
    DFJK_CUBLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)G, nsig, nsig, &one,
                            b.phi.as<double>(), (int)G, b.Pc.as<double>(), nsig, &zero,
                            b.X.as<double>(), (int)G));
    rho_kernel<<<(unsigned)((ng + 2 * kRhoPairs - 1) / (2 * kRhoPairs)), kRhoPairs * kRhoLanes, 0, bs>>>(
        b.X.as<double>(), b.phi.as<double>(), b.dphi.as<double>(), nsig, G, ng,
        b.vr.as<double>(), b.vg.as<double>());
    DFJK_LAUNCHED();
    pbe_kernel<<<(unsigned)nblk, kPtThreads, 0, bs>>>(b.vr.as<double>(), b.vg.as<double>(),
                                                      w + g0, G, ng, xp.x_scale, xp.c_scale,
                                                      xp.rho_thresh, ws.ered.as<double>() + k * nblk);
    DFJK_LAUNCHED();
    if (Vxc) {
      w_kernel<<<(unsigned)((plane + 255) / 256), 256, 0, bs>>>(
          b.phi.as<double>(), b.dphi.as<double>(), b.vr.as<double>(), b.vg.as<double>(), nsig,
          G, ng, b.W.as<double>());
      DFJK_LAUNCHED();
      // Vc = Phi^T W, scattered into this branch's V
      DFJK_CUBLAS(cublasDgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, nsig, nsig, (int)G, &one,
                              b.phi.as<double>(), (int)G, b.W.as<double>(), (int)G, &zero,
                              b.Vc.as<double>(), nsig));
      scatter_v_kernel<<<(unsigned)(((int64_t)nsig * nsig + 255) / 256), 256, 0, bs>>>(
          b.Vc.as<double>(), nsig, map, nao, Vacc);
      DFJK_LAUNCHED();
    }
  }
  // join: s waits for every branch
  for (int q = 0; q < nb; ++q) {
    DFJK_CUDA(cudaEventRecord(c.xc_done[q], c.xc_stream[q]));
    DFJK_CUDA(cudaStreamWaitEvent(s, c.xc_done[q], 0));
  }
  if (Vxc) {
    symmetrize_sum_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(ws.Vacc.as<double>(),
                                                                        nb, nao, Vxc);
    DFJK_LAUNCHED();
  }
}

double xc_energy_fock(const Context& c, const OrbView& ov, const double* pts, const double* w,
                      const double* P, double* Vxc, const XcParams& xp, XcWork& ws,
                      cudaStream_t s) {
  const int nao = ov.nao;
  const XcChunks& ch = ws.ch;
  const int64_t G = ch.G;
  const int64_t nchunk = (int64_t)ch.g0.size();
  const int64_t nblk = (G + kPtThreads - 1) / kPtThreads;
  const int64_t plane_max = (int64_t)std::max(ch.max_ao, 1) * G;
  const size_t sq = (size_t)std::max(ch.max_ao, 1) * std::max(ch.max_ao, 1) * sizeof(double);
  for (int q = 0; q < std::min(std::max(ws.nbr, 1), kXcBranches); ++q) {
    XcBranch& b = ws.br[q];
    b.phi.ensure(plane_max * sizeof(double));
    b.dphi.ensure(3 * plane_max * sizeof(double));
    b.X.ensure(plane_max * sizeof(double));
    b.W.ensure(plane_max * sizeof(double));
    b.Pc.ensure(sq);
    b.Vc.ensure(sq);
    b.vr.ensure(G * sizeof(double));
    b.vg.ensure(3 * G * sizeof(double));
  }
  // the context's branch streams, events and handles are made here on first
  // use, never during a capture
  Context& cx = const_cast<Context&>(c);
  for (int q = 0; q < kXcBranches; ++q) {
    if (!cx.xc_stream[q]) DFJK_CUDA(cudaStreamCreateWithFlags(&cx.xc_stream[q], cudaStreamNonBlocking));
    if (!cx.xc_done[q]) DFJK_CUDA(cudaEventCreateWithFlags(&cx.xc_done[q], cudaEventDisableTiming));
    if (!cx.xc_blas[q]) DFJK_CUBLAS(cublasCreate(&cx.xc_blas[q]));
    cx.xc_ws[q].ensure(kXcBlasWorkspace);
  }
  if (!cx.xc_fork) DFJK_CUDA(cudaEventCreateWithFlags(&cx.xc_fork, cudaEventDisableTiming));
  ws.ered.ensure((size_t)std::max<int64_t>(nchunk, 1) * nblk * sizeof(double));
  if (Vxc) ws.Vacc.ensure((size_t)std::max(ws.nbr, 1) * nao * nao * sizeof(double));
  const void* args[4] = {P, Vxc, pts, w};
  const bool same = std::equal(args, args + 4, ws.g_args);
  if (ws.exec && same) {
    DFJK_CUDA(cudaGraphLaunch(ws.exec, s));
    count_launch(ws.graph_kernels);
  } else if (!ws.graph_off && ws.calls > 0 && Vxc) {
    // capture this call's work (the buffers above are already sized, and the
    // first, direct call let cuBLAS set up its workspace outside capture)
    if (ws.exec) {
      DFJK_CUDA(cudaGraphExecDestroy(ws.exec));
      ws.exec = nullptr;
    }
    if (!ws.cap) DFJK_CUDA(cudaStreamCreateWithFlags(&ws.cap, cudaStreamNonBlocking));
    const int64_t k0 = dfjk_kernel_launches();
    cudaGraph_t graph = nullptr;
    bool ok;
    {
      // no other thread of the library synchronizes the device meanwhile
      std::lock_guard<std::recursive_mutex> cap(capture_mutex());
      ok = cudaStreamBeginCapture(ws.cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      if (ok) {
        try {
          xc_enqueue(c, ov, pts, w, P, Vxc, xp, ws, ws.cap);
        } catch (...) {
          ok = false;
        }
        const cudaError_t ec = cudaStreamEndCapture(ws.cap, &graph);
        ok = ok && ec == cudaSuccess && graph;
      }
    }
    if (ok) ok = cudaGraphInstantiate(&ws.exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    if (ok) {
      ws.graph_kernels = dfjk_kernel_launches() - k0;
      std::copy(args, args + 4, ws.g_args);
      DFJK_CUDA(cudaGraphLaunch(ws.exec, s));
    } else {
      // the same kernels, launched directly
      ws.exec = nullptr;
      ws.graph_off = true;
      xc_enqueue(c, ov, pts, w, P, Vxc, xp, ws, s);
    }
  } else {
    xc_enqueue(c, ov, pts, w, P, Vxc, xp, ws, s);
  }
  ++ws.calls;
  std::vector<double> e((size_t)nchunk * nblk);
  if (!e.empty())
    DFJK_CUDA(cudaMemcpyAsync(e.data(), ws.ered.p, e.size() * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
  DFJK_CUDA(cudaStreamSynchronize(s));
  double sum = 0.0;
  for (double v : e) sum += v;
  return sum;
}

}  // namespace dfjk

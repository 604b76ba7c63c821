// Closed-shell Kohn-Sham SCF on the device around a built DF J/K plan
// (include/dfscf.h). The reference is dftax's _scf_solve (dftax/ks/scf.py:
// 279-391) with the KS energy of dftax/ks/energy.py:700-723:
//
//   E(P) = Tr(P Hcore) + E_J + a_x E_K + E_xc + E_nn,
//   F(P) = Hcore + J(P) - a_x/2 K(P) + Vxc(P)          (sym(dE/dP), scf.py:42-46)
//
// Per iteration, on the density P_k (from aufbau orbitals, so P_k = 2 C_occ
// C_occ^T and J, K come from the plan's J/K of C_occ with weight 2):
//   err = X^T (F P S - S P F) X, |err| (scf.py:350-351);
//   Pulay DIIS over a circular buffer of m Fock and error matrices, the
//   (m+1) system with unfilled slots masked to the identity and a 1e-10 ridge
//   on the filled ones (scf.py:245-273), solved on the host;
//   optional level shift b (S - S P S / 2) (scf.py:367);
//   X^T F X diagonalized in float64 (cuSOLVER syevd), C = X C', P_{k+1} =
//   2 C_occ C_occ^T (scf.py:319-327); or, with the purification option, the
//   same aufbau projector of X^T F X by SP2 iterations (GEMMs), C_occ from a
//   projected Cholesky QR, and the eigensolver once at the end for the
//   orbitals and their energies;
//   E(P_{k+1}) and F(P_{k+1}) together; converged when |E_{k+1} - E_k| < e_tol
//   and |err_k| < d_tol (scf.py:371).
// X is the canonical orthonormalizer U s^-1/2 over the overlap eigenvalues
// above lindep (scf.py:73-90); the guess is the core Hamiltonian's aufbau
// density (guess.py:605-606) or the caller's P0.
// Matrices are column-major n x n on the device (the symmetric ones are the
// same either way); the host synchronizes a few times per iteration for
// scalars (norms, traces, the DIIS row) and the m x m DIIS solve.
#include "scf.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>

namespace dfjk {
double energy(Plan& p, const double* P, int nspin, double hf, double hf_lr, double* F,
              cudaStream_t s);
}  // namespace dfjk

struct dfscf {
  dfjk::Plan* p = nullptr;
  dfjk::Context* c = nullptr;
  int nao = 0, nocc = 0, natom = 0, nmo = 0, nshell = 0;
  dfscf_options o{};
  double e_nn = 0.0;
  int64_t npts = 0;
  dfjk::DevBuf atom_xyz, atom_z, pts, wts, out0;
  dfjk::OrbView ov{};
  dfjk::DevBuf S, T, V, H, X;
  dfjk::DevBuf P, C, eps, F, J, K, Vxc, Cocc, wocc;
  dfjk::DevBuf dF, dE, A1, A2, Fo, work, info, vec;
  dfjk::DevBuf Fx;                                   // the DIIS Fock matrix of the iteration
  dfjk::DevBuf sp_X, sp_X2, sp_Z, sp_Y, sp_Q, sp_st, sp_info, sp_work;   // purification
  bool sp_have_Q = false;      // sp_Q holds the last occupied orbitals (X^T-basis)
  int sp_steps = 16;           // projection steps the last converged density took
  dfjk::XcWork xcw;
  std::vector<double> B;   // DIIS error overlaps, m x m
  dfscf_result res{};
  bool have_orbitals = false;
  bool orbitals_current = false;   // C / eps diagonalize the Fock matrix of the last density
  bool fx_valid = false;           // Fx holds the last run's final DIIS Fock matrix
  int64_t tuned_chunk = 0;   // XC points per chunk chosen by the autotuner (0: not tuned)
};

namespace dfjk {
namespace {

__global__ void scale_cols_kernel(const double* __restrict__ U, const double* __restrict__ w, int n,
                                  int first, int nkeep, double* __restrict__ X) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= (int64_t)n * nkeep) return;
  const int64_t r = i % n, k = i / n;
  X[i] = U[(first + k) * (int64_t)n + r] / sqrt(w[first + k]);
}

__global__ void fill_upper_kernel(double* __restrict__ A, int n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= (int64_t)n * n) return;
  const int64_t r = i % n, c = i / n;   // column-major (r, c)
  if (r < c) A[i] = A[c + r * (int64_t)n];
}

// F = H + J + a K + Vxc (elementwise)
__global__ void fock_kernel(const double* __restrict__ H, const double* __restrict__ J,
                            const double* __restrict__ K, const double* __restrict__ Vxc, double a,
                            int64_t n, double* __restrict__ F) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) F[i] = H[i] + J[i] + (K ? a * K[i] : 0.0) + (Vxc ? Vxc[i] : 0.0);
}

// y += x
__global__ void add_inplace_kernel(const double* __restrict__ x, int64_t n, double* y) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) y[i] += x[i];
}

// D = B - B^T (column-major n x n)
__global__ void antisym_kernel(const double* __restrict__ Bm, int n, double* __restrict__ D) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= (int64_t)n * n) return;
  const int64_t r = i % n, c = i / n;
  D[i] = Bm[i] - Bm[c + r * (int64_t)n];
}

unsigned blocks(int64_t n) { return (unsigned)((n + 255) / 256); }

// --- density by purification (SP2) -----------------------------------------
// Second-order spectral projection (A. M. N. Niklasson, Phys. Rev. B 66,
// 155115 (2002)), trace-correcting form: X_0 maps the spectrum of the
// orthonormal-basis Fock matrix A into [0, 1] with the lowest eigenvalues
// nearest 1; each step applies x^2 or 2x - x^2, whichever brings the trace
// nearer nocc. With a gap between the nocc-th and the next eigenvalue the
// eigenvalues go to 1 (occupied) and 0 (virtual): X is then the aufbau
// projector C'_occ C'_occ^T that the eigensolver path builds.

// Gershgorin bounds of the symmetric m x m matrix A (column-major):
// out[0] <= every eigenvalue <= out[1]. One block; thread r sums rows r,
// r + 1024, ... (a warp reads 32 consecutive rows of one column at a time).
__global__ void __launch_bounds__(1024) gershgorin_kernel(const double* __restrict__ A, int m,
                                                          double* __restrict__ out) {
  __shared__ double slo[1024], shi[1024];
  double lo = INFINITY, hi = -INFINITY;
  for (int r = threadIdx.x; r < m; r += 1024) {
    double off = 0.0;
    for (int c = 0; c < m; ++c)
      if (c != r) off += fabs(A[(int64_t)c * m + r]);
    const double d = A[(int64_t)r * m + r];
    lo = fmin(lo, d - off);
    hi = fmax(hi, d + off);
  }
  slo[threadIdx.x] = lo;
  shi[threadIdx.x] = hi;
  __syncthreads();
  for (int w = 512; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      slo[threadIdx.x] = fmin(slo[threadIdx.x], slo[threadIdx.x + w]);
      shi[threadIdx.x] = fmax(shi[threadIdx.x], shi[threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = slo[0];
    out[1] = shi[0];
  }
}

// X_0 = (hi I - A) / (hi - lo) with b = {lo, hi} (zero when hi = lo, which
// then fails the trace test and falls back to the eigensolver)
__global__ void sp2_init_kernel(const double* __restrict__ A, int m, const double* __restrict__ b,
                                double* __restrict__ X) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= (int64_t)m * m) return;
  const int64_t r = i % m, c = i / m;
  const double w = b[1] - b[0];
  X[i] = w > 0.0 ? ((r == c ? b[1] : 0.0) - A[i]) / w : 0.0;
}

// One projection step from X (in) and Z = X X to Xn (out; a separate
// buffer, since every block first reads the diagonals of X and Z): the
// traces t1 = Tr X and t2 = Tr Z, reduced by every block in the same fixed
// order so all take the same branch, then Xn = sym(Z) when Tr X^2 is nearer
// nocc than Tr(2X - X^2), else 2X - sym(Z). Block 0 records {t1, t2, branch}.
constexpr int kSp2Threads = 512;
__global__ void __launch_bounds__(kSp2Threads) sp2_step_kernel(const double* __restrict__ X,
                                                              const double* __restrict__ Z, int m,
                                                              int nocc, double* __restrict__ Xn,
                                                              double* __restrict__ rec) {
  __shared__ double s1[kSp2Threads], s2[kSp2Threads];
  double a = 0.0, b = 0.0;
  for (int r = threadIdx.x; r < m; r += kSp2Threads) {
    a += X[(int64_t)r * m + r];
    b += Z[(int64_t)r * m + r];
  }
  s1[threadIdx.x] = a;
  s2[threadIdx.x] = b;
  __syncthreads();
  for (int w = kSp2Threads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s1[threadIdx.x] += s1[threadIdx.x + w];
      s2[threadIdx.x] += s2[threadIdx.x + w];
    }
    __syncthreads();
  }
  const double t1 = s1[0], t2 = s2[0], N = (double)nocc;
  const bool sq = fabs(t2 - N) < fabs(2.0 * t1 - t2 - N);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    rec[0] = t1;
    rec[1] = t2;
    rec[2] = sq ? 1.0 : 0.0;
  }
  const int64_t mm = (int64_t)m * m;
  for (int64_t i = blockIdx.x * (int64_t)kSp2Threads + threadIdx.x; i < mm;
       i += (int64_t)gridDim.x * kSp2Threads) {
    const int64_t r = i % m, c = i / m;
    const double z = 0.5 * (Z[i] + Z[c + r * (int64_t)m]);
    Xn[i] = sq ? z : 2.0 * X[i] - z;
  }
}

// deterministic start vectors in [-1, 1): splitmix64 (Steele, Lea and Flood,
// OOPSLA 2014) of the element index
__global__ void fill_hash_kernel(double* __restrict__ R, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t z = (uint64_t)i + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  R[i] = (double)(z >> 11) * 0x1.0p-52 - 1.0;
}

// adds the milliseconds of the device work enqueued on s since the last mark
struct PartTimer {
  cudaStream_t s;
  std::chrono::steady_clock::time_point t0;
  explicit PartTimer(cudaStream_t st) : s(st) { mark(); }
  void mark() {
    DFJK_CUDA(cudaStreamSynchronize(s));
    t0 = std::chrono::steady_clock::now();
  }
  void add(double& acc) {
    DFJK_CUDA(cudaStreamSynchronize(s));
    const auto t1 = std::chrono::steady_clock::now();
    acc += std::chrono::duration<double, std::milli>(t1 - t0).count();
    t0 = t1;
  }
};

double ddot(Context& c, const double* a, const double* b, int64_t n, cudaStream_t s) {
  double r = 0.0;
  DFJK_CUBLAS(cublasSetStream(c.cublas, s));
  DFJK_CUBLAS(cublasDdot(c.cublas, (int)n, a, 1, b, 1, &r));
  return r;
}

void gemm(Context& c, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k,
          double alpha, const double* A, int lda, const double* B, int ldb, double beta, double* C,
          int ldc, cudaStream_t s) {
  DFJK_CUBLAS(cublasSetStream(c.cublas, s));
  DFJK_CUBLAS(cublasDgemm(c.cublas, ta, tb, m, n, k, &alpha, A, lda, B, ldb, &beta, C, ldc));
}

// symmetric eigensolver: A (n x n, overwritten by eigenvectors), w (n)
void syevd(dfscf& f, double* A, int n, double* w, cudaStream_t s) {
  Context& c = *f.c;
  DFJK_CUSOLVER(cusolverDnSetStream(c.cusolver, s));
  int lwork = 0;
  DFJK_CUSOLVER(cusolverDnDsyevd_bufferSize(c.cusolver, CUSOLVER_EIG_MODE_VECTOR,
                                            CUBLAS_FILL_MODE_LOWER, n, A, n, w, &lwork));
  f.work.ensure((size_t)std::max(lwork, 1) * sizeof(double));
  f.info.ensure(sizeof(int));
  DFJK_CUSOLVER(cusolverDnDsyevd(c.cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, A,
                                 n, w, f.work.as<double>(), lwork, f.info.as<int>()));
  int h = 0;
  DFJK_CUDA(cudaMemcpyAsync(&h, f.info.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  DFJK_CUDA(cudaStreamSynchronize(s));
  if (h != 0) fail(DFJK_ERR_NUMERIC, "Fock / overlap eigensolver failed (info=%d)", h);
}

XcParams xc_params(const dfscf& f) {
  XcParams xp;
  xp.x_scale = f.o.x_scale;
  xp.c_scale = f.o.c_scale;
  xp.rho_thresh = f.o.rho_thresh;
  return xp;
}

bool has_xc(const dfscf& f) { return f.npts > 0 && (f.o.x_scale != 0.0 || f.o.c_scale != 0.0); }

// E(P) and F(P) into f.F; J, K through the C_occ of f.C (from_orbitals) or
// through the plan's density path for a general symmetric P
double energy_fock(dfscf& f, const double* P, bool from_orbitals, double* Fout, cudaStream_t s) {
  Context& c = *f.c;
  const int64_t n = f.nao, nn = n * n;
  const double hf = f.o.hf_coeff;
  double e_coul;
  PartTimer tm(s);
  if (from_orbitals) {
    // C_occ row-major [nao][nocc] for the plan's J/K; weight 2 per orbital
    const double one = 1.0, zero = 0.0;
    DFJK_CUBLAS(cublasSetStream(c.cublas, s));
    DFJK_CUBLAS(cublasDgeam(c.cublas, CUBLAS_OP_T, CUBLAS_OP_N, f.nocc, f.nao, &one, f.C.as<double>(),
                            f.nao, &zero, f.C.as<double>(), f.nocc, f.Cocc.as<double>(), f.nocc));
    jk_compute(*f.p, f.Cocc.as<double>(), f.wocc.as<double>(), f.nocc, f.J.as<double>(),
               hf != 0.0 ? f.K.as<double>() : nullptr, s);
    e_coul = 0.5 * ddot(c, P, f.J.as<double>(), nn, s);
    if (hf != 0.0) e_coul -= 0.25 * hf * ddot(c, P, f.K.as<double>(), nn, s);
    fock_kernel<<<blocks(nn), 256, 0, s>>>(f.H.as<double>(), f.J.as<double>(),
                                           hf != 0.0 ? f.K.as<double>() : nullptr, nullptr,
                                           -0.5 * hf, nn, Fout);
    DFJK_LAUNCHED();
  } else {
    // the plan's DFCoulomb energy and gradient (J - a_x/2 K) of any symmetric P
    e_coul = energy(*f.p, P, 1, hf, 0.0, f.J.as<double>(), s);
    fock_kernel<<<blocks(nn), 256, 0, s>>>(f.H.as<double>(), f.J.as<double>(), nullptr, nullptr,
                                           0.0, nn, Fout);
    DFJK_LAUNCHED();
  }
  tm.add(f.res.ms_jk);
  double e_xc = 0.0;
  if (has_xc(f)) {
    e_xc = xc_energy_fock(c, f.ov, f.pts.as<double>(), f.wts.as<double>(), P, f.Vxc.as<double>(),
                          xc_params(f), f.xcw, s);
    add_inplace_kernel<<<blocks(nn), 256, 0, s>>>(f.Vxc.as<double>(), nn, Fout);
    DFJK_LAUNCHED();
    tm.add(f.res.ms_xc);
  }
  const double e_one = ddot(c, P, f.H.as<double>(), nn, s);
  f.res.e_one = e_one;
  f.res.e_coul = e_coul;
  f.res.e_xc = e_xc;
  f.res.e_nn = f.e_nn;
  return e_one + e_coul + e_xc + f.e_nn;
}

// orbitals of F into f.C / f.eps and (write_P) the aufbau density into f.P
void make_density_eig(dfscf& f, const double* Fm, cudaStream_t s, bool write_P = true) {
  Context& c = *f.c;
  PartTimer tm(s);
  const int n = f.nao, m = f.nmo;
  // Fo = X^T F X
  gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, n, m, n, 1.0, Fm, n, f.X.as<double>(), n, 0.0, f.A1.as<double>(),
       n, s);
  gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, m, m, n, 1.0, f.X.as<double>(), n, f.A1.as<double>(), n, 0.0,
       f.Fo.as<double>(), m, s);
  syevd(f, f.Fo.as<double>(), m, f.eps.as<double>(), s);
  // C = X C'
  gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, n, m, m, 1.0, f.X.as<double>(), n, f.Fo.as<double>(), m, 0.0,
       f.C.as<double>(), n, s);
  if (write_P) {
    // P = 2 C_occ C_occ^T (lower by SYRK, then mirrored)
    const double two = 2.0, zero = 0.0;
    DFJK_CUBLAS(cublasSetStream(c.cublas, s));
    DFJK_CUBLAS(cublasDsyrk(c.cublas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, n, f.nocc, &two,
                            f.C.as<double>(), n, &zero, f.P.as<double>(), n));
    fill_upper_kernel<<<blocks((int64_t)n * n), 256, 0, s>>>(f.P.as<double>(), n);
    DFJK_LAUNCHED();
    ++f.res.n_eig;
  }
  tm.add(f.res.ms_diag);
  f.have_orbitals = true;
  f.orbitals_current = true;
}

constexpr int kSp2Max = 96;     // projection steps before giving up (no gap)

// The aufbau density of F by SP2 purification into f.P, with C_occ (only
// the occupied columns of f.C). Returns false, with f.P untouched, when the
// projection does not converge to a rank-nocc projector.
bool sp2_density(dfscf& f, const double* Fm, cudaStream_t s) {
  Context& c = *f.c;
  PartTimer tm(s);
  const int n = f.nao, m = f.nmo, k = f.nocc;
  const int64_t mm = (int64_t)m * m;
  gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, n, m, n, 1.0, Fm, n, f.X.as<double>(), n, 0.0, f.A1.as<double>(),
       n, s);
  gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, m, m, n, 1.0, f.X.as<double>(), n, f.A1.as<double>(), n, 0.0,
       f.Fo.as<double>(), m, s);
  double* Xb[2] = {f.sp_X.as<double>(), f.sp_X2.as<double>()};
  double* Z = f.sp_Z.as<double>();
  double* st = f.sp_st.as<double>();   // [0..1] bounds, then 3 per step
  gershgorin_kernel<<<1, 1024, 0, s>>>(f.Fo.as<double>(), m, st);
  DFJK_LAUNCHED();
  sp2_init_kernel<<<blocks(mm), 256, 0, s>>>(f.Fo.as<double>(), m, st, Xb[0]);
  DFJK_LAUNCHED();
  const unsigned grid =
      (unsigned)std::min<int64_t>((mm + 4 * kSp2Threads - 1) / (4 * kSp2Threads), 4 * 148);
  // Stop on the idempotency error e = Tr X - Tr X^2 = sum l (1 - l): below
  // m 1e-15, or once it is below 1e-9 and no longer falling (the rounding
  // floor; steps enqueued after that point keep X at the floor). The first
  // host check comes after as many steps as the last converged projection
  // took (the spectra of consecutive iterations are alike), then every 4.
  std::vector<double> hs(3 * kSp2Max);
  double e1 = INFINITY, e2 = INFINITY, t1_last = 0.0;
  bool done = false;
  int it = 0, cur = 0;
  while (it < kSp2Max && !done) {
    const int g = std::min(it == 0 ? std::max(f.sp_steps, 4) : 4, kSp2Max - it);
    for (int j = 0; j < g; ++j) {
      gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, Xb[cur], m, Xb[cur], m, 0.0, Z, m, s);
      sp2_step_kernel<<<grid, kSp2Threads, 0, s>>>(Xb[cur], Z, m, k, Xb[cur ^ 1],
                                                   st + 2 + 3 * (it + j));
      DFJK_LAUNCHED();
      cur ^= 1;
    }
    DFJK_CUDA(cudaMemcpyAsync(hs.data(), st + 2 + 3 * it, 3 * g * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
    DFJK_CUDA(cudaStreamSynchronize(s));
    bool bad = false;
    for (int j = 0; j < g && !done; ++j) {
      const double e = std::fabs(hs[3 * j] - hs[3 * j + 1]);
      t1_last = hs[3 * j];
      if (!std::isfinite(e)) {
        bad = true;
        break;
      }
      if (e < 1e-15 * m || (e < 1e-9 && e >= e2)) {
        done = true;
        f.sp_steps = it + j + 1;
      }
      e2 = e1;
      e1 = e;
    }
    if (bad) break;
    it += g;
  }
  const double* Xs = Xb[cur];
  if (!done || !(std::fabs(t1_last - k) < 1e-6)) {
    tm.add(f.res.ms_diag);
    return false;
  }
  // C'_occ: X applied to the last occupied orbitals (or to fixed
  // pseudo-random vectors), orthonormalized by Cholesky QR, twice; the second
  // pass projects out what the first left outside range(X)
  double* Y = f.sp_Y.as<double>();
  double* Q = f.sp_Q.as<double>();
  double* M = f.A2.as<double>();   // k x k
  const int64_t mk = (int64_t)m * k;
  if (!f.sp_have_Q) {
    fill_hash_kernel<<<blocks(mk), 256, 0, s>>>(Q, mk);
    DFJK_LAUNCHED();
  }
  f.sp_have_Q = false;
  const double one = 1.0, zero = 0.0, mone = -1.0;
  DFJK_CUSOLVER(cusolverDnSetStream(c.cusolver, s));
  int lwork = 0;
  DFJK_CUSOLVER(cusolverDnDpotrf_bufferSize(c.cusolver, CUBLAS_FILL_MODE_LOWER, k, M, k, &lwork));
  f.sp_work.ensure((size_t)std::max(lwork, 1) * sizeof(double));
  for (int pass = 0; pass < 2; ++pass) {
    gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, m, k, m, 1.0, Xs, m, Q, m, 0.0, Y, m, s);
    DFJK_CUBLAS(cublasSetStream(c.cublas, s));
    DFJK_CUBLAS(cublasDsyrk(c.cublas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, k, m, &one, Y, m, &zero,
                            M, k));
    DFJK_CUSOLVER(cusolverDnDpotrf(c.cusolver, CUBLAS_FILL_MODE_LOWER, k, M, k,
                                   f.sp_work.as<double>(), lwork, f.sp_info.as<int>() + pass));
    // Y <- Y L^-T, then Q = Y
    DFJK_CUBLAS(cublasDtrsm(c.cublas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T,
                            CUBLAS_DIAG_NON_UNIT, m, k, &one, M, k, Y, m));
    DFJK_CUDA(cudaMemcpyAsync(Q, Y, mk * sizeof(double), cudaMemcpyDeviceToDevice, s));
  }
  // |X Q - Q|_F: Q must lie in range(X)
  gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, m, k, m, 1.0, Xs, m, Q, m, 0.0, Y, m, s);
  DFJK_CUBLAS(cublasDaxpy(c.cublas, (int)mk, &mone, Q, 1, Y, 1));
  double res = 0.0;
  DFJK_CUBLAS(cublasDnrm2(c.cublas, (int)mk, Y, 1, &res));
  int hinfo[2] = {0, 0};
  DFJK_CUDA(cudaMemcpyAsync(hinfo, f.sp_info.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
  DFJK_CUDA(cudaStreamSynchronize(s));
  if (hinfo[0] != 0 || hinfo[1] != 0 || !(res < 1e-10 * std::sqrt((double)k))) {
    tm.add(f.res.ms_diag);
    return false;
  }
  f.sp_have_Q = true;
  // C_occ = X C'_occ (first k columns of f.C), P = 2 C_occ C_occ^T
  gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, n, k, m, 1.0, f.X.as<double>(), n, Q, m, 0.0, f.C.as<double>(),
       n, s);
  const double two = 2.0;
  DFJK_CUBLAS(cublasSetStream(c.cublas, s));
  DFJK_CUBLAS(cublasDsyrk(c.cublas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, n, k, &two,
                          f.C.as<double>(), n, &zero, f.P.as<double>(), n));
  fill_upper_kernel<<<blocks((int64_t)n * n), 256, 0, s>>>(f.P.as<double>(), n);
  DFJK_LAUNCHED();
  tm.add(f.res.ms_diag);
  f.orbitals_current = false;
  return true;
}

// the aufbau density of F into f.P with C_occ in f.C, by the configured route
void make_density(dfscf& f, const double* Fm, cudaStream_t s) {
  if (f.o.density == 1 && f.nocc < f.nmo && sp2_density(f, Fm, s)) return;
  make_density_eig(f, Fm, s);
}

// err = X^T (F P S - S P F) X into f.Fo's slot of dE; returns |err|
double commutator(dfscf& f, const double* Fm, const double* Pm, double* err, cudaStream_t s) {
  Context& c = *f.c;
  const int n = f.nao, m = f.nmo;
  gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, 1.0, Fm, n, Pm, n, 0.0, f.A1.as<double>(), n, s);
  gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, 1.0, f.A1.as<double>(), n, f.S.as<double>(), n, 0.0,
       f.A2.as<double>(), n, s);
  antisym_kernel<<<blocks((int64_t)n * n), 256, 0, s>>>(f.A2.as<double>(), n, f.A1.as<double>());
  DFJK_LAUNCHED();
  gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, n, m, n, 1.0, f.A1.as<double>(), n, f.X.as<double>(), n, 0.0,
       f.A2.as<double>(), n, s);
  gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, m, m, n, 1.0, f.X.as<double>(), n, f.A2.as<double>(), n, 0.0, err,
       m, s);
  double r = 0.0;
  DFJK_CUBLAS(cublasSetStream(c.cublas, s));
  DFJK_CUBLAS(cublasDnrm2(c.cublas, m * m, err, 1, &r));
  return r;
}

// DIIS coefficients of the filled slots (scf.py:245-273), host
std::vector<double> diis_solve(const std::vector<double>& Bm, int count, int m) {
  const int N = m + 1;
  std::vector<double> A((size_t)N * N, 0.0), rhs(N, 0.0);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) {
      const bool v = i < count && j < count;
      A[(size_t)i * N + j] = v ? Bm[(size_t)i * m + j] : (i == j ? 1.0 : 0.0);
    }
  for (int i = 0; i < count; ++i) A[(size_t)i * N + i] += 1e-10;
  for (int i = 0; i < m; ++i) {
    const double b = i < count ? -1.0 : 0.0;
    A[(size_t)i * N + m] = b;
    A[(size_t)m * N + i] = b;
  }
  rhs[m] = -1.0;
  // Gaussian elimination with partial pivoting
  std::vector<int> piv(N);
  for (int k = 0; k < N; ++k) {
    int p = k;
    for (int i = k + 1; i < N; ++i)
      if (std::fabs(A[(size_t)i * N + k]) > std::fabs(A[(size_t)p * N + k])) p = i;
    if (A[(size_t)p * N + k] == 0.0) fail(DFJK_ERR_NUMERIC, "singular DIIS system");
    if (p != k) {
      for (int j = 0; j < N; ++j) std::swap(A[(size_t)k * N + j], A[(size_t)p * N + j]);
      std::swap(rhs[k], rhs[p]);
    }
    for (int i = k + 1; i < N; ++i) {
      const double l = A[(size_t)i * N + k] / A[(size_t)k * N + k];
      if (l == 0.0) continue;
      for (int j = k; j < N; ++j) A[(size_t)i * N + j] -= l * A[(size_t)k * N + j];
      rhs[i] -= l * rhs[k];
    }
  }
  std::vector<double> x(N);
  for (int i = N - 1; i >= 0; --i) {
    double v = rhs[i];
    for (int j = i + 1; j < N; ++j) v -= A[(size_t)i * N + j] * x[j];
    x[i] = v / A[(size_t)i * N + i];
  }
  x.resize(m);
  return x;
}

void run(dfscf& f, const double* P0, cudaStream_t s) {
  Context& c = *f.c;
  const int n = f.nao, m = f.nmo, md = f.o.diis_space;
  const int64_t nn = (int64_t)n * n, mm = (int64_t)m * m;
  f.res = dfscf_result{};
  f.fx_valid = false;
  f.res.nmo = f.nmo;
  f.res.nocc = f.nocc;
  bool orbitals;
  if (P0) {
    DFJK_CUDA(cudaMemcpyAsync(f.P.p, P0, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
    orbitals = false;
  } else {
    make_density_eig(f, f.H.as<double>(), s);   // core-Hamiltonian guess
    orbitals = true;
  }
  double e_prev = energy_fock(f, f.P.as<double>(), orbitals, f.F.as<double>(), s);
  f.B.assign((size_t)md * md, 0.0);
  int it = 0;
  bool converged = false;
  double derr = INFINITY;
  while (it < f.o.max_iter && !converged) {
    PartTimer tm(s);
    const int slot = it % md;
    double* dFs = f.dF.as<double>() + slot * nn;
    double* dEs = f.dE.as<double>() + slot * mm;
    derr = commutator(f, f.F.as<double>(), f.P.as<double>(), dEs, s);
    DFJK_CUDA(cudaMemcpyAsync(dFs, f.F.p, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
    // the new row of error overlaps: B[slot][j] = <err_slot, err_j>
    const int count = std::min(it + 1, md);
    std::vector<double> row(md, 0.0);
    for (int j = 0; j < count; ++j)
      row[j] = ddot(c, dEs, f.dE.as<double>() + j * mm, mm, s);
    for (int j = 0; j < count; ++j) {
      f.B[(size_t)slot * md + j] = row[j];
      f.B[(size_t)j * md + slot] = row[j];
    }
    std::vector<double> coef = diis_solve(f.B, count, md);
    // F_ext = sum_i c_i F_i over the filled slots 0 .. count-1 only: the
    // others hold whatever the recycled buffer held, and 0 times a NaN
    // pattern is NaN
    f.vec.ensure((size_t)md * sizeof(double));
    DFJK_CUDA(cudaMemcpyAsync(f.vec.p, coef.data(), count * sizeof(double), cudaMemcpyHostToDevice,
                              s));
    {
      const double one = 1.0, zero = 0.0;
      DFJK_CUBLAS(cublasSetStream(c.cublas, s));
      DFJK_CUBLAS(cublasDgemv(c.cublas, CUBLAS_OP_N, (int)nn, count, &one, f.dF.as<double>(),
                              (int)nn, f.vec.as<double>(), 1, &zero, f.A2.as<double>(), 1));
    }
    double* Fext = f.A2.as<double>();
    if (f.o.level_shift != 0.0) {
      // F_ext + b (S - S P S / 2)
      gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, 1.0, f.S.as<double>(), n, f.P.as<double>(), n, 0.0,
           f.A1.as<double>(), n, s);
      gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, -0.5 * f.o.level_shift, f.A1.as<double>(), n,
           f.S.as<double>(), n, 1.0, Fext, n, s);
      const double b = f.o.level_shift;
      DFJK_CUBLAS(cublasDaxpy(c.cublas, (int)nn, &b, f.S.as<double>(), 1, Fext, 1));
    }
    // the DIIS Fock moves to its own buffer before make_density reuses A1/A2
    DFJK_CUDA(cudaMemcpyAsync(f.Fx.p, Fext, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
    f.fx_valid = true;
    tm.add(f.res.ms_diis);
    make_density(f, f.Fx.as<double>(), s);
    const double e = energy_fock(f, f.P.as<double>(), true, f.F.as<double>(), s);
    converged = std::fabs(e - e_prev) < f.o.e_tol && derr < f.o.d_tol;
    e_prev = e;
    ++it;
  }
  // when the last density came from the projection, the orbitals and
  // energies of the last DIIS Fock matrix are computed by the first
  // dfscf_get_orbitals (the batch engine, which reads only densities, skips it)
  f.res.e_tot = e_prev;
  f.res.derr = derr;
  f.res.xc_chunk = f.xcw.ch.G;
  f.res.xc_graph = f.xcw.exec != nullptr ? 1 : 0;
  f.res.xc_gemm_flop = has_xc(f) ? f.xcw.ch.gemm_flop : 0.0;
  f.res.n_iter = it;
  f.res.converged = converged ? 1 : 0;
}

// Points per XC chunk, chosen by timing: the chunk size sets the shapes of the
// two DGEMMs per chunk (G x nsig x nsig) and the launches per evaluation.
// Candidates 2048, 4096, 8192 and 16384 points are timed on the core-guess
// density (three evaluations each: a direct one, the graph capture, and a
// timed graph replay) for the first molecule of each (nao / 128, log2 points,
// XC streams) bucket; the choice is kept for the process, so later molecules
// of that size (solves in a batch included) use it without timing.
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, int64_t>& tuned() {
  static auto* m = new std::map<std::tuple<int, int, int>, int64_t>();
  return *m;
}

void autotune_chunk(dfscf& f, const int (&nout)[8], const std::vector<double>& pv,
                    cudaStream_t s) {
  int lg = 0;
  while ((int64_t(1) << (lg + 1)) <= f.npts) ++lg;
  const std::tuple<int, int, int> key{(f.nao + 127) / 128, lg, f.xcw.nbr};
  int64_t best = 0;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = tuned().find(key);
    if (it != tuned().end()) best = it->second;
  }
  if (best == 0) {
    make_density_eig(f, f.H.as<double>(), s);   // core-guess density to time on
    double best_ms = INFINITY;
    for (int64_t G : {2048, 4096, 8192, 16384}) {
      if ((int64_t)6 * f.nao * G * 8 > ((int64_t)3 << 30)) continue;
      // as the SCF runs it: the first call launches directly, the second
      // captures the CUDA graph, the timed ones replay it
      xc_chunk(f.p->orb, nout, pv, G, f.o.ao_thresh, f.xcw);
      for (int rep = 0; rep < 2; ++rep)
        xc_energy_fock(*f.c, f.ov, f.pts.as<double>(), f.wts.as<double>(), f.P.as<double>(),
                       f.Vxc.as<double>(), xc_params(f), f.xcw, s);
      const auto t0 = std::chrono::steady_clock::now();
      xc_energy_fock(*f.c, f.ov, f.pts.as<double>(), f.wts.as<double>(), f.P.as<double>(),
                     f.Vxc.as<double>(), xc_params(f), f.xcw, s);
      const double ms =
          std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      if (ms < best_ms) {
        best_ms = ms;
        best = G;
      }
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tuned().emplace(key, best);
  }
  f.tuned_chunk = best;
  xc_chunk(f.p->orb, nout, pv, best, f.o.ao_thresh, f.xcw);   // also a fresh graph state
}

}  // namespace
}  // namespace dfjk

using namespace dfjk;

extern "C" {

void dfscf_default_options(dfscf_options* o) {
  if (!o) return;
  *o = dfscf_options{};
  o->hf_coeff = 0.25;
  o->x_scale = 0.75;
  o->c_scale = 1.0;
  o->e_tol = 1e-8;
  o->d_tol = 1e-6;
  o->lindep = 1e-7;
  o->level_shift = 0.0;
  o->rho_thresh = 1e-10;
  o->ao_thresh = 1e-14;
  o->max_iter = 128;
  o->diis_space = 8;
  o->grid_chunk = 0;
  o->xc_streams = 0;
  o->density = 1;
}

dfjk_status dfscf_create(dfjk_plan* pl, int32_t natom, const double* atom_xyz,
                         const double* atom_charge, int64_t npoint, const double* grid_xyz,
                         const double* grid_w, int32_t nocc, const dfscf_options* opts,
                         dfscf** out, void* stream) {
  if (!pl || !out) return DFJK_ERR_INVALID;
  *out = nullptr;
  dfscf* f = new (std::nothrow) dfscf;
  if (!f) return DFJK_ERR_MEMORY;
  Context* c = pl->p.ctx;
  dfjk_status st = guard(c, [&] {
    Plan& p = pl->p;
    if (!p.built) fail(DFJK_ERR_STATE, "dfscf_create before dfjk_build");
    if (p.lr) fail(DFJK_ERR_UNSUPPORTED, "the SCF does not take range-separated plans");
    for (int l : p.orb.l)
      if (l > kXcMaxL) fail(DFJK_ERR_UNSUPPORTED, "the SCF's AO evaluation takes l <= %d (got %d)",
                            kXcMaxL, l);
    if (natom <= 0 || !atom_xyz || !atom_charge) fail(DFJK_ERR_INVALID, "no atoms");
    if (npoint < 0 || (npoint > 0 && (!grid_xyz || !grid_w))) fail(DFJK_ERR_INVALID, "bad grid");
    if (nocc <= 0 || nocc > p.nao) fail(DFJK_ERR_INVALID, "nocc=%d for nao=%d", nocc, p.nao);
    DFJK_CUDA(cudaSetDevice(c->device));
    f->p = &p;
    f->c = c;
    if (opts) f->o = *opts;
    else dfscf_default_options(&f->o);
    if (f->o.diis_space < 1 || f->o.max_iter < 0) fail(DFJK_ERR_INVALID, "invalid SCF options");
    if (f->o.xc_streams < 0 || f->o.xc_streams > kXcBranches)
      fail(DFJK_ERR_INVALID, "xc_streams must be 0..%d", kXcBranches);
    f->xcw.nbr = f->o.xc_streams > 0 ? f->o.xc_streams : kXcBranches;
    if (f->o.density != 0 && f->o.density != 1) fail(DFJK_ERR_INVALID, "density must be 0 or 1");
    for (int64_t i = 0; i < 3 * (int64_t)natom; ++i)
      if (!std::isfinite(atom_xyz[i])) fail(DFJK_ERR_NUMERIC, "non-finite atom coordinate");
    for (int64_t i = 0; i < 3 * npoint; ++i)
      if (!std::isfinite(grid_xyz[i])) fail(DFJK_ERR_NUMERIC, "non-finite grid point");
    f->nao = p.nao;
    f->nocc = nocc;
    f->natom = natom;
    f->npts = npoint;
    f->nshell = p.orb.n;

    upload(f->atom_xyz, std::vector<double>(atom_xyz, atom_xyz + 3 * natom));
    upload(f->atom_z, std::vector<double>(atom_charge, atom_charge + natom));
    if (!(f->o.ao_thresh >= 0.0)) fail(DFJK_ERR_INVALID, "ao_thresh must be >= 0");
    std::vector<double> pv, wv;
    int nout[8];
    for (int l = 0; l < 8; ++l) nout[l] = p.orb.spherical ? 2 * l + 1 : ncart(l);
    if (npoint > 0) {
      // spatially sorted chunks with their non-negligible shells
      pv.assign(grid_xyz, grid_xyz + 3 * npoint);
      wv.assign(grid_w, grid_w + npoint);
      xc_sort(pv, wv);
      const int64_t G = f->o.grid_chunk > 0 ? (f->o.grid_chunk + 255) / 256 * 256 : 8192;
      xc_chunk(p.orb, nout, pv, G, f->o.ao_thresh, f->xcw);
      upload(f->pts, pv);
      upload(f->wts, wv);
    }
    double enn = 0.0;
    for (int a = 0; a < natom; ++a)
      for (int b = 0; b < a; ++b) {
        const double dx = atom_xyz[3 * a] - atom_xyz[3 * b], dy = atom_xyz[3 * a + 1] - atom_xyz[3 * b + 1],
                     dz = atom_xyz[3 * a + 2] - atom_xyz[3 * b + 2];
        enn += atom_charge[a] * atom_charge[b] / std::sqrt(dx * dx + dy * dy + dz * dz);
      }
    f->e_nn = enn;
    // orbital shells as the AO and one-electron kernels read them
    upload(f->out0, p.orb.out0);
    OrbView& ov = f->ov;
    ov.sh = ShellView{p.orb.d_l.as<int>(), p.orb.d_nprim.as<int>(), p.orb.d_prim0.as<int>(),
                      p.orb.d_cen.as<double>(), p.orb.d_pexp.as<double>(), p.orb.d_pcoef.as<double>()};
    ov.out0 = f->out0.as<int>();
    ov.c2s = p.c2s_orb.dev.as<double>();
    for (int l = 0; l < 8; ++l) {
      ov.c2s_off[l] = p.c2s_orb.off[l];
      ov.nout[l] = p.orb.spherical ? 2 * l + 1 : ncart(l);
    }
    ov.nao = p.nao;
    const int64_t n = p.nao, nn = n * n;
    for (DevBuf* b : {&f->S, &f->T, &f->V, &f->H, &f->P, &f->F, &f->J, &f->K, &f->Vxc, &f->A1, &f->A2})
      b->alloc(nn * sizeof(double));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    launch_one_electron(*c, ov, f->nshell, p.orb.l, natom, f->atom_xyz.as<double>(),
                        f->atom_z.as<double>(), f->S.as<double>(), f->T.as<double>(),
                        f->V.as<double>(), s);
    DFJK_CUBLAS(cublasSetStream(c->cublas, s));
    const double one = 1.0;
    DFJK_CUBLAS(cublasDgeam(c->cublas, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, (int)n, &one,
                            f->T.as<double>(), (int)n, &one, f->V.as<double>(), (int)n,
                            f->H.as<double>(), (int)n));
    check_finite(p, f->H.as<double>(), nn, s, "the one-electron integrals");
    // canonical orthonormalizer X = U s^-1/2 over s > lindep
    DFJK_CUDA(cudaMemcpyAsync(f->A1.p, f->S.p, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
    DevBuf w;
    w.alloc(n * sizeof(double));
    syevd(*f, f->A1.as<double>(), (int)n, w.as<double>(), s);
    std::vector<double> hw(n);
    DFJK_CUDA(cudaMemcpyAsync(hw.data(), w.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    DFJK_CUDA(cudaStreamSynchronize(s));
    int first = 0;
    while (first < n && !(hw[first] > f->o.lindep)) ++first;
    f->nmo = (int)(n - first);
    if (f->nmo < nocc) fail(DFJK_ERR_NUMERIC, "only %d orbitals kept for %d occupied", f->nmo, nocc);
    const int64_t m = f->nmo;
    f->X.alloc(n * m * sizeof(double));
    scale_cols_kernel<<<blocks(n * m), 256, 0, s>>>(f->A1.as<double>(), w.as<double>(), (int)n,
                                                    first, (int)m, f->X.as<double>());
    DFJK_LAUNCHED();
    f->C.alloc(n * m * sizeof(double));
    f->eps.alloc(m * sizeof(double));
    f->Fo.alloc(m * m * sizeof(double));
    f->Cocc.alloc(n * nocc * sizeof(double));
    f->Fx.alloc(nn * sizeof(double));
    if (f->o.density == 1) {
      f->sp_X.alloc(m * m * sizeof(double));
      f->sp_X2.alloc(m * m * sizeof(double));
      f->sp_Z.alloc(m * m * sizeof(double));
      f->sp_Y.alloc(m * nocc * sizeof(double));
      f->sp_Q.alloc(m * nocc * sizeof(double));
      f->sp_st.alloc((2 + 3 * kSp2Max) * sizeof(double));
      f->sp_info.alloc(2 * sizeof(int));
    }
    upload(f->wocc, std::vector<double>(nocc, 2.0));
    f->dF.alloc((size_t)f->o.diis_space * nn * sizeof(double));
    f->dE.alloc((size_t)f->o.diis_space * m * m * sizeof(double));
    DFJK_CUDA(cudaMemsetAsync(f->dE.p, 0, (size_t)f->o.diis_space * m * m * sizeof(double), s));
    DFJK_CUDA(cudaMemsetAsync(f->dF.p, 0, (size_t)f->o.diis_space * nn * sizeof(double), s));
    if (npoint > 0 && f->o.grid_chunk <= 0 && has_xc(*f)) autotune_chunk(*f, nout, pv, s);
    DFJK_CUDA(cudaStreamSynchronize(s));
  });
  if (st != DFJK_OK) {
    delete f;
    return st;
  }
  *out = f;
  return DFJK_OK;
}

dfjk_status dfscf_destroy(dfscf* f) {
  if (!f) return DFJK_OK;
  cudaSetDevice(f->c->device);
  // no device synchronization: the buffers go back to the library's cache,
  // which synchronizes before it hands one out again unless the device has
  // been synchronized since (solves on other streams keep running)
  delete f;
  return DFJK_OK;
}

dfjk_status dfscf_run(dfscf* f, const double* P0, const dfscf_options* ro, void* stream) {
  if (!f) return DFJK_ERR_INVALID;
  return guard(f->c, [&] {
    if (ro) {
      if (ro->max_iter < 0) fail(DFJK_ERR_INVALID, "max_iter=%d", ro->max_iter);
      f->o.max_iter = ro->max_iter;
      f->o.e_tol = ro->e_tol;
      f->o.d_tol = ro->d_tol;
      f->o.level_shift = ro->level_shift;
    }
    DFJK_CUDA(cudaSetDevice(f->c->device));
    run(*f, P0, static_cast<cudaStream_t>(stream));
  });
}

dfjk_status dfscf_get_result(const dfscf* f, dfscf_result* r) {
  if (!f || !r) return DFJK_ERR_INVALID;
  *r = f->res;
  return DFJK_OK;
}

dfjk_status dfscf_get_density(dfscf* f, double* P, void* stream) {
  if (!f) return DFJK_ERR_INVALID;
  return guard(f->c, [&] {
    if (P)
      DFJK_CUDA(cudaMemcpyAsync(P, f->P.p, (size_t)f->nao * f->nao * sizeof(double),
                                cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream)));
  });
}

dfjk_status dfscf_get_orbitals(dfscf* f, double* eps, double* C, void* stream) {
  if (!f) return DFJK_ERR_INVALID;
  return guard(f->c, [&] {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!f->orbitals_current && f->fx_valid) {
      // the last density came from the projection: diagonalize that run's
      // last DIIS Fock matrix now (the density stays; the run's timings too)
      DFJK_CUDA(cudaSetDevice(f->c->device));
      const double ms = f->res.ms_diag;
      make_density_eig(*f, f->Fx.as<double>(), s, false);
      f->res.ms_diag = ms;
    }
    if (!f->have_orbitals) fail(DFJK_ERR_STATE, "no orbitals before dfscf_run");
    if (eps)
      DFJK_CUDA(cudaMemcpyAsync(eps, f->eps.p, (size_t)f->nmo * sizeof(double),
                                cudaMemcpyDeviceToDevice, s));
    if (C)
      DFJK_CUDA(cudaMemcpyAsync(C, f->C.p, (size_t)f->nao * f->nmo * sizeof(double),
                                cudaMemcpyDeviceToDevice, s));
  });
}

dfjk_status dfscf_one_electron(dfscf* f, double* S, double* T, double* V, void* stream) {
  if (!f) return DFJK_ERR_INVALID;
  return guard(f->c, [&] {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t b = (size_t)f->nao * f->nao * sizeof(double);
    if (S) DFJK_CUDA(cudaMemcpyAsync(S, f->S.p, b, cudaMemcpyDeviceToDevice, s));
    if (T) DFJK_CUDA(cudaMemcpyAsync(T, f->T.p, b, cudaMemcpyDeviceToDevice, s));
    if (V) DFJK_CUDA(cudaMemcpyAsync(V, f->V.p, b, cudaMemcpyDeviceToDevice, s));
  });
}

dfjk_status dfscf_xc(dfscf* f, const double* P, double* exc, double* Vxc, void* stream) {
  if (!f || !P || !exc) return DFJK_ERR_INVALID;
  return guard(f->c, [&] {
    DFJK_CUDA(cudaSetDevice(f->c->device));
    if (!has_xc(*f)) {
      *exc = 0.0;
      if (Vxc)
        DFJK_CUDA(cudaMemsetAsync(Vxc, 0, (size_t)f->nao * f->nao * sizeof(double),
                                  static_cast<cudaStream_t>(stream)));
      return;
    }
    *exc = xc_energy_fock(*f->c, f->ov, f->pts.as<double>(), f->wts.as<double>(), P, Vxc,
                          xc_params(*f), f->xcw, static_cast<cudaStream_t>(stream));
  });
}

dfjk_status dfscf_energy_fock(dfscf* f, const double* P, double* e, double* F, void* stream) {
  if (!f || !P || !e) return DFJK_ERR_INVALID;
  return guard(f->c, [&] {
    DFJK_CUDA(cudaSetDevice(f->c->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    *e = energy_fock(*f, P, false, F ? F : f->A2.as<double>(), s);
    DFJK_CUDA(cudaStreamSynchronize(s));
  });
}

dfjk_status dfjk_becke_partition(dfjk_ctx* h, const double* pts, const int32_t* owner,
                                 const double* raw, int64_t n, int32_t natom,
                                 const double* atom_xyz, const double* bragg, double* w,
                                 void* stream) {
  if (!h) return DFJK_ERR_INVALID;
  return guard(&h->c, [&] {
    if (n < 0 || natom <= 0 || !atom_xyz || !bragg) fail(DFJK_ERR_INVALID, "bad partition input");
    if (n > 0 && (!pts || !owner || !raw || !w)) fail(DFJK_ERR_INVALID, "null grid array");
    DFJK_CUDA(cudaSetDevice(h->c.device));
    launch_becke_partition(pts, owner, raw, n, atom_xyz, bragg, natom, w,
                           static_cast<cudaStream_t>(stream));
  });
}

}  // extern "C"

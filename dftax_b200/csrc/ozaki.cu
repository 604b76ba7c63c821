// Mixed precision (precision = DFJK_MIXED): the three large products of the DF
// path on the int8 tensor cores with exact accumulation (ozaki_gemm.cu):
//   B[r][x] = sum_P (ij|P)[r][P] L[P][x]      (build, per raw row chunk)
//   X[m][x][i] = sum_n B_x[m][n] C'[n][i]     (K half transform, per call)
//   K[m][n] = sum_(x,i) X[m][x][i] X[n][x][i]  (K accumulation, per call)
// Both operands of each product are split into signed int8 digits (a 7-bit
// leading digit, then balanced 8-bit digits) under a per-row exponent;
// outputs are float64. The integrals, the metric, its factor L, the stored B
// and J stay float64.
//
// Accuracy findings behind the digit counts (device runs on water clusters,
// against the float64 path of the same plan):
//   * storing the 3-center tensor or B in float32 moves E_J by 1.3 uHa already
//     for (H2O)_4 (oracle simulation);
//   * split-bf16 products accumulated in fp32 on the tensor cores bias K
//     toward zero (relative -3e-6 with one 64-deep k tile per partial, -2.7e-4
//     with long partials; E off by 76 uHa .. 5.9 mHa for (H2O)_32);
//   * int8 digits with int32 accumulation are exact: what is left is the
//     digit truncation, 2^-(8D) of 2^e (at most 2^(2-8D) of the row maximum)
//     for D digits;
//   * the half transform B_x C is well conditioned: 4 digits keep K within
//     1e-9 relative for (H2O)_32;
//   * the build product (ij|P) L is not: the columns of L for small metric
//     eigenvalues cancel the smooth part of each (ij|P) row, which amplifies
//     the truncation by up to the metric's condition number. With four 7-bit
//     digits (2^-29), E moved by 1.5e-5 Ha for (H2O)_8 and 1.0e-4 Ha for
//     (H2O)_32; the build uses 5 digits (2^-40): 4e-8 Ha for (H2O)_32;
//   * K = X X^T sums nfit * nocc products per element, with strong
//     cancellation off the diagonal: with four 7-bit digits E moved by 3.1e-6
//     Ha for (H2O)_32, so it uses 5 digits (2^-40).
#include "ozaki.h"

#include <algorithm>
#include <cmath>

namespace dfjk {

namespace {

__device__ __forceinline__ int row_exponent(double vmax) {
  // |value| * 2^-e < 1/2 for every value of the row
  return vmax > 0.0 ? ilogb(vmax) + 2 : 0;
}

// ND signed digits of t = v 2^-e (|t| < 1/2): a 7-bit leading digit, then
// balanced 8-bit digits,
//   t = d_0 2^-7 + sum_(s>=1) d_s 2^-(7+8s) + r,   |r| <= 2^-(8 ND),
// with |d_0| <= 65 and -128 <= d_s <= 127. They are the balanced base-256
// digits of the integer N = rint(t 2^(7+8(ND-1))) (half to even, |N| < 2^39).
// N comes from adding 1.5 * 2^52 to the exactly scaled value (the sum's
// mantissa then holds N), with no float64 <-> int conversion; adding 128 to
// every byte of N below the top digit turns each of those bytes into its
// digit + 128, so the digits are read off with byte operations.
// With 7 digits N reaches 2^54, past the 2^51 where adding 1.5 * 2^52
// rounds correctly: there the exactly scaled value is converted to an integer
// with round-half-even (cvt.rni.s64.f64), which is exact below 2^63.
template <int ND>
__device__ __forceinline__ long long digit_biased(double v, int e) {
  constexpr double kRound = 6755399441055744.0;   // 1.5 * 2^52
  long long bias = 0;
#pragma unroll
  for (int s = 0; s < ND - 1; ++s) bias |= 128LL << (8 * s);
  // v 2^sh: a power-of-two multiply while that power is a normal double
  const int sh = 7 + 8 * (ND - 1) - e;
  const double t = (sh >= -1022 && sh <= 1023)
                       ? v * __longlong_as_double((long long)(sh + 1023) << 52)
                       : ldexp(v, sh);
  if constexpr (7 + 8 * (ND - 1) > 51) return __double2ll_rn(t) + bias;
  return __double_as_longlong(t + kRound) - __double_as_longlong(kRound) + bias;
}

template <int ND>
__device__ __forceinline__ void digits(double v, int e, int8_t* d) {
  const long long m = digit_biased<ND>(v, e);
#pragma unroll
  for (int s = 1; s < ND; ++s) d[s] = (int8_t)(((m >> (8 * (ND - 1 - s))) & 0xFF) ^ 0x80);
  d[0] = (int8_t)(m >> (8 * (ND - 1)));
}

// the four digits of digits<4> packed into a word, d_0 in the low byte
__device__ __forceinline__ uint32_t digits4_word(double v, int e) {
  const uint32_t m = (uint32_t)digit_biased<4>(v, e) ^ 0x808080u;   // bytes d_3 d_2 d_1 d_0
  return __byte_perm(m, 0, 0x0123);
}

// Digit planes of the square B_x: A[d][x][m][nao_p] (4 digits) with row
// exponents ea[x][m], for XB fitted directions and one AO m per block. Row m
// of B_x is gathered through m's list of (row of B, n) entries (both
// triangles, screened pairs absent); pass 1 takes the row maxima, pass 2
// (re-reading the same rows, now in L2) packs the four digits of each value
// into one 32-bit word of a shared-memory row per direction, and the rows go
// out as one 32-bit word of 4 consecutive n per digit plane (a 4 x 4 byte
// transpose). Loads are issued kU at a time per thread so the gathers overlap.
// (Holding the values in registers between the passes, with 1024-thread
// blocks, was measured 1.5x slower: the per-block setup then dominates.)
template <int XB>
__global__ void __launch_bounds__(256) kplanes_kernel(const double* __restrict__ B, int64_t ldb,
                                                      const int* __restrict__ kptr,
                                                      const int* __restrict__ krow,
                                                      const int* __restrict__ kn, int nao,
                                                      int64_t nao_p, int64_t nfit,
                                                      int* __restrict__ ea, int64_t plane,
                                                      int8_t* __restrict__ out) {
  constexpr int G = 256 / XB;   // list entries in flight per block
  constexpr int kU = 8;
  // [XB][W] words, W = nao_p + 4: rows stay 16-byte aligned and start 4 banks apart
  extern __shared__ __align__(16) uint32_t sw[];
  __shared__ double red[G][XB];
  __shared__ int sh_e[XB];
  const int64_t W = nao_p + 4;
  const int m = blockIdx.x;
  const int64_t x0 = (int64_t)blockIdx.y * XB;
  const int lx = threadIdx.x % XB, g = threadIdx.x / XB;
  const int64_t x = x0 + lx;
  const bool xin = x < nfit;
  const int e0 = kptr[m], e1 = kptr[m + 1];
  double mx = 0.0;
  if (xin) {
    int e = e0 + g;
    for (; e + (kU - 1) * G < e1; e += kU * G) {
      int r[kU];
      double v[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) r[u] = krow[e + u * G];
#pragma unroll
      for (int u = 0; u < kU; ++u) v[u] = B[(int64_t)r[u] * ldb + x];
#pragma unroll
      for (int u = 0; u < kU; ++u) mx = fmax(mx, fabs(v[u]));
    }
    for (; e < e1; e += G) mx = fmax(mx, fabs(B[(int64_t)krow[e] * ldb + x]));
  }
  red[g][lx] = mx;
  // zero the staging rows (screened n and the padding stay zero)
  const int64_t nvec = XB * W / 4;
  for (int64_t q = threadIdx.x; q < nvec; q += 256) reinterpret_cast<uint4*>(sw)[q] = make_uint4(0, 0, 0, 0);
  __syncthreads();
  if (threadIdx.x < XB) {
    double v = 0.0;
    for (int j = 0; j < G; ++j) v = fmax(v, red[j][threadIdx.x]);
    const int ex = row_exponent(v);
    sh_e[threadIdx.x] = ex;
    if (x0 + threadIdx.x < nfit) ea[(x0 + threadIdx.x) * nao + m] = ex;
  }
  __syncthreads();
  const int ex = sh_e[lx];
  auto pack = [&](double v) { return digits4_word(v, ex); };
  if (xin) {
    uint32_t* row = sw + lx * W;
    int e = e0 + g;
    for (; e + (kU - 1) * G < e1; e += kU * G) {
      int r[kU], n[kU];
      double v[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        r[u] = krow[e + u * G];
        n[u] = kn[e + u * G];
      }
#pragma unroll
      for (int u = 0; u < kU; ++u) v[u] = B[(int64_t)r[u] * ldb + x];
#pragma unroll
      for (int u = 0; u < kU; ++u) row[n[u]] = pack(v[u]);
    }
    for (; e < e1; e += G) row[kn[e]] = pack(B[(int64_t)krow[e] * ldb + x]);
  }
  __syncthreads();
  const int64_t nq = nao_p / 4;   // groups of 4 n per row
  for (int64_t q = threadIdx.x; q < XB * nq; q += 256) {
    const int j = (int)(q / nq);
    const int64_t c = q % nq;
    if (x0 + j >= nfit) continue;
    const uint4 w = *reinterpret_cast<const uint4*>(sw + j * W + 4 * c);
    // byte d of the 4 words -> word of plane d
    const uint32_t lo01 = __byte_perm(w.x, w.y, 0x5140), hi01 = __byte_perm(w.x, w.y, 0x7362);
    const uint32_t lo23 = __byte_perm(w.z, w.w, 0x5140), hi23 = __byte_perm(w.z, w.w, 0x7362);
    const uint32_t dw[4] = {__byte_perm(lo01, lo23, 0x5410), __byte_perm(lo01, lo23, 0x7632),
                            __byte_perm(hi01, hi23, 0x5410), __byte_perm(hi01, hi23, 0x7632)};
    const int64_t o = ((x0 + j) * nao + m) * nao_p;
#pragma unroll
    for (int d = 0; d < 4; ++d) reinterpret_cast<uint32_t*>(out + d * plane + o)[c] = dw[d];
  }
}

// Digit planes of row-major rows with a per-row exponent: planes[d][row][kp]
// (k < ncols from src[row * ld + k], zero up to kp), e_out[row]. One block per row.
template <int ND>
__global__ void __launch_bounds__(256) split_rows_kernel(const double* __restrict__ src, int64_t ld,
                                                         int64_t ncols, int64_t kp,
                                                         int* __restrict__ e_out,
                                                         int64_t plane_stride,
                                                         int8_t* __restrict__ planes,
                                                         int* __restrict__ nonfinite) {
  __shared__ double red[256];
  const int64_t row = blockIdx.x;
  const double* r = src + row * ld;
  double mx = 0.0;
  bool bad = false;
  for (int64_t k = threadIdx.x; k < ncols; k += 256) {
    const double v = r[k];
    bad |= !isfinite(v);
    mx = fmax(mx, fabs(v));
  }
  red[threadIdx.x] = mx;
  // digits of a NaN or infinity would be finite and wrong: the caller is told
  if (__syncthreads_or(bad) && threadIdx.x == 0 && nonfinite) atomicExch(nonfinite, 1);
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  const int e = row_exponent(red[0]);
  if (threadIdx.x == 0) e_out[row] = e;
  int8_t* dst = planes + row * kp;
  for (int64_t k = threadIdx.x; k < kp; k += 256) {
    int8_t d[ND] = {};
    if (k < ncols) digits<ND>(r[k], e, d);
#pragma unroll
    for (int s = 0; s < ND; ++s) dst[s * plane_stride + k] = d[s];
  }
}

// ND-digit planes of k slices of a row-major matrix X (nrows x kt, ld kt):
// planes[d][z][row][ks] for slice z = blockIdx.y (zero past kt), one exponent
// per (slice, row): e_out[z * nrows + row]. One block per (row, slice).
template <int ND>
__global__ void __launch_bounds__(256) split_slices_kernel(const double* __restrict__ X, int64_t kt,
                                                           int64_t nrows, int64_t ks,
                                                           int* __restrict__ e_out, int64_t plane,
                                                           int8_t* __restrict__ planes) {
  __shared__ double red[256];
  const int64_t row = blockIdx.x, z = blockIdx.y;
  const int64_t k0 = z * ks;
  const int64_t nk = kt - k0 < ks ? kt - k0 : ks;
  const double* r = X + row * kt + k0;
  double mx = 0.0;
  for (int64_t k = threadIdx.x; k < nk; k += 256) mx = fmax(mx, fabs(r[k]));
  red[threadIdx.x] = mx;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  const int e = row_exponent(red[0]);
  if (threadIdx.x == 0) e_out[z * nrows + row] = e;
  int8_t* dst = planes + (z * nrows + row) * ks;
  for (int64_t k = threadIdx.x; k < ks; k += 256) {
    int8_t d[ND] = {};
    if (k < nk) digits<ND>(r[k], e, d);
#pragma unroll
    for (int s = 0; s < ND; ++s) dst[s * plane + k] = d[s];
  }
}

// K[i] = (beta0 ? 0 : K[i]) + sign * sum_z part[z][i], z in a fixed order
// K[m][j] = sign * sum_z part[z][m][j] (or += with beta0 = 0) for j <= m, in
// slice order, mirrored to K[j][m]: the slice products computed only the
// tiles that reach the lower triangle, and K comes out exactly symmetric
__global__ void reduce_slices_kernel(const double* __restrict__ part, int64_t nslice, int64_t nao,
                                     double sign, int beta0, double* __restrict__ K) {
  const int64_t n = nao * nao;
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t m = i / nao, j = i % nao;
  if (j > m) return;
  double acc = 0.0;
  for (int64_t z = 0; z < nslice; ++z) acc += part[z * n + i];
  const int64_t t = j * nao + m;
  K[i] = beta0 ? sign * acc : K[i] + sign * acc;
  if (t != i) K[t] = beta0 ? sign * acc : K[t] + sign * acc;
}

// 4-digit planes of C'^T: Ct[d][i][n] from Cp[n][i] (nao x nsel), exponents eb[i]
__global__ void __launch_bounds__(256) c_digits_kernel(const double* __restrict__ Cp, int nao,
                                                       int64_t nsel, int64_t nao_p,
                                                       int* __restrict__ eb,
                                                       int8_t* __restrict__ out) {
  __shared__ double red[256];
  const int64_t i = blockIdx.x;
  double mx = 0.0;
  for (int n = threadIdx.x; n < nao; n += blockDim.x) mx = fmax(mx, fabs(Cp[(int64_t)n * nsel + i]));
  red[threadIdx.x] = mx;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  const int e = row_exponent(red[0]);
  if (threadIdx.x == 0) eb[i] = e;
  const int64_t plane = nsel * nao_p;
  for (int64_t n = threadIdx.x; n < nao_p; n += blockDim.x) {
    int8_t d[4] = {0, 0, 0, 0};
    if (n < nao) digits<4>(Cp[n * nsel + i], e, d);
#pragma unroll
    for (int s = 0; s < 4; ++s) out[s * plane + i * nao_p + n] = d[s];
  }
}

void check_oz_err(Plan& p, cudaStream_t s) {
  int h = 0;
  DFJK_CUDA(cudaMemcpyAsync(&h, p.ws_oz_err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  DFJK_CUDA(cudaStreamSynchronize(s));
  if (h) fail(DFJK_ERR_CUDA, "tensor-core pipeline gave up waiting (code %d)", h);
}

}  // namespace

template <int XB>
static void launch_kplanes(Plan& p, int64_t plane, cudaStream_t s) {
  const size_t smem = (size_t)4 * XB * (p.nao_p16 + 4);
  DFJK_CUDA(cudaFuncSetAttribute(kplanes_kernel<XB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  const int64_t nxb = (p.nfit + XB - 1) / XB;
  for (int64_t b0 = 0; b0 < nxb; b0 += 65535) {
    const int64_t nb = std::min<int64_t>(65535, nxb - b0);
    const int64_t x0 = b0 * XB;
    dim3 grid((unsigned)p.nao, (unsigned)nb);
    kplanes_kernel<XB><<<grid, 256, smem, s>>>(
        p.d_B.as<double>() + x0, p.ldb, p.d_kptr.as<int>(), p.d_krow.as<int>(), p.d_kn.as<int>(),
        p.nao, p.nao_p16, p.nfit - x0, p.d_oz_ea.as<int>() + x0 * p.nao, plane,
        p.d_oz_a.as<int8_t>() + x0 * p.nao * p.nao_p16);
    DFJK_LAUNCHED();
  }
}

void build_ozaki_planes(Plan& p, cudaStream_t s) {
  p.nao_p16 = (p.nao + 15) / 16 * 16;
  const int64_t nfit = p.nfit, nao = p.nao;
  const int64_t plane = nfit * nao * p.nao_p16;
  p.d_oz_a.ensure((size_t)kOzKDigits * plane);
  p.d_oz_ea.ensure((size_t)nfit * nao * sizeof(int));
  // 16 directions per block while the staging rows fit in 160 KB of shared memory
  if ((size_t)4 * 16 * (p.nao_p16 + 4) <= (size_t)160 << 10) launch_kplanes<16>(p, plane, s);
  else if ((size_t)4 * 4 * (p.nao_p16 + 4) <= (size_t)200 << 10) launch_kplanes<4>(p, plane, s);
  else fail(DFJK_ERR_UNSUPPORTED, "mixed precision supports nao <= 12800");
}

// split_rows_kernel with the build product's digit count of the plan
static void split_rows(const Plan& p, unsigned nrow, const double* src, int64_t ld, int64_t ncols,
                       int64_t kp, int* e, int64_t plane, int8_t* planes, int* flag,
                       cudaStream_t s) {
  if (build_digits(p) == kOzB64Digits)
    split_rows_kernel<kOzB64Digits><<<nrow, 256, 0, s>>>(src, ld, ncols, kp, e, plane, planes, flag);
  else
    split_rows_kernel<kOzBDigits><<<nrow, 256, 0, s>>>(src, ld, ncols, kp, e, plane, planes, flag);
  DFJK_LAUNCHED();
}

void ozaki_prepare_l(Plan& p, cudaStream_t s) {
  p.naux_p16 = (p.naux + 15) / 16 * 16;
  const int64_t plane = p.ldb * p.naux_p16;
  p.ws_oz_l.ensure((size_t)build_digits(p) * plane);
  p.ws_oz_el.ensure((size_t)p.ldb * sizeof(int));
  // L is column-major naux x ldb: column x (contiguous over P) is row x of L^T
  // one flag for every digit split of this build (L and the raw rows),
  // read with the pipeline's error flag by ozaki_check at the end
  p.ws_flag.ensure(sizeof(int));
  DFJK_CUDA(cudaMemsetAsync(p.ws_flag.p, 0, sizeof(int), s));
  split_rows(p, (unsigned)p.ldb, p.d_L.as<double>(), p.naux, p.naux, p.naux_p16,
             p.ws_oz_el.as<int>(), plane, p.ws_oz_l.as<int8_t>(), p.ws_flag.as<int>(), s);
  p.ws_oz_err.ensure(sizeof(int));
  DFJK_CUDA(cudaMemsetAsync(p.ws_oz_err.p, 0, sizeof(int), s));
}

void ozaki_check(Plan& p, cudaStream_t s) {
  int h[2] = {0, 0};
  DFJK_CUDA(cudaMemcpyAsync(&h[0], p.ws_oz_err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  DFJK_CUDA(cudaMemcpyAsync(&h[1], p.ws_flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  DFJK_CUDA(cudaStreamSynchronize(s));
  if (h[0]) fail(DFJK_ERR_CUDA, "tensor-core pipeline gave up waiting (code %d)", h[0]);
  if (h[1]) fail(DFJK_ERR_NUMERIC, "non-finite values in the 3-center integrals or the metric factor");
}

// Digit planes of nr raw 3-center rows (ld naux): planes[d * plane_stride +
// row * naux_p16 + k], row exponents e[row]
void ozaki_split_raw(Plan& p, const double* raw, int64_t nr, int8_t* planes, int64_t plane_stride,
                     int* e, cudaStream_t s) {
  if (nr <= 0) return;
  p.naux_p16 = (p.naux + 15) / 16 * 16;
  split_rows(p, (unsigned)nr, raw, p.naux, p.naux, p.naux_p16, e, plane_stride, planes,
             p.ws_flag.as<int>(), s);
}

// Bout[r][x] (ld ldb) = sum_P raw[r][P] L[P][x] for nr rows given as digit
// planes (layout of ozaki_split_raw) and their row exponents
void ozaki_bgemm(Plan& p, const int8_t* planes, int64_t plane_stride, const int* e, int64_t nr,
                 double* Bout, cudaStream_t s) {
  if (nr <= 0) return;
  const int ND = build_digits(p);
  const OzakiShape shape = ND == kOzB64Digits ? kOzBuild64 : kOzBuild;
  const OzakiShapeInfo sh = ozaki_shape(shape);
  if (sh.digits != ND) fail(DFJK_ERR_INVALID, "build product: digit count of the shape");
  const int bk = sh.box_k;
  const int64_t kp = p.naux_p16;
  OzakiMaps maps;
  const int64_t lplane = p.ldb * kp;
  for (int d = 0; d < ND; ++d)
    ozaki_map(&maps.b[d], p.ws_oz_l.as<int8_t>() + d * lplane, p.naux, p.ldb, 1, kp, lplane, bk,
              sh.box_b);
  OzakiArgs a{};
  a.N = (int)p.ldb;
  a.ktiles = (int)((p.naux + bk - 1) / bk);
  a.plane0 = 0;
  a.ea_stride = 0;
  a.eb = p.ws_oz_el.as<int>();
  a.ld_out = p.ldb;
  a.batch_stride_out = 0;
  a.err = p.ws_oz_err.as<int>();
  // row blocks of at most 65535 pairs of 128-row tiles (grid y)
  const int64_t step = (int64_t)65535 * 256;
  for (int64_t m0 = 0; m0 < nr; m0 += step) {
    const int64_t mr = std::min(step, nr - m0);
    ozaki_map_out(&maps.out, Bout + m0 * p.ldb, p.ldb, 1, mr, p.ldb, p.ldb);
    for (int d = 0; d < ND; ++d)
      ozaki_map(&maps.a[d], planes + d * plane_stride + m0 * kp, p.naux, mr, 1, kp, plane_stride,
                bk, 128);
    a.M = (int)mr;
    a.ea = e + m0;
    a.out = Bout + m0 * p.ldb;
    ozaki_launch(shape, maps, a, 1, s);
  }
  // checked once per build (ozaki_check)
}

void ozaki_prepare_c(Plan& p, const double* Cp, int64_t nsel, cudaStream_t s) {
  p.ws_oz_c.ensure((size_t)kOzKDigits * nsel * p.nao_p16);
  p.ws_oz_eb.ensure((size_t)nsel * sizeof(int));
  c_digits_kernel<<<(unsigned)nsel, 256, 0, s>>>(Cp, p.nao, nsel, p.nao_p16, p.ws_oz_eb.as<int>(),
                                                 p.ws_oz_c.as<int8_t>());
  DFJK_LAUNCHED();
  p.ws_oz_err.ensure(sizeof(int));
  DFJK_CUDA(cudaMemsetAsync(p.ws_oz_err.p, 0, sizeof(int), s));
}

// X[m][x - x0][i] (float64, ld n * nsel) for fitted directions [x0, x0 + n)
void ozaki_k1(Plan& p, int64_t nsel, int64_t x0, int64_t n, double* X, cudaStream_t s) {
  constexpr int ND = kOzKDigits;
  // every tile of occupied columns streams all B_x planes: take 96-column
  // tiles when they need fewer tiles than 80-column ones (81 columns: 1, not 2)
  const int64_t t80 = (nsel + ozaki_shape(kOzHalf).bn - 1) / ozaki_shape(kOzHalf).bn;
  const int64_t t96 = (nsel + ozaki_shape(kOzHalfWide).bn - 1) / ozaki_shape(kOzHalfWide).bn;
  const OzakiShape shape = t96 < t80 ? kOzHalfWide : kOzHalf;
  const OzakiShapeInfo sh = ozaki_shape(shape);
  const int bk = sh.box_k;
  const int64_t nao = p.nao, nao_p = p.nao_p16;
  const int64_t plane = p.nfit * nao * nao_p;
  OzakiMaps maps;
  for (int d = 0; d < ND; ++d) {
    ozaki_map(&maps.a[d], p.d_oz_a.as<int8_t>() + d * plane, nao, nao, p.nfit, nao_p, nao * nao_p,
              bk, 128);
    ozaki_map(&maps.b[d], p.ws_oz_c.as<int8_t>() + d * nsel * nao_p, nao, nsel, 1, nao_p,
              nsel * nao_p, bk, sh.box_b);
  }
  OzakiArgs a{};
  a.M = (int)nao;
  a.N = (int)nsel;
  a.ktiles = (int)((nao + bk - 1) / bk);
  a.ea = p.d_oz_ea.as<int>();
  a.ea_stride = nao;
  a.eb = p.ws_oz_eb.as<int>();
  a.out = X;
  a.ld_out = n * nsel;
  a.batch_stride_out = nsel;
  a.err = p.ws_oz_err.as<int>();
  // several fitted directions per CTA (one TMEM allocation and one copy ring
  // for all of them) while the grid still fills the device four times over
  int sm = 148;
  cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, p.ctx->device);
  const int64_t tiles = ((nsel + sh.bn - 1) / sh.bn) * ((nao + 127) / 128);
  a.zper = (int)std::max<int64_t>(1, std::min<int64_t>(16, tiles * n / (4 * (int64_t)sm)));
  const int64_t zstep = (int64_t)65535 * a.zper;
  for (int64_t z0 = 0; z0 < n; z0 += zstep) {
    const int64_t nz = std::min<int64_t>(zstep, n - z0);
    a.plane0 = (int)(x0 + z0);
    a.out = X + z0 * nsel;
    // X[m][z][i] leaves through TMA tensor stores when its strides allow
    a.tma_out = ozaki_out_mappable(a.out, a.batch_stride_out, a.ld_out) ? 1 : 0;
    if (a.tma_out) ozaki_map_out(&maps.out, a.out, nsel, nz, nao, a.batch_stride_out, a.ld_out);
    ozaki_launch(shape, maps, a, (int)nz, s);
  }
  check_oz_err(p, s);
}

// K (+)= sign * X X^T for one chunk of X (nao x kt, row-major): k in slices of
// kOzSlice bytes, each with its own row exponents and its own float64 partial
// (full square, exactly symmetric: both triangles come from the same integer
// sums), then summed in a fixed order, so K is bit-reproducible.
void ozaki_syrk(Plan& p, const double* X, int64_t kt, double sign, bool beta0, double* K,
                cudaStream_t s) {
  constexpr int ND = kOzSDigits;
  constexpr int64_t KS = kOzSlice;
  static_assert(KS <= kOzMaxK, "a k slice must stay within the exact int32 range");
  const OzakiShapeInfo sh = ozaki_shape(kOzSyrk);
  const int bk = sh.box_k;
  const int64_t nao = p.nao;
  const int64_t nsl = (kt + KS - 1) / KS;
  const int64_t plane = nsl * nao * KS;
  p.ws_oz_x.ensure((size_t)ND * plane);
  p.ws_oz_ex.ensure((size_t)nsl * nao * sizeof(int));
  p.ws_oz_kp.ensure((size_t)nsl * nao * nao * sizeof(double));
  split_slices_kernel<ND><<<dim3((unsigned)nao, (unsigned)nsl), 256, 0, s>>>(
      X, kt, nao, KS, p.ws_oz_ex.as<int>(), plane, p.ws_oz_x.as<int8_t>());
  DFJK_LAUNCHED();
  OzakiMaps maps;
  for (int d = 0; d < ND; ++d) {
    const int8_t* base = p.ws_oz_x.as<int8_t>() + d * plane;
    ozaki_map(&maps.a[d], base, KS, nao, nsl, KS, nao * KS, bk, 128);
    ozaki_map(&maps.b[d], base, KS, nao, nsl, KS, nao * KS, bk, sh.box_b);
  }
  OzakiArgs a{};
  a.M = (int)nao;
  a.N = (int)nao;
  a.ktiles = (int)(KS / bk);
  a.ea = p.ws_oz_ex.as<int>();
  a.ea_stride = nao;
  a.eb = p.ws_oz_ex.as<int>();
  a.eb_stride = nao;
  a.b_batched = 1;
  a.ld_out = nao;
  a.batch_stride_out = nao * nao;
  a.err = p.ws_oz_err.as<int>();
  a.lower = 1;
  for (int64_t z0 = 0; z0 < nsl; z0 += 65535) {
    const int64_t nz = std::min<int64_t>(65535, nsl - z0);
    a.plane0 = (int)z0;
    a.out = p.ws_oz_kp.as<double>() + z0 * nao * nao;
    ozaki_launch(kOzSyrk, maps, a, (int)nz, s);
  }
  const int64_t n = nao * nao;
  reduce_slices_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p.ws_oz_kp.as<double>(), nsl,
                                                                   nao, sign, beta0 ? 1 : 0, K);
  DFJK_LAUNCHED();
  check_oz_err(p, s);
}

}  // namespace dfjk

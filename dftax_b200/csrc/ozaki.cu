// Mixed-precision K half transform (precision = DFJK_MIXED) on the int8
// tensor cores with exact accumulation (ozaki_gemm.cu).
//
// Accuracy findings behind this design (device runs on water clusters):
//   * storing the 3-center tensor or B in float32 moves E_J by 1.3 uHa already
//     for (H2O)_4 (oracle simulation), so J and B stay float64;
//   * split-bf16 products accumulated in fp32 on the tensor cores bias K
//     toward zero (relative -3e-6 with one 64-deep k tile per partial, -2.7e-4
//     with long partials; E off by 76 uHa .. 5.9 mHa for (H2O)_32), so fp32
//     accumulation cannot hold 1 uHa at these sizes;
//   * int8 digits with int32 accumulation are exact: what is left is the
//     digit truncation (2^-27 of each row's largest value).
// The half transform X[x][m][i] = sum_n B_x[m][n] C[n][i] therefore runs on
// int8 digit planes of the square B_x (built once per geometry) and of C
// (per call), and the float64 DSYRK of the float64 path finishes K.
#include "ozaki.h"

#include <algorithm>
#include <cmath>

namespace dfjk {

namespace {

__device__ __forceinline__ int row_exponent(double vmax) {
  // |value| * 2^-e < 1/2 for every value of the row
  return vmax > 0.0 ? ilogb(vmax) + 2 : 0;
}

// four signed 7-bit digits: t = v 2^-e = sum_s d_s 2^(-7(s+1)) + O(2^-29)
__device__ __forceinline__ void digits4(double v, int e, int8_t (&d)[4]) {
  double t = ldexp(v, -e);
  const double sc[4] = {0x1p7, 0x1p14, 0x1p21, 0x1p28};
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const double q = rint(t * sc[s]);
    d[s] = (int8_t)q;
    t -= q / sc[s];
  }
}

// max |B_x[m][n]| over n for every (x, m), as float bits (atomicMax on the
// non-negative float's integer image); 32 x 32 (n, x) tiles through shared memory
__global__ void __launch_bounds__(256) rowmax_kernel(const double* __restrict__ B, int64_t ldb,
                                                     const int* __restrict__ rowmap, int nao,
                                                     int64_t nfit, unsigned* __restrict__ rowmax) {
  __shared__ float tile[32][33];
  const int64_t n0 = (int64_t)blockIdx.x * 32, x0 = (int64_t)blockIdx.z * 32;
  const int m = blockIdx.y;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int j = ty; j < 32; j += 8) {
    const int64_t n = n0 + j, x = x0 + tx;
    float v = 0.f;
    if (n < nao && x < nfit) {
      const int r = rowmap[(int64_t)m * nao + n];
      if (r >= 0) v = (float)fabs(B[(int64_t)r * ldb + x]);
    }
    tile[j][tx] = v;
  }
  __syncthreads();
  if (ty == 0) {
    float mx = 0.f;
    for (int j = 0; j < 32; ++j) mx = fmaxf(mx, tile[j][tx]);
    const int64_t x = x0 + tx;
    if (x < nfit && mx > 0.f) atomicMax(rowmax + x * nao + m, __float_as_uint(mx));
  }
}

// int8 digit planes A[d][x][m][nao_p] and row exponents ea[x][m]
__global__ void __launch_bounds__(256) digits_kernel(const double* __restrict__ B, int64_t ldb,
                                                     const int* __restrict__ rowmap, int nao,
                                                     int64_t nao_p, int64_t nfit,
                                                     const unsigned* __restrict__ rowmax,
                                                     int* __restrict__ ea, int64_t plane_bytes,
                                                     int8_t* __restrict__ out) {
  __shared__ double tile[32][33];
  const int64_t n0 = (int64_t)blockIdx.x * 32, x0 = (int64_t)blockIdx.z * 32;
  const int m = blockIdx.y;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int j = ty; j < 32; j += 8) {
    const int64_t n = n0 + j, x = x0 + tx;
    double v = 0.0;
    if (n < nao && x < nfit) {
      const int r = rowmap[(int64_t)m * nao + n];
      if (r >= 0) v = B[(int64_t)r * ldb + x];
    }
    tile[j][tx] = v;
  }
  __syncthreads();
  for (int j = ty; j < 32; j += 8) {
    const int64_t x = x0 + j, n = n0 + tx;
    if (x >= nfit || n >= nao_p) continue;
    const int e = row_exponent((double)__uint_as_float(rowmax[x * nao + m]));
    if (blockIdx.x == 0 && tx == 0) ea[x * nao + m] = e;
    int8_t d[4];
    digits4(tile[tx][j], e, d);
    const int64_t o = (x * nao + m) * nao_p + n;
#pragma unroll
    for (int s = 0; s < 4; ++s) out[s * plane_bytes + o] = d[s];
  }
}

// digit planes of C^T: Ct[d][i][n] from Cp[n][i] (nao x nsel), exponents eb[i]
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
    if (n < nao) digits4(Cp[n * nsel + i], e, d);
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

void build_ozaki_planes(Plan& p, cudaStream_t s) {
  p.nao_p16 = (p.nao + 15) / 16 * 16;
  const int64_t nfit = p.nfit, nao = p.nao;
  const int64_t plane = nfit * nao * p.nao_p16;
  p.d_oz_a.ensure((size_t)kOzDigits * plane);
  p.d_oz_rowmax.ensure((size_t)nfit * nao * sizeof(unsigned));
  p.d_oz_ea.ensure((size_t)nfit * nao * sizeof(int));
  DFJK_CUDA(cudaMemsetAsync(p.d_oz_rowmax.p, 0, (size_t)nfit * nao * sizeof(unsigned), s));
  const int64_t step = (int64_t)65535 * 32;
  for (int64_t x0 = 0; x0 < nfit; x0 += step) {
    const int64_t nx = std::min(step, nfit - x0);
    dim3 grid((unsigned)((p.nao_p16 + 31) / 32), (unsigned)nao, (unsigned)((nx + 31) / 32));
    rowmax_kernel<<<grid, 256, 0, s>>>(p.d_B.as<double>() + x0, p.ldb, p.d_rowmap.as<int>(), p.nao,
                                       nx, p.d_oz_rowmax.as<unsigned>() + x0 * nao);
    DFJK_LAUNCHED();
    digits_kernel<<<grid, 256, 0, s>>>(p.d_B.as<double>() + x0, p.ldb, p.d_rowmap.as<int>(), p.nao,
                                       p.nao_p16, nx, p.d_oz_rowmax.as<unsigned>() + x0 * nao,
                                       p.d_oz_ea.as<int>() + x0 * nao, plane,
                                       p.d_oz_a.as<int8_t>() + x0 * nao * p.nao_p16);
    DFJK_LAUNCHED();
  }
}

void ozaki_prepare_c(Plan& p, const double* Cp, int64_t nsel, cudaStream_t s) {
  p.ws_oz_c.ensure((size_t)kOzDigits * nsel * p.nao_p16);
  p.ws_oz_eb.ensure((size_t)nsel * sizeof(int));
  c_digits_kernel<<<(unsigned)nsel, 256, 0, s>>>(Cp, p.nao, nsel, p.nao_p16, p.ws_oz_eb.as<int>(),
                                                 p.ws_oz_c.as<int8_t>());
  DFJK_LAUNCHED();
  p.ws_oz_err.ensure(sizeof(int));
  DFJK_CUDA(cudaMemsetAsync(p.ws_oz_err.p, 0, sizeof(int), s));
}

// X[m][x - x0][i] (float64, ld n * nsel) for fitted directions [x0, x0 + n)
void ozaki_k1(Plan& p, int64_t nsel, int64_t x0, int64_t n, double* X, cudaStream_t s) {
  const int64_t nao = p.nao, nao_p = p.nao_p16;
  const int64_t plane = p.nfit * nao * nao_p;
  OzakiMaps maps;
  for (int d = 0; d < kOzDigits; ++d) {
    ozaki_map(&maps.a[d], p.d_oz_a.as<int8_t>() + d * plane, nao, nao, p.nfit, nao_p, nao * nao_p,
              128);
    ozaki_map(&maps.b[d], p.ws_oz_c.as<int8_t>() + d * nsel * nao_p, nao, nsel, 1, nao_p,
              nsel * nao_p, kOzBN);
  }
  OzakiArgs a{};
  a.M = (int)nao;
  a.N = (int)nsel;
  a.ktiles = (int)((nao + 127) / 128);
  a.ea = p.d_oz_ea.as<int>();
  a.ea_stride = nao;
  a.eb = p.ws_oz_eb.as<int>();
  a.out = X;
  a.ld_out = n * nsel;
  a.batch_stride_out = nsel;
  a.err = p.ws_oz_err.as<int>();
  for (int64_t z0 = 0; z0 < n; z0 += 65535) {
    const int64_t nz = std::min<int64_t>(65535, n - z0);
    a.plane0 = (int)(x0 + z0);
    a.out = X + z0 * nsel;
    ozaki_launch(maps, a, (int)nz, s);
  }
  check_oz_err(p, s);
}

}  // namespace dfjk

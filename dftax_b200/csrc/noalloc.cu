// J without device allocation: dfjk_j_noalloc.
//
// Some callers cannot allocate device memory while they run. An XLA FFI
// handler executes inside a JAX program whose allocator has already reserved
// most of the GPU's memory for itself, so a cudaMalloc from the handler can
// fail or take memory XLA has promised to other buffers; a serving loop may
// forbid cudaMalloc/cudaFree on its hot path because they synchronize the
// device and have unbounded latency. This entry point computes J exactly as
// dfjk_jk does (same B, same algorithm) but its scratch lives in a file-scope
// __device__ array of fixed size, so the call allocates nothing.
//
// Limits and sharing:
//   * the scratch holds kParts partial rows of gamma plus gamma itself, for B
//     with at most kMaxFit columns (the plan's fitted dimension rounded up to
//     8); larger plans are rejected with DFJK_ERR_UNSUPPORTED. Its size is
//     (kParts + 1) * kMaxFit doubles = 16.8 MB per device. dfjk_create looks
//     up its address with the context's device current, which loads this
//     file's module: the 16.8 MB are taken then, not by a later call of the
//     entry point, and stay until the process exits;
//   * every call on a device uses the same array and leaves its contents
//     behind; each call overwrites all the scratch it reads, so nothing needs
//     clearing, but two calls whose kernels overlap on the GPU (different
//     streams, no ordering between them) race on it.
#include "internal.h"

#include <algorithm>

namespace dfjk {
namespace {

constexpr int64_t kMaxFit = 8192;
constexpr int kParts = 256;
constexpr int kThreads = 256;
constexpr int kCols = kThreads * 8;          // columns per CTA (4 double2 per thread)
constexpr int kRowBatch = 32;                // rows whose density weights a CTA stages at once

__device__ __align__(256) double g_scratch[(kParts + 1) * kMaxFit];

// Partial gamma over a row range; the density weight of each row,
// w_r sum_i w_i C[m][i] C[n][i], is formed in the CTA (no dvec array).
__global__ void __launch_bounds__(kThreads) gamma_part_noalloc(
    const double* __restrict__ B, int64_t ldb, int64_t nrows, const double* __restrict__ C,
    const double* __restrict__ w, int64_t ncol, const int* __restrict__ rm,
    const int* __restrict__ rn, const int8_t* __restrict__ kind, int64_t rows_per_cta,
    double* __restrict__ part) {
  __shared__ double dsh[kRowBatch];
  const int64_t r0 = blockIdx.x * rows_per_cta;
  const int64_t r1 = min(nrows, r0 + rows_per_cta);
  const int64_t c0 = (int64_t)blockIdx.y * kCols + 2 * threadIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 acc[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) acc[j] = make_double2(0.0, 0.0);
  for (int64_t rb = r0; rb < r1; rb += kRowBatch) {
    for (int q = warp; q < kRowBatch; q += kThreads / 32) {
      const int64_t r = rb + q;
      double s = 0.0;
      if (r < r1) {
        const double* cm = C + (int64_t)rm[r] * ncol;
        const double* cn = C + (int64_t)rn[r] * ncol;
        for (int64_t i = lane; i < ncol; i += 32) s += (w ? w[i] : 1.0) * cm[i] * cn[i];
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) dsh[q] = (r < r1) ? (kind[r] == 2 ? 2.0 : 1.0) * s : 0.0;
    }
    __syncthreads();
    const int64_t nb = min((int64_t)kRowBatch, r1 - rb);
    for (int q = 0; q < nb; ++q) {
      const double d = dsh[q];
      const double* row = B + (rb + q) * ldb;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int64_t c = c0 + j * 2 * kThreads;
        if (c < ldb) {
          const double2 b = __ldcs(reinterpret_cast<const double2*>(row + c));
          acc[j].x += d * b.x;
          acc[j].y += d * b.y;
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int64_t c = c0 + j * 2 * kThreads;
    if (c < ldb) *reinterpret_cast<double2*>(part + blockIdx.x * ldb + c) = acc[j];
  }
}

__global__ void gamma_reduce_noalloc(const double* __restrict__ part, int64_t nparts, int64_t ldb,
                                     double* __restrict__ gamma) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= ldb) return;
  double s = 0.0;
  for (int64_t p = 0; p < nparts; ++p) s += part[p * ldb + c];
  gamma[c] = s;
}

__global__ void j_rows_noalloc(const double* __restrict__ B, int64_t ldb, int64_t nrows,
                               const double* __restrict__ gamma, const int* __restrict__ rm,
                               const int* __restrict__ rn, const int8_t* __restrict__ kind,
                               int64_t nao, double* __restrict__ J) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (gridDim.x * (int64_t)blockDim.x) >> 5;
  for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; r < nrows; r += nwarps) {
    const double* row = B + r * ldb;
    double s = 0.0;
    for (int64_t c = 2 * lane; c < ldb; c += 64) {
      const double2 b = __ldcs(reinterpret_cast<const double2*>(row + c));
      const double2 g = __ldg(reinterpret_cast<const double2*>(gamma + c));
      s += b.x * g.x + b.y * g.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0 && kind[r] != 0) {
      const int m = rm[r], n = rn[r];
      J[(int64_t)m * nao + n] = s;
      J[(int64_t)n * nao + m] = s;
    }
  }
}

}  // namespace

double* noalloc_scratch_address() {
  void* ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
  if (e != cudaSuccess)
    fail(DFJK_ERR_CUDA, "cudaGetSymbolAddress of the no-alloc scratch failed: %s",
         cudaGetErrorString(e));
  return static_cast<double*>(ptr);
}

void j_noalloc(Plan& p, const double* C, const double* w, int64_t ncol, double* J, cudaStream_t s) {
  if (p.ldb > kMaxFit)
    fail(DFJK_ERR_UNSUPPORTED,
         "dfjk_j_noalloc supports at most %lld fitted columns; this plan has %lld (use dfjk_jk)",
         (long long)kMaxFit, (long long)p.ldb);
  double* scratch = p.ctx->noalloc_scratch;
  if (!scratch) fail(DFJK_ERR_STATE, "the context has no no-alloc scratch address");
  const int dev = p.ctx->device;
  double* part = scratch;
  double* gamma = scratch + (int64_t)kParts * kMaxFit;
  DFJK_CUDA(cudaMemsetAsync(J, 0, (size_t)p.nao * p.nao * sizeof(double), s));
  if (p.nrows == 0) return;
  const int64_t ycols = (p.ldb + kCols - 1) / kCols;
  int64_t xparts = std::min<int64_t>(kParts, p.nrows);
  const int64_t rows_per = (p.nrows + xparts - 1) / xparts;
  xparts = (p.nrows + rows_per - 1) / rows_per;
  gamma_part_noalloc<<<dim3((unsigned)xparts, (unsigned)ycols), kThreads, 0, s>>>(
      p.d_B.as<double>(), p.ldb, p.nrows, C, w, ncol, p.d_row_m.as<int>(), p.d_row_n.as<int>(),
      p.d_row_w.as<int8_t>(), rows_per, part);
  DFJK_LAUNCHED();
  gamma_reduce_noalloc<<<(unsigned)((p.ldb + 255) / 256), 256, 0, s>>>(part, xparts, p.ldb, gamma);
  DFJK_LAUNCHED();
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t warps = std::min<int64_t>(p.nrows, (int64_t)sms * 64);
  j_rows_noalloc<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, s>>>(
      p.d_B.as<double>(), p.ldb, p.nrows, gamma, p.d_row_m.as<int>(), p.d_row_n.as<int>(),
      p.d_row_w.as<int8_t>(), p.nao, J);
  DFJK_LAUNCHED();
}

}  // namespace dfjk

extern "C" dfjk_status dfjk_j_noalloc(dfjk_plan* pl, const double* C, const double* w, int64_t ncol,
                                      double* J, void* stream) {
  if (!pl) return DFJK_ERR_INVALID;
  dfjk::Context* c = pl->p.ctx;
  return dfjk::guard(c, [&] {
    if (!pl->p.built) dfjk::fail(DFJK_ERR_STATE, "dfjk_j_noalloc before dfjk_build");
    if (!C || !J || ncol <= 0) dfjk::fail(DFJK_ERR_INVALID, "C or J is null or ncol=%lld", (long long)ncol);
    if (pl->p.opts.precision != DFJK_FP64)
      dfjk::fail(DFJK_ERR_UNSUPPORTED, "dfjk_j_noalloc needs a float64 plan");
    if (pl->p.opts.streamed)
      dfjk::fail(DFJK_ERR_UNSUPPORTED, "dfjk_j_noalloc needs B held in device memory (not streamed)");
    DFJK_CUDA(cudaSetDevice(c->device));
    dfjk::j_noalloc(pl->p, C, w, ncol, J, static_cast<cudaStream_t>(stream));
  });
}

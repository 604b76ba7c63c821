// J and K contractions over the fitted tensor B.
//
// B is row-major [nrows][ldb]: one row per AO pair (m, n) of a kept shell
// pair, one column per kept metric direction (B = (mn|P) L, L L^T = V+).
//
//   J: dvec[r] = w_r D[m, n]             (w_r = 2 off-diagonal pair, else 1)
//      gamma   = B^T dvec                 (stream B once; CTA partials + reduce)
//      J[m, n] = J[n, m] = B[r] . gamma   (stream B again; warp per row)
//   K: X[m][x][i] = sum_{(r, n) in list(m)} B[r][x] C'[n][i]   (half transform)
//      K = X X^T over the (x, i) index, C' = C sqrt|w|
// Float64 plans run both K products on the float64 tensor cores (mma.sync
// m8n8k4 f64: the gathered half transform, then a split-k X X^T); mixed plans
// run them on the int8 tensor cores (ozaki.cu). J is float64 in both.
// which are the P-gradients of dftax's DFCoulomb.energy (terms.py:592-613):
// J = int3c (V+ gamma), K = einsum("mlP,PQ,nsQ,ls->mn") (hybrid.py:23-41).
#include "internal.h"

#include <algorithm>
#include <cmath>

namespace dfjk {

// ---------------------------------------------------------------------------
// J
// ---------------------------------------------------------------------------

__global__ void dvec_from_c_kernel(const double* __restrict__ C, const double* __restrict__ w,
                                   int64_t ncol, const int* __restrict__ rm,
                                   const int* __restrict__ rn, const int8_t* __restrict__ kind,
                                   int64_t nrows, double* __restrict__ dvec) {
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= nrows) return;
  const int m = rm[warp], n = rn[warp];
  const double* cm = C + (int64_t)m * ncol;
  const double* cn = C + (int64_t)n * ncol;
  double s = 0.0;
  for (int64_t i = lane; i < ncol; i += 32) s += (w ? w[i] : 1.0) * cm[i] * cn[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) dvec[warp] = (kind[warp] == 2 ? 2.0 : 1.0) * s;
}

__global__ void dvec_from_density_kernel(const double* __restrict__ D, int64_t nao,
                                         const int* __restrict__ rm, const int* __restrict__ rn,
                                         const int8_t* __restrict__ kind, int64_t nrows,
                                         double* __restrict__ dvec) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= nrows) return;
  const int m = rm[r], n = rn[r];
  // off-diagonal pairs stand for both (m, n) and (n, m)
  const double v = kind[r] == 2 ? D[(int64_t)m * nao + n] + D[(int64_t)n * nao + m]
                                : D[(int64_t)m * nao + n];
  dvec[r] = v;
}

// gamma partials: CTA (bx, by) sums rows [r0, r1) for columns [by*2048, +2048)
constexpr int kGtThreads = 256;
constexpr int kGtCols = kGtThreads * 8;

__global__ void __launch_bounds__(kGtThreads) gamma_partial_kernel(
    const double* __restrict__ B, int64_t ldb, int64_t nrows, const double* __restrict__ dvec,
    int64_t rows_per_cta, double* __restrict__ part) {
  const int64_t r0 = blockIdx.x * rows_per_cta;
  const int64_t r1 = min(nrows, r0 + rows_per_cta);
  const int64_t c0 = (int64_t)blockIdx.y * kGtCols + 2 * threadIdx.x;
  double2 acc[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) acc[j] = make_double2(0.0, 0.0);
  for (int64_t r = r0; r < r1; ++r) {
    const double d = __ldg(dvec + r);
    const double* row = B + r * ldb;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t c = c0 + j * 2 * kGtThreads;
      if (c < ldb) {
        const double2 b = __ldcs(reinterpret_cast<const double2*>(row + c));
        acc[j].x += d * b.x;
        acc[j].y += d * b.y;
      }
    }
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int64_t c = c0 + j * 2 * kGtThreads;
    if (c < ldb) *reinterpret_cast<double2*>(part + blockIdx.x * ldb + c) = acc[j];
  }
}

__global__ void reduce_rows_kernel(const double* __restrict__ part, int64_t nparts, int64_t ldb,
                                   double* __restrict__ out) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= ldb) return;
  double s = 0.0;
  for (int64_t p = 0; p < nparts; ++p) s += part[p * ldb + c];
  out[c] = s;
}

// J rows: one warp per row, J[m, n] and J[n, m]
__global__ void j_rows_kernel(const double* __restrict__ B, int64_t ldb, int64_t nrows,
                              const double* __restrict__ gamma, const int* __restrict__ rm,
                              const int* __restrict__ rn, const int8_t* __restrict__ kind,
                              int64_t nao, double* __restrict__ J) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (gridDim.x * (int64_t)blockDim.x) >> 5;
  for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; r < nrows; r += nwarps) {
    const double* row = B + r * ldb;
    // four 16-byte loads in flight per lane (ldb is a multiple of 8 and c is
    // even, so c + 192 < ldb keeps all four pairs inside the row)
    double s4[4] = {0.0, 0.0, 0.0, 0.0};
    int64_t c = 2 * lane;
    for (; c + 192 < ldb; c += 256) {
      double2 b[4], g[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        b[u] = __ldcs(reinterpret_cast<const double2*>(row + c + 64 * u));
        g[u] = __ldg(reinterpret_cast<const double2*>(gamma + c + 64 * u));
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) s4[u] += b[u].x * g[u].x + b[u].y * g[u].y;
    }
    for (; c < ldb; c += 64) {
      const double2 b = __ldcs(reinterpret_cast<const double2*>(row + c));
      const double2 g = __ldg(reinterpret_cast<const double2*>(gamma + c));
      s4[0] += b.x * g.x + b.y * g.y;
    }
    double s = (s4[0] + s4[1]) + (s4[2] + s4[3]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
      const int k = kind[r];
      if (k == 0) continue;
      const int m = rm[r], n = rn[r];
      J[(int64_t)m * nao + n] = s;
      J[(int64_t)n * nao + m] = s;
    }
  }
}

static int num_sms(int dev) {
  int n = 0;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 148;
}

__global__ void add_to_kernel(const double* __restrict__ x, int64_t n, double* __restrict__ y) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) y[i] += x[i];
}

// gamma (+)= Bc^T dvec over nrows rows of Bc: fixed-order partial sums
static void gamma_rows(Plan& p, const double* Bc, int64_t nrows, const double* dvec, double* out,
                       bool add, cudaStream_t s) {
  const int sms = num_sms(p.ctx->device);
  const int64_t ycols = (p.ldb + kGtCols - 1) / kGtCols;
  int64_t xparts = std::max<int64_t>(1, (int64_t)sms * 4 / ycols);
  xparts = std::min<int64_t>(xparts, std::max<int64_t>(1, nrows));
  const int64_t rows_per = (nrows + xparts - 1) / xparts;
  xparts = (nrows + rows_per - 1) / rows_per;
  DevBuf& part = p.ws_part;
  part.ensure((size_t)(std::max<int64_t>(xparts, 1) + (add ? 1 : 0)) * p.ldb * sizeof(double));
  double* sum = part.as<double>() + xparts * p.ldb;   // the chunk's gamma when adding
  gamma_partial_kernel<<<dim3((unsigned)xparts, (unsigned)ycols), kGtThreads, 0, s>>>(
      Bc, p.ldb, nrows, dvec, rows_per, part.as<double>());
  DFJK_LAUNCHED();
  reduce_rows_kernel<<<(unsigned)((p.ldb + 255) / 256), 256, 0, s>>>(part.as<double>(), xparts,
                                                                     p.ldb, add ? sum : out);
  DFJK_LAUNCHED();
  if (add) {
    add_to_kernel<<<(unsigned)((p.ldb + 255) / 256), 256, 0, s>>>(sum, p.ldb, out);
    DFJK_LAUNCHED();
  }
}

// gamma = B^T dvec into `gamma` (ldb doubles)
static void gamma_from_dvec(Plan& p, const double* dvec, double* gamma, cudaStream_t s) {
  if (p.opts.streamed) {
    DFJK_CUDA(cudaMemsetAsync(gamma, 0, p.ldb * sizeof(double), s));
    for_each_b_chunk(p, s, [&](int64_t r0, int64_t nr, const double* Bc) {
      if (nr > 0) gamma_rows(p, Bc, nr, dvec + r0, gamma, true, s);
    });
    return;
  }
  const int sms = num_sms(p.ctx->device);
  const int64_t ycols = (p.ldb + kGtCols - 1) / kGtCols;
  int64_t xparts = std::max<int64_t>(1, (int64_t)sms * 4 / ycols);
  xparts = std::min<int64_t>(xparts, std::max<int64_t>(1, p.nrows));
  const int64_t rows_per = (p.nrows + xparts - 1) / xparts;
  xparts = (p.nrows + rows_per - 1) / rows_per;
  DevBuf& part = p.ws_part;
  part.ensure((size_t)std::max<int64_t>(xparts, 1) * p.ldb * sizeof(double));
  if (p.nrows > 0) {
    gamma_partial_kernel<<<dim3((unsigned)xparts, (unsigned)ycols), kGtThreads, 0, s>>>(
        p.d_B.as<double>(), p.ldb, p.nrows, dvec, rows_per, part.as<double>());
    DFJK_LAUNCHED();
    reduce_rows_kernel<<<(unsigned)((p.ldb + 255) / 256), 256, 0, s>>>(part.as<double>(), xparts,
                                                                       p.ldb, gamma);
    DFJK_LAUNCHED();
  } else {
    DFJK_CUDA(cudaMemsetAsync(gamma, 0, p.ldb * sizeof(double), s));
  }
}

static void j_from_gamma(Plan& p, const double* gamma, double* J, cudaStream_t s) {
  DFJK_CUDA(cudaMemsetAsync(J, 0, (size_t)p.nao * p.nao * sizeof(double), s));
  if (p.nrows == 0) return;
  const int sms = num_sms(p.ctx->device);
  if (p.opts.streamed) {
    for_each_b_chunk(p, s, [&](int64_t r0, int64_t nr, const double* Bc) {
      if (nr == 0) return;
      const int64_t warps = std::min<int64_t>(nr, (int64_t)sms * 64);
      j_rows_kernel<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, s>>>(
          Bc, p.ldb, nr, gamma, p.d_row_m.as<int>() + r0, p.d_row_n.as<int>() + r0,
          p.d_row_w.as<int8_t>() + r0, p.nao, J);
      DFJK_LAUNCHED();
    });
    return;
  }
  const int64_t warps = std::min<int64_t>(p.nrows, (int64_t)sms * 64);
  j_rows_kernel<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, s>>>(
      p.d_B.as<double>(), p.ldb, p.nrows, gamma, p.d_row_m.as<int>(), p.d_row_n.as<int>(),
      p.d_row_w.as<int8_t>(), p.nao, J);
  DFJK_LAUNCHED();
}

// ---------------------------------------------------------------------------
// K: half transform X[m][x][i] = sum_{(r, n) in list(m)} B[r][x0 + x] C'[n][i]
// ---------------------------------------------------------------------------

// Block tile 64 (x) x 80 (i), 16 list entries per k chunk, on the float64
// tensor cores (mma.sync m8n8k4 f64: tcgen05 has no float64 kind). Eight
// warps as 4 (x, 16 rows) x 2 (i, 40 columns); a warp holds 2 x 5 fragments
// of 8 x 8. Shared rows are padded to 68 / 84 doubles so that the fragment
// loads (k = lane % 4, row = lane / 4) fall in distinct banks.
constexpr int kHtX = 64, kHtI = 80, kHtK = 16, kHtPX = 68, kHtPI = 84;

__device__ __forceinline__ void dmma_8x8x4(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
  // src-size 0 fills the 8 shared bytes with zeros (gmem must still be a valid address)
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(
                   static_cast<unsigned>(__cvta_generic_to_shared(smem))),
               "l"(gmem), "r"(valid ? 8 : 0)
               : "memory");
}

// The list of m is entries [kbeg[m], kend[m]) (kend == nullptr: up to
// kbeg[m + 1]); entry e reads B row krow[e] - row0. accumulate: X += instead
// of X = (a streamed plan sums the chunks of B rows).
__global__ void __launch_bounds__(256) half_transform_kernel(
    const double* __restrict__ B, int64_t ldb, int64_t x0, int64_t xc, const double* __restrict__ Cp,
    int64_t ncol, const int* __restrict__ kbeg, const int* __restrict__ kend,
    const int* __restrict__ krow, const int* __restrict__ kn, int64_t row0, int accumulate,
    double* __restrict__ X) {
  // two buffers: chunk c + 1 is copied (cp.async) while chunk c is multiplied
  __shared__ double Bs[2][kHtK][kHtPX];
  __shared__ double Cs[2][kHtK][kHtPI];
  const int m = blockIdx.x;
  const int64_t xt = (int64_t)blockIdx.y * kHtX;   // within the chunk
  const int64_t it = (int64_t)blockIdx.z * kHtI;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wx = (warp & 3) * 16, wi = (warp >> 2) * 40;
  const int fr = lane >> 2, fk = lane & 3;   // fragment row / k of this lane
  double acc[2][5][2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 5; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  const int e0 = kbeg[m], e1 = kend ? kend[m] : kbeg[m + 1];
  // kHtK list entries: rows of B (x tile) and rows of C' (i tile)
  auto stage = [&](int buf, int e) {
    for (int q = threadIdx.x; q < kHtK * kHtX; q += 256) {
      const int k = q / kHtX, x = q % kHtX;
      const bool ok = e + k < e1 && xt + x < xc;
      cp_async8(&Bs[buf][k][x], ok ? B + ((int64_t)krow[e + k] - row0) * ldb + x0 + xt + x : B, ok);
    }
    for (int q = threadIdx.x; q < kHtK * kHtI; q += 256) {
      const int k = q / kHtI, i = q % kHtI;
      const bool ok = e + k < e1 && it + i < ncol;
      cp_async8(&Cs[buf][k][i], ok ? Cp + (int64_t)kn[e + k] * ncol + it + i : Cp, ok);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  if (e0 < e1) stage(0, e0);
  int buf = 0;
  for (int e = e0; e < e1; e += kHtK, buf ^= 1) {
    if (e + kHtK < e1) {
      stage(buf ^ 1, e + kHtK);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kHtK; kk += 4) {
      double af[2], bf[5];
#pragma unroll
      for (int a = 0; a < 2; ++a) af[a] = Bs[buf][kk + fk][wx + 8 * a + fr];
#pragma unroll
      for (int b = 0; b < 5; ++b) bf[b] = Cs[buf][kk + fk][wi + 8 * b + fr];
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 5; ++b) dmma_8x8x4(acc[a][b], af[a], bf[b]);
    }
    __syncthreads();
  }
  // accumulator (a, b, r) holds x = wx + 8a + lane / 4, i = wi + 8b + 2 (lane % 4) + r
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    const int64_t x = xt + wx + 8 * a + fr;
    if (x >= xc) continue;
#pragma unroll
    for (int b = 0; b < 5; ++b)
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int64_t i = it + wi + 8 * b + 2 * fk + r;
        if (i < ncol) {
          double* o = X + ((int64_t)m * xc + x) * ncol + i;
          *o = accumulate ? *o + acc[a][b][r] : acc[a][b][r];
        }
      }
  }
}

// [kb[m], ke[m]): the entries of m's K list whose rows lie in [r0, r1) (each
// list is in ascending row order)
__global__ void list_bounds_kernel(const int* __restrict__ kptr, const int* __restrict__ krow,
                                   int64_t nao, int64_t r0, int64_t r1, int* __restrict__ kb,
                                   int* __restrict__ ke) {
  const int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (m >= nao) return;
  auto lower = [&](int lo, int hi, int64_t v) {
    while (lo < hi) {
      const int mid = lo + (hi - lo) / 2;
      if (krow[mid] < v) lo = mid + 1;
      else hi = mid;
    }
    return lo;
  };
  const int lo = kptr[m], hi = kptr[m + 1];
  kb[m] = lower(lo, hi, r0);
  ke[m] = lower(lo, hi, r1);
}

// K partials on the float64 tensor cores: for the lower-triangle tile pair
// (tm >= tn, 64 x 64) of blockIdx.x and the k slice blockIdx.y,
// part[slice][tm*64 + r][tn*64 + c] = sum_k X[tm*64 + r][k] X[tn*64 + c][k]
// over the slice (X row-major, nao x kt). Same fragment layout and cp.async
// double buffering as the half transform; rows are staged k-major.
constexpr int kSyT = 64, kSyK = 16, kSyP = 68;

__global__ void __launch_bounds__(256) syrk_part_kernel(const double* __restrict__ X, int64_t nao,
                                                        int64_t kt, int64_t kslice,
                                                        const int2* __restrict__ tiles,
                                                        double* __restrict__ part) {
  __shared__ double As[2][kSyK][kSyP];
  __shared__ double Bs[2][kSyK][kSyP];
  const int2 tp = tiles[blockIdx.x];
  const int64_t r0 = (int64_t)tp.x * kSyT, c0 = (int64_t)tp.y * kSyT;
  const int64_t k0 = (int64_t)blockIdx.y * kslice;
  const int64_t k1 = k0 + kslice < kt ? k0 + kslice : kt;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wr = (warp & 3) * 16, wc = (warp >> 2) * 32;
  const int fr = lane >> 2, fk = lane & 3;
  double acc[2][4][2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  auto stage = [&](int buf, int64_t k) {
    for (int q = threadIdx.x; q < kSyT * kSyK; q += 256) {
      const int r = q / kSyK, kk = q % kSyK;
      const bool ka = k + kk < k1;
      const bool oa = ka && r0 + r < nao, ob = ka && c0 + r < nao;
      cp_async8(&As[buf][kk][r], oa ? X + (r0 + r) * kt + k + kk : X, oa);
      cp_async8(&Bs[buf][kk][r], ob ? X + (c0 + r) * kt + k + kk : X, ob);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  if (k0 < k1) stage(0, k0);
  int buf = 0;
  for (int64_t k = k0; k < k1; k += kSyK, buf ^= 1) {
    if (k + kSyK < k1) {
      stage(buf ^ 1, k + kSyK);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kSyK; kk += 4) {
      double af[2], bf[4];
#pragma unroll
      for (int a = 0; a < 2; ++a) af[a] = As[buf][kk + fk][wr + 8 * a + fr];
#pragma unroll
      for (int b = 0; b < 4; ++b) bf[b] = Bs[buf][kk + fk][wc + 8 * b + fr];
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) dmma_8x8x4(acc[a][b], af[a], bf[b]);
    }
    __syncthreads();
  }
  double* out = part + (int64_t)blockIdx.y * nao * nao;
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    const int64_t r = r0 + wr + 8 * a + fr;
    if (r >= nao) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int64_t c = c0 + wc + 8 * b + 2 * fk + q;
        if (c < nao) out[r * nao + c] = acc[a][b][q];
      }
  }
}

// K[i][j] = (beta0 ? 0 : K[i][j]) + sign * sum_s part[s][max(i,j)][min(i,j)], s in order
__global__ void syrk_reduce_kernel(const double* __restrict__ part, int64_t nsplit, int64_t nao,
                                   double sign, int beta0, double* __restrict__ K) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nao * nao) return;
  const int64_t i = t / nao, j = t % nao;
  const int64_t src = i >= j ? i * nao + j : j * nao + i;
  double acc = 0.0;
  for (int64_t s = 0; s < nsplit; ++s) acc += part[s * nao * nao + src];
  K[t] = beta0 ? sign * acc : K[t] + sign * acc;
}

__global__ void scale_cols_kernel(const double* __restrict__ C, const double* __restrict__ w,
                                  int64_t nao, int64_t ncol, const int* __restrict__ sel,
                                  int64_t nsel, double* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nao * nsel) return;
  const int64_t m = i / nsel, j = i % nsel;
  const int col = sel[j];
  const double f = w ? sqrt(fabs(w[col])) : 1.0;
  out[i] = C[m * ncol + col] * f;
}

__global__ void symmetrize_kernel(double* __restrict__ K, int64_t n) {
  // cuBLAS filled the column-major lower triangle = row-major upper (j >= i)
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n * n) return;
  const int64_t i = t / n, j = t % n;
  if (j < i) K[t] = K[j * n + i];
}

// K (+)= sign * X X^T (float64, full square) for X nao x kt row-major: lower
// 64 x 64 tile pairs times k slices, enough blocks for several waves, then a
// fixed-order sum of the slices (bit-reproducible).
static void syrk_fp64(Plan& p, const double* X, int64_t kt, double sign, bool beta0, double* K,
                      cudaStream_t s) {
  const int64_t nao = p.nao;
  const int64_t nt = (nao + kSyT - 1) / kSyT;
  std::vector<int2> tl;
  for (int64_t a = 0; a < nt; ++a)
    for (int64_t b = 0; b <= a; ++b) tl.push_back(make_int2((int)a, (int)b));
  int sm = 148;
  cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, p.ctx->device);
  const int64_t want = 4 * (int64_t)sm;
  int64_t nsplit = std::max<int64_t>(1, (want + (int64_t)tl.size() - 1) / (int64_t)tl.size());
  nsplit = std::min<int64_t>(nsplit, std::max<int64_t>(1, kt / 1024));
  nsplit = std::min<int64_t>(nsplit, 65535);
  const int64_t kslice = ((kt + nsplit - 1) / nsplit + kSyK - 1) / kSyK * kSyK;
  nsplit = (kt + kslice - 1) / kslice;
  p.ws_syrk_tiles.ensure(tl.size() * sizeof(int2));
  DFJK_CUDA(cudaMemcpyAsync(p.ws_syrk_tiles.p, tl.data(), tl.size() * sizeof(int2),
                            cudaMemcpyHostToDevice, s));
  p.ws_syrk.ensure((size_t)nsplit * nao * nao * sizeof(double));
  syrk_part_kernel<<<dim3((unsigned)tl.size(), (unsigned)nsplit), 256, 0, s>>>(
      X, nao, kt, kslice, p.ws_syrk_tiles.as<int2>(), p.ws_syrk.as<double>());
  DFJK_LAUNCHED();
  syrk_reduce_kernel<<<(unsigned)((nao * nao + 255) / 256), 256, 0, s>>>(
      p.ws_syrk.as<double>(), nsplit, nao, sign, beta0 ? 1 : 0, K);
  DFJK_LAUNCHED();
}

// K (+)= sign * X X^T for the selected columns of C (scaled by sqrt|w|)
// fuse (streamed plans only, may be null): gamma = B^T dvec is also summed
// in the first pass over B's chunks (one rebuild of B fewer per J/K call);
// its dvec is cleared once gamma is done.
struct GammaFuse {
  const double* dvec = nullptr;
  double* gamma = nullptr;
};

static void k_accumulate(Plan& p, const double* C, const double* w, int64_t ncol,
                         const std::vector<int>& sel, double sign, bool first, double* K,
                         cudaStream_t s, GammaFuse* fuse = nullptr) {
  Context& c = *p.ctx;
  const int64_t nao = p.nao, nsel = (int64_t)sel.size();
  if (nsel == 0) return;
  DevBuf& dsel = p.ws_sel;
  DevBuf& Cp = p.ws_Cp;
  dsel.ensure(sel.size() * sizeof(int));
  DFJK_CUDA(cudaMemcpyAsync(dsel.p, sel.data(), sel.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  Cp.ensure((size_t)nao * nsel * sizeof(double));
  scale_cols_kernel<<<(unsigned)((nao * nsel + 255) / 256), 256, 0, s>>>(C, w, nao, ncol,
                                                                         dsel.as<int>(), nsel,
                                                                         Cp.as<double>());
  DFJK_LAUNCHED();
  // x chunking so that X (nao * xc * nsel doubles) stays within budget; a
  // streamed plan rebuilds B once per x chunk, so it takes up to half the
  // free device memory
  int64_t budget = (int64_t)6 << 30;
  if (p.opts.streamed) {
    size_t fr = 0, tot = 0;
    DFJK_CUDA(cudaMemGetInfo(&fr, &tot));
    budget = std::max<int64_t>(budget, (int64_t)(fr / 2));
  }
  int64_t xc = budget / (nao * nsel * (int64_t)sizeof(double));
  xc = std::max<int64_t>(kHtX, xc / kHtX * kHtX);
  xc = std::min<int64_t>(xc, (p.nfit + kHtX - 1) / kHtX * kHtX);
  DevBuf& X = p.ws_X;
  X.ensure((size_t)nao * xc * nsel * sizeof(double));
  DFJK_CUBLAS(cublasSetStream(c.cublas, s));
  bool beta0 = first;
  for (int64_t x0 = 0; x0 < p.nfit; x0 += xc) {
    const int64_t n = std::min(xc, p.nfit - x0);
    dim3 grid((unsigned)nao, (unsigned)((n + kHtX - 1) / kHtX), (unsigned)((nsel + kHtI - 1) / kHtI));
    p.timer.mark(kPhKhalf, s);
    const bool oz = p.opts.precision == DFJK_MIXED && !p.opts.streamed;
    if (p.opts.streamed) {
      // X = sum over chunks of B rows of the half transform of each chunk
      DFJK_CUDA(cudaMemsetAsync(X.p, 0, (size_t)nao * n * nsel * sizeof(double), s));
      p.ws_kb.ensure(nao * sizeof(int));
      p.ws_ke.ensure(nao * sizeof(int));
      const bool with_gamma = fuse && fuse->dvec;
      if (with_gamma) DFJK_CUDA(cudaMemsetAsync(fuse->gamma, 0, p.ldb * sizeof(double), s));
      for_each_b_chunk(p, s, [&](int64_t r0, int64_t nr, const double* Bc) {
        if (with_gamma && nr > 0) gamma_rows(p, Bc, nr, fuse->dvec + r0, fuse->gamma, true, s);
        list_bounds_kernel<<<(unsigned)((nao + 255) / 256), 256, 0, s>>>(
            p.d_kptr.as<int>(), p.d_krow.as<int>(), nao, r0, r0 + nr, p.ws_kb.as<int>(),
            p.ws_ke.as<int>());
        DFJK_LAUNCHED();
        half_transform_kernel<<<grid, 256, 0, s>>>(Bc, p.ldb, x0, n, Cp.as<double>(), nsel,
                                                   p.ws_kb.as<int>(), p.ws_ke.as<int>(),
                                                   p.d_krow.as<int>(), p.d_kn.as<int>(), r0, 1,
                                                   X.as<double>());
        DFJK_LAUNCHED();
      });
      if (with_gamma) fuse->dvec = nullptr;   // gamma is complete
    } else if (oz) {
      if (x0 == 0) ozaki_prepare_c(p, Cp.as<double>(), nsel, s);
      ozaki_k1(p, nsel, x0, n, X.as<double>(), s);   // int8 tensor cores, exact accumulation
    } else {
      half_transform_kernel<<<grid, 256, 0, s>>>(p.d_B.as<double>(), p.ldb, x0, n, Cp.as<double>(),
                                                 nsel, p.d_kptr.as<int>(), nullptr,
                                                 p.d_krow.as<int>(), p.d_kn.as<int>(), 0, 0,
                                                 X.as<double>());
      DFJK_LAUNCHED();
    }
    p.timer.mark(kPhKhalf, s);
    p.timer.mark(kPhKsyrk, s);
    if (oz) {
      ozaki_syrk(p, X.as<double>(), n * nsel, sign, beta0, K, s);   // full square, int8 tensor cores
    } else {
      syrk_fp64(p, X.as<double>(), n * nsel, sign, beta0, K, s);
    }
    p.timer.mark(kPhKsyrk, s);
    beta0 = false;
  }
}

static void k_compute(Plan& p, const double* C, const double* w, int64_t ncol, double* K,
                      cudaStream_t s, GammaFuse* fuse = nullptr) {
  std::vector<int> pos, neg;
  if (w) {
    std::vector<double> hw(ncol);
    DFJK_CUDA(cudaMemcpyAsync(hw.data(), w, ncol * sizeof(double), cudaMemcpyDeviceToHost, s));
    DFJK_CUDA(cudaStreamSynchronize(s));
    for (int64_t i = 0; i < ncol; ++i) {
      if (!std::isfinite(hw[i])) fail(DFJK_ERR_NUMERIC, "non-finite weight");
      if (hw[i] > 0) pos.push_back((int)i);
      else if (hw[i] < 0) neg.push_back((int)i);
    }
  } else {
    for (int64_t i = 0; i < ncol; ++i) pos.push_back((int)i);
  }
  if (pos.empty() && neg.empty()) {
    DFJK_CUDA(cudaMemsetAsync(K, 0, (size_t)p.nao * p.nao * sizeof(double), s));
    return;
  }
  k_accumulate(p, C, w, ncol, pos, 1.0, true, K, s, fuse);
  k_accumulate(p, C, w, ncol, neg, -1.0, pos.empty(), K, s, fuse);
  const int64_t n = p.nao;
  symmetrize_kernel<<<(unsigned)((n * n + 255) / 256), 256, 0, s>>>(K, n);
  DFJK_LAUNCHED();
}

void jk_compute(Plan& p, const double* C, const double* w, int64_t ncol, double* J, double* K,
                cudaStream_t s) {
  for (int ph = kPhJ; ph <= kPhKsyrk; ++ph) p.timer.reset(ph);
  if (J) {
    p.timer.mark(kPhJ, s);
    DevBuf& dvec = p.ws_dvec;
    DevBuf& gamma = p.ws_gamma;
    dvec.ensure(std::max<int64_t>(p.nrows, 1) * sizeof(double));
    gamma.ensure(p.ldb * sizeof(double));
    if (p.nrows > 0) {
      dvec_from_c_kernel<<<(unsigned)((p.nrows * 32 + 255) / 256), 256, 0, s>>>(
          C, w, ncol, p.d_row_m.as<int>(), p.d_row_n.as<int>(), p.d_row_w.as<int8_t>(), p.nrows,
          dvec.as<double>());
      DFJK_LAUNCHED();
    }
    if (p.opts.streamed && K) {
      // one pass over B's chunks gives gamma and the K half transform; J
      // takes a second
      GammaFuse fuse{dvec.as<double>(), gamma.as<double>()};
      k_compute(p, C, w, ncol, K, s, &fuse);
      if (fuse.dvec) gamma_from_dvec(p, dvec.as<double>(), gamma.as<double>(), s);
      j_from_gamma(p, gamma.as<double>(), J, s);
      p.timer.mark(kPhJ, s);
      return;
    }
    gamma_from_dvec(p, dvec.as<double>(), gamma.as<double>(), s);
    j_from_gamma(p, gamma.as<double>(), J, s);
    p.timer.mark(kPhJ, s);
  }
  if (K) k_compute(p, C, w, ncol, K, s);
}

// ---------------------------------------------------------------------------
// DFCoulomb.energy and its gradient
// ---------------------------------------------------------------------------

__global__ void add_kernel(const double* __restrict__ a, const double* __restrict__ b, int64_t n,
                           double* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] + b[i];
}

__global__ void dot_kernel(const double* __restrict__ a, const double* __restrict__ b, int64_t n,
                           double* __restrict__ out) {
  __shared__ double sh[256];
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += a[i] * b[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

__global__ void axpy_kernel(const double* __restrict__ x, double a, int64_t n, double* __restrict__ y) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) y[i] += a * x[i];
}

static double dot(const double* a, const double* b, int64_t n, cudaStream_t s) {
  DevBuf r;
  r.alloc(sizeof(double));
  dot_kernel<<<1, 256, 0, s>>>(a, b, n, r.as<double>());
  DFJK_LAUNCHED();
  double h = 0;
  DFJK_CUDA(cudaMemcpyAsync(&h, r.p, sizeof(double), cudaMemcpyDeviceToHost, s));
  DFJK_CUDA(cudaStreamSynchronize(s));
  return h;
}

// K of a symmetric density Q (device, nao x nao): Q = V diag(l) V^T on the
// device, K(Q) = sum_k l_k K(v_k v_k^T) over |l_k| > 1e-14 max|l|.
// Eigen-factor of a symmetric Q (nao x nao): Ct row-major with Q = Ct diag(dw) Ct^T,
// eigenvalues below 1e-14 of the largest set to zero, so K(Q) = k_compute(Ct, dw).
static void density_factor(Plan& p, const double* Q, DevBuf& Ct, DevBuf& dw, cudaStream_t s) {
  Context& c = *p.ctx;
  const int64_t n = p.nao;
  DevBuf V, wv, work, info;
  V.alloc((size_t)n * n * sizeof(double));
  wv.alloc(n * sizeof(double));
  DFJK_CUDA(cudaMemcpyAsync(V.p, Q, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  DFJK_CUSOLVER(cusolverDnSetStream(c.cusolver, s));
  int lwork = 0;
  DFJK_CUSOLVER(cusolverDnDsyevd_bufferSize(c.cusolver, CUSOLVER_EIG_MODE_VECTOR,
                                            CUBLAS_FILL_MODE_LOWER, (int)n, V.as<double>(), (int)n,
                                            wv.as<double>(), &lwork));
  work.alloc((size_t)std::max(lwork, 1) * sizeof(double));
  info.alloc(sizeof(int));
  DFJK_CUSOLVER(cusolverDnDsyevd(c.cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER,
                                 (int)n, V.as<double>(), (int)n, wv.as<double>(), work.as<double>(),
                                 lwork, info.as<int>()));
  std::vector<double> hw(n);
  int hinfo = 0;
  DFJK_CUDA(cudaMemcpyAsync(hw.data(), wv.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  DFJK_CUDA(cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  DFJK_CUDA(cudaStreamSynchronize(s));
  if (hinfo != 0) fail(DFJK_ERR_NUMERIC, "density eigensolver failed (info=%d)", hinfo);
  double big = 0.0;
  for (double v : hw) big = std::max(big, std::fabs(v));
  // eigenvectors are the columns of the column-major V, i.e. rows of the
  // row-major view: C[m][k] = V[k*n + m]; transpose into a row-major C
  Ct.alloc((size_t)n * n * sizeof(double));
  DFJK_CUBLAS(cublasSetStream(c.cublas, s));
  const double one = 1.0, zero = 0.0;
  DFJK_CUBLAS(cublasDgeam(c.cublas, CUBLAS_OP_T, CUBLAS_OP_N, (int)n, (int)n, &one, V.as<double>(),
                          (int)n, &zero, V.as<double>(), (int)n, Ct.as<double>(), (int)n));
  std::vector<double> wsel(n, 0.0);
  for (int64_t k = 0; k < n; ++k)
    if (std::fabs(hw[k]) > 1e-14 * big) wsel[k] = hw[k];
  upload(dw, wsel);
}

// hf_lr: the long-range exchange of range-separated hybrids through the plan's
// long-range fit (terms.py:604-612)
void gamma_from_density(Plan& p, const double* Ptot, double* gamma, cudaStream_t s) {
  DevBuf dvec;
  dvec.alloc(std::max<int64_t>(p.nrows, 1) * sizeof(double));
  if (p.nrows > 0) {
    dvec_from_density_kernel<<<(unsigned)((p.nrows + 255) / 256), 256, 0, s>>>(
        Ptot, p.nao, p.d_row_m.as<int>(), p.d_row_n.as<int>(), p.d_row_w.as<int8_t>(), p.nrows,
        dvec.as<double>());
    DFJK_LAUNCHED();
  }
  gamma_from_dvec(p, dvec.as<double>(), gamma, s);
}

double energy(Plan& p, const double* P, int nspin, double hf, double hf_lr, double* F,
              cudaStream_t s) {
  const int64_t n = p.nao, nn = n * n;
  DevBuf Ptot, dvec, gamma, J;
  const double* Pt = P;
  if (nspin == 2) {
    Ptot.alloc(nn * sizeof(double));
    add_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(P, P + nn, nn, Ptot.as<double>());
    DFJK_LAUNCHED();
    Pt = Ptot.as<double>();
  }
  check_finite(p, P, nn * nspin, s, "the density");
  dvec.alloc(std::max<int64_t>(p.nrows, 1) * sizeof(double));
  gamma.alloc(p.ldb * sizeof(double));
  if (p.nrows > 0) {
    dvec_from_density_kernel<<<(unsigned)((p.nrows + 255) / 256), 256, 0, s>>>(
        Pt, n, p.d_row_m.as<int>(), p.d_row_n.as<int>(), p.d_row_w.as<int8_t>(), p.nrows,
        dvec.as<double>());
    DFJK_LAUNCHED();
  }
  gamma_from_dvec(p, dvec.as<double>(), gamma.as<double>(), s);
  double e = 0.5 * dot(gamma.as<double>(), gamma.as<double>(), p.ldb, s);
  if (F) {
    J.alloc(nn * sizeof(double));
    j_from_gamma(p, gamma.as<double>(), J.as<double>(), s);
    for (int sp = 0; sp < nspin; ++sp)
      DFJK_CUDA(cudaMemcpyAsync(F + sp * nn, J.p, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
  }
  if (hf != 0.0 || hf_lr != 0.0) {
    DevBuf K, Ct, dw;
    K.alloc(nn * sizeof(double));
    for (int sp = 0; sp < nspin; ++sp) {
      const double* Ps = P + sp * nn;
      density_factor(p, Ps, Ct, dw, s);
      const struct { Plan* plan; double coeff; } terms[2] = {{&p, hf},
                                                             {p.lr ? &p.lr->p : nullptr, hf_lr}};
      for (const auto& t : terms) {
        if (t.coeff == 0.0) continue;
        k_compute(*t.plan, Ct.as<double>(), dw.as<double>(), n, K.as<double>(), s);
        const double tr = dot(Ps, K.as<double>(), nn, s);
        // exchange quadratic (terms.py:500-509)
        e += (nspin == 1 ? -0.25 : -0.5) * t.coeff * tr;
        if (F) {
          const double a = (nspin == 1 ? -0.5 : -1.0) * t.coeff;
          axpy_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(K.as<double>(), a, nn,
                                                                    F + sp * nn);
          DFJK_LAUNCHED();
        }
      }
    }
  }
  DFJK_CUDA(cudaStreamSynchronize(s));
  return e;
}

}  // namespace dfjk

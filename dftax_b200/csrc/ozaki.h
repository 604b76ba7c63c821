// Exact-accumulation int8 tensor-core GEMM (tcgen05 kind::i8) for the
// mixed-precision products of the DF path.
#pragma once

#include <cuda.h>

#include "internal.h"

namespace dfjk {

constexpr int kOzKDigits = 4;      // K half transform: 2^-32 of each row's scale
constexpr int kOzBDigits = 5;      // B = (ij|P) L, mixed precision: 2^-40 (see ozaki.cu)
constexpr int kOzB64Digits = 7;    // B = (ij|P) L, float64 plans: 2^-56 of each row's scale
constexpr int kOzSDigits = 5;      // K = X X^T: 2^-40
constexpr int kOzMaxDigits = 7;
// longest exact dot product: 5 digits, order 4 sums 2*65*128 + 3*128*128 per k
constexpr int64_t kOzMaxK = 32640;
// 7 digits: order 6 sums 2*65*128 + 5*128*128 = 98560 per k, below 2^31 for k <= 21788
constexpr int64_t kOzMaxK7 = 21788;
constexpr int64_t kOzSlice = 8192;  // k bytes per slice of the K = X X^T product

// The products and the tile shape each one runs with (ozaki_gemm.cu).
// kOzHalfWide: the half transform with 96 occupied columns per tile, used when
// it needs fewer tiles than 80 columns would (each tile streams every B_x plane)
// kOzBuild64: the build product of float64 plans, 7 digits on SM pairs
enum OzakiShape { kOzBuild = 0, kOzHalf = 1, kOzSyrk = 2, kOzHalfWide = 3, kOzBuild64 = 4 };

// digits per value of the build product B = (ij|P) L of a plan
inline int build_digits(const Plan& p) {
  return p.opts.precision == DFJK_MIXED ? kOzBDigits : kOzB64Digits;
}
struct OzakiShapeInfo {
  int digits, box_k, bn, stages;   // digits per value, k tile bytes, n tile, ring depth
  int box_b;                       // B rows per copy: bn, or bn / 2 on SM pairs
};
OzakiShapeInfo ozaki_shape(OzakiShape shape);

struct OzakiMaps {
  CUtensorMap a[kOzMaxDigits];   // A digit planes, box (box_k, 128 rows, 1)
  CUtensorMap b[kOzMaxDigits];   // B digit planes, box (box_k, box_b rows, 1)
  CUtensorMap out;               // float64 output when tma_out: box (16, 1, 32), 128-byte swizzle
};

struct OzakiArgs {
  int M, N;                // output extent (rows of A, rows of B)
  int ktiles;              // k tiles of the shape's box_k bytes
  int plane0;              // A plane of blockIdx.z == 0
  const int* ea;           // exponent per A row: ea[(plane0 + z) * ea_stride + row]
  int64_t ea_stride;
  const int* eb;           // exponent per B row: eb[(b_batched ? plane0 + z : 0) * eb_stride + col]
  int64_t eb_stride;
  int b_batched;           // 1: B planes and exponents follow blockIdx.z like A's
  double* out;             // out[z * batch_stride + row * ld + col]
  int64_t ld_out, batch_stride_out;
  int* err;                // set non-zero when a bounded wait gives up
  int zper;                // batches per CTA (one TMEM allocation, one ring); 0 or 1: one
  int zcount;              // batches of the launch (set by ozaki_launch)
  int tma_out;             // half transform: 1 writes through maps.out (the build product always does)
  int lower;               // 1: tiles wholly above the diagonal (n0 > m0 + 127) are skipped
};

// 3-D int8 tensor map over [d2][d1][d0] (d0 contiguous; strides in bytes),
// box (box_k, box1, 1) with the swizzle that matches box_k
void ozaki_map(CUtensorMap* m, const void* base, int64_t d0, int64_t d1, int64_t d2,
               int64_t stride1, int64_t stride2, int box_k, int box1);

// float64 output map over [rows][batches][cols] (strides in elements), and
// whether a base and strides allow one (16-byte alignment)
bool ozaki_out_mappable(const double* base, int64_t batch_stride, int64_t ld);
void ozaki_map_out(CUtensorMap* m, double* base, int64_t cols, int64_t batches, int64_t rows,
                   int64_t batch_stride, int64_t ld);

// grid (ceil(N/bn), ceil(M/128), ceil(nbatch / a.zper)): nbatch batches (grid_z);
// the build product: clusters of two CTAs, grid (2 ceil(N/bn), ceil(M/256)), one batch
void ozaki_launch(OzakiShape shape, const OzakiMaps& maps, const OzakiArgs& a, int grid_z,
                  cudaStream_t s);

// The bounded wait of the tensor-core pipelines, made to run out: one block
// waits limit_ns on a barrier nothing completes (a second warp with the
// pipelines' own 4 s limit returns when the first one's timeout is flagged);
// fails with the pipelines' timeout error. waited_ms[0..1]: each warp's wait.
constexpr int kWaitSelftestCode = 90;
void wait_selftest(const Context& c, int64_t limit_ns, double* waited_ms, cudaStream_t s);

}  // namespace dfjk

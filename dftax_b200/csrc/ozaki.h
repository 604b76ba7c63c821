// Exact-accumulation int8 tensor-core GEMM (tcgen05 kind::i8) for the
// mixed-precision products of the DF path.
#pragma once

#include <cuda.h>

#include "internal.h"

namespace dfjk {

constexpr int kOzBN = 80;          // n tile
constexpr int kOzKDigits = 4;      // K half transform: 28 bits per value
constexpr int kOzBDigits = 6;      // B = (ij|P) L: 42 bits per value (see ozaki.cu)
constexpr int kOzSDigits = 5;      // K = X X^T: 35 bits per value
constexpr int kOzMaxDigits = 6;
constexpr int64_t kOzSlice = 8192;  // k bytes per slice of the K = X X^T product

struct OzakiMaps {
  CUtensorMap a[kOzMaxDigits];   // A digit planes, box (k tile bytes, 128 rows, 1)
  CUtensorMap b[kOzMaxDigits];   // B digit planes, box (k tile bytes, kOzBN rows, 1)
};

struct OzakiArgs {
  int M, N;                // output extent (rows of A, rows of B)
  int ktiles;              // k tiles of ozaki_box_k(ndig) bytes
  int plane0;              // A plane of blockIdx.z == 0
  const int* ea;           // exponent per A row: ea[(plane0 + z) * ea_stride + row]
  int64_t ea_stride;
  const int* eb;           // exponent per B row: eb[(b_batched ? plane0 + z : 0) * eb_stride + col]
  int64_t eb_stride;
  int b_batched;           // 1: B planes and exponents follow blockIdx.z like A's
  double* out;             // out[z * batch_stride + row * ld + col]
  int64_t ld_out, batch_stride_out;
  int* err;                // set non-zero when a bounded wait gives up
};

// k tile (bytes) of the kernel that runs ndig digits per value: 128 (4 digits,
// 128-byte swizzle) or 64 (5 and 6 digits, 64-byte swizzle)
int ozaki_box_k(int ndig);

// 3-D int8 tensor map over [d2][d1][d0] (d0 contiguous; strides in bytes),
// box (box_k, box1, 1) with the swizzle that matches box_k
void ozaki_map(CUtensorMap* m, const void* base, int64_t d0, int64_t d1, int64_t d2,
               int64_t stride1, int64_t stride2, int box_k, int box1);

// grid (ceil(N/kOzBN), ceil(M/128), grid_z); ndig is 4, 5 or 6
void ozaki_launch(int ndig, const OzakiMaps& maps, const OzakiArgs& a, int grid_z, cudaStream_t s);

}  // namespace dfjk

// Exact-accumulation int8 tensor-core GEMM (tcgen05 kind::i8) for the
// mixed-precision K half transform.
#pragma once

#include <cuda.h>

#include "internal.h"

namespace dfjk {

constexpr int kOzDigits = 4;     // signed 7-bit digits per value (28 bits)
constexpr int kOzBN = 80;        // n tile (occupied orbitals)

struct OzakiMaps {
  CUtensorMap a[kOzDigits];   // A digit planes, box (128 k, 128 rows, 1)
  CUtensorMap b[kOzDigits];   // B digit planes, box (128 k, kOzBN rows, 1)
};

struct OzakiArgs {
  int M, N;                // output extent (rows of A, rows of B)
  int ktiles;              // k tiles of 128
  int plane0;              // A plane of blockIdx.z == 0
  const int* ea;           // exponent per A row: ea[(plane0 + z) * ea_stride + row]
  int64_t ea_stride;
  const int* eb;           // exponent per B row
  double* out;             // out[z * batch_stride + row * ld + col]
  int64_t ld_out, batch_stride_out;
  int* err;                // set non-zero when a bounded wait gives up
};

// 3-D int8 tensor map over [d2][d1][d0] (d0 contiguous; strides in bytes)
void ozaki_map(CUtensorMap* m, const void* base, int64_t d0, int64_t d1, int64_t d2,
               int64_t stride1, int64_t stride2, int box1);

// grid (ceil(N/kOzBN), ceil(M/128), grid_z)
void ozaki_launch(const OzakiMaps& maps, const OzakiArgs& a, int grid_z, cudaStream_t s);

}  // namespace dfjk

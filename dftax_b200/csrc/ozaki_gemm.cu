// Exact-accumulation int8 GEMM on the 5th-generation tensor cores.
//
//   D[m][n] = 2^(ea[m] + eb[n]) * sum_k a[m][k] b[n][k]
// where every value is stored as four signed 7-bit digits under its row's
// exponent: a = 2^ea * sum_s d_s 2^(-7(s+1)), |d_s| <= 64 (Ozaki-style
// splitting). The ten digit products of combined order o = s + t <= 3 are
// accumulated EXACTLY in int32 (kind::i8 MMA), one tensor-memory accumulator
// per order; the epilogue combines them in float64 with weights 2^(-7(o+2)).
// The only error is the truncation of the digit expansion (2^-27 of the row
// maximum); unlike fp32 accumulation there is no rounding drift with k.
// (Float32 accumulation of split-bf16 products was measured to bias K toward
// zero by ~1e-6 per 24 MMAs, growing with the k length; that path was dropped.)
//
// Tiles: 128 (m) x 80 (n) x 128 (k, bytes), K-major operands, TMA with the
// 128-byte swizzle into a 2-stage mbarrier ring (4 digit planes per operand
// per stage, 104 KB). Warp 0 lane 0 issues copies, warp 1 lane 0 issues MMAs
// (4 per k tile per digit pair), all four warps drain tensor memory
// (warp w owns rows 32w..32w+31). Every wait is bounded (4 s of
// %globaltimer); a timeout sets *err, skips the remaining work, drains the
// copies in flight (bounded) and still frees the tensor memory.
#include "ozaki.h"

#include <mutex>

namespace dfjk {

namespace {

constexpr int kBM = 128, kBK = 128, kStages = 2, kD = kOzDigits, kBN = kOzBN;
constexpr uint32_t kTmemCols = 512;        // 4 order accumulators at 128-column stride
constexpr unsigned long long kWaitNs = 4000000000ull;

__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool mbar_try(uint32_t addr, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(addr), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity, int* err, int code) {
  if (mbar_try(addr, parity)) return true;
  const uint64_t t0 = now_ns();
  while (true) {
    if (mbar_try(addr, parity)) return true;
    if (*reinterpret_cast<volatile int*>(err) != 0) return false;
    if (now_ns() - t0 > kWaitNs) {
      atomicCAS(err, 0, code);
      return false;
    }
    __nanosleep(64);
  }
}

__device__ __forceinline__ void mbar_init(uint32_t addr, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(addr), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t addr, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(addr), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, uint32_t mbar,
                                            int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(mbar), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

// K-major, 128-byte swizzle: 8-row atoms of 1024 B (SBO), 16 B leading
// offset, descriptor version 1 (sm_100)
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                        uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   mbar)
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = (int)r[i];
}

__global__ void __launch_bounds__(128, 1) ozaki_gemm_i8(const __grid_constant__ OzakiMaps maps,
                                                        OzakiArgs a) {
  constexpr uint32_t A_TILE = kBM * kBK;   // 16 KB
  constexpr uint32_t B_TILE = kBN * kBK;   // 10 KB
  constexpr uint32_t STAGE = kD * (A_TILE + B_TILE);
  // S32 accumulator (c_format 2), signed int8 A and B (format 1), N>>3, M>>4
  constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kBN >> 3) << 17) |
                             ((uint32_t)(kBM >> 4) << 24);
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kStages * STAGE);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n0 = blockIdx.x * kBN, m0 = blockIdx.y * kBM, z = blockIdx.z;
  const int nk = a.ktiles;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(smem_u32(&bars[s]), 1);
      mbar_init(smem_u32(&bars[kStages + s]), 1);
    }
    mbar_init(smem_u32(&bars[2 * kStages]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (threadIdx.x == 0 && nk > 0) {
    int issued = 0;
    bool ok = true;
    for (int i = 0; i < nk && ok; ++i) {
      const int s = i % kStages;
      if (i >= kStages) ok = mbar_wait(smem_u32(&bars[kStages + s]), ((i / kStages) - 1) & 1, a.err, 1);
      if (!ok) break;
      const uint32_t full = smem_u32(&bars[s]);
      mbar_expect_tx(full, STAGE);
      uint8_t* st = smem + s * STAGE;
#pragma unroll
      for (int d = 0; d < kD; ++d) {
        tma_load_3d(smem_u32(st + d * A_TILE), &maps.a[d], full, i * kBK, m0, a.plane0 + z);
        tma_load_3d(smem_u32(st + kD * A_TILE + d * B_TILE), &maps.b[d], full, i * kBK, n0, 0);
      }
      ++issued;
    }
    if (!ok) {
      for (int i = issued - kStages > 0 ? issued - kStages : 0; i < issued; ++i) {
        const uint64_t t0 = now_ns();
        while (!mbar_try(smem_u32(&bars[i % kStages]), (i / kStages) & 1) && now_ns() - t0 < kWaitNs)
          __nanosleep(64);
      }
    }
  } else if (threadIdx.x == 32 && nk > 0) {
    bool ok = true;
    // digit pairs (s, t) with s + t <= 3, and their order accumulator
    const int pa[10] = {0, 0, 1, 0, 1, 2, 0, 1, 2, 3};
    const int pb[10] = {0, 1, 0, 2, 1, 0, 3, 2, 1, 0};
    const int po[10] = {0, 1, 1, 2, 2, 2, 3, 3, 3, 3};
    const int first[10] = {1, 1, 0, 1, 0, 0, 1, 0, 0, 0};   // first pair of its order
    for (int i = 0; i < nk; ++i) {
      const int s = i % kStages;
      ok = mbar_wait(smem_u32(&bars[s]), (i / kStages) & 1, a.err, 2);
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t base = smem_u32(smem + s * STAGE);
      const uint32_t bbase = base + kD * A_TILE;
#pragma unroll
      for (int t = 0; t < 10; ++t) {
        const uint64_t ad = sw128_desc(base + pa[t] * A_TILE);
        const uint64_t bd = sw128_desc(bbase + pb[t] * B_TILE);
        const uint32_t dcol = tmem + (uint32_t)(po[t] * 128);
#pragma unroll
        for (int k = 0; k < kBK / 32; ++k)
          umma_i8(dcol, ad + (uint64_t)(2 * k), bd + (uint64_t)(2 * k), IDESC,
                  (i > 0 || !first[t] || k > 0) ? 1u : 0u);
      }
      umma_commit(smem_u32(&bars[kStages + s]));
    }
    if (ok) umma_commit(smem_u32(&bars[2 * kStages]));
  }
  __syncwarp();

  bool have = nk > 0 && mbar_wait(smem_u32(&bars[2 * kStages]), 0, a.err, 3);
  have = __all_sync(0xffffffffu, have);   // tcgen05.ld is warp-collective
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (have) {
    const int row = m0 + warp * 32 + lane;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    const int era = row < a.M ? a.ea[(int64_t)(a.plane0 + z) * a.ea_stride + row] : 0;
    double* orow = a.out + (int64_t)z * a.batch_stride_out + (int64_t)row * a.ld_out;
    for (int c = 0; c < kBN; c += 16) {
      int v0[16], v1[16], v2[16], v3[16];
      tmem_ld16(trow + c, v0);
      tmem_ld16(trow + 128 + c, v1);
      tmem_ld16(trow + 256 + c, v2);
      tmem_ld16(trow + 384 + c, v3);
      if (row >= a.M) continue;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int col = n0 + c + j;
        if (col >= a.N) break;
        // sum_o acc_o 2^(-7(o+2)), exact in float64 up to the final rounding
        const double v = (double)v0[j] * 0x1p-14 + (double)v1[j] * 0x1p-21 +
                         (double)v2[j] * 0x1p-28 + (double)v3[j] * 0x1p-35;
        orow[col] = ldexp(v, era + a.eb[col]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                 : "memory");
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                 CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                 CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static EncodeTiled fn = nullptr;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    DFJK_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (!p || q != cudaDriverEntryPointSuccess)
      fail(DFJK_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    fn = reinterpret_cast<EncodeTiled>(p);
  }
  return fn;
}

constexpr size_t kSmem = kStages * (size_t)kD * (kBM * kBK + kBN * kBK) + 1024 + 256;

}  // namespace

void ozaki_map(CUtensorMap* m, const void* base, int64_t d0, int64_t d1, int64_t d2,
               int64_t stride1, int64_t stride2, int box1) {
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (stride1 % 16) || (stride2 % 16))
    fail(DFJK_ERR_INVALID, "tensor map: base or strides not 16-byte aligned");
  cuuint64_t dims[3] = {(cuuint64_t)d0, (cuuint64_t)d1, (cuuint64_t)d2};
  cuuint64_t strides[2] = {(cuuint64_t)stride1, (cuuint64_t)stride2};
  cuuint32_t box[3] = {(cuuint32_t)kBK, (cuuint32_t)box1, 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = encode_fn()(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims,
                           strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(DFJK_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
}

void ozaki_launch(const OzakiMaps& maps, const OzakiArgs& a, int grid_z, cudaStream_t s) {
  if (grid_z <= 0 || a.M <= 0 || a.N <= 0) return;
  dim3 grid((a.N + kBN - 1) / kBN, (a.M + kBM - 1) / kBM, grid_z);
  DFJK_CUDA(cudaFuncSetAttribute(ozaki_gemm_i8, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSmem));
  ozaki_gemm_i8<<<grid, 128, kSmem, s>>>(maps, a);
  DFJK_LAUNCHED();
}

}  // namespace dfjk

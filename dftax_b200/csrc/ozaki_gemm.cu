// Exact-accumulation int8 GEMM on the 5th-generation tensor cores.
//
//   D[m][n] = 2^(ea[m] + eb[n]) * sum_k a[m][k] b[n][k]
// where every value is stored as ND signed int8 digits under its row's
// exponent (Ozaki-style splitting): a = 2^ea * (d_0 2^-7 + sum_(s>=1) d_s
// 2^-(7+8s)), a 7-bit leading digit and balanced 8-bit digits after it. Digit
// s times digit t weighs 2^-(14+8(s+t)), so the ND(ND+1)/2 products of
// combined order o = s + t < ND are accumulated EXACTLY in int32 (kind::i8
// MMA), one tensor-memory accumulator per order, and the epilogue combines
// them in float64 with weights 2^-(14+8o). Exactness needs k * (sum over an
// order of |d_s d_t|) < 2^31: k <= kOzMaxK. The only error is the truncation
// of the digit expansion (2^-(8 ND) of 2^e, at most 2^(2-8ND) of the row
// maximum); unlike fp32 accumulation there is no rounding drift with k. (Float32 accumulation of split-bf16 products was
// measured to bias K toward zero by ~1e-6 per 24 MMAs, growing with the k
// length; that path was dropped.)
//
// Tiles: 128 (m) x BN (n) x BK (k, bytes), K-major operands, TMA with the
// BK-byte swizzle into an ST-stage mbarrier ring (ND digit planes per operand
// per stage). Two shapes are compiled: ND 4, BK 128, BN 80, two 104 KB stages
// (K half transform: n = occupied orbitals, 160 = 2 x 80 for (H2O)_32), and
// ND 5, BK 64, BN 96, three 70 KB stages (build product and K = X X^T;
// 5 x 96 of the 512 TMEM columns). Warp 0 lane 0 issues
// copies, warp 1 lane 0 issues MMAs (BK/32 per digit pair per k tile), all
// four warps drain tensor memory (warp w owns rows 32w..32w+31). Every wait
// is bounded (4 s of %globaltimer); a timeout sets *err, skips the remaining
// work, drains the copies in flight (bounded) and still frees the tensor
// memory.
#include "ozaki.h"

#include <mutex>

namespace dfjk {

namespace {

constexpr int kBM = 128;
constexpr uint32_t kTmemCols = 512;
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

// K-major shared-memory descriptor (sm_100, version 1) for BK-byte rows with
// the BK-byte swizzle: 8-row atoms of 8 * BK bytes (SBO), leading offset
// unused (1); layout type 2 = 128-byte swizzle, 4 = 64-byte swizzle
template <int BK>
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t saddr) {
  static_assert(BK == 128 || BK == 64, "k tile must be 64 or 128 bytes");
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)((8 * BK) >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)(BK == 128 ? 2 : 4) << 61;
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

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int* v) {
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

template <int ND, int BK, int BN, int ST>
__global__ void __launch_bounds__(192, 1) ozaki_gemm_i8(const __grid_constant__ OzakiMaps maps,
                                                        OzakiArgs a) {
  constexpr uint32_t A_TILE = kBM * BK;
  constexpr uint32_t B_TILE = BN * BK;
  constexpr uint32_t STAGE = ND * (A_TILE + B_TILE);
  constexpr int KSTEPS = BK / 32;   // one kind::i8 MMA covers 32 bytes of k
  // accumulator o at column o * ACC (128 when they fit, else packed at BN)
  constexpr uint32_t ACC = (ND * 128 <= (int)kTmemCols) ? 128 : BN;
  static_assert(ND * ACC <= kTmemCols, "order accumulators exceed tensor memory");
  static_assert(A_TILE % 1024 == 0 && B_TILE % 1024 == 0, "tiles must keep 1 KB alignment");
  // S32 accumulator (c_format 2), signed int8 A and B (format 1), N>>3, M>>4
  constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                             ((uint32_t)(kBM >> 4) << 24);
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  // barriers: full[ST], empty[ST], done (accumulators of a batch final),
  // drained (the epilogue warps have read them)
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + ST * STAGE);
  uint64_t* empty = full + ST;
  uint64_t* done = empty + ST;
  uint64_t* drained = done + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drained + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n0 = blockIdx.x * BN, m0 = blockIdx.y * kBM;
  const int nk = a.ktiles;
  const int zper = a.zper > 0 ? a.zper : 1;
  const int z0 = blockIdx.z * zper;
  const int nz = (a.zcount - z0) < zper ? (a.zcount - z0) : zper;   // batches of this CTA

  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    mbar_init(smem_u32(done), 1);
    mbar_init(smem_u32(drained), 4);
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
    // producer: the k tiles of every batch of this CTA through one ring
    int issued = 0;
    bool ok = true;
    for (int zi = 0; zi < nz && ok; ++zi) {
      const int z = z0 + zi;
      const int bz = a.b_batched ? a.plane0 + z : 0;
      for (int i = 0; i < nk; ++i, ++issued) {
        const int s = issued % ST;
        if (issued >= ST) ok = mbar_wait(smem_u32(&empty[s]), ((issued / ST) - 1) & 1, a.err, 1);
        if (!ok) break;
        const uint32_t fb = smem_u32(&full[s]);
        mbar_expect_tx(fb, STAGE);
        uint8_t* st = smem + s * STAGE;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
          tma_load_3d(smem_u32(st + d * A_TILE), &maps.a[d], fb, i * BK, m0, a.plane0 + z);
          tma_load_3d(smem_u32(st + ND * A_TILE + d * B_TILE), &maps.b[d], fb, i * BK, n0, bz);
        }
      }
    }
    if (!ok) {
      for (int q = issued - ST > 0 ? issued - ST : 0; q < issued; ++q) {
        const uint64_t t0 = now_ns();
        while (!mbar_try(smem_u32(&full[q % ST]), (q / ST) & 1) && now_ns() - t0 < kWaitNs)
          __nanosleep(64);
      }
    }
  } else if (threadIdx.x == 32 && nk > 0) {
    // MMA issuer: one accumulator set per batch, reused once the epilogue drained it
    bool ok = true;
    int it = 0;
    for (int zi = 0; zi < nz && ok; ++zi) {
      if (zi > 0) ok = mbar_wait(smem_u32(drained), (zi - 1) & 1, a.err, 4);
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int i = 0; i < nk; ++i, ++it) {
        const int s = it % ST;
        ok = mbar_wait(smem_u32(&full[s]), (it / ST) & 1, a.err, 2);
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t base = smem_u32(smem + s * STAGE);
        const uint32_t bbase = base + ND * A_TILE;
        // digit pairs (sa, o - sa) of order o into accumulator o
#pragma unroll
        for (int o = 0; o < ND; ++o) {
          const uint32_t dcol = tmem + (uint32_t)o * ACC;
#pragma unroll
          for (int sa = 0; sa <= o; ++sa) {
            const uint64_t ad = kmajor_desc<BK>(base + sa * A_TILE);
            const uint64_t bd = kmajor_desc<BK>(bbase + (o - sa) * B_TILE);
#pragma unroll
            for (int k = 0; k < KSTEPS; ++k)
              umma_i8(dcol, ad + (uint64_t)(2 * k), bd + (uint64_t)(2 * k), IDESC,
                      (i > 0 || sa > 0 || k > 0) ? 1u : 0u);
          }
        }
        umma_commit(smem_u32(&empty[s]));
      }
      // also after a failed wait: done then tracks the MMAs already issued,
      // so tensor memory is not read or freed under them
      umma_commit(smem_u32(done));
    }
  } else if (warp >= 2) {
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31
    const int q = warp & 3;
    const int row = m0 + q * 32 + lane;
    const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16);
    for (int zi = 0; zi < nz && nk > 0; ++zi) {
      const int z = z0 + zi;
      bool have = false;
      // bounded by time only: the MMAs must be finished before TMEM is read or freed
      const uint64_t t0 = now_ns();
      while (!(have = mbar_try(smem_u32(done), zi & 1))) {
        if (now_ns() - t0 > kWaitNs) {
          atomicCAS(a.err, 0, 3);
          break;
        }
        __nanosleep(64);
      }
      have = have && *reinterpret_cast<volatile int*>(a.err) == 0;
      have = __all_sync(0xffffffffu, have);   // tcgen05.ld is warp-collective
      if (!have) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int bz = a.b_batched ? a.plane0 + z : 0;
      const int era = row < a.M ? a.ea[(int64_t)(a.plane0 + z) * a.ea_stride + row] : 0;
      double* orow = a.out + (int64_t)z * a.batch_stride_out + (int64_t)row * a.ld_out;
      const int* ebz = a.eb + (int64_t)bz * a.eb_stride;
      for (int c = 0; c < BN; c += 16) {
        int v[ND][16];
#pragma unroll
        for (int o = 0; o < ND; ++o) tmem_ld16(trow + (uint32_t)o * ACC + c, v[o]);
        if (row >= a.M) continue;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = n0 + c + j;
          if (col >= a.N) break;
          // sum_o acc_o 2^-(14+8o), highest order first
          double t = 0.0;
#pragma unroll
          for (int o = ND - 1; o >= 0; --o) t = t * 0x1p-8 + (double)v[o][j];
          orow[col] = ldexp(t, era + ebz[col] - 14);
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(drained)) : "memory");
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

template <int ND, int BK, int BN, int ST>
constexpr size_t smem_bytes() {
  return (size_t)ST * ND * (kBM * BK + BN * BK) + 1024 + 256;
}

template <int ND, int BK, int BN, int ST>
void launch(const OzakiMaps& maps, const OzakiArgs& a, int grid_z, cudaStream_t s) {
  constexpr size_t smem = smem_bytes<ND, BK, BN, ST>();
  static_assert(smem <= 232448, "stages exceed the shared memory of one CTA");
  OzakiArgs b = a;
  b.zcount = grid_z;
  if (b.zper < 1) b.zper = 1;
  dim3 grid((a.N + BN - 1) / BN, (a.M + kBM - 1) / kBM, (grid_z + b.zper - 1) / b.zper);
  DFJK_CUDA(cudaFuncSetAttribute(ozaki_gemm_i8<ND, BK, BN, ST>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  ozaki_gemm_i8<ND, BK, BN, ST><<<grid, 192, smem, s>>>(maps, b);
  DFJK_LAUNCHED();
}

}  // namespace

// digits, k tile bytes, n tile, stages of each product (see ozaki.h)
OzakiShapeInfo ozaki_shape(OzakiShape shape) {
  switch (shape) {
    case kOzHalf: return {kOzKDigits, 128, 80, 2};
    case kOzBuild: return {kOzBDigits, 64, 96, 3};
    case kOzSyrk: return {kOzSDigits, 64, 96, 3};
  }
  fail(DFJK_ERR_INVALID, "unknown int8 GEMM shape %d", (int)shape);
}

void ozaki_map(CUtensorMap* m, const void* base, int64_t d0, int64_t d1, int64_t d2,
               int64_t stride1, int64_t stride2, int box_k, int box1) {
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (stride1 % 16) || (stride2 % 16))
    fail(DFJK_ERR_INVALID, "tensor map: base or strides not 16-byte aligned");
  if (box_k != 64 && box_k != 128) fail(DFJK_ERR_INVALID, "tensor map: k box must be 64 or 128");
  cuuint64_t dims[3] = {(cuuint64_t)d0, (cuuint64_t)d1, (cuuint64_t)d2};
  cuuint64_t strides[2] = {(cuuint64_t)stride1, (cuuint64_t)stride2};
  cuuint32_t box[3] = {(cuuint32_t)box_k, (cuuint32_t)box1, 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = encode_fn()(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims,
                           strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           box_k == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(DFJK_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
}

void ozaki_launch(OzakiShape shape, const OzakiMaps& maps, const OzakiArgs& a, int grid_z,
                  cudaStream_t s) {
  if (grid_z <= 0 || a.M <= 0 || a.N <= 0) return;
  static_assert(kOzKDigits == 4 && kOzBDigits == 5 && kOzSDigits == 5,
                "the compiled shapes follow the digit counts");
  switch (shape) {
    case kOzHalf: launch<4, 128, 80, 2>(maps, a, grid_z, s); return;
    case kOzBuild:
    case kOzSyrk: launch<5, 64, 96, 3>(maps, a, grid_z, s); return;
  }
  fail(DFJK_ERR_INVALID, "unknown int8 GEMM shape %d", (int)shape);
}

}  // namespace dfjk

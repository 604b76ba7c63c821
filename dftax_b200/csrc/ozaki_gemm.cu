// Exact-accumulation int8 GEMM on the 5th-generation tensor cores.
//
//   D[m][n] = 2^(ea[m] + eb[n]) * sum_k a[m][k] b[n][k]
// where every value is stored as ND signed int8 digits under its row's
// exponent (Ozaki-style splitting): a = 2^ea * (d_0 2^-7 + sum_(s>=1) d_s
// 2^-(7+8s)), a 7-bit leading digit and balanced 8-bit digits after it. Digit
// s times digit t weighs 2^-(14+8(s+t)), so the ND(ND+1)/2 products of
// combined order o = s + t < ND are accumulated EXACTLY in int32 (kind::i8
// MMA), one tensor-memory accumulator per order, and the epilogue combines
// them exactly in int64 with weights 2^-(14+8o) before one rounding to
// float64. Exactness needs k * (sum over an
// order of |d_s d_t|) < 2^31: k <= kOzMaxK. The only error is the truncation
// of the digit expansion (2^-(8 ND) of 2^e, at most 2^(2-8ND) of the row
// maximum); unlike fp32 accumulation there is no rounding drift with k. (Float32 accumulation of split-bf16 products was
// measured to bias K toward zero by ~1e-6 per 24 MMAs, growing with the k
// length; that path was dropped.)
//
// Tiles: 128 (m) x BN (n) x BK (k, bytes), K-major operands, TMA with the
// BK-byte swizzle into an ST-stage mbarrier ring (ND digit planes per operand
// per stage). Two shapes are compiled: ND 4, BK 64, BN 80, three 52 KB stages
// and 64 KB of output staging for TMA stores (K half transform: n = occupied
// orbitals, 160 = 2 x 80 for (H2O)_32), and
// ND 5, BK 64, BN 96, three 70 KB stages (K = X X^T; 5 x 96 of the 512 TMEM
// columns). The build product runs on SM pairs (ozaki_gemm_i8_pair below,
// M = 256, four 55 KB stages). Warp 0 lane 0 issues
// copies, warp 1 lane 0 issues MMAs (BK/32 per digit pair per k tile), and
// eight warps drain tensor memory (warps w and w + 4 own rows 32 (w % 4) ..
// + 31, alternate 16-column chunks each). Every wait
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

__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity, int* err, int code,
                                          unsigned long long limit_ns = kWaitNs) {
  if (mbar_try(addr, parity)) return true;
  const uint64_t t0 = now_ns();
  while (true) {
    if (mbar_try(addr, parity)) return true;
    if (*reinterpret_cast<volatile int*>(err) != 0) return false;
    if (now_ns() - t0 > limit_ns) {
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

__device__ __forceinline__ void tmem_ld16_issue(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// keeps every use of r after the preceding tcgen05.wait::ld
__device__ __forceinline__ void reg_fence16(uint32_t* r) {
  asm volatile(""
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                 "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
               :
               : "memory");
}

// sum_o acc_o 2^-(14+8o) 2^e: the orders combine exactly in int64 (order 0
// is below 2^28 and order 1 below 2^30 for k <= kOzMaxK, so the sum stays
// below 2^60) and round once to float64; 5 int-to-float64 conversions and 4
// float64 FMAs per value made the epilogue the slowest part of a tile
// x 2^e: a multiply by the power of two while 2^e is a normal double (the
// product rounds as ldexp's result does), ldexp beyond; ldexp itself per
// value cost more than the rest of the epilogue arithmetic
__device__ __forceinline__ double scale_pow2(double x, int e) {
  if (e >= -1022 && e <= 1023) return x * __longlong_as_double((long long)(e + 1023) << 52);
  return ldexp(x, e);
}

// Past 5 digits the int64 sum would overflow (order 0 times 2^48 for 7
// digits): orders 0-3 and orders 4.. are summed apart in int64, each below
// 2^53 and so exact as a float64 (order 0 < 2^28, the others < 2^31), and one
// FMA joins them with a single rounding.
template <int ND>
__device__ __forceinline__ double combine_orders(const uint32_t (&v)[ND][16], int j, int e) {
  if constexpr (ND <= 5) {
    long long s = (int)v[0][j];
#pragma unroll
    for (int o = 1; o < ND; ++o) s = s * 256 + (int)v[o][j];
    return scale_pow2((double)s, e - 14 - 8 * (ND - 1));
  } else {
    static_assert(ND <= 8, "the low part holds at most four orders");
    long long hi = (int)v[0][j];
#pragma unroll
    for (int o = 1; o < 4; ++o) hi = hi * 256 + (int)v[o][j];
    long long lo = (int)v[4][j];
#pragma unroll
    for (int o = 5; o < ND; ++o) lo = lo * 256 + (int)v[o][j];
    constexpr double kLoScale = (double)(1LL << (8 * (ND - 4)));
    return scale_pow2(fma((double)hi, kLoScale, (double)lo), e - 14 - 8 * (ND - 1));
  }
}

__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, uint32_t src, int c0, int c1,
                                             int c2) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(src), "r"(c0), "r"(c1), "r"(c2)
               : "memory");
}

// one lane's 128-byte row of a 32 x 16 float64 block in shared memory, in the
// 128-byte swizzle of the output tensor maps (16-byte chunk j at j ^ (row % 8))
template <int ND>
__device__ __forceinline__ void stage_row(uint8_t* buf, int lane, const uint32_t (&v)[ND][16],
                                          int era, const int* ecol) {
#pragma unroll
  for (int j = 0; j < 16; j += 2) {
    const double r0 = combine_orders<ND>(v, j, era + ecol[j]);
    const double r1 = combine_orders<ND>(v, j + 1, era + ecol[j + 1]);
    *reinterpret_cast<double2*>(buf + lane * 128 + (((j >> 1) ^ (lane & 7)) << 4)) =
        make_double2(r0, r1);
  }
}

template <int ND, int BK, int BN, int ST, bool TOUT>
__global__ void __launch_bounds__(320, 1) ozaki_gemm_i8(const __grid_constant__ OzakiMaps maps,
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
  // TOUT: per epilogue warp two 32 x 16 float64 staging blocks after the ring
  // (outputs leave through maps.out); barriers: full[ST], empty[ST], done
  // (accumulators of a batch final), drained (the epilogue warps have read them)
  constexpr uint32_t STG_BYTES = TOUT ? 8 * 2 * 4096 : 0;
  static_assert(BN % 16 == 0, "16-column epilogue chunks");
  uint8_t* stg = smem + ST * STAGE;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + ST * STAGE + STG_BYTES);
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
  // a symmetric product needs only the tiles that reach the lower triangle;
  // the whole CTA leaves before any barrier or tensor memory is set up
  if (a.lower && n0 > m0 + kBM - 1) return;

  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    mbar_init(smem_u32(done), 1);
    mbar_init(smem_u32(drained), 8);
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
    // epilogue, eight warps: warp w reads TMEM lanes 32 (w % 4) .. + 31 and
    // the 16-column chunks h, h + 2, ... of them, h = (w - 2) / 4
    const int q = warp & 3, h = (warp - 2) >> 2;
    const int row0 = m0 + q * 32, row = row0 + lane;
    const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16);
    int nst = 0;   // TOUT: blocks this warp has handed to TMA (double buffer index)
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
      for (int c = 16 * h; c < BN; c += 32) {
        uint32_t v[ND][16];
#pragma unroll
        for (int o = 0; o < ND; ++o) tmem_ld16_issue(trow + (uint32_t)o * ACC + c, v[o]);
        tmem_ld_wait();
#pragma unroll
        for (int o = 0; o < ND; ++o) reg_fence16(v[o]);
        if constexpr (TOUT) {
          // columns past N read exponent 0; the tensor map clips them and rows past M
          int ecol[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) ecol[j] = n0 + c + j < a.N ? ebz[n0 + c + j] : 0;
          uint8_t* buf = stg + (uint32_t)((warp - 2) * 2 + (nst & 1)) * 4096;
          // the block handed over two chunks ago has been read out of this buffer
          if (lane == 0) asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
          __syncwarp();
          stage_row<ND>(buf, lane, v, era, ecol);
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          __syncwarp();
          if (lane == 0) {
            tma_store_3d(&maps.out, smem_u32(buf), n0 + c, z, row0);
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
          }
          ++nst;
        } else {
          if (row >= a.M) continue;
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int col = n0 + c + j;
            if (col >= a.N) break;
            orow[col] = combine_orders<ND>(v, j, era + ebz[col]);
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(drained)) : "memory");
    }
    // the staging blocks must be read out before the CTA's shared memory goes
    if (TOUT && lane == 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                 : "memory");
}

// ---------------------------------------------------------------------------
// Two-SM form of the same product (tcgen05 cta_group::2, M = 256) for the
// build product B = (ij|P) L. A cluster of two CTAs (consecutive in x, so a
// pair and the n tiles after it share A rows in L2) shares an n tile: each CTA
// loads its own 128 rows of A and half of the BN rows of B, the leader (rank 0)
// issues the MMAs, which read A from each CTA's shared memory and B from both
// halves, and each CTA's TMEM receives its 128 rows x BN columns. Per MMA a
// CTA thus reads (128 + BN/2) * 32 bytes of operands instead of
// (128 + BN) * 32, and its TMA writes (128 + BN/2) * BK bytes per digit and k
// tile instead of (128 + BN) * BK: shared-memory bandwidth, not the tensor
// pipe, bounds the one-SM kernel at BN = 96, and TMEM (5 orders x BN of 512
// columns) caps BN.
//   * both CTAs' TMA loads complete on the leader's full barrier (its cluster
//     address from mapa; cta_group::2 form of the tiled copy);
//   * the leader's commits arrive on both CTAs' empty / done barriers
//     (tcgen05.commit multicast);
//   * TMEM is allocated and freed cta_group::2 by warp 0 of each CTA;
//   * cluster barriers after the setup and before the teardown keep the peer's
//     shared memory alive while the leader's MMAs may still read it.
//   * eight epilogue warps (two per TMEM lane quarter, half the columns each)
//     combine the orders and stage 32 x 16 float64 blocks in the idle stage
//     memory for TMA tensor stores.
// Every mbarrier wait is bounded as in the one-SM kernel.
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %cluster_ctarank;" : "=r"(r));
  return r;
}

__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t leader_addr(uint32_t cta_addr) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, 0;" : "=r"(r) : "r"(cta_addr));
  return r;
}

__device__ __forceinline__ void tma_load_3d_pair(uint32_t dst, const CUtensorMap* map,
                                                 uint32_t leader_mbar, int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(leader_mbar), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

__device__ __forceinline__ void umma_i8_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                             uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
      : "memory");
}

__device__ __forceinline__ void umma_commit_pair(uint32_t mbar) {
  const uint16_t both = 0x3;
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64"
      " [%0], %1;" ::"r"(mbar),
      "h"(both)
      : "memory");
}

template <int ND, int BK, int BN, int ST>
__global__ void __launch_bounds__(320, 1) ozaki_gemm_i8_pair(const __grid_constant__ OzakiMaps maps,
                                                             OzakiArgs a) {
  constexpr int BH = BN / 2;                 // B rows loaded by each CTA
  constexpr uint32_t A_TILE = kBM * BK;
  constexpr uint32_t B_TILE = BH * BK;
  constexpr uint32_t STAGE = ND * (A_TILE + B_TILE);
  constexpr int KSTEPS = BK / 32;
  constexpr uint32_t ACC = (ND * 128 <= (int)kTmemCols) ? 128 : BN;
  constexpr uint32_t STG = 32 * 128;         // one warp's 32 x 16 float64 block
  static_assert(ND * ACC <= kTmemCols, "order accumulators exceed tensor memory");
  static_assert(A_TILE % 1024 == 0 && B_TILE % 1024 == 0, "tiles must keep 1 KB alignment");
  static_assert(BN % 32 == 0, "two-SM i8 MMA needs N a multiple of 32");
  static_assert((BN / 2) % 16 == 0, "each epilogue warp takes whole 16-column chunks");
  static_assert(4 * (BN / 16) * STG <= ST * STAGE, "output staging exceeds the stage memory");
  // S32 accumulator, signed int8 A and B, N>>3, M = 256 >> 4
  constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                             ((uint32_t)(256 >> 4) << 24);
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + ST * STAGE);
  uint64_t* empty = full + ST;
  uint64_t* done = empty + ST;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  int* ebs = reinterpret_cast<int*>(tmem_slot + 4);   // exponents of the n tile's columns
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  const bool leader = rank == 0;
  // blockIdx.x = 2 * (n tile) + rank, blockIdx.y = pair of m tiles
  const int n0 = (blockIdx.x >> 1) * BN, m0 = (blockIdx.y * 2 + (int)rank) * kBM;
  const int nk = a.ktiles;

  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    mbar_init(smem_u32(done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  cluster_sync();   // both CTAs' barriers exist before any load or commit targets them
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (threadIdx.x == 0 && nk > 0) {
    // producer of this CTA: its A rows and its half of B, counted on the leader's barrier
    int issued = 0;
    bool ok = true;
    for (int i = 0; i < nk; ++i, ++issued) {
      const int s = i % ST;
      if (i >= ST) ok = mbar_wait(smem_u32(&empty[s]), ((i / ST) - 1) & 1, a.err, 1);
      if (!ok) break;
      const uint32_t fb = leader_addr(smem_u32(&full[s]));
      if (leader) mbar_expect_tx(smem_u32(&full[s]), 2 * STAGE);
      uint8_t* st = smem + s * STAGE;
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        tma_load_3d_pair(smem_u32(st + d * A_TILE), &maps.a[d], fb, i * BK, m0, a.plane0);
        tma_load_3d_pair(smem_u32(st + ND * A_TILE + d * B_TILE), &maps.b[d], fb, i * BK,
                         n0 + (int)rank * BH, 0);
      }
    }
    if (!ok && leader) {
      // the copies in flight complete on the leader's barriers (bounded)
      for (int q = issued - ST > 0 ? issued - ST : 0; q < issued; ++q) {
        const uint64_t t0 = now_ns();
        while (!mbar_try(smem_u32(&full[q % ST]), (q / ST) & 1) && now_ns() - t0 < kWaitNs)
          __nanosleep(64);
      }
    }
  } else if (threadIdx.x == 32 && nk > 0 && leader) {
    bool ok = true;
    for (int i = 0; i < nk; ++i) {
      const int s = i % ST;
      ok = mbar_wait(smem_u32(&full[s]), (i / ST) & 1, a.err, 2);
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t base = smem_u32(smem + s * STAGE);
      const uint32_t bbase = base + ND * A_TILE;
#pragma unroll
      for (int o = 0; o < ND; ++o) {
        const uint32_t dcol = tmem + (uint32_t)o * ACC;
#pragma unroll
        for (int sa = 0; sa <= o; ++sa) {
          const uint64_t ad = kmajor_desc<BK>(base + sa * A_TILE);
          const uint64_t bd = kmajor_desc<BK>(bbase + (o - sa) * B_TILE);
#pragma unroll
          for (int k = 0; k < KSTEPS; ++k)
            umma_i8_pair(dcol, ad + (uint64_t)(2 * k), bd + (uint64_t)(2 * k), IDESC,
                         (i > 0 || sa > 0 || k > 0) ? 1u : 0u);
        }
      }
      umma_commit_pair(smem_u32(&empty[s]));
    }
    // also after a failed wait: done then tracks the MMAs already issued
    umma_commit_pair(smem_u32(done));
  } else if (warp >= 2 && nk > 0) {
    // epilogue, eight warps: warp w reads TMEM lanes 32 (w % 4) .. + 31 of this
    // CTA (rows row0 .. row0 + 31) and columns h BN/2 .. of them, h = (w - 2) / 4,
    // and stores them through shared memory with TMA
    const int q = warp & 3, h = (warp - 2) >> 2;
    const int row0 = m0 + q * 32, row = row0 + lane;
    const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16);
    for (int j = threadIdx.x - 64; j < BN; j += 256) ebs[j] = n0 + j < a.N ? a.eb[n0 + j] : 0;
    asm volatile("bar.sync 1, 256;" ::: "memory");   // the eight epilogue warps
    bool have = false;
    const uint64_t t0 = now_ns();
    while (!(have = mbar_try(smem_u32(done), 0))) {
      if (now_ns() - t0 > kWaitNs) {
        atomicCAS(a.err, 0, 3);
        break;
      }
      __nanosleep(64);
    }
    have = have && *reinterpret_cast<volatile int*>(a.err) == 0;
    have = __all_sync(0xffffffffu, have);   // tcgen05.ld is warp-collective
    if (have) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int era = row < a.M ? a.ea[row] : 0;
      // the stage memory is idle once done has fired: every copy landed and
      // every MMA that read it (in either CTA) has completed
      uint8_t* stg = smem + (uint32_t)q * (BN / 16) * STG;
      for (int c = h * (BN / 2); c < (h + 1) * (BN / 2); c += 16) {
        uint32_t v[ND][16];
#pragma unroll
        for (int o = 0; o < ND; ++o) tmem_ld16_issue(trow + (uint32_t)o * ACC + c, v[o]);
        tmem_ld_wait();
#pragma unroll
        for (int o = 0; o < ND; ++o) reg_fence16(v[o]);
        uint8_t* buf = stg + (uint32_t)(c / 16) * STG;
        stage_row<ND>(buf, lane, v, era, ebs + c);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) {
          // rows past M and columns past N are clipped by the tensor map
          tma_store_3d(&maps.out, smem_u32(buf), n0 + c, 0, row0);
          asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        }
      }
      if (lane == 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
      __syncwarp();
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  cluster_sync();   // the leader's MMAs are done before either CTA frees or leaves
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
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

template <int ND, int BK, int BN, int ST, bool TOUT>
constexpr size_t smem_bytes() {
  return (size_t)ST * ND * (kBM * BK + BN * BK) + (TOUT ? 8 * 2 * 4096 : 0) + 1024 + 256;
}

template <int ND, int BK, int BN, int ST, bool TOUT>
void launch(const OzakiMaps& maps, const OzakiArgs& a, int grid_z, cudaStream_t s) {
  constexpr size_t smem = smem_bytes<ND, BK, BN, ST, TOUT>();
  static_assert(smem <= 232448, "stages exceed the shared memory of one CTA");
  OzakiArgs b = a;
  b.zcount = grid_z;
  if (b.zper < 1) b.zper = 1;
  dim3 grid((a.N + BN - 1) / BN, (a.M + kBM - 1) / kBM, (grid_z + b.zper - 1) / b.zper);
  DFJK_CUDA(cudaFuncSetAttribute(ozaki_gemm_i8<ND, BK, BN, ST, TOUT>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  ozaki_gemm_i8<ND, BK, BN, ST, TOUT><<<grid, 320, smem, s>>>(maps, b);
  DFJK_LAUNCHED();
}

template <int ND, int BK, int BN, int ST>
constexpr size_t smem_bytes_pair() {
  return (size_t)ST * ND * (kBM * BK + (BN / 2) * BK) + 1024 + 128 + 4 * BN;
}

// clusters of two CTAs along x: grid (2 * ceil(N/BN), ceil(M/256)), one batch
template <int ND, int BK, int BN, int ST>
void launch_pair(const OzakiMaps& maps, const OzakiArgs& a, cudaStream_t s) {
  constexpr size_t smem = smem_bytes_pair<ND, BK, BN, ST>();
  static_assert(smem <= 232448, "stages exceed the shared memory of one CTA");
  OzakiArgs b = a;
  b.zcount = 1;
  b.zper = 1;
  const int mpairs = (a.M + 2 * kBM - 1) / (2 * kBM);
  if (mpairs > 65535) fail(DFJK_ERR_INVALID, "two-SM int8 GEMM: too many row tiles");
  auto* kern = ozaki_gemm_i8_pair<ND, BK, BN, ST>;
  DFJK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2 * ((a.N + BN - 1) / BN), mpairs, 1);
  cfg.blockDim = dim3(320, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  DFJK_CUDA(cudaLaunchKernelEx(&cfg, kern, maps, b));
  DFJK_LAUNCHED();
}

}  // namespace

// digits, k tile bytes, n tile, stages and B rows per copy of each product
// (see ozaki.h); the build product runs on SM pairs, each CTA copying half of
// the n tile
OzakiShapeInfo ozaki_shape(OzakiShape shape) {
  switch (shape) {
    case kOzHalf: return {kOzKDigits, 64, 80, 3, 80};
    case kOzHalfWide: return {kOzKDigits, 64, 96, 2, 96};
    case kOzBuild: return {kOzBDigits, 64, 96, 4, 48};
    case kOzSyrk: return {kOzSDigits, 64, 96, 3, 96};
    // 7 orders x 64 columns = 448 of the 512 TMEM columns; three 70 KB stages
    case kOzBuild64: return {kOzB64Digits, 64, 64, 3, 32};
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

bool ozaki_out_mappable(const double* base, int64_t batch_stride, int64_t ld) {
  return !(reinterpret_cast<uintptr_t>(base) & 15) && (batch_stride * 8) % 16 == 0 &&
         (ld * 8) % 16 == 0;
}

void ozaki_map_out(CUtensorMap* m, double* base, int64_t cols, int64_t batches, int64_t rows,
                   int64_t batch_stride, int64_t ld) {
  if (!ozaki_out_mappable(base, batch_stride, ld))
    fail(DFJK_ERR_INVALID, "output tensor map: base or strides not 16-byte aligned");
  cuuint64_t dims[3] = {(cuuint64_t)cols, (cuuint64_t)batches, (cuuint64_t)rows};
  cuuint64_t strides[2] = {(cuuint64_t)(batch_stride * 8), (cuuint64_t)(ld * 8)};
  cuuint32_t box[3] = {16, 1, 32};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = encode_fn()(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides, box, es,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(DFJK_ERR_CUDA, "cuTensorMapEncodeTiled (output) failed (%d)", (int)r);
}

void ozaki_launch(OzakiShape shape, const OzakiMaps& maps, const OzakiArgs& a, int grid_z,
                  cudaStream_t s) {
  if (grid_z <= 0 || a.M <= 0 || a.N <= 0) return;
  static_assert(kOzKDigits == 4 && kOzBDigits == 5 && kOzSDigits == 5 && kOzB64Digits == 7,
                "the compiled shapes follow the digit counts");
  switch (shape) {
    case kOzHalf:
      if (a.tma_out) launch<4, 64, 80, 3, true>(maps, a, grid_z, s);
      else launch<4, 64, 80, 3, false>(maps, a, grid_z, s);
      return;
    case kOzHalfWide:
      // two stages: three would not leave room for the output staging
      if (a.tma_out) launch<4, 64, 96, 2, true>(maps, a, grid_z, s);
      else launch<4, 64, 96, 2, false>(maps, a, grid_z, s);
      return;
    case kOzBuild:
      if (grid_z != 1) fail(DFJK_ERR_INVALID, "the two-SM build product takes one batch");
      launch_pair<5, 64, 96, 4>(maps, a, s);
      return;
    case kOzBuild64:
      if (grid_z != 1) fail(DFJK_ERR_INVALID, "the two-SM build product takes one batch");
      launch_pair<7, 64, 64, 3>(maps, a, s);
      return;
    case kOzSyrk: launch<5, 64, 96, 3, false>(maps, a, grid_z, s); return;
  }
  fail(DFJK_ERR_INVALID, "unknown int8 GEMM shape %d", (int)shape);
}

// ---------------------------------------------------------------------------
// Self-test of the bounded wait
// ---------------------------------------------------------------------------

namespace {

// Warp 0 waits on an mbarrier that no thread arrives at, with the given limit;
// warp 1 waits on it with the pipelines' own limit and must return as soon as
// warp 0's timeout is flagged. Nothing else is in flight, so the block only
// has to return.
__global__ void wait_selftest_kernel(int* err, unsigned long long limit_ns,
                                     unsigned long long* waited) {
  __shared__ __align__(8) uint64_t bar;
  const uint32_t a = smem_u32(&bar);
  if (threadIdx.x == 0) mbar_init(a, 1);
  __syncthreads();
  const int warp = threadIdx.x / 32;
  const uint64_t t0 = now_ns();
  mbar_wait(a, 0, err, kWaitSelftestCode + warp, warp == 0 ? limit_ns : kWaitNs);
  __syncwarp();
  if ((threadIdx.x & 31) == 0) waited[warp] = now_ns() - t0;
}

}  // namespace

void wait_selftest(const Context& c, int64_t limit_ns, double* waited_ms, cudaStream_t s) {
  (void)c;
  DevBuf buf;
  buf.alloc(32);
  DFJK_CUDA(cudaMemsetAsync(buf.p, 0, 32, s));
  int* err = buf.as<int>();
  auto* waited = reinterpret_cast<unsigned long long*>(buf.as<char>() + 16);
  wait_selftest_kernel<<<1, 64, 0, s>>>(err, (unsigned long long)limit_ns, waited);
  DFJK_LAUNCHED();
  int h = 0;
  unsigned long long w[2] = {0, 0};
  DFJK_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  DFJK_CUDA(cudaMemcpyAsync(w, waited, sizeof(w), cudaMemcpyDeviceToHost, s));
  DFJK_CUDA(cudaStreamSynchronize(s));
  if (waited_ms)
    for (int i = 0; i < 2; ++i) waited_ms[i] = 1e-6 * (double)w[i];
  if (h) fail(DFJK_ERR_CUDA, "tensor-core pipeline gave up waiting (code %d)", h);
}

}  // namespace dfjk

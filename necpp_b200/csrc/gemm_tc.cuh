// Trailing update of the mixed-precision LU on the 5th-generation tensor
// cores: C -= A * B for complex64 A (m x kb), B (kb x n), C (m x n), all
// row-major, as ONE real GEMM with FP32 accumulation in TMEM, in one of two
// operand formats (the engine picks one per factorisation).
//
// Split BF16 (SplitBf16).  Each complex FP32 operand is split into BF16 hi/lo
// parts (x = hi + lo + O(2^-16 x)); with K' = 6 * kbp (kbp = kb rounded up
// to 64):
//   A'[i]    = [ Ar_hi | Ai_hi | Ar_hi | Ai_hi | Ar_lo | Ai_lo ]          (m rows)
//   B'[2j]   = [ Br_hi |-Bi_hi | Br_lo |-Bi_lo | Br_hi |-Bi_hi ]  -> Re(AB)_j
//   B'[2j+1] = [ Bi_hi | Br_hi | Bi_lo | Br_lo | Bi_hi | Br_hi ]  -> Im(AB)_j
// Products kept: hi*hi + hi*lo + lo*hi (the lo*lo term, ~2^-16 relative, is
// dropped).
//
// TF32 (Tf32).  One pass, K' = 2 * kbp, the operands rounded to
// TF32 (10-bit mantissa, round to nearest) in FP32 containers:
//   A'[i] = [ Ar | Ai ],  B'[2j] = [ Br | -Bi ],  B'[2j+1] = [ Bi | Br ].
// TF32 runs at half the BF16 rate, so this issues 2/3 of the split form's
// tensor cycles and moves 2/3 of its operand bytes; the factor's error is
// ~2^-11 instead of ~2^-16, which costs the refinement a step.
//
// Either way D = A' B'^T (m x 2n) holds (Re, Im) of A*B interleaved per
// column: the accumulator row of output row i is a contiguous run of
// complex values of C's row i, and the FP64 refinement of the solve removes
// the update's rounding.
//
// Kernel: persistent, one CTA per SM, 6 warps:
//   warp 0  TMA producer: A' (128 x 128 B) and B' (256 x 128 B) tiles, 128B
//           swizzle, into a 4-stage shared-memory ring (48 KB per stage);
//   warp 1  MMA issuer: tcgen05.mma.cta_group::1, M=128 N=256, four
//           instructions of 32 B of K per stage (K=16 BF16 or K=8 TF32),
//           accumulating in one of two 128 x 256 FP32 TMEM buffers;
//   warps 2-5 epilogue: tcgen05.ld of the finished buffer (32 rows x 32
//           columns per load), negated into a 128B-swizzled 4 KB staging
//           tile in shared memory (two per warp), and added to C by a TMA
//           bulk tensor reduction (cp.reduce.async.bulk.tensor .add.f32):
//           the read-modify-write of C happens in L2, fully coalesced, while
//           the MMA warp fills the other accumulator.
// Every wait on an mbarrier is bounded; on timeout the kernel records an
// error bit and winds down (outstanding TMA copies are waited for, TMEM is
// freed).  TMA loads never use cluster multicast.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace necb {
namespace tc {

// The two operand formats: element type, K' per complex K (kKMul), the
// instruction descriptor's A/B format code (1 = BF16, 2 = TF32)
struct SplitBf16 {
  using T = __nv_bfloat16;
  static constexpr int kKMul = 6;
  static constexpr uint32_t kFormat = 1;
};
struct Tf32 {
  using T = float;  // TF32 values in FP32 containers
  static constexpr int kKMul = 2;
  static constexpr uint32_t kFormat = 2;
};
// BK: operand elements per 128-byte row of a stage; KP: the complex K of an
// update is padded to a multiple of KP, and K' = F::kKMul * (padded K)
template <class F>
__host__ __device__ constexpr int bk() {
  return 128 / (int)sizeof(typename F::T);
}
constexpr int BM = 128, BN = 256, KP = 64, STAGES = 4;
constexpr int A_BYTES = BM * 128;               // 16 KB
constexpr int B_BYTES = BN * 128;               // 32 KB
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;  // 48 KB
constexpr int THREADS = 192;
constexpr int EPI_WARPS = 4;
constexpr int EPI_TILE_BYTES = 32 * 32 * 4;  // 32 rows x 128 B
constexpr int EPI_BYTES = EPI_WARPS * 2 * EPI_TILE_BYTES;  // 32 KB
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + EPI_BYTES + 1024 /*align*/ + 256 /*barriers*/;
static_assert(SMEM_BYTES <= 232448, "dynamic shared memory per CTA");
constexpr uint32_t TMEM_COLS = 512;  // two 256-column FP32 accumulators
constexpr long long kWaitLimit = 1LL << 20;

enum : int { kStatTimeout = 1 << 12 };

// ---- PTX helpers --------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait; false on timeout
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (long long i = 0; i < kWaitLimit; i++)
    if (mbar_try(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int c0, int c1, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(map), "r"(c0), "r"(c1), "r"(bar)
      : "memory");
}
// C[box at (x, y)] += smem tile, reduced in L2 (no multicast; C is local)
__device__ __forceinline__ void tma_reduce_add_2d(const CUtensorMap* map, int c0, int c1, uint32_t src) {
  asm volatile("cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(map),
               "r"(c0), "r"(c1), "r"(src)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// at most one committed group still reading its shared-memory source
__device__ __forceinline__ void bulk_wait_read1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// K-major, 128B-swizzled operand tile: rows of 128 B, 8-row atoms of 1 KB
// (leading offset 16 B, stride offset 1 KB, descriptor version 1).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  uint64_t d = (uint64_t)((addr & 0x3FFFF) >> 4);
  d |= (uint64_t)1 << 16;          // leading byte offset (16 B units)
  d |= (uint64_t)(1024 >> 4) << 32; // stride byte offset
  d |= (uint64_t)1 << 46;          // version
  d |= (uint64_t)2 << 61;          // SWIZZLE_128B
  return d;
}
// instruction descriptor: FP32 accumulator (bits 4-5 = 1), A and B format
// (bits 7-9, 10-12: 1 = BF16, 2 = TF32), both K-major, N >> 3 at bit 17,
// M >> 4 at bit 24; M = 128, N = 256
template <class F>
__host__ __device__ constexpr uint32_t idesc() {
  return (1u << 4) | (F::kFormat << 7) | (F::kFormat << 10) | ((uint32_t)(BN >> 3) << 17) |
         ((uint32_t)(BM >> 4) << 24);
}

template <class F>
__device__ __forceinline__ void mma_op(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  if constexpr (F::kFormat == 2)
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc<F>()), "r"(accumulate)
        : "memory");
  else
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc<F>()), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ---- operand packing ----------------------------------------------------
__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}
// x rounded to TF32 (nearest, ties away), kept in an FP32 container
__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// A' entries of one complex value a at column k of an A' row (kbp: the
// padded complex K, so the parts sit kbp apart)
template <class F>
__device__ __forceinline__ void put_a(typename F::T* row, int kbp, int k, float2 a) {
  if constexpr (F::kFormat == 2) {
    row[k] = to_tf32(a.x);
    row[kbp + k] = to_tf32(a.y);
  } else {
    __nv_bfloat16 rh, rl, ih, il;
    split_bf16(a.x, rh, rl);
    split_bf16(a.y, ih, il);
    row[0 * kbp + k] = rh;
    row[1 * kbp + k] = ih;
    row[2 * kbp + k] = rh;
    row[3 * kbp + k] = ih;
    row[4 * kbp + k] = rl;
    row[5 * kbp + k] = il;
  }
}
// B' entries of one complex value b at column k of rows 2j (re) and 2j+1 (im)
template <class F>
__device__ __forceinline__ void put_b(typename F::T* re, typename F::T* im, int kbp, int k, float2 b) {
  if constexpr (F::kFormat == 2) {
    const float br = to_tf32(b.x), bi = to_tf32(b.y);
    re[k] = br;
    re[kbp + k] = -bi;
    im[k] = bi;
    im[kbp + k] = br;
  } else {
    __nv_bfloat16 rh, rl, ih, il;
    split_bf16(b.x, rh, rl);
    split_bf16(b.y, ih, il);
    const __nv_bfloat16 nih = __hneg(ih), nil = __hneg(il);
    re[0 * kbp + k] = rh;
    re[1 * kbp + k] = nih;
    re[2 * kbp + k] = rl;
    re[3 * kbp + k] = nil;
    re[4 * kbp + k] = rh;
    re[5 * kbp + k] = nih;
    im[0 * kbp + k] = ih;
    im[1 * kbp + k] = rh;
    im[2 * kbp + k] = il;
    im[3 * kbp + k] = rl;
    im[4 * kbp + k] = ih;
    im[5 * kbp + k] = rh;
  }
}

// A' from A (m x kb complex, row-major lda): one thread per (row, k)
template <class F>
__global__ void pack_a_kernel(const float2* A, int64_t lda, int m, int kb, int kbp, typename F::T* Ap) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)m * kbp) return;
  const int i = (int)(idx / kbp), k = (int)(idx - (int64_t)i * kbp);
  const float2 a = k < kb ? A[(int64_t)i * lda + k] : make_float2(0.f, 0.f);
  put_a<F>(Ap + (int64_t)i * F::kKMul * kbp, kbp, k, a);
}

// B' from B (kb x n complex, row-major ldb): tile of 64 k x 32 columns
// through shared memory so both the reads (along n) and the writes (along k)
// are contiguous.
template <class F>
__global__ void __launch_bounds__(256)
    pack_b_kernel(const float2* B, int64_t ldb, int kb, int kbp, int n, typename F::T* Bp) {
  __shared__ float2 t[64][33];
  const int j0 = blockIdx.x * 32, k0 = blockIdx.y * 64;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int kk = ty; kk < 64; kk += 8) {
    const int k = k0 + kk, j = j0 + tx;
    t[kk][tx] = (k < kb && j < n) ? B[(int64_t)k * ldb + j] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const int64_t K2 = F::kKMul * (int64_t)kbp;
  // each warp writes rows (2j, 2j+1) for 4 columns j; lane covers k pairs
  for (int jj = ty; jj < 32; jj += 8) {
    const int j = j0 + jj;
    if (j >= n) continue;
    typename F::T* re = Bp + (int64_t)(2 * j) * K2 + k0;
    for (int kk = tx; kk < 64; kk += 32) put_b<F>(re, re + K2, kbp, kk, t[kk][jj]);
  }
}

// ---- the GEMM -----------------------------------------------------------
// Tile order of the persistent loop: bands of `group` m-tiles; inside a band
// the walk goes down the band's m-tiles for one n-tile, then to the next
// n-tile.  The CTAs resident at one time then share a few B' tiles (each is
// read from DRAM once per band and by the band's other CTAs from L2) and
// the band's A' tiles stay in L2 while the band sweeps n, instead of every
// m-row of tiles sweeping all of B' while the C traffic evicts it.
__device__ __forceinline__ void tile_coords(int tile, int m_tiles, int n_tiles, int group, int& mt, int& nt) {
  const int per_band = group * n_tiles;
  const int band = tile / per_band;
  const int m0 = band * group;
  const int gm = min(group, m_tiles - m0);  // m-tiles in this band (the last may be short)
  const int local = tile - band * per_band;
  mt = m0 + local % gm;
  nt = local / gm;
}

// C (m x n complex, row-major; tmC views it as m rows x 2n FP32 with 32 x 32
// boxes, 128B swizzle) -= D, D = A' B'^T, K' = kdim (multiple of 64)
template <class F>
__global__ void __launch_bounds__(THREADS, 1)
    gemm_tc_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const __grid_constant__ CUtensorMap tmC, int m, int n, int kdim, int group, int* status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  uint8_t* epi = smem + STAGES * STAGE_BYTES;  // 1 KB aligned (the swizzle atom)
  uint64_t* bars = reinterpret_cast<uint64_t*>(epi + EPI_BYTES);
  // bars: full[STAGES], empty[STAGES], tfull[2], tempty[2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 4);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m_tiles = (m + BM - 1) / BM;
  const int n_tiles = (2 * n + BN - 1) / BN;
  const int total = m_tiles * n_tiles;
  constexpr int BK = bk<F>();
  const int kblocks = kdim / BK;

  auto bar = [&](int i) { return smem_u32(bars + i); };
  const int FULL = 0, EMPTY = STAGES, TFULL = 2 * STAGES, TEMPTY = 2 * STAGES + 2;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(bar(FULL + s), 1);
      mbar_init(bar(EMPTY + s), 1);
    }
    for (int a = 0; a < 2; a++) {
      mbar_init(bar(TFULL + a), 1);
      mbar_init(bar(TEMPTY + a), 128);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmA) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmB) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmC) : "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      int it = 0;
      for (int tile = blockIdx.x; tile < total && !*abort_flag; tile += gridDim.x) {
        int mt, nt;
      tile_coords(tile, m_tiles, n_tiles, group, mt, nt);
        for (int kb = 0; kb < kblocks; kb++, it++) {
          const int s = it % STAGES;
          const uint32_t ph = (it / STAGES) & 1;
          if (!mbar_wait(bar(EMPTY + s), ph ^ 1)) {
            atomicOr(status, kStatTimeout);
            *abort_flag = 1;
            break;
          }
          uint8_t* a_dst = smem + s * STAGE_BYTES;
          uint8_t* b_dst = a_dst + A_BYTES;
          mbar_expect_tx(bar(FULL + s), STAGE_BYTES);
          tma_load_2d(smem_u32(a_dst), &tmA, kb * BK, mt * BM, bar(FULL + s));
          tma_load_2d(smem_u32(b_dst), &tmB, kb * BK, nt * BN, bar(FULL + s));
        }
      }
      // drain: every issued stage must have landed before the CTA may exit
      for (int k = 0; k < STAGES && it > 0; k++) {
        const int j = it - 1 - k;
        if (j < 0) break;
        mbar_wait(bar(FULL + (j % STAGES)), (j / STAGES) & 1);
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      int it = 0, tc = 0;
      for (int tile = blockIdx.x; tile < total && !*abort_flag; tile += gridDim.x, tc++) {
        const int acc = tc & 1;
        const uint32_t aph = (tc >> 1) & 1;
        if (!mbar_wait(bar(TEMPTY + acc), aph ^ 1)) {
          atomicOr(status, kStatTimeout);
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
        for (int kb = 0; kb < kblocks; kb++, it++) {
          const int s = it % STAGES;
          const uint32_t ph = (it / STAGES) & 1;
          if (!mbar_wait(bar(FULL + s), ph)) {
            atomicOr(status, kStatTimeout);
            *abort_flag = 1;
            break;
          }
          tc_fence_after();
          const uint32_t a_addr = smem_u32(smem + s * STAGE_BYTES);
          const uint32_t b_addr = a_addr + A_BYTES;
#pragma unroll
          for (int k = 0; k < 4; k++)
            mma_op<F>(d_tmem, smem_desc(a_addr + k * 32), smem_desc(b_addr + k * 32), (kb | k) != 0);
          mma_commit(bar(EMPTY + s));  // frees the stage once these MMAs retire
        }
        if (*abort_flag) break;
        mma_commit(bar(TFULL + acc));  // accumulator ready for the epilogue
      }
    }
  } else {
    // ---------------- epilogue (warps 2..5) ----------------
    const int q = warp & 3;  // TMEM lane quarter this warp may access
    uint8_t* stage0 = epi + (warp - 2) * 2 * EPI_TILE_BYTES;
    // this lane's row in a staging tile; 16-byte chunk j sits at j ^ (row % 8)
    const uint32_t row_off = (uint32_t)lane * 128;
    const uint32_t swz = (uint32_t)(lane & 7);
    int tc = 0, issued = 0;
    for (int tile = blockIdx.x; tile < total; tile += gridDim.x, tc++) {
      const int acc = tc & 1;
      const uint32_t aph = (tc >> 1) & 1;
      bool ok = mbar_wait(bar(TFULL + acc), aph);
      if (!ok || *abort_flag) {
        if (!ok) {
          atomicOr(status, kStatTimeout);
          *abort_flag = 1;
        }
        break;
      }
      tc_fence_after();
      int mt, nt;
      tile_coords(tile, m_tiles, n_tiles, group, mt, nt);
      const int y = mt * BM + q * 32;  // first C row of this warp's quarter
      const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * BN);
#pragma unroll 1
      for (int c = 0; c < BN / 32; c++) {
        uint32_t r[32];
        tmem_ld32(taddr + c * 32, r);
        if (c == BN / 32 - 1) {
          // the accumulator is in registers: hand TMEM back to the MMA warp
          tc_fence_before();
          mbar_arrive(bar(TEMPTY + acc));
        }
        const int x = nt * BN + c * 32;  // first FP32 column of the box
        if (y >= m || x >= 2 * n) continue;  // box entirely outside C
        uint8_t* st = stage0 + (issued & 1) * EPI_TILE_BYTES;
        if (lane == 0) bulk_wait_read1();  // the reduction that used st two boxes ago has read it
        __syncwarp();
#pragma unroll
        for (int j = 0; j < 8; j++) {
          float4 v = make_float4(-__uint_as_float(r[4 * j]), -__uint_as_float(r[4 * j + 1]),
                                 -__uint_as_float(r[4 * j + 2]), -__uint_as_float(r[4 * j + 3]));
          *reinterpret_cast<float4*>(st + row_off + (((uint32_t)j ^ swz) << 4)) = v;
        }
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
          tma_reduce_add_2d(&tmC, x, y, smem_u32(st));
          bulk_commit();
        }
        issued++;
      }
    }
    // every reduction must be complete (not only read) before the CTA exits
    if (lane == 0) bulk_wait_all();
    __syncwarp();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS) : "memory");
  }
}

}  // namespace tc
}  // namespace necb

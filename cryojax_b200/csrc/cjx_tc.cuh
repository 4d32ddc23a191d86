// Blackwell tensor-core building blocks: mbarriers with bounded waits, 2-D
// TMA tile loads (no multicast), tcgen05.mma (kind::f16, one CTA, M = 128)
// with the accumulator in tensor memory, and tcgen05.ld for the epilogue.
//
// Shared-memory operand layout: K-major tiles of 64 16-bit elements per row
// (one 128-byte row), 128-byte swizzle, written by TMA with
// CU_TENSOR_MAP_SWIZZLE_128B; every tile starts on a 1024-byte boundary.
// The matching UMMA shared-memory descriptor has the canonical K-major
// SWIZZLE_128B form: stride between 8-row groups (SBO) 1024 bytes, leading
// offset 16 bytes (unused when swizzled), descriptor version 1, layout type
// 2.  One MMA consumes K = 16 (32 bytes of a row); the k-th MMA of a 64-wide
// k-block starts 32 k bytes into the swizzle atom.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cjx {
namespace tc {

constexpr int BM = 128;  // rows per tile (TMEM lanes)
constexpr int BK = 64;   // 16-bit elements per k-block (one 128-byte swizzle row)
// A wait that has not completed after this long reports an error and
// gives up instead of spinning on.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;

// Error codes written to the status word by a kernel that gave up.
constexpr int kErrWaitFull = 101, kErrWaitEmpty = 102, kErrWaitDone = 103, kErrDrain = 104, kErrSelfTest = 105;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
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

// Wait for the phase of `bar` with the given parity.  Gives up (returns
// false) when another thread of the CTA raised `abort_flag`, or after
// kWaitLimitNs, in which case it raises the flag and records `code`.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag, int* status,
                                          int code, uint64_t limit_ns = kWaitLimitNs) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (abort_flag && *abort_flag) return false;
    if (globaltimer_ns() - t0 > limit_ns) {
      if (abort_flag) *abort_flag = 1;
      if (status) atomicCAS(status, 0, code);
      return false;
    }
  }
}

// 2-D tiled TMA load of box (x = inner coordinate, y = outer) into shared
// memory, completing on `bar`.  x * element size is a multiple of 16 bytes
// at every call site (x is a multiple of 64 16-bit elements).
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void prefetch_tma_map(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// K-major, 128-byte swizzled operand descriptor for a tile at shared address saddr.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr & 0x3FFFFu) >> 4);  // start address, 16-byte units
  d |= static_cast<uint64_t>(1) << 16;                 // leading byte offset (16 B; unused when swizzled)
  d |= static_cast<uint64_t>(1024 >> 4) << 32;         // stride byte offset: 8 rows x 128 B
  d |= static_cast<uint64_t>(1) << 46;                 // descriptor version
  d |= static_cast<uint64_t>(2) << 61;                 // layout: 128-byte swizzle
  return d;
}

// Instruction descriptor of tcgen05.mma kind::f16: FP32 accumulate, A and B
// both BF16 (fmt 1) or both FP16 (fmt 0), both K-major, shape M x N.
__host__ __device__ constexpr uint32_t f16_idesc(int m, int n, int fmt) {
  return (1u << 4) | (static_cast<uint32_t>(fmt) << 7) | (static_cast<uint32_t>(fmt) << 10) |
         (static_cast<uint32_t>(n >> 3) << 17) | (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

// Arrive on `bar` once every tcgen05 operation issued so far by this thread has completed.
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Warp-wide: allocate `ncols` (power of two >= 32) TMEM columns; the address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// Warp-wide: 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__host__ __device__ constexpr int stages_for(int bn) { return bn >= 256 ? 4 : (bn >= 128 ? 5 : 6); }
__host__ __device__ constexpr uint32_t stage_bytes(int bn) { return (BM + bn) * BK * 2; }
__host__ __device__ constexpr size_t gemm_smem_bytes(int bn) {
  return 1024 + static_cast<size_t>(stages_for(bn)) * stage_bytes(bn) + 256;
}

// The main loop of one 128 x BN output tile over k-blocks [kb0, kb1):
// thread 0 of warp 0 issues the TMA loads, thread 0 of warp 1 the MMAs, and
// on return the accumulator sits in TMEM (columns [tmem, tmem + BN)) once
// the `done` barrier completes.  All four warps must call it.
template <int BN>
struct TileMainloop {
  static constexpr int kStages = stages_for(BN);
  static constexpr uint32_t kABytes = BM * BK * 2;
  static constexpr uint32_t kStageBytes = stage_bytes(BN);

  uint8_t* tiles;     // kStages x (A tile, B tile), 1024-byte aligned
  uint64_t* bars;     // full[kStages], empty[kStages], done
  uint32_t* tmem_slot;
  volatile int* abort_flag;
  int* consumed;      // k-blocks whose MMAs were issued (for the drain on abort)

  __device__ void carve(uint8_t* smem_raw) {
    uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    tiles = base;
    bars = reinterpret_cast<uint64_t*>(base + kStages * kStageBytes);
    tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 1);
    abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    consumed = const_cast<int*>(abort_flag) + 1;
  }
  __device__ uint32_t full(int s) const { return smem_u32(bars + s); }
  __device__ uint32_t empty(int s) const { return smem_u32(bars + kStages + s); }
  __device__ uint32_t done() const { return smem_u32(bars + 2 * kStages); }
  __device__ uint32_t a_tile(int s) const { return smem_u32(tiles + s * kStageBytes); }
  __device__ uint32_t b_tile(int s) const { return smem_u32(tiles + s * kStageBytes + kABytes); }

  // Barrier init + TMEM allocation; ends with a CTA-wide barrier.
  __device__ uint32_t setup(const CUtensorMap* ta, const CUtensorMap* tb) {
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
      for (int s = 0; s < kStages; ++s) {
        mbar_init(full(s), 1);
        mbar_init(empty(s), 1);
      }
      mbar_init(done(), 1);
      *abort_flag = 0;
      *consumed = 0;
      fence_barrier_init();
      prefetch_tma_map(ta);
      prefetch_tma_map(tb);
    }
    if (warp == 1) tmem_alloc(tmem_slot, BN < 32 ? 32 : BN);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    return *tmem_slot;
  }

  // Producer / MMA roles; other threads fall through.  Returns after the
  // caller's role is done (not after the MMAs complete).
  __device__ void run(const CUtensorMap* ta, const CUtensorMap* tb, int m0, int n0, int kb0, int kb1,
                      uint32_t tmem, uint32_t idesc, int* status, int* issued_out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0 && lane == 0) {
      int issued = 0;
      for (int kb = kb0; kb < kb1; ++kb) {
        const int i = kb - kb0, s = i % kStages;
        const uint32_t ph = (i / kStages) & 1;
        if (!mbar_wait(empty(s), ph ^ 1, abort_flag, status, kErrWaitEmpty)) break;
        mbar_arrive_expect_tx(full(s), kStageBytes);
        tma_load_2d(a_tile(s), ta, full(s), kb * BK, m0);
        tma_load_2d(b_tile(s), tb, full(s), kb * BK, n0);
        ++issued;
      }
      *issued_out = issued;
    } else if (warp == 1 && lane == 0) {
      int i = 0;
      for (int kb = kb0; kb < kb1; ++kb, ++i) {
        const int s = i % kStages;
        const uint32_t ph = (i / kStages) & 1;
        if (!mbar_wait(full(s), ph, abort_flag, status, kErrWaitFull)) break;
        tc_fence_after();
        const uint64_t da = sw128_desc(a_tile(s)), db = sw128_desc(b_tile(s));
#pragma unroll
        for (int k = 0; k < BK / 16; ++k)
          umma_f16(tmem, da + 2 * k, db + 2 * k, idesc, (i > 0 || k > 0) ? 1u : 0u);
        umma_commit(empty(s));
        *consumed = i + 1;
      }
      umma_commit(done());
    }
    __syncwarp();
  }

  // Every warp: wait for the accumulator (lane 0 polls, the warp follows).
  __device__ bool wait_done(int* status) {
    const int lane = threadIdx.x & 31;
    int ok = 0;
    if (lane == 0) ok = mbar_wait(done(), 0, abort_flag, status, kErrWaitDone) ? 1 : 0;
    ok = __shfl_sync(0xffffffffu, ok, 0);
    tc_fence_after();
    return ok != 0;
  }

  // End of the CTA: after an abort, wait (bounded) for the loads still in
  // flight and for the MMAs issued, then free TMEM.
  __device__ void teardown(uint32_t tmem, int issued, int* status) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    tc_fence_before();
    __syncthreads();
    if (*abort_flag) {
      if (warp == 0 && lane == 0) {
        for (int i = *consumed; i < issued; ++i)
          mbar_wait(full(i % kStages), (i / kStages) & 1, nullptr, status, kErrDrain);
      }
      if (warp == 1 && lane == 0) mbar_wait(done(), 0, nullptr, status, kErrDrain);
      __syncthreads();
    }
    if (warp == 1) tmem_dealloc(tmem, BN < 32 ? 32 : BN);
  }
};

}  // namespace tc
}  // namespace cjx

// Tile staging through the tensor memory accelerator (TMA): bulk tensor
// copies from a state buffer in this GPU's HBM into shared memory, completed
// on an mbarrier.  No cluster multicast: every copy reads this GPU's own
// memory into its own CTA.
//
// A state buffer is addressed as a 4-D tensor (x, y, z, field) of FP32 with
// extents (nx, ny, nz, nf) and byte strides (4 nx, 4 nx ny, 4 N): the
// structure-of-arrays layout of the resident state.  A map fixes the box
// (bx, by, bz, bf) one copy moves; coordinates outside the tensor read zero.
// The rules the hardware imposes and the host checks before making a map:
// every stride a multiple of 16 bytes (nx % 4 == 0), the base 16-byte
// aligned, the box's inner extent bx * 4 bytes a multiple of 16, and -- the
// rule nothing checks at run time -- the x coordinate of every copy a
// multiple of 4 elements (16 bytes).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <mutex>

namespace pu {
namespace tma {

// ---- host ----------------------------------------------------------------

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links no driver library); null if the driver does not have it.
inline PFN_cuTensorMapEncodeTiled_v12000 encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    else
      cudaGetLastError();
  });
  return fn;
}

// A map of the FP32 state buffer `base` ((nf, nz, ny, nx), x fastest) with
// box (bx, by, bz, bf).  False when the buffer or box breaks a TMA rule.
inline bool encode_state(CUtensorMap *m, const void *base, int nx, int ny, int nz, int nf, uint32_t bx, uint32_t by,
                         uint32_t bz, uint32_t bf) {
  auto enc = encoder();
  if (!enc || !base || nx % 4 != 0 || (reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
  if ((bx * 4) % 16 != 0 || bx > 256 || by > 256 || bz > 256 || bf > 256 || !bx || !by || !bz || !bf) return false;
  const cuuint64_t dims[4] = {cuuint64_t(nx), cuuint64_t(ny), cuuint64_t(nz), cuuint64_t(nf)};
  const cuuint64_t strides[3] = {cuuint64_t(nx) * 4, cuuint64_t(nx) * ny * 4, cuuint64_t(nx) * ny * nz * 4};
  const cuuint32_t box[4] = {bx, by, bz, bf};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<void *>(base), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// ---- device --------------------------------------------------------------

__device__ __forceinline__ uint32_t saddr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// One thread: an mbarrier expecting one arrival, made visible to the
// asynchronous proxy.
__device__ __forceinline__ void mbar_init(uint64_t *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// The arrival of the issuing thread, announcing `bytes` of copies to come.
__device__ __forceinline__ void mbar_expect(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}

// A box of `map` at (x, y, z, f) into shared memory at dst (16-byte aligned;
// x a multiple of 4 elements), completing on bar.
__device__ __forceinline__ void load_4d(void *dst, const CUtensorMap *map, int x, int y, int z, int f, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(saddr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(f), "r"(saddr(bar))
      : "memory");
}

// The GPU's nanosecond timer.
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// How long a wait on a tile copy may take before the block gives up: a copy
// lands in microseconds even under full load; a poll of try_wait that does
// not see it suspends the thread for ~4 us (measured on B200).
constexpr uint64_t WAIT_LIMIT_NS = 20000000ull;   // 20 ms

// Waits for phase `parity` of bar for at most limit_ns; false if it did not
// complete (the caller reports the error and gives up the tile).  The poll
// count is capped too (2^20 polls, ~4 s), in case the timer stood still.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit_ns = WAIT_LIMIT_NS) {
  const uint32_t a = saddr(bar);
  const uint64_t t0 = globaltimer_ns();
  for (int it = 0; it < (1 << 20); it++) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
    if (globaltimer_ns() - t0 > limit_ns) return false;
  }
  return false;
}

}  // namespace tma
}  // namespace pu

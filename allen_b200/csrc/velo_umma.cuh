// Fifth-generation tensor cores (tcgen05) for the seed gate's network: shared-memory operand
// tiles in the canonical no-swizzle K-major layout, the instruction and shared-memory matrix
// descriptors, tcgen05.mma issued by one thread with its completion tracked by an mbarrier, the
// accumulator in tensor memory (TMEM) read back with tcgen05.ld.  sm_100a only; 1-GPU code
// (nothing here reads another GPU's memory).
//
// Tile layout (bf16, `rows` x K, K a multiple of 16): 8 x 8 core matrices of 128 contiguous
// bytes (8 rows of 16 bytes); element (r, k) at byte (r / 8) * (K / 8) * 128 + (k / 8) * 128 +
// (r % 8) * 16 + (k % 8) * 2.  In the descriptor's terms: leading-dimension byte offset (between
// the two core matrices of one K step) 128, stride-dimension byte offset (between 8-row groups)
// K / 8 * 128; one MMA of K = 16 starts at the tile plus 256 bytes per K step.
#pragma once

#include <stdint.h>

namespace velo {
  namespace umma {

    __device__ __forceinline__ uint32_t smem_addr(const void* p)
    {
      return static_cast<uint32_t>(__cvta_generic_to_shared(p));
    }

    __host__ __device__ constexpr unsigned tile_offset(unsigned r, unsigned k, unsigned K)
    {
      return (r / 8u) * (K / 8u) * 128u + (k / 8u) * 128u + (r % 8u) * 16u + (k % 8u) * 2u;
    }

    // Shared-memory matrix descriptor: start address, leading and stride byte offsets (16-byte
    // units), version 1 (sm_100), no swizzle.  `tile` 16-byte aligned; k_step selects K columns
    // 16 k_step .. 16 k_step + 15.
    __device__ __forceinline__ uint64_t desc(const void* tile, unsigned K, unsigned k_step)
    {
      const uint32_t a = smem_addr(tile) + 256u * k_step;
      uint64_t d = uint64_t((a >> 4) & 0x3FFFu);
      d |= uint64_t((128u >> 4) & 0x3FFFu) << 16;
      d |= uint64_t(((K / 8u * 128u) >> 4) & 0x3FFFu) << 32;
      d |= uint64_t(1) << 46;
      return d;
    }

    // Instruction descriptor of kind::f16: fp32 accumulator, bf16 A and B, both K-major, M x N.
    __host__ __device__ constexpr uint32_t idesc_bf16(unsigned M, unsigned N)
    {
      return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
    }

    // D[tmem] (+)= A x B^T, issued by the calling thread.
    __device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, bool accumulate)
    {
      asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate ? 1u : 0u)
        : "memory");
    }

    // The mbarrier arrives once every MMA this thread issued before has completed.
    __device__ __forceinline__ void commit(uint64_t* bar)
    {
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                   : "memory");
    }

    __device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
    {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }

    // Waits for the phase with parity `phase` to complete, at most `limit` polls; false if not.
    __device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned phase, unsigned limit)
    {
      for (unsigned i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
          "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
          : "=r"(done)
          : "r"(smem_addr(bar)), "r"(phase)
          : "memory");
        if (done) return true;
      }
      return false;
    }

    // Generic-proxy writes to shared memory made visible to the tensor cores (async proxy).
    __device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
    __device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
    __device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

    // TMEM allocation by one full warp: the base address lands in *dst (shared memory).
    __device__ __forceinline__ void alloc(uint32_t* dst, unsigned columns)
    {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)), "r"(columns)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    __device__ __forceinline__ void dealloc(uint32_t taddr, unsigned columns)
    {
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(columns) : "memory");
    }

    // 32 consecutive fp32 columns of this thread's TMEM lane (lane = the warp's 32-lane slice +
    // lane index), then the wait for the load.
    __device__ __forceinline__ void load32(uint32_t taddr, float (&v)[32])
    {
      uint32_t r[32];
      asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (unsigned i = 0; i < 32; ++i)
        v[i] = __uint_as_float(r[i]);
    }

  } // namespace umma
} // namespace velo

// Fifth-generation tensor-core (tcgen05) building blocks for sm_100a:
// shared-memory operand descriptors, instruction descriptors, TMEM
// allocation, MMA issue/commit, TMEM loads and a bounded mbarrier wait.
//
// Operand layout.  Every bf16 operand lives in shared memory as a grid of
// 8 x 16-byte "core matrices" with no swizzle.  A buffer of R rows and C
// columns (row = first index) stores element (r, c) at
//     ((c / 8) * (R / 8) + r / 8) * 128 + (r % 8) * 16 + (c % 8) * 2
// i.e. 8 consecutive columns of one row form one 16-byte line, 8 rows form a
// 128-byte core matrix, core matrices run down the rows first.  The same
// buffer serves as
//   * a K-major operand whose M/N index is the buffer row and whose K index
//     is the buffer column (SBO = 128 B between row blocks, LBO = 16 R bytes
//     between column blocks; K step s starts 32 R s bytes in), or
//   * an MN-major operand whose K index is the buffer row and whose M/N index
//     is the buffer column (LBO = 128 B between row blocks, SBO = 16 R bytes
//     between column blocks; K step s starts 256 s bytes in),
// which is what lets the backward pass use the forward pass's activations
// and weights transposed without a second copy.
#pragma once
#include <cstdint>

namespace zsph {
namespace umma {

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (r, c) in an R-row core-matrix buffer
__host__ __device__ __forceinline__ uint32_t core_off(int R, int r, int c) {
  return (uint32_t)((((c >> 3) * (R >> 3) + (r >> 3)) << 7) + ((r & 7) << 4) + ((c & 7) << 1));
}

// Shared-memory matrix descriptor (no swizzle): start address, leading and
// stride byte offsets in 16-byte units, descriptor version 1 at bit 46.
__device__ __forceinline__ uint64_t sdesc(uint32_t start, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((start >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}
// K step `k` (16 elements) of a buffer used K-major / MN-major (see above)
__device__ __forceinline__ uint64_t kmaj(const void* buf, int R, int k) {
  return sdesc(saddr(buf) + (uint32_t)(32 * R * k), (uint32_t)(16 * R), 128u);
}
__device__ __forceinline__ uint64_t mnmaj(const void* buf, int R, int k) {
  return sdesc(saddr(buf) + (uint32_t)(256 * k), 128u, (uint32_t)(16 * R));
}

// Instruction descriptor for kind::f16 with bf16 A and B, f32 accumulator:
// D format bits [4,6) = 1, A format [7,10) = 1, B format [10,13) = 1,
// A/B major bits 15/16 (1 = MN-major), N >> 3 at [17,23), M >> 4 at [24,29).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A * B, one CTA, issued by a single thread.
__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, bool acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"((uint32_t)acc)
      : "memory");
}
// arrive once on `bar` when every MMA this thread issued so far has completed
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
               : "memory");
}

// TMEM allocation (whole warp), address written to shared memory
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes -> visible to the tensor core
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 TMEM lanes x 32-bit, N consecutive columns per thread (N = 16 or 32),
// followed by the wait that makes the registers valid.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(saddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
constexpr int kMbarPolls = 1 << 22;  // each poll suspends briefly: far above any MMA chain here
// bounded wait for the phase with the given parity to complete
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (int i = 0; i < kMbarPolls; ++i)
    if (mbar_try(bar, parity)) return true;
  return false;
}

}  // namespace umma
}  // namespace zsph

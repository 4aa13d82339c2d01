// mc_umma.cuh - the sm_100a tensor-core pieces the guiding MLP uses:
// shared-memory matrix descriptors, the kind::f16 instruction descriptor,
// tcgen05.mma issue/commit, TMEM allocation and loads, and bounded mbarrier
// waits. Written from the PTX ISA's descriptions of these instructions.
//
// Operand layout (both operands K-major, no swizzle): an R x K bf16 matrix is
// stored as 8x8 core matrices of 128 contiguous bytes (8 rows of 16 bytes);
// core matrices adjacent in K are 128 bytes apart (leading byte offset) and
// 8-row groups are K*16 bytes apart (stride byte offset). One MMA consumes
// K = 16, i.e. two core matrices along K, so successive K steps advance the
// start address by 256 bytes.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace mc {
namespace umma {

// Byte offset of element (row r, column k) in the K-major layout above.
__device__ __forceinline__ uint32_t kmaj_off(int r, int k, int K) {
    return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: start address, leading byte offset (K
// direction, 128 B), stride byte offset (8-row groups), descriptor version 1,
// no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, int K) {
    const uint64_t lbo = 128u >> 4;
    const uint64_t sbo = (uint64_t)(K * 16) >> 4;
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: BF16 A and B (both K-major), FP32 D,
// shape M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A * B^T over one K = 16 slice (single thread issues).
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
        "}"
        :
        : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// D = A(R x K, at sa) * B(N x K, at sb)^T, K a multiple of 16; accumulate
// into D when acc != 0. Issued by one thread.
__device__ __forceinline__ void gemm_k(uint32_t d_tmem, uint32_t sa, uint32_t sb, int K, uint32_t idesc, uint32_t acc) {
    for (int s = 0; s < K / 16; s++) {
        mma_bf16(d_tmem, smem_desc(sa + 256u * s, K), smem_desc(sb + 256u * s, K), idesc, (s > 0 || acc) ? 1u : 0u);
    }
}

// An MMA operand in shared memory, stored in the K-major layout above as a
// matrix of rows x C columns (kmaj_off with K = C). Used with K along its
// columns it is a K-major operand; used with K along its rows it is the same
// bytes read as an MN-major operand (no swizzle): an 8 x 8 core matrix is 8
// K-rows of 8 MN-consecutive elements, MN-adjacent core matrices are 128
// bytes apart (the descriptor's stride byte offset) and K-adjacent ones C*16
// bytes (its leading byte offset). That is how the weight gradients read the
// activations and output gradients, and the data gradients the forward
// weights, without transposed copies.
struct Operand {
    uint32_t addr, lbo, sbo, kstep;  // kstep: start-address advance per K = 16
};
__device__ __forceinline__ Operand kmajor(uint32_t addr, int C) { return {addr, 128u, (uint32_t)C * 16u, 256u}; }
__device__ __forceinline__ Operand mnmajor(uint32_t addr, int C) {
    return {addr, (uint32_t)C * 16u, 128u, 2u * (uint32_t)C * 16u};
}

__device__ __forceinline__ uint64_t smem_desc_raw(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction-descriptor bits of an MN-major A (bit 15) or B (bit 16).
constexpr uint32_t kMajorA_MN = 1u << 15;
constexpr uint32_t kMajorB_MN = 1u << 16;

// D (+)= A * B^T over K (a multiple of 16) with operands of either major-ness
// (the instruction descriptor's major bits must agree). One thread issues.
__device__ __forceinline__ void gemm_op(uint32_t d_tmem, Operand A, Operand B, int K, uint32_t idesc, uint32_t acc) {
    for (int s = 0; s < K / 16; s++) {
        mma_bf16(d_tmem, smem_desc_raw(A.addr + A.kstep * s, A.lbo, A.sbo), smem_desc_raw(B.addr + B.kstep * s, B.lbo, B.sbo),
                 idesc, (s > 0 || acc) ? 1u : 0u);
    }
}

// Arrive on an mbarrier when every MMA this thread issued so far has finished.
__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy writes to shared memory become visible to the tensor core.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for the phase of the given parity; gives up after `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit) {
    const uint32_t a = smem_u32(bar);
    for (long long i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// TMEM allocation by one full warp; the column base lands in *dst (shared).
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (the warp reads its
// 32-lane slice; taddr carries the warp's first lane in bits 16..31), with
// the wait for completion inside the same asm so no use can precede it.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// 32 consecutive FP32 columns of this thread's TMEM lane, as raw bits.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
}

// Two floats -> max(., 0) as a bf16 pair (round to nearest even), lo in the
// low half.
__device__ __forceinline__ uint32_t relu_bf16x2(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

// Eight floats -> eight bf16 (round to nearest even) packed in a uint4, lowest
// column in the lowest address.
__device__ __forceinline__ uint4 pack8_bf16(const float* f) {
    uint4 u;
    __nv_bfloat162 p0 = __floats2bfloat162_rn(f[0], f[1]);
    __nv_bfloat162 p1 = __floats2bfloat162_rn(f[2], f[3]);
    __nv_bfloat162 p2 = __floats2bfloat162_rn(f[4], f[5]);
    __nv_bfloat162 p3 = __floats2bfloat162_rn(f[6], f[7]);
    u.x = *reinterpret_cast<uint32_t*>(&p0);
    u.y = *reinterpret_cast<uint32_t*>(&p1);
    u.z = *reinterpret_cast<uint32_t*>(&p2);
    u.w = *reinterpret_cast<uint32_t*>(&p3);
    return u;
}

__device__ __forceinline__ void unpack8_bf16(uint4 u, float* f) {
    const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int i = 0; i < 4; i++) {
        f[2 * i] = __uint_as_float(w[i] << 16);
        f[2 * i + 1] = __uint_as_float(w[i] & 0xFFFF0000u);
    }
}

}  // namespace umma
}  // namespace mc

// tcgen05.cuh -- inline PTX for the 5th-generation tensor cores (tcgen05:
// MMA with the accumulator in tensor memory, TMEM allocation, loads and
// stores) and the TF32 split used for FP32-class products (3xTF32).
//
// Shared-memory operands use the no-swizzle K-major canonical layout: a
// core matrix is 8 rows x 16 bytes (4 tf32 along K), K-adjacent core
// matrices are LBO = 128 bytes apart, 8-row groups SBO bytes apart.
#pragma once
#include <cuda_fp16.h>

#include <cstdint>
#include <cstring>

#include "ptx.cuh"

namespace h3d {

// ------------------------------------------------------------- tf32 split
__host__ __device__ inline float tf32_round(float f) {
    uint32_t u;
#ifdef __CUDA_ARCH__
    u = __float_as_uint(f);
#else
    std::memcpy(&u, &f, 4);
#endif
    u = (u + 0x1000u) & 0xFFFFE000u;
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float r;
    std::memcpy(&r, &u, 4);
    return r;
#endif
}

// hi + lo ~ v to ~2^-21 relative, both exact tf32 values
__host__ __device__ inline void tf32_split(double v, float &hi, float &lo) {
    hi = tf32_round((float)v);
    lo = tf32_round((float)(v - (double)hi));
}
__host__ __device__ inline void tf32_split_f(float v, float &hi, float &lo) {
    hi = tf32_round(v);
    lo = tf32_round(v - hi);
}
// the same split with lo left in FP32: v - hi is exact, and the tensor core
// reads only its tf32 part, which drops less than 2^-21 |v|
__host__ __device__ inline void tf32_split_fast(float v, float &hi, float &lo) {
    hi = tf32_round(v);
    lo = v - hi;
}

// byte offset of element (row, kk) in a no-swizzle K-major operand whose
// rows hold KC elements (8-row groups SBO = KC / 4 * 128 bytes apart)
__host__ __device__ inline uint32_t canon_off(int row, int kk, int KC) {
    return (uint32_t)((row >> 3) * (KC / 4) * 128 + (kk >> 2) * 128 + (row & 7) * 16 + (kk & 3) * 4);
}

// ------------------------------------------------ FP16 hi/lo operands
// FP16 hi/lo of a pair (x, y), each as a packed pair (x in the low half):
// hi = x rounded to 11 significant bits in FP32 (exact in FP16 in its
// normal range), lo = x - hi (exact in FP32) rounded to FP16 -- two
// conversions per pair
__device__ __forceinline__ uint2 f16_split2(float x, float y) {
    const float hx = tf32_round(x), hy = tf32_round(y);
    const __half2 hi = __floats2half2_rn(hx, hy);
    const __half2 lo = __floats2half2_rn(x - hx, y - hy);
    return make_uint2(*reinterpret_cast<const uint32_t *>(&hi), *reinterpret_cast<const uint32_t *>(&lo));
}

// 2^(13 - e) for mx in [2^e, 2^(e+1)): scales the largest entry into
// [2^13, 2^14) (1 for mx = 0 or not finite)
__device__ __forceinline__ float pow2_scale_13(float mx) {
    const uint32_t b = __float_as_uint(mx);
    const int ex = (int)((b >> 23) & 0xffu);
    if (mx <= 0.f || ex == 0xff) return 1.f;
    int e = (ex == 0 ? -126 : ex - 127);
    e = max(-100, min(100, e));
    return __uint_as_float((uint32_t)(127 + 13 - e) << 23);
}

// 1 / s for a power of two s (exact)
__device__ __forceinline__ float pow2_inv(float s) {
    return __uint_as_float((254u - ((__float_as_uint(s) >> 23) & 0xffu)) << 23);
}

// ------------------------------------------------------------ tcgen05 PTX
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    // start address, LBO, SBO (all >> 4), version 1 (sm_100), no swizzle
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::tf32, fp32 accumulator, A and B K-major, M rows (64 or 128), N columns
__host__ __device__ constexpr uint32_t umma_idesc_tf32(int n, int m = 128) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// kind::f16 with FP16 A and B, fp32 accumulator, K-major, M rows, N columns
__host__ __device__ constexpr uint32_t umma_idesc_f16(int n, int m = 128) {
    return (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// D (TMEM) (+)= A (shared memory) B^T (shared memory)
__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// D (TMEM) (+)= A (TMEM: lane = row, one tf32 per column) B^T (shared memory)
__device__ __forceinline__ void umma_tf32_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t idesc,
                                             uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(tmem_d), "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// kind::f16: D (TMEM) (+)= A (TMEM: lane = row, two fp16 per column) B^T (shared memory), K = 16
__device__ __forceinline__ void umma_f16_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(tmem_d), "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// kind::f16: D (TMEM) (+)= A (shared memory) B^T (shared memory), K = 16
__device__ __forceinline__ void umma_f16_ss(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// arrive on `bar` once every tcgen05 operation this thread issued so far has completed
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes made visible to the async proxy (the tensor core)
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// warp-wide TMEM allocation of `cols` columns (a power of two >= 32); the
// base address is written to *slot
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols) : "memory");
}

// 16 consecutive fp32 columns of this warp's 32 TMEM lanes (lane = thread);
// the values may be used only after tmem_wait_ld()
__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, float *v) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7]),
          "=f"(v[8]), "=f"(v[9]), "=f"(v[10]), "=f"(v[11]), "=f"(v[12]), "=f"(v[13]), "=f"(v[14]), "=f"(v[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld32_nowait(uint32_t taddr, float *v) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7]),
          "=f"(v[8]), "=f"(v[9]), "=f"(v[10]), "=f"(v[11]), "=f"(v[12]), "=f"(v[13]), "=f"(v[14]), "=f"(v[15]),
          "=f"(v[16]), "=f"(v[17]), "=f"(v[18]), "=f"(v[19]), "=f"(v[20]), "=f"(v[21]), "=f"(v[22]), "=f"(v[23]),
          "=f"(v[24]), "=f"(v[25]), "=f"(v[26]), "=f"(v[27]), "=f"(v[28]), "=f"(v[29]), "=f"(v[30]), "=f"(v[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld8_nowait(uint32_t taddr, float *v) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
                 : "r"(taddr));
}
// waits for this thread's outstanding TMEM loads; the registers they fill
// pass through the statement so that no use of them is scheduled before it
__device__ __forceinline__ void tmem_wait_ld(float (&v)[32]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+f"(v[0]), "+f"(v[1]), "+f"(v[2]), "+f"(v[3]), "+f"(v[4]), "+f"(v[5]), "+f"(v[6]), "+f"(v[7]),
                   "+f"(v[8]), "+f"(v[9]), "+f"(v[10]), "+f"(v[11]), "+f"(v[12]), "+f"(v[13]), "+f"(v[14]),
                   "+f"(v[15]), "+f"(v[16]), "+f"(v[17]), "+f"(v[18]), "+f"(v[19]), "+f"(v[20]), "+f"(v[21]),
                   "+f"(v[22]), "+f"(v[23]), "+f"(v[24]), "+f"(v[25]), "+f"(v[26]), "+f"(v[27]), "+f"(v[28]),
                   "+f"(v[29]), "+f"(v[30]), "+f"(v[31])
                 :
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_ld(float (&v)[16]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+f"(v[0]), "+f"(v[1]), "+f"(v[2]), "+f"(v[3]), "+f"(v[4]), "+f"(v[5]), "+f"(v[6]), "+f"(v[7]),
                   "+f"(v[8]), "+f"(v[9]), "+f"(v[10]), "+f"(v[11]), "+f"(v[12]), "+f"(v[13]), "+f"(v[14]),
                   "+f"(v[15])
                 :
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_ld(float (&v)[8]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+f"(v[0]), "+f"(v[1]), "+f"(v[2]), "+f"(v[3]), "+f"(v[4]), "+f"(v[5]), "+f"(v[6]), "+f"(v[7])
                 :
                 : "memory");
}

// 16 / 32 consecutive fp32 columns into this warp's 32 TMEM lanes (lane =
// thread); complete once tmem_wait_st() returns
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float (&v)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16};" ::"r"(taddr),
        "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]), "f"(v[8]),
        "f"(v[9]), "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15])
        : "memory");
}
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const float (&v)[32]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};" ::"r"(
            taddr),
        "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]), "f"(v[8]),
        "f"(v[9]), "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15]), "f"(v[16]),
        "f"(v[17]), "f"(v[18]), "f"(v[19]), "f"(v[20]), "f"(v[21]), "f"(v[22]), "f"(v[23]), "f"(v[24]),
        "f"(v[25]), "f"(v[26]), "f"(v[27]), "f"(v[28]), "f"(v[29]), "f"(v[30]), "f"(v[31])
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

}  // namespace h3d

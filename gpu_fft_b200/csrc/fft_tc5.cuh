// fft_tc5.cuh — radix-16 FFT stages on the fifth-generation tensor cores
// (sm_100a: tcgen05.mma with accumulators in tensor memory).
//
// One radix-16 stage of a column tile is a batch of 16-point DFTs
// y = F x, F[j][o] = exp(-+ 2 pi i j o / 16).  In real form, with the 16
// inputs of one butterfly as a row of 32 values [Re x_0..15 | Im x_0..15]
// and the outputs as [Re y_0..15 | Im y_0..15], the batch is the product
// Y = X B of an (M x 32) matrix X by the constant 32 x 32 matrix
//   B = [[Re F, Im F], [-Im F, Re F]].
// FP32 accuracy from TF32 operands (10-bit mantissas): X = Xh + Xl with
// Xh = X rounded to TF32 and Xl = X - Xh (exact; the tensor core reads its
// top 10 mantissa bits), B = Bh + Bl likewise, and
//   Y ~ Xl Bh + Xh Bl + Xh Bh
// (the dropped Xl Bl term is below 2^-21 relative), accumulated in FP32.
//
// Tensor memory: every block of 128 butterflies (one per lane, 128 lanes)
// owns 96 columns: Xh (32), Xl (32) and Y (32).  Each thread holds one
// butterfly, writes its 64 operand values to its own lane (tcgen05.st),
// and after a block barrier one thread issues, per block, 12 MMAs of
// M = 128, N = 32, K = 8 (kind::tf32, A from tensor memory, B from shared
// memory), commits them to an mbarrier, and every thread reads its 32
// outputs back (tcgen05.ld).
//
// B in shared memory, K-major without swizzle: element (k, n) at byte
//   (k / 8) * 1024 + ((k % 8) / 4) * 128 + (n / 8) * 256 + (n % 8) * 16 + (k % 4) * 4,
// i.e. 8 x 16-byte core matrices with the two K halves of one MMA 128 bytes
// apart (leading byte offset) and 8-row groups of N 256 bytes apart (stride
// byte offset); the MMA of K-step s starts at byte s * 1024.
#pragma once
#include <cstdint>

namespace gpufft {
namespace tc5 {

constexpr uint32_t kTmemCols = 512;   // the whole tensor memory of the SM (one CTA per SM)
constexpr int kColsPerBlock = 96;     // Xh, Xl, Y of one 128-butterfly block
constexpr int kMaxBlocks = 5;         // 5 x 96 <= 512

// per-CTA state (static shared memory, one instance per kernel)
struct __align__(128) State {
    float b[2][1024];   // Bh, Bl in the MMA layout above
    uint64_t bar;       // MMA completion
    uint32_t tmem;      // tensor-memory base address
    uint32_t phase;     // MMA groups completed so far
    int err;            // a bounded wait ran out
};
__device__ __forceinline__ State &state() {
    __shared__ State s;
    return s;
}

__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint32_t rna_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
    return r;
}

// ---- allocation (one whole warp) ----
__device__ __forceinline__ void tmem_alloc(uint32_t *dst) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(saddr(dst)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(kTmemCols) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

// 16 consecutive columns of this thread's lane (lane field of taddr = the warp's quarter)
__device__ __forceinline__ void st16(uint32_t taddr, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};\n" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
        "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}
__device__ __forceinline__ void ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
}

// shared-memory matrix descriptor: K-major, no swizzle, LBO 128 B, SBO 256 B
__device__ __forceinline__ uint64_t bdesc(uint32_t smem_byte_addr) {
    return (uint64_t)((smem_byte_addr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(256 >> 4) << 32) |
           (1ull << 46);  // descriptor version 1 (sm_100); base offset 0, layout "no swizzle" (0)
}
// instruction descriptor: D F32, A and B TF32, both K-major, N = 32, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma(uint32_t d, uint32_t a, uint64_t b, bool acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n}\n" ::"r"(d),
        "r"(a), "l"(b), "r"(kIdesc), "r"((uint32_t)acc)
        : "memory");
}
__device__ __forceinline__ void commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(saddr(bar))
                 : "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait (about 2 s of global timer)
__device__ __forceinline__ bool bar_wait(uint64_t *bar, uint32_t parity) {
    if (bar_try(bar, parity)) return true;
    unsigned long long t0, t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t0));
    while (true) {
        for (int i = 0; i < 64; ++i)
            if (bar_try(bar, parity)) return true;
        asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
        if (t - t0 > 2000000000ull) return false;
    }
}

// Kernel prologue (every thread of the CTA): B for the transform direction,
// the barrier, and the tensor memory (allocated by warp 0).
template <bool FWD>
__device__ __forceinline__ void setup() {
    State &s = state();
    for (int idx = threadIdx.x; idx < 1024; idx += blockDim.x) {
        const int k = idx >> 5, n = idx & 31;
        const int j = k & 15, o = n & 15;
        double sn, c;
        sincospi((double)((j * o) & 15) / 8.0, &sn, &c);
        const double im = FWD ? -sn : sn;
        const double v = k < 16 ? (n < 16 ? c : im) : (n < 16 ? -im : c);
        const uint32_t hi = rna_tf32((float)v);
        const uint32_t lo = rna_tf32((float)(v - (double)__uint_as_float(hi)));
        const int at = (k >> 3) * 256 + ((k & 7) >> 2) * 32 + (n >> 3) * 64 + (n & 7) * 4 + (k & 3);
        s.b[0][at] = __uint_as_float(hi);
        s.b[1][at] = __uint_as_float(lo);
    }
    // the generic-proxy writes of B are read by the tensor core (async proxy)
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(saddr(&s.bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        s.phase = 0;
        s.err = 0;
    }
    if (threadIdx.x < 32) tmem_alloc(&s.tmem);
    fence_before();
    __syncthreads();
    fence_after();
}
// Kernel epilogue (every thread): frees the tensor memory.  Returns true
// when no wait ran out.
__device__ __forceinline__ bool teardown() {
    State &s = state();
    fence_before();
    __syncthreads();
    if (threadIdx.x < 32) {
        fence_after();
        tmem_dealloc(s.tmem);
    }
    return s.err == 0;
}

// The MMAs of nblk blocks (one thread): Y = Xl Bh + Xh Bl + Xh Bh, K = 32 in
// four steps of 8, then one commit to the barrier.
__device__ __forceinline__ void issue(int nblk) {
    State &s = state();
    fence_after();
    const uint32_t bh = saddr(&s.b[0][0]), bl = saddr(&s.b[1][0]);
    for (int q = 0; q < nblk; ++q) {
        const uint32_t xh = s.tmem + (uint32_t)(q * kColsPerBlock), xl = xh + 32, y = xh + 64;
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) mma(y, xl + 8 * ks, bdesc(bh + 1024 * ks), ks > 0);
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) mma(y, xh + 8 * ks, bdesc(bl + 1024 * ks), true);
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) mma(y, xh + 8 * ks, bdesc(bh + 1024 * ks), true);
    }
    commit(&s.bar);
}

}  // namespace tc5
}  // namespace gpufft

// fast_queue.cu — instantiations of the queue-scheduled Pass A
// (fft_queue.cuh): 512 consumer threads (two z-rows per warp, 32-row items)
// plus one copy-issuing warp, one CTA per SM; ring depth 2 or 3.
#include "fast_registry.h"
#include "fft_queue.cuh"

namespace gpufft {
namespace fast {

// (Ny, Nz/2, consumer threads, y radix variant, ring depth, columns per column item)
// (QA_ENTRY_FB: the forward's row items written back by bulk stores as well)
#define QA_ENTRY_X(T, DT, NY, M, NT, VY, NBUF, WY, FB)                                                          \
    {2, NBUF, DT, NY, M, 2, WY, NT + 32, VY, 0, q::QShape<T, NY, M, NT, NBUF, WY>::smem_bytes(),                \
     (const void *)q::pass_a_queue<T, NY, M, NT, true, VY, NBUF, WY, FB>,                                       \
     (const void *)q::pass_a_queue<T, NY, M, NT, false, VY, NBUF, WY, FB>, nullptr, nullptr}
#define QA_ENTRY(T, DT, NY, M, NT, VY, NBUF, WY) QA_ENTRY_X(T, DT, NY, M, NT, VY, NBUF, WY, 0)
#define QA_ENTRY_FB(T, DT, NY, M, NT, VY, NBUF, WY) QA_ENTRY_X(T, DT, NY, M, NT, VY, NBUF, WY, 1)

const VariantA kVariantsA_f32q[] = {
    // 512^2 planes, B200, ms per launch at 512^3 (forward / inverse, queue
    // depth 24-32): 16 consumer warps, 16-column items, 3-deep ring of 72 KB
    // buffers 0.396 / 0.407; 2-deep 0.412 / 0.435.  Measured and dropped:
    // 8 consumer warps (16-row items) 0.425 / 0.473; 8-column items with a
    // 4-deep ring 0.475 / 0.520 (8 warps) and 0.457 / 0.500 (16 warps); the y
    // FFT as 16 x 16 x 2 0.403 / 0.441; the y FFT alternating with a 64 KB
    // scratch tile (two barriers per item fewer, 2-deep ring) 0.406 / 0.417;
    // two groups of 8 consumer warps, each on its own 16-row or 8-column
    // items (barrier waits of one group overlapping the other's work), 4- or
    // 5-deep ring of 40 KB buffers 0.467-0.476 / 0.484-0.492
    // Row items of both directions written back by bulk stores from the copy
    // warp: 0.369 / 0.369 (forward by the consumers' own stores 0.384, and
    // 0.408 for the inverse before its rows went by bulk store too).  At
    // 512 x 128 and in FP64 the forward's bulk stores were slower (the copy
    // warp waits for each before it publishes): 0.470 against 0.443 ms.
    // The inverse's column items with their even rows by tensor store as
    // well: inverse 0.354 (forward with the same: 0.371 against 0.369).
    QA_ENTRY_X(float, 0, 512, 256, 512, 0, 3, 16, 3),
    QA_ENTRY_X(float, 0, 512, 256, 512, 0, 2, 16, 3),

    // 512 x 128 planes (1024 x 512 x 256): the row FFT is 16 x 8; queue depth
    // 32: 0.464 / 0.445 ms (depth 16: 0.517 / 0.626), the cluster form 0.484 / 0.442
    // (the inverse's column items with their even rows by tensor store:
    // 0.433 against 0.431; four rows per warp, 8 lanes a row, so that no lane
    // idles in the radix-16 step: 0.456 / 0.440 against 0.449 / 0.430 --
    // not registered)
    QA_ENTRY(float, 0, 512, 128, 512, 0, 3, 16),
    QA_ENTRY(float, 0, 512, 128, 256, 0, 3, 16),
    // 360 x 240 planes (384 x 360 x 480): the row FFT is 16 x 15 (prime-factor
    // radix 15), 4-deep ring of 52 KB buffers; ms per launch: 20-row items on
    // 10 consumer warps 0.230 / 0.235 (an 11-warp CTA gets 168 registers a
    // thread), 24-row items on 12 warps 0.270 / 0.224 (13 warps get 128 and
    // the forward spills), 18-row items on 9 warps 0.236 / 0.245
    // (the inverse's column items with their even rows by tensor store:
    // inverse 0.232 against 0.235; the forward's rows by bulk store as well:
    // forward 0.230 against 0.222 -- not used)
    QA_ENTRY_X(float, 0, 360, 240, 320, 0, 4, 16, 2),
    QA_ENTRY(float, 0, 360, 240, 320, 0, 4, 16),
    QA_ENTRY(float, 0, 360, 240, 384, 0, 4, 16),
    QA_ENTRY(float, 0, 360, 240, 288, 0, 4, 16),
};
const int kNumVariantsA_f32q = sizeof(kVariantsA_f32q) / sizeof(kVariantsA_f32q[0]);

// Pass B fed by tensor copies: (Nx, consumer threads, radix variant, ring depth
// [, columns per tile: 128-byte rows when omitted])
#define TB_ENTRY_W(T, DT, NX, NT, V, NBUF, WW)                                                                    \
    {3, DT, NX, q::BShape<T, NX, NT, NBUF, WW>::W, NT, V, q::BShape<T, NX, NT, NBUF, WW>::smem_bytes(),          \
     (const void *)q::pass_b_tma<T, NX, NT, true, V, NBUF, false, WW>,                                            \
     (const void *)q::pass_b_tma<T, NX, NT, false, V, NBUF, false, WW>,                                           \
     (const void *)q::pass_b_tma<T, NX, NT, true, V, NBUF, true, WW>,                                             \
     (const void *)q::pass_b_tma<T, NX, NT, false, V, NBUF, true, WW>}
#define TB_ENTRY(T, DT, NX, NT, V, NBUF) TB_ENTRY_W(T, DT, NX, NT, V, NBUF, 0)

const VariantB kVariantsB_f32q[] = {
    // 512^3 on B200, ms per launch (fwd / inv): 2-deep ring 0.184 / 0.183
    // (the tile written back in place and stored by tensor copies from thread
    // 0, its buffer refilled one tile later in a 3-deep ring: 0.192-0.195),
    // 3-deep 0.211 / 0.210 (256 threads) and 0.207 / 0.207 (512 threads),
    // against 0.204 / 0.203 for the cp.async double buffer
    TB_ENTRY(float, 0, 512, 256, 1, 2),
    TB_ENTRY(float, 0, 512, 512, 1, 2),
    TB_ENTRY(float, 0, 512, 256, 0, 2),
    TB_ENTRY(float, 0, 512, 256, 1, 3),
    TB_ENTRY(float, 0, 512, 512, 1, 3),
    // radix-16 stages on tcgen05 (v = 3, fft_tc5.cuh): only plans made with
    // GPUFFT_PLAN_TC_SPLIT use it.  512^3: 0.360 / 0.360 ms, 1.8e-7 from the
    // plain pass (mma.sync forms 0.427-0.503 ms).  Fusing Xh [Bh | Bl] into
    // N = 64 MMAs with per-block barriers: 0.374 ms and 3.8e-7, not kept.
    // Pipelining tiles in a 3-deep ring (tile k's first tensor-core stage on
    // the tensor cores while the CTA runs tile k-1's last stage): 0.365 ms,
    // no better, not kept.
    TB_ENTRY(float, 0, 512, 512, 3, 2),
    // Nx = 384 (384 x 360 x 480): two boxes of 192 rows per tile; ms per
    // launch: 3-deep ring 0.0945, 2-deep 0.103 (256 or 512 threads), against
    // 0.108 for the cp.async double buffer
    TB_ENTRY(float, 0, 384, 256, 0, 3),
    TB_ENTRY(float, 0, 384, 256, 0, 2),
    TB_ENTRY(float, 0, 384, 512, 0, 2),
    // (Nx = 1024, 8-column tiles of 64-byte rows in a 2-deep ring of 64 KB,
    // TB_ENTRY_W(float, 0, 1024, 256, 0, 2, 8): 0.216 ms per launch at
    // 1024x512x256 against 0.221 for pass_b_pipe1, but 3.36 against 1.85 ms
    // at 1024^3, where the two halves of a 128-byte line no longer meet in
    // L2 -- not registered)
    // (Nx = 1024, one 128 KB tile buffer refilled during the last stage by
    // tensor copies: 0.226 ms per launch at 1024x512x256 against 0.222 for
    // the same scheme with cp.async, pass_b_pipe1 -- not registered)
};
const int kNumVariantsB_f32q = sizeof(kVariantsB_f32q) / sizeof(kVariantsB_f32q[0]);

// FP64: 16-row items on 8 consumer warps (the radix-16 row butterflies need
// 64 registers of data), 8-column (128-byte) items, a 2-deep ring (three
// 72 KB buffers and the 16 KB of tables do not fit)
const VariantA kVariantsA_f64q[] = {
    // the forward's column items written back by tensor stores of every row
    // from the copy warp: forward 0.769 against 0.801 ms (the inverse's the
    // same way: 0.797 against 0.786 -- not used); the forward's row items by
    // bulk stores as well, each awaited at the end of the copy warp's
    // iteration: forward 0.720
    QA_ENTRY_X(double, 1, 512, 256, 256, 0, 2, 8, 5),
    QA_ENTRY_X(double, 1, 512, 256, 256, 0, 2, 8, 4),
    QA_ENTRY(double, 1, 512, 256, 256, 0, 2, 8),
    // 512 x 128 planes (1024 x 512 x 256): two 74 KB buffers
    // (forward column items by tensor stores: 0.966 against 1.001 ms forward;
    // and the forward's row items by bulk stores: 0.921)
    QA_ENTRY_X(double, 1, 512, 128, 256, 0, 2, 8, 5),
    QA_ENTRY_X(double, 1, 512, 128, 256, 0, 2, 8, 4),
    QA_ENTRY(double, 1, 512, 128, 256, 0, 2, 8),
    // 360 x 240 planes (384 x 360 x 480): 12-row items on 6 consumer warps,
    // two boxes of 180 rows per column item, 2- or 3-deep ring of 51 KB buffers
    // (forward column items by tensor stores: 0.440 against 0.454 ms forward;
    // the forward's row items by bulk stores as well: 0.447 -- not used)
    QA_ENTRY_X(double, 1, 360, 240, 192, 0, 3, 8, 4),
    QA_ENTRY(double, 1, 360, 240, 192, 0, 3, 8),
    QA_ENTRY(double, 1, 360, 240, 192, 0, 2, 8),
};
const int kNumVariantsA_f64q = sizeof(kVariantsA_f64q) / sizeof(kVariantsA_f64q[0]);

const VariantB kVariantsB_f64q[] = {
    TB_ENTRY(double, 1, 512, 256, 0, 2),
    TB_ENTRY(double, 1, 512, 512, 0, 2),
    // Nx = 384, 8-column tiles of 48 KB: 3-deep ring 0.192 ms per launch,
    // 2-deep 0.210, the cp.async double buffer 0.216.  (Nx = 1024, one 128 KB
    // buffer refilled during the last stage: 0.462 against 0.433 for the
    // same scheme with cp.async -- not registered)
    TB_ENTRY(double, 1, 384, 256, 0, 3),
    TB_ENTRY(double, 1, 384, 256, 0, 2),
    // (Nx = 1024, 4-column tiles of 64-byte rows in a 2-deep ring: 0.535 ms
    // per launch at 1024x512x256 against 0.432 for pass_b_pipe1 -- not registered)
};
const int kNumVariantsB_f64q = sizeof(kVariantsB_f64q) / sizeof(kVariantsB_f64q[0]);

}  // namespace fast
}  // namespace gpufft

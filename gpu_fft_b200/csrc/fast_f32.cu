// fast_f32.cu — FP32 instantiations of the compile-time specialised passes.
// Tile shapes: column tiles of 8 or 16 complex (64/128-byte rows), row tiles
// of whole rows per warp, 256 threads per CTA; see fft_fast.cuh.
#include "fast_entries.h"

namespace gpufft {
namespace fast {

const VariantA kVariantsA_f32[] = {
    A_ENTRY(float, 0, 512, 256, 2, 8, 256, 0, 0, 3),
    A_ENTRY(float, 0, 512, 256, 2, 16, 256, 0, 0, 2),
    A_ENTRY(float, 0, 512, 256, 2, 8, 256, 0, 0, 4),
    A_ENTRY(float, 0, 512, 256, 2, 8, 256, 1, 0, 3),
    // 1024x512x256 planes: four rows per warp and 16-column tiles, 2-CTA
    // clusters: 0.484 / 0.442 ms per launch against 0.573 / 0.519 for two
    // rows and 8-column tiles
    A_ENTRY(float, 0, 512, 128, 4, 16, 256, 0, 0, 2),
    A_ENTRY(float, 0, 512, 128, 2, 16, 256, 0, 0, 2),
    A_ENTRY(float, 0, 512, 128, 4, 8, 256, 0, 0, 2),
    A_ENTRY(float, 0, 512, 128, 2, 8, 256, 0, 0, 2),
    // plane held in the cluster's shared memory: correct, measured slower at 512^3
    // (one 180 KB CTA per SM leaves 28 SMs idle); kept as an autotuning candidate
    D_ENTRY(float, 0, 512, 256, 2, 8, 512, 8, 0, 0, 1),
    A_ENTRY(float, 0, 1024, 512, 1, 8, 256, 0, 0, 2),
    A_ENTRY(float, 0, 1024, 512, 1, 16, 512, 0, 0, 1),
    // 384x360x480 planes: two rows per warp and 16-column tiles at two CTAs
    // per SM (it spills some, which costs less than the occupancy it buys):
    // 0.322 / 0.315 ms per launch against 0.53 for the generic kernels and
    // 0.51 / 0.56 for one 232-register CTA per SM
    A_ENTRY(float, 0, 360, 240, 2, 16, 256, 0, 0, 2),
    A_ENTRY(float, 0, 360, 240, 2, 8, 256, 0, 0, 2),
    A_ENTRY(float, 0, 360, 240, 1, 8, 256, 0, 0, 1),
    A_ENTRY(float, 0, 256, 128, 2, 8, 256, 0, 0, 2),
    A_ENTRY(float, 0, 192, 96, 1, 8, 256, 0, 0, 2),
    A_ENTRY(float, 0, 160, 80, 2, 8, 256, 0, 0, 2),
    A_ENTRY(float, 0, 128, 64, 4, 8, 256, 0, 0, 2),
    A_ENTRY(float, 0, 128, 32, 4, 8, 256, 0, 0, 2),
    A_ENTRY(float, 0, 96, 48, 2, 8, 256, 0, 0, 2),
    A_ENTRY(float, 0, 64, 32, 4, 8, 256, 0, 0, 2),
    // column tiles copied ahead by cp.async: 1024^2 planes, split Pass A,
    // 4.02 / 3.95 ms against 4.23 / 4.11 (at 512^2 it was 4% slower)
    AC_ENTRY(float, 0, 1024, 512, 1, 16, 512, 0, 0, 1),
};
const int kNumVariantsA_f32 = sizeof(kVariantsA_f32) / sizeof(kVariantsA_f32[0]);

const VariantB kVariantsB_f32[] = {
    // 512: cp.async double-buffered tiles first (0.209 ms per launch at 512^3
    // vs 0.275 ms for the best single-buffered kernel, on B200)
    P_ENTRY(float, 0, 512, 16, 256, 1, 2),
    P_ENTRY(float, 0, 512, 16, 512, 1, 1),
    P_ENTRY(float, 0, 512, 8, 512, 0, 2),
    B_ENTRY(float, 0, 512, 16, 256, 1, 2),
    B_ENTRY(float, 0, 512, 16, 256, 0, 3),
    // 128-byte tile rows matter more than double buffering at Nx = 1024
    // (2.36 ms per launch at 1024^3 against 3.57 ms for 8-column tiles); the
    // one 128 KB tile buffer refilled during the last stage: 1.83 ms
    Q_ENTRY(float, 0, 1024, 16, 512, 0, 1),
    B_ENTRY(float, 0, 1024, 16, 512, 0, 1),
    B_ENTRY(float, 0, 1024, 16, 1024, 0, 1),
    B_ENTRY(float, 0, 1024, 8, 256, 0, 2),
    P_ENTRY(float, 0, 1024, 8, 256, 0, 2),
    P_ENTRY(float, 0, 384, 16, 256, 0, 2),
    B_ENTRY(float, 0, 384, 16, 256, 0, 2),
    P_ENTRY(float, 0, 256, 16, 256, 0, 2),
    B_ENTRY(float, 0, 256, 16, 256, 0, 2),
    B_ENTRY(float, 0, 192, 16, 256, 0, 2),
    B_ENTRY(float, 0, 160, 16, 256, 0, 2),
    P_ENTRY(float, 0, 128, 16, 256, 0, 2),
    B_ENTRY(float, 0, 128, 16, 256, 0, 2),
    B_ENTRY(float, 0, 96, 16, 256, 0, 2),
    B_ENTRY(float, 0, 64, 16, 256, 0, 2),
    // one refilled tile buffer (measured at 512^3: 0.219 / 0.253 ms against
    // 0.207 for the double-buffered kernel; at 1024^3 1.88 ms with 1024 threads)
    Q_ENTRY(float, 0, 1024, 16, 1024, 0, 1),
    Q_ENTRY(float, 0, 512, 16, 256, 1, 2),
    Q_ENTRY(float, 0, 512, 16, 512, 1, 1),
    // tensor-core radix-16 stages (v = 2): only plans made with
    // GPUFFT_PLAN_TC_SPLIT use these, and they use nothing else
    P_ENTRY(float, 0, 512, 16, 512, 2, 1),
    P_ENTRY(float, 0, 512, 16, 256, 2, 2),
    B_ENTRY(float, 0, 512, 16, 256, 2, 2),
    Q_ENTRY(float, 0, 1024, 16, 512, 2, 1),
    B_ENTRY(float, 0, 1024, 16, 512, 2, 1),
};
const int kNumVariantsB_f32 = sizeof(kVariantsB_f32) / sizeof(kVariantsB_f32[0]);

}  // namespace fast
}  // namespace gpufft

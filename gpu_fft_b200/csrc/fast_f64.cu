// fast_f64.cu — FP64 instantiations of the compile-time specialised passes.
// Tile shapes: column tiles of 4 or 8 complex (64/128-byte rows), row tiles
// of whole rows per warp, 256 threads per CTA; see fft_fast.cuh.
#include "fast_entries.h"

namespace gpufft {
namespace fast {

const VariantA kVariantsA_f64[] = {
    A_ENTRY(double, 1, 512, 256, 2, 8, 256, 0, 0, 2),
    A_ENTRY(double, 1, 512, 256, 2, 4, 256, 0, 0, 2),
    // 1024x512x256: planes of 512 x 129
    // four rows per warp at 128 registers: 1.04 / 0.97 ms per launch on
    // 2-CTA clusters against 1.03 / 1.08 for two rows
    A_ENTRY(double, 1, 512, 128, 4, 8, 256, 0, 0, 2),
    A_ENTRY(double, 1, 512, 128, 2, 8, 256, 0, 0, 1),
    A_ENTRY(double, 1, 512, 128, 2, 4, 256, 0, 0, 1),
    // 384x360x480 planes: spills about 800 bytes at 255 registers and is
    // still faster than the generic kernels (0.79 / 0.90 ms per launch
    // against 0.96 / 0.96)
    A_ENTRY(double, 1, 360, 240, 2, 8, 256, 0, 0, 1),
    // 128^3 (the 256^2 plane spills even at 255 registers: generic)
    A_ENTRY(double, 1, 128, 64, 4, 8, 256, 0, 0, 1),
};
const int kNumVariantsA_f64 = sizeof(kVariantsA_f64) / sizeof(kVariantsA_f64[0]);

const VariantB kVariantsB_f64[] = {
    P_ENTRY(double, 1, 512, 8, 256, 0, 2),
    P_ENTRY(double, 1, 512, 4, 256, 0, 2),
    B_ENTRY(double, 1, 512, 8, 256, 0, 2),
    B_ENTRY(double, 1, 512, 4, 256, 0, 2),
    Q_ENTRY(double, 1, 512, 8, 256, 0, 2),
    B_ENTRY(double, 1, 128, 8, 256, 0, 2),
    // 1024 (8 x 16-byte complex = 128-byte tile rows), 384, 256
    Q_ENTRY(double, 1, 1024, 8, 512, 0, 1),
    B_ENTRY(double, 1, 1024, 8, 512, 0, 1),
    B_ENTRY(double, 1, 1024, 4, 256, 0, 1),
    P_ENTRY(double, 1, 384, 8, 256, 0, 1),
    B_ENTRY(double, 1, 384, 8, 256, 0, 1),
    P_ENTRY(double, 1, 256, 8, 256, 0, 1),
    B_ENTRY(double, 1, 256, 8, 256, 0, 1),
};
const int kNumVariantsB_f64 = sizeof(kVariantsB_f64) / sizeof(kVariantsB_f64[0]);

}  // namespace fast
}  // namespace gpufft

// fast_f32_3s.cu — FP32 specialisations for the 3-smooth lengths 2^a 3^b of
// the serving mix (32..486) that the main table (fast_f32.cu) does not cover:
// Pass A of cubic grids (Ny = n, Nz/2 = n/2) and Pass B of length n.  A
// separate translation unit, so the two tables compile in parallel.  Pass A
// entries are kept only where they beat the generic kernels (measured R2C+C2R,
// B200): 32-72^3 1.5x, 108^3 1.3x, 144^3 1.35x, 288^3 1.4x, 432^3 1.2x; at
// 162, 216, 324 and 486 (many radix-3 stages) the generic Pass A was as fast.
#include "fast_entries.h"

namespace gpufft {
namespace fast {

const VariantA kVariantsA_f32s[] = {
    A_ENTRY(float, 0, 32, 16, 4, 8, 256, 0, 0, 2),
    A_ENTRY(float, 0, 36, 18, 4, 8, 256, 0, 0, 2),
    A_ENTRY(float, 0, 48, 24, 4, 8, 256, 0, 0, 2),
    A_ENTRY(float, 0, 54, 27, 4, 8, 256, 0, 0, 2),
    A_ENTRY(float, 0, 72, 36, 2, 8, 256, 0, 0, 2),
    A_ENTRY(float, 0, 108, 54, 2, 8, 256, 0, 0, 2),
    A_ENTRY(float, 0, 144, 72, 2, 8, 256, 0, 0, 2),
    A_ENTRY(float, 0, 288, 144, 2, 8, 256, 0, 0, 2),
    A_ENTRY(float, 0, 432, 216, 1, 8, 256, 0, 0, 2),
};
const int kNumVariantsA_f32s = sizeof(kVariantsA_f32s) / sizeof(kVariantsA_f32s[0]);

const VariantB kVariantsB_f32s[] = {
    P_ENTRY(float, 0, 32, 16, 512, 0, 1),
    B_ENTRY(float, 0, 32, 8, 256, 0, 2),
    P_ENTRY(float, 0, 36, 16, 512, 0, 1),
    B_ENTRY(float, 0, 36, 8, 256, 0, 2),
    P_ENTRY(float, 0, 48, 16, 512, 0, 1),
    B_ENTRY(float, 0, 48, 8, 256, 0, 2),
    P_ENTRY(float, 0, 54, 16, 512, 0, 1),
    B_ENTRY(float, 0, 54, 8, 256, 0, 2),
    P_ENTRY(float, 0, 72, 16, 512, 0, 1),
    B_ENTRY(float, 0, 72, 8, 256, 0, 2),
    P_ENTRY(float, 0, 108, 16, 512, 0, 1),
    B_ENTRY(float, 0, 108, 8, 256, 0, 2),
    P_ENTRY(float, 0, 144, 16, 512, 0, 1),
    B_ENTRY(float, 0, 144, 8, 256, 0, 2),
    P_ENTRY(float, 0, 162, 16, 512, 0, 1),
    B_ENTRY(float, 0, 162, 8, 256, 0, 2),
    P_ENTRY(float, 0, 216, 16, 512, 0, 1),
    B_ENTRY(float, 0, 216, 8, 256, 0, 2),
    P_ENTRY(float, 0, 288, 16, 512, 0, 1),
    B_ENTRY(float, 0, 288, 8, 256, 0, 2),
    P_ENTRY(float, 0, 324, 16, 512, 0, 1),
    B_ENTRY(float, 0, 324, 8, 256, 0, 2),
    P_ENTRY(float, 0, 432, 16, 512, 0, 1),
    B_ENTRY(float, 0, 432, 8, 256, 0, 2),
    P_ENTRY(float, 0, 486, 16, 512, 0, 1),
    B_ENTRY(float, 0, 486, 8, 256, 0, 2),
};
const int kNumVariantsB_f32s = sizeof(kVariantsB_f32s) / sizeof(kVariantsB_f32s[0]);

}  // namespace fast
}  // namespace gpufft

// fast_f64.cu — FP64 instantiations of the compile-time specialised passes.
// Tile shapes: column tiles of 4 or 8 complex (64/128-byte rows), row tiles
// of whole rows per warp, 256 threads per CTA; see fft_fast.cuh.
#include "fast_entries.h"

namespace gpufft {
namespace fast {

const VariantA kVariantsA_f64[] = {
    A_ENTRY(double, 1, 512, 256, 2, 8, 256, 0, 0, 2),
    A_ENTRY(double, 1, 512, 256, 2, 4, 256, 0, 0, 2),
};
const int kNumVariantsA_f64 = sizeof(kVariantsA_f64) / sizeof(kVariantsA_f64[0]);

const VariantB kVariantsB_f64[] = {
    P_ENTRY(double, 1, 512, 8, 256, 0, 2),
    P_ENTRY(double, 1, 512, 4, 256, 0, 2),
    B_ENTRY(double, 1, 512, 8, 256, 0, 2),
    B_ENTRY(double, 1, 512, 4, 256, 0, 2),
    B_ENTRY(double, 1, 128, 8, 256, 0, 2),
};
const int kNumVariantsB_f64 = sizeof(kVariantsB_f64) / sizeof(kVariantsB_f64[0]);

}  // namespace fast
}  // namespace gpufft

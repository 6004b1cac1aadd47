// fast_f64.cu — FP64 instantiations of the compile-time specialised passes.
// Tile shapes: column tiles of 4 or 8 complex (64/128-byte rows), row tiles
// of whole rows per warp, 256 threads per CTA; see fft_fast.cuh.
#include "fast_registry.h"
#include "fft_fast.cuh"

namespace gpufft {
namespace fast {

#define A_ENTRY(T, DT, NY, M, RW, WY, NT, VY, VZ, MINB)                                                      \
    {0, 0, DT, NY, M, RW, WY, NT, VY, VZ, PassAShape<T, NY, M, RW, WY, NT, VY, VZ>::smem_bytes(),              \
     (const void *)pass_a_fast<T, NY, M, RW, WY, NT, true, VY, VZ, MINB>,                                     \
     (const void *)pass_a_fast<T, NY, M, RW, WY, NT, false, VY, VZ, MINB>}
#define D_ENTRY(T, DT, NY, M, RW, WY, NT, K, VY, VZ, MINB)                                                   \
    {1, K, DT, NY, M, RW, WY, NT, VY, VZ, PassADsmemShape<T, NY, M, RW, WY, NT, K, VY, VZ>::smem_bytes(),        \
     (const void *)pass_a_dsmem<T, NY, M, RW, WY, NT, K, true, VY, VZ, MINB>,                                    \
     (const void *)pass_a_dsmem<T, NY, M, RW, WY, NT, K, false, VY, VZ, MINB>}
#define P_ENTRY(T, DT, NX, W, NT, V, MINB)                                                                    \
    {1, DT, NX, W, NT, V, (size_t)(((NX + 1) / 2 * 2) + 2 * NX * W) * sizeof(cx_t<T>),                          \
     (const void *)pass_b_pipe<T, NX, W, NT, true, V, MINB>, (const void *)pass_b_pipe<T, NX, W, NT, false, V, MINB>,  \
     (const void *)pass_b_pipe<T, NX, W, NT, true, V, MINB, true>,                                                  \
     (const void *)pass_b_pipe<T, NX, W, NT, false, V, MINB, true>}
#define B_ENTRY(T, DT, NX, W, NT, V, MINB)                                                                    \
    {0, DT, NX, W, NT, V, (size_t)(NX + NX * W) * sizeof(cx_t<T>), (const void *)pass_b_fast<T, NX, W, NT, true, V, MINB>, \
     (const void *)pass_b_fast<T, NX, W, NT, false, V, MINB>,                                                       \
     (const void *)pass_b_fast<T, NX, W, NT, true, V, MINB, true>,                                                  \
     (const void *)pass_b_fast<T, NX, W, NT, false, V, MINB, true>}

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

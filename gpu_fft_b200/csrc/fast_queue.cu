// fast_queue.cu — instantiations of the queue-scheduled Pass A
// (fft_queue.cuh): 512 consumer threads (two z-rows per warp, 32-row items)
// plus one copy-issuing warp, one CTA per SM; ring depth 2 or 3.
#include "fast_registry.h"
#include "fft_queue.cuh"

namespace gpufft {
namespace fast {

#define QA_ENTRY(T, DT, NY, M, VY, NBUF)                                                                           \
    {2, NBUF, DT, NY, M, 2, q::QShape<T, NY, M, 512, NBUF>::WY, 544, VY, 0,                                       \
     q::QShape<T, NY, M, 512, NBUF>::smem_bytes(), (const void *)q::pass_a_queue<T, NY, M, 512, true, VY, NBUF>, \
     (const void *)q::pass_a_queue<T, NY, M, 512, false, VY, NBUF>, nullptr, nullptr}

const VariantA kVariantsA_f32q[] = {
    QA_ENTRY(float, 0, 512, 256, 0, 2),
    QA_ENTRY(float, 0, 512, 256, 0, 3),
};
const int kNumVariantsA_f32q = sizeof(kVariantsA_f32q) / sizeof(kVariantsA_f32q[0]);

// Pass B fed by tensor copies: (Nx, consumer threads, radix variant, ring depth)
#define TB_ENTRY(T, DT, NX, NT, V, NBUF)                                                                          \
    {3, DT, NX, q::BShape<T, NX, NT, NBUF>::W, NT, V, q::BShape<T, NX, NT, NBUF>::smem_bytes(),                  \
     (const void *)q::pass_b_tma<T, NX, NT, true, V, NBUF, false>,                                                \
     (const void *)q::pass_b_tma<T, NX, NT, false, V, NBUF, false>,                                               \
     (const void *)q::pass_b_tma<T, NX, NT, true, V, NBUF, true>, (const void *)q::pass_b_tma<T, NX, NT, false, V, NBUF, true>}

const VariantB kVariantsB_f32q[] = {
    TB_ENTRY(float, 0, 512, 256, 1, 3),
    TB_ENTRY(float, 0, 512, 512, 1, 3),
    TB_ENTRY(float, 0, 512, 256, 0, 3),
    TB_ENTRY(float, 0, 512, 256, 1, 2),
};
const int kNumVariantsB_f32q = sizeof(kVariantsB_f32q) / sizeof(kVariantsB_f32q[0]);

}  // namespace fast
}  // namespace gpufft

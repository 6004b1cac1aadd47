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

}  // namespace fast
}  // namespace gpufft

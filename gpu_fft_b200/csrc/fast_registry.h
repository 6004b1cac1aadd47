// fast_registry.h — table of the compile-time specialised kernels.
//
// Each entry names one instantiation of fast::pass_a_fast / fast::pass_b_fast
// (forward and inverse) with its shape parameters and shared-memory size.  The
// plan looks up the entries matching its axis lengths; when several match it
// either takes the first (the default) or, when autotuning, times them.
#pragma once
#include <cstddef>

namespace gpufft {
namespace fast {

struct VariantA {
    int kind;        // 0: plane exchanged through L2 (cluster size chosen at plan time)
                     // 1: plane held in the cluster's shared memory (cluster size = k)
                     // 2: persistent queue of row and column items fed by bulk / tensor
                     //    copies (fft_queue.cuh; k = ring depth, nt counts the copy-issuing warp)
    int k;           // cluster size of kind 1
    int dtype;       // GPUFFT_FLOAT / GPUFFT_DOUBLE
    int ny, m;       // Ny and Nz/2
    int rw, wy, nt;  // rows per warp in the row phase, columns per column tile, threads per CTA
    int vy, vz;      // radix-list variants of the y and z/2 axes
    size_t smem;     // dynamic shared memory per CTA
    const void *kfwd, *kinv;
    const void *kfwd_x, *kinv_x;  // the same with the y columns in the exchange layout (or null)
};

struct VariantB {
    int kind;  // 0: tiles loaded by the first FFT stage; 1: tiles double-buffered by cp.async;
               // 2: one tile buffer refilled by cp.async during the last stage;
               // 3: tiles brought in by tensor copies, NBUF-deep ring (fft_queue.cuh;
               //    nt counts the copy-issuing warp)
    int dtype;
    int nx;
    int w, nt, v;
    size_t smem;
    const void *kfwd, *kinv;
    const void *kfwd_epi, *kinv_epi;  // the same with the x-pass epilogue (scale, dealiasing)
};

// all entries of one precision (defined in fast_f32.cu / fast_f64.cu)
extern const VariantA kVariantsA_f32[];
extern const int kNumVariantsA_f32;
extern const VariantB kVariantsB_f32[];
extern const int kNumVariantsB_f32;
extern const VariantA kVariantsA_f32s[];  // 3-smooth lengths (fast_f32_3s.cu)
extern const int kNumVariantsA_f32s;
extern const VariantB kVariantsB_f32s[];
extern const int kNumVariantsB_f32s;
extern const VariantA kVariantsA_f32q[];  // queue-scheduled Pass A (fast_queue.cu)
extern const int kNumVariantsA_f32q;
extern const VariantB kVariantsB_f32q[];  // tensor-copy Pass B (fast_queue.cu)
extern const int kNumVariantsB_f32q;
extern const VariantA kVariantsA_f64q[];  // FP64 queue form and tensor-copy x pass (fast_queue.cu)
extern const int kNumVariantsA_f64q;
extern const VariantB kVariantsB_f64q[];
extern const int kNumVariantsB_f64q;
extern const VariantA kVariantsA_f64[];
extern const int kNumVariantsA_f64;
extern const VariantB kVariantsB_f64[];
extern const int kNumVariantsB_f64;

}  // namespace fast
}  // namespace gpufft

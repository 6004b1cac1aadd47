// gpufft_internal.h — the plan object shared by the host translation units.
#pragma once
#include <cstdarg>
#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "fast_registry.h"
#include "fft_kernels.cuh"

namespace gpufft {

struct Plan {
    int64_t nx = 0, ny = 0, nz = 0;
    int dtype = 0;
    int device = 0;
    void *tw_dev = nullptr;     // x, y, z twiddle tables back to back
    void *stage_dev = nullptr;  // per-stage tables of the specialised kernels
    PassAParams pa{};
    PassBParams pb{};
    size_t smem_a = 0, smem_b = 0;
    int grid_a = 0, grid_b = 0;
    int occ_a = 0, occ_b = 0;
    // compile-time specialised kernels, when the registry has this shape
    const fast::VariantA *fa = nullptr;
    const fast::VariantB *fb = nullptr;
    int grid_fa = 0, grid_fb = 0, k_fa = 1, occ_fa = 0, occ_fb = 0;
    int idx_a = 0, idx_b = 0;  // registry candidate in use per pass (-1 = generic kernels)
    int kfix = 0;              // specialised Pass A cluster size (0: chosen from the L2 size;
                               // -1: split Pass A, z rows and y columns in two launches)
    bool split_a = false;      // specialised Pass A runs as two launches (kfix == -1)
    bool tc_split = false;     // x pass on the tensor-core radix-16 kernels (GPUFFT_PLAN_TC_SPLIT)
    bool tuned = false;
    // queue-scheduled Pass A (kind 2, fft_queue.cuh): counters, the forward and
    // inverse item lists and the full unpack table in one allocation
    void *q_dev = nullptr;
    int q_depth = 0;     // planes between a plane's first and second phase in the lists
    int q_nitems = 0;    // items per launch
    int q_need = 0;      // first-phase items per plane (forward)
    int q_extra = 0;     // test hook: items a plane's second phase waits for beyond those that exist
    const int *q_items_f = nullptr, *q_items_i = nullptr;
    const void *q_unp = nullptr;    // forward unpack factors
    const void *q_unp_i = nullptr;  // inverse pack factors
    const void *q_rtw = nullptr;  // the row FFT's step-1 twiddles
};

int set_error(int code, const char *fmt, ...);
const char *last_error();
// Raises a kernel's dynamic shared memory limit on the current device to at
// least `bytes`.  Never lowers it: plans of different sizes share the generic
// kernels, and a later, smaller plan must not undo an earlier plan's limit.
cudaError_t raise_smem_limit(const void *fn, size_t bytes);
// slab-decomposed plans (dist.cu), for the reference-shaped process-wide plans
struct DistPlan;
int dist_exec(DistPlan *D, void *data, cudaStream_t s, bool fwd);
void dist_free(DistPlan *D);
int plan_create(Plan **out, int64_t nx, int64_t ny, int64_t nz, int dtype, int flags);
int plan_destroy(Plan *P);
int plan_exec(const Plan *P, void *data, void *stream, bool forward);
int plan_exec_ex(const Plan *P, void *data, void *stream, bool forward, double scale, int dealias);
int plan_exec_pass(const Plan *P, void *data, void *stream, int pass, bool forward);
int plan_launches(const Plan *P);
// Slab decomposition: whether P's Pass A has exchange-layout kernels, and a
// Pass A whose y columns write (forward) or read (inverse) the all-to-all's
// layout in `xch` -- chunk y / nyl, element (x * nyl + y % nyl) * Nh + kz --
// instead of the field
bool plan_has_xch(const Plan *P);
int plan_exec_pass_a_xch(const Plan *P, void *data, void *xch, int nyl, long long chunk, void *stream, bool forward);
int plan_describe(const Plan *P, char *buf, int len);
int plan_autotune(Plan *P, void *scratch, void *stream);
// P takes Q's kernel choice (same grid, precision and form; Q tuned already)
int plan_adopt(Plan *P, const Plan *Q);
int wisdom_save(const char *path);
int wisdom_load(const char *path);

}  // namespace gpufft

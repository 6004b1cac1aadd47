// s16.cu — host side of the precision form (fft_s16.cuh): plans for BF16 /
// FP16 storage with per-pencil FP32 scales, conversion kernels, C ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/gpufft_b200.h"
#include "fft_s16.cuh"
#include "gpufft_internal.h"

namespace gpufft {
namespace s16 {

struct VarA {
    int fmt, ny, m, rw, wy, nt, vy, vz;
    size_t smem;
    const void *kfwd, *kinv;
};
struct VarB {
    int fmt, nx, w, nt, v;
    size_t smem;
    const void *kfwd, *kinv;
    int pipe = 0;  // 1: cp.async double-buffered (needs 16-byte aligned rows and data)
};

#define S16_A(FMT, NY, M, RW, WY, NT, MINB)                                                                     \
    {FMT, NY, M, RW, WY, NT, 0, 0, PassA16Shape<NY, M, RW, WY, NT>::smem_bytes(),                               \
     (const void *)pass_a_s16<FMT, NY, M, RW, WY, NT, true, 0, 0, MINB>,                                       \
     (const void *)pass_a_s16<FMT, NY, M, RW, WY, NT, false, 0, 0, MINB>}
#define S16_B(FMT, NX, W, NT, MINB)                                                                             \
    {FMT, NX, W, NT, 0, (size_t)(NX + NX * W) * sizeof(float2) + (size_t)NX * W * sizeof(float),                \
     (const void *)pass_b_s16<FMT, NX, W, NT, true, 0, MINB>, (const void *)pass_b_s16<FMT, NX, W, NT, false, 0, MINB>}

static const VarA kA[] = {
    S16_A(0, 1024, 512, 1, 8, 256, 2), S16_A(1, 1024, 512, 1, 8, 256, 2),
    S16_A(0, 1024, 512, 1, 16, 512, 1), S16_A(1, 1024, 512, 1, 16, 512, 1),
    S16_A(0, 512, 256, 2, 8, 256, 2),  S16_A(1, 512, 256, 2, 8, 256, 2),
    S16_A(0, 384, 192, 1, 8, 256, 1),  S16_A(1, 384, 192, 1, 8, 256, 1),
    S16_A(0, 256, 128, 2, 8, 256, 2),  S16_A(1, 256, 128, 2, 8, 256, 2),
    S16_A(0, 192, 96, 1, 8, 256, 2),   S16_A(1, 192, 96, 1, 8, 256, 2),
    S16_A(0, 128, 64, 4, 8, 256, 2),   S16_A(1, 128, 64, 4, 8, 256, 2),
    S16_A(0, 96, 48, 2, 8, 256, 2),    S16_A(1, 96, 48, 2, 8, 256, 2),
    S16_A(0, 64, 32, 4, 8, 256, 2),    S16_A(1, 64, 32, 4, 8, 256, 2),
};
#define S16_P(FMT, NX, W, NT, MINB)                                                                             \
    {FMT, NX, W, NT, 0, PassB16PipeShape<NX, W>::smem_bytes(), (const void *)pass_b_s16_pipe<FMT, NX, W, NT, true, 0, MINB>, \
     (const void *)pass_b_s16_pipe<FMT, NX, W, NT, false, 0, MINB>, 1}

static const VarB kB[] = {
    S16_P(0, 512, 16, 256, 1), S16_P(1, 512, 16, 256, 1), S16_P(0, 256, 16, 256, 1), S16_P(1, 256, 16, 256, 1),
    S16_P(0, 1024, 8, 256, 1), S16_P(1, 1024, 8, 256, 1),
    S16_B(0, 1024, 8, 256, 2), S16_B(1, 1024, 8, 256, 2),
    S16_B(0, 1024, 16, 512, 1), S16_B(1, 1024, 16, 512, 1), S16_B(0, 512, 16, 256, 2), S16_B(1, 512, 16, 256, 2),
    S16_B(0, 256, 16, 256, 2), S16_B(1, 256, 16, 256, 2), S16_B(0, 128, 16, 256, 2), S16_B(1, 128, 16, 256, 2),
    S16_B(0, 64, 16, 256, 2),  S16_B(1, 64, 16, 256, 2),  S16_B(0, 384, 8, 256, 2),  S16_B(1, 384, 8, 256, 2),
    S16_B(0, 192, 16, 256, 2), S16_B(1, 192, 16, 256, 2), S16_B(0, 96, 16, 256, 2),  S16_B(1, 96, 16, 256, 2),
};

struct Plan16 {
    int64_t nx = 0, ny = 0, nz = 0;
    int fmt = 0;
    int device = 0;
    const VarA *va = nullptr;
    const VarB *vb = nullptr;
    const VarB *vb_plain = nullptr;  // for data that is not 16-byte aligned when vb is a pipelined entry
    void *tables = nullptr;  // twz | stz | sty | stw (float2)
    float *ms = nullptr, *ms2 = nullptr;
    const float2 *twz = nullptr, *stz = nullptr, *sty = nullptr, *stw = nullptr;
    int K = 1, grid_a = 0, grid_b = 0, grid_b_plain = 0;
};

static std::vector<float> stage_table_f32(int n) {
    const fast::Fac f = fast::factor(n, 0);
    std::vector<float> t(2 * (size_t)std::max(n, 1), 0.f);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    int p = 1;
    for (int s = 0; s < f.n; ++s) {
        const int R = f.r[s], off = fast::stage_offset(f, s);
        for (int j = 1; j < R; ++j)
            for (int k = 0; k < p; ++k) {
                const long long e = ((long long)j * k) % ((long long)p * R);
                const long double ang = two_pi * (long double)e / (long double)(p * R);
                const size_t at = (size_t)off + (size_t)(j - 1) * p + k;
                t[2 * at] = (float)cosl(ang);
                t[2 * at + 1] = (float)(-sinl(ang));
            }
        p *= R;
    }
    return t;
}

static void plan16_free(Plan16 *P) {
    if (!P) return;
    if (P->tables) cudaFree(P->tables);
    if (P->ms) cudaFree(P->ms);
    if (P->ms2) cudaFree(P->ms2);
    delete P;
}

static int plan16_create(Plan16 **out, int64_t nx, int64_t ny, int64_t nz, int fmt) {
    if (!out) return set_error(GPUFFT_ERR_INVALID, "plan pointer is NULL");
    *out = nullptr;
    if (nx < 1 || ny < 1 || nz < 2 || nz % 2) return set_error(GPUFFT_ERR_INVALID, "bad grid for a 16-bit plan");
    if (fmt != 0 && fmt != 1) return set_error(GPUFFT_ERR_INVALID, "format %d is neither 0 (bf16) nor 1 (fp16)", fmt);
    const int m = (int)(nz / 2);
    const VarA *va = nullptr;
    const VarB *vb = nullptr;
    // first matching entry, or the i-th with GPUFFT_VARIANT16_A / _B (measurement)
    const char *ea = std::getenv("GPUFFT_VARIANT16_A"), *eb = std::getenv("GPUFFT_VARIANT16_B");
    int skip_a = ea ? std::max(0, std::atoi(ea)) : 0, skip_b = eb ? std::max(0, std::atoi(eb)) : 0;
    for (const auto &v : kA)
        if (v.fmt == fmt && v.ny == ny && v.m == m && skip_a-- == 0) { va = &v; break; }
    const int64_t nh16 = nz / 2 + 1;
    const bool rows16 = (ny * nh16) % 4 == 0;  // 16-bit rows start on 16-byte boundaries
    for (const auto &v : kB)
        if (v.fmt == fmt && v.nx == nx && (!v.pipe || rows16) && skip_b-- == 0) { vb = &v; break; }
    const VarB *vb_plain = nullptr;
    for (const auto &v : kB)
        if (v.fmt == fmt && v.nx == nx && !v.pipe) { vb_plain = &v; break; }
    if (vb && !vb_plain) vb = nullptr;
    if (!va || !vb)
        return set_error(GPUFFT_ERR_UNSUPPORTED,
                         "16-bit storage form: grid %lldx%lldx%lld has no compiled kernels (cubic 64, 96, 128, "
                         "192, 256, 384, 512 and 1024 are built)", (long long)nx, (long long)ny, (long long)nz);
    Plan16 *P = new (std::nothrow) Plan16();
    if (!P) return set_error(GPUFFT_ERR_OOM, "host allocation failed");
    P->nx = nx; P->ny = ny; P->nz = nz; P->fmt = fmt; P->va = va; P->vb = vb; P->vb_plain = vb_plain;
    cudaGetDevice(&P->device);
    // tables: w_Nz (unpack roots), stage tables of Nz/2, Ny and Nx
    std::vector<float> t;
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int e = 0; e < (int)nz; ++e) {
        const long double ang = two_pi * (long double)e / (long double)nz;
        t.push_back((float)cosl(ang));
        t.push_back((float)(-sinl(ang)));
    }
    const size_t oz = t.size() / 2;
    auto a1 = stage_table_f32(m);
    t.insert(t.end(), a1.begin(), a1.end());
    const size_t oy = t.size() / 2;
    auto a2 = stage_table_f32((int)ny);
    t.insert(t.end(), a2.begin(), a2.end());
    const size_t ox = t.size() / 2;
    auto a3 = stage_table_f32((int)nx);
    t.insert(t.end(), a3.begin(), a3.end());
    const int64_t nh = nz / 2 + 1;
    cudaError_t e = cudaMalloc(&P->tables, t.size() * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&P->ms, sizeof(float) * (size_t)(nx * nh));
    if (e == cudaSuccess) e = cudaMalloc(&P->ms2, sizeof(float) * (size_t)(ny * nh));
    if (e != cudaSuccess) {
        plan16_free(P);
        return set_error(GPUFFT_ERR_OOM, "16-bit plan tables: %s", cudaGetErrorString(e));
    }
    e = cudaMemcpy(P->tables, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice);
    const float2 *tb = (const float2 *)P->tables;
    P->twz = tb;
    P->stz = tb + oz;
    P->sty = tb + oy;
    P->stw = tb + ox;
    for (const void *k : {va->kfwd, va->kinv})
        if (e == cudaSuccess) e = raise_smem_limit(k, va->smem);
    for (const VarB *b : {vb, vb_plain})
        for (const void *k : {b->kfwd, b->kinv})
            if (e == cudaSuccess) e = raise_smem_limit(k, b->smem);
    if (e != cudaSuccess) {
        plan16_free(P);
        return set_error(GPUFFT_ERR_CUDA, "16-bit plan set-up: %s", cudaGetErrorString(e));
    }
    int sms = 0, occa = 0, occb = 0, l2 = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, P->device);
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, P->device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occa, va->kfwd, va->nt, va->smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occb, vb->kfwd, vb->nt, vb->smem);
    occa = std::max(occa, 1);
    occb = std::max(occb, 1);
    // cluster size as for the FP32 plan: planes in flight within half of L2
    const long long plane = (long long)ny * nh * 4;
    const int resident = occa * std::max(sms, 1);
    const int tiles_y = (m + va->wy - 1) / va->wy;
    const int kcap = std::max(1, std::min({8, tiles_y, (int)ny}));
    int K = 1;
    while (K < kcap && (long long)(resident / K) * plane > (long long)std::max(l2, 1 << 20) / 2) K *= 2;
    while (K < kcap && nx * K < resident) K *= 2;
    P->K = std::min(K, kcap);
    {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        cfg.gridDim = dim3(P->K * (unsigned)nx, 1, 1);
        cfg.blockDim = dim3(va->nt, 1, 1);
        cfg.dynamicSmemBytes = va->smem;
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = P->K;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int mc = 0;
        if (cudaOccupancyMaxActiveClusters(&mc, va->kfwd, &cfg) != cudaSuccess || mc < 1) {
            cudaGetLastError();
            mc = std::max(1, resident / P->K);
        }
        P->grid_a = P->K * (int)std::min<long long>(nx, mc);
    }
    const long long tiles = (ny * nh + vb->w - 1) / vb->w;
    P->grid_b = (int)std::min<long long>(tiles, (long long)occb * sms);
    int occp = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occp, vb_plain->kfwd, vb_plain->nt, vb_plain->smem);
    P->grid_b_plain = (int)std::min<long long>((ny * nh + vb_plain->w - 1) / vb_plain->w, (long long)std::max(occp, 1) * sms);
    *out = P;
    return GPUFFT_SUCCESS;
}

static int launch_a(const Plan16 &P, void *data, float *scales, cudaStream_t s, bool fwd) {
    PassA16Params prm;
    prm.data = (uint32_t *)data;
    prm.rs = scales;
    prm.ms = P.ms;
    prm.ms2 = P.ms2;
    prm.twz = P.twz;
    prm.stz = P.stz;
    prm.sty = P.sty;
    prm.nx = (int)P.nx;
    prm.K = P.K;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim = dim3(P.grid_a, 1, 1);
    cfg.blockDim = dim3(P.va->nt, 1, 1);
    cfg.dynamicSmemBytes = P.va->smem;
    cfg.stream = s;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = P.K;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void *args[] = {&prm};
    const cudaError_t e = cudaLaunchKernelExC(&cfg, fwd ? P.va->kfwd : P.va->kinv, args);
    return e == cudaSuccess ? GPUFFT_SUCCESS : set_error(GPUFFT_ERR_CUDA, "16-bit pass A: %s", cudaGetErrorString(e));
}

static int launch_b(const Plan16 &P, void *data, float *scales, cudaStream_t s, bool fwd) {
    PassB16Params prm;
    prm.data = (uint32_t *)data;
    prm.ks = scales;
    prm.ms = P.ms;
    prm.ms2 = P.ms2;
    prm.stw = P.stw;
    prm.nh = (int)(P.nz / 2 + 1);
    prm.ncols = P.ny * prm.nh;
    // a pipelined entry copies 16-byte chunks: unaligned data takes the plain kernel
    const bool plain = P.vb->pipe && ((uintptr_t)data % 16 != 0);
    const VarB &b = plain ? *P.vb_plain : *P.vb;
    prm.ntiles = (prm.ncols + b.w - 1) / b.w;
    void *args[] = {&prm};
    const cudaError_t e =
        cudaLaunchKernel(fwd ? b.kfwd : b.kinv, dim3(plain ? P.grid_b_plain : P.grid_b), dim3(b.nt), args, b.smem, s);
    return e == cudaSuccess ? GPUFFT_SUCCESS : set_error(GPUFFT_ERR_CUDA, "16-bit pass B: %s", cudaGetErrorString(e));
}

// ---- conversions between FP32 and the 16-bit storage form (a warp per row / pencil)
template <int FMT>
__global__ void quantize_rows(const float2 *src, uint32_t *dst, float *rs, long long rows, int nh, int nz) {
    const long long row = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (row >= rows) return;
    const float2 *r = src + row * nh;
    float m = 0.f;
    for (int n = lane; n < nh; n += 32) {
        float2 v = r[n];
        if (2 * n >= nz) v.x = 0.f;       // padding cells
        if (2 * n + 1 >= nz) v.y = 0.f;
        m = fmaxf(m, amax(v));
    }
    m = warp_max(m);
    const float inv = inv_of(m);
    for (int n = lane; n < nh; n += 32) {
        float2 v = r[n];
        if (2 * n >= nz) v.x = 0.f;
        if (2 * n + 1 >= nz) v.y = 0.f;
        Fmt<FMT>::store(dst + row * nh + n, mulf(v, inv));
    }
    if (lane == 0) rs[row] = m;
}

// element i of rows of `nh` 32-bit pairs, scale index = scale_of(i)
template <int FMT>
__global__ void dequantize(const uint32_t *src, const float *scales, float2 *dst, long long count, int nh,
                           long long ny_nh, int per_row) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x) {
        // real space: scale per row (i / nh); spectrum: per x-pencil (i % (Ny*Nh))
        const float sc = per_row ? scales[i / nh] : scales[i % ny_nh];
        dst[i] = mulf(Fmt<FMT>::load(src + i), sc);
    }
}

}  // namespace s16
}  // namespace gpufft

using namespace gpufft;
using namespace gpufft::s16;

extern "C" int gpufft_plan16_create(gpufft_plan16 *plan, int64_t nx, int64_t ny, int64_t nz, int format) {
    Plan16 *P = nullptr;
    const int rc = plan16_create(&P, nx, ny, nz, format);
    if (plan) *plan = reinterpret_cast<gpufft_plan16>(P);
    return rc;
}

extern "C" int gpufft_plan16_destroy(gpufft_plan16 plan) {
    plan16_free(reinterpret_cast<Plan16 *>(plan));
    return GPUFFT_SUCCESS;
}

extern "C" int64_t gpufft_plan16_scale_count(gpufft_plan16 plan) {
    const Plan16 *P = reinterpret_cast<const Plan16 *>(plan);
    if (!P) return -1;
    return std::max<int64_t>(P->nx * P->ny, P->ny * (P->nz / 2 + 1));
}

extern "C" int gpufft_exec16_pass(gpufft_plan16 plan, void *data, float *scales, void *stream, int pass, int forward) {
    const Plan16 *P = reinterpret_cast<const Plan16 *>(plan);
    if (!P) return set_error(GPUFFT_ERR_NOT_INIT, "no 16-bit plan");
    if (!data || !scales) return set_error(GPUFFT_ERR_INVALID, "data and scales must be device pointers");
    if (((uintptr_t)data) % 4 || ((uintptr_t)scales) % 4) return set_error(GPUFFT_ERR_INVALID, "misaligned pointer");
    if (pass != 0 && pass != 1) return set_error(GPUFFT_ERR_INVALID, "pass must be 0 (A) or 1 (B)");
    return pass == 0 ? launch_a(*P, data, scales, (cudaStream_t)stream, forward != 0)
                     : launch_b(*P, data, scales, (cudaStream_t)stream, forward != 0);
}

static int exec16(gpufft_plan16 plan, void *data, float *scales, void *stream, bool fwd) {
    const Plan16 *P = reinterpret_cast<const Plan16 *>(plan);
    if (!P) return set_error(GPUFFT_ERR_NOT_INIT, "no 16-bit plan");
    if (!data || !scales) return set_error(GPUFFT_ERR_INVALID, "data and scales must be device pointers");
    if (((uintptr_t)data) % 4 || ((uintptr_t)scales) % 4) return set_error(GPUFFT_ERR_INVALID, "misaligned pointer");
    cudaStream_t s = (cudaStream_t)stream;
    int rc = fwd ? launch_a(*P, data, scales, s, true) : launch_b(*P, data, scales, s, false);
    if (rc == GPUFFT_SUCCESS) rc = fwd ? launch_b(*P, data, scales, s, true) : launch_a(*P, data, scales, s, false);
    return rc;
}

extern "C" int gpufft_exec16_r2c(gpufft_plan16 plan, void *data, float *scales, void *stream) {
    return exec16(plan, data, scales, stream, true);
}

extern "C" int gpufft_exec16_c2r(gpufft_plan16 plan, void *data, float *scales, void *stream) {
    return exec16(plan, data, scales, stream, false);
}

extern "C" int gpufft_quantize16(gpufft_plan16 plan, const float *field, void *data, float *row_scales, void *stream) {
    const Plan16 *P = reinterpret_cast<const Plan16 *>(plan);
    if (!P) return set_error(GPUFFT_ERR_NOT_INIT, "no 16-bit plan");
    const long long rows = P->nx * P->ny;
    const int nh = (int)(P->nz / 2 + 1);
    const int block = 256, rpb = block / 32;
    const unsigned grid = (unsigned)((rows + rpb - 1) / rpb);
    if (P->fmt == 0)
        quantize_rows<0><<<grid, block, 0, (cudaStream_t)stream>>>((const float2 *)field, (uint32_t *)data, row_scales,
                                                                    rows, nh, (int)P->nz);
    else
        quantize_rows<1><<<grid, block, 0, (cudaStream_t)stream>>>((const float2 *)field, (uint32_t *)data, row_scales,
                                                                    rows, nh, (int)P->nz);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GPUFFT_SUCCESS : set_error(GPUFFT_ERR_CUDA, "quantize: %s", cudaGetErrorString(e));
}

extern "C" int gpufft_dequantize16(gpufft_plan16 plan, const void *data, const float *scales, float *out, int spectrum,
                                   void *stream) {
    const Plan16 *P = reinterpret_cast<const Plan16 *>(plan);
    if (!P) return set_error(GPUFFT_ERR_NOT_INIT, "no 16-bit plan");
    const int nh = (int)(P->nz / 2 + 1);
    const long long count = P->nx * P->ny * nh;
    if (P->fmt == 0)
        dequantize<0><<<1184, 256, 0, (cudaStream_t)stream>>>((const uint32_t *)data, scales, (float2 *)out, count, nh,
                                                               P->ny * nh, spectrum ? 0 : 1);
    else
        dequantize<1><<<1184, 256, 0, (cudaStream_t)stream>>>((const uint32_t *)data, scales, (float2 *)out, count, nh,
                                                               P->ny * nh, spectrum ? 0 : 1);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GPUFFT_SUCCESS : set_error(GPUFFT_ERR_CUDA, "dequantize: %s", cudaGetErrorString(e));
}

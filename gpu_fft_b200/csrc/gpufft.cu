// gpufft.cu — host side of libgpufft_b200.so: plans, twiddle tables, launches
// and the C ABI declared in include/gpufft_b200.h.
//
// A plan replaces what GPU_FFT's INIT_GPU_FFT sets up
// (GPU_FFT/src/initialize_GPU_FFT/GPU_FFT_init.cu:41-93): instead of three
// cuFFT plans and a field-sized scratch buffer it holds a radix factorisation
// per axis, the tile shapes of the two passes, the cluster size of Pass A and
// three FP64-computed twiddle tables (rounded once to the storage type).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <tuple>
#include <new>
#include <string>
#include <vector>

#include "../../include/gpufft_b200.h"
#include "fft_fast.cuh"
#include "fft_kernels.cuh"
#include "fft_queue.cuh"
#include "gpufft_internal.h"

namespace gpufft {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;

cudaError_t raise_smem_limit(const void *fn, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, size_t> limit;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    size_t &cur = limit[std::make_pair(dev, fn)];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

int set_error(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

const char *last_error() { return g_last_error.c_str(); }

static int cuda_error(cudaError_t e, const char *what) {
    return set_error(GPUFFT_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// factorisation and tile feasibility
// ---------------------------------------------------------------------------
// Radix list for a length-n FFT: the power-of-two part split into as few
// stages of at most 16 as possible with balanced sizes (512 -> 8,8,8;
// 1024 -> 16,8,8), then pairs of 3s as 9s, then the odd primes 3, 5, 7, 11, 13.
bool factorize(int n, std::vector<int> &radices) {
    radices.clear();
    if (n < 1) return false;
    int a = 0, r = n;
    while (r % 2 == 0) { r /= 2; ++a; }
    if (a > 0) {
        const int k = (a + 3) / 4;
        for (int s = 0; s < k; ++s) {
            const int bits = a / k + (s < a % k ? 1 : 0);
            radices.push_back(1 << bits);
        }
    }
    while (r % 9 == 0) { radices.push_back(9); r /= 9; }  // pairs of 3s: radix-9 stages
    for (int p : {3, 5, 7, 11, 13})
        while (r % p == 0) { radices.push_back(p); r /= p; }
    return r == 1;
}

static void fill_axis(AxisPlan &ax, int n, const std::vector<int> &radices, int tabmul) {
    std::memset(&ax, 0, sizeof(ax));
    ax.n = n;
    ax.nst = (int)radices.size();
    int p = 1;
    for (int s = 0; s < ax.nst; ++s) {
        const int R = radices[s];
        ax.radix[s] = R;
        ax.p[s] = p;
        ax.pdiv[s] = make_fastdiv((uint32_t)p);
        ax.twstep[s] = tabmul * (n / (p * R));
        p *= R;
    }
}

// ---------------------------------------------------------------------------
// twiddle tables: w[e] = exp(-2 pi i e / L), e < L, computed in long double
// on the reduced angle and rounded once to the storage type
// ---------------------------------------------------------------------------
template <typename T>
static std::vector<T> twiddle_table(int L) {
    std::vector<T> t(2 * (size_t)L);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int e = 0; e < L; ++e) {
        const long double ang = two_pi * (long double)e / (long double)L;
        t[2 * e] = (T)cosl(ang);
        t[2 * e + 1] = (T)(-sinl(ang));
    }
    return t;
}

// Per-stage table of the specialised kernels for length n (fft_fast.cuh,
// stage_offset): stage s with radix R after sub-length p holds
// exp(-2 pi i j k / (p R)) at offset + (j-1)*p + k.  Padded to n entries.
template <typename T>
static std::vector<T> stage_table(int n, int variant) {
    const fast::Fac f = fast::factor(n, variant);
    std::vector<T> t(2 * (size_t)std::max(n, 1), (T)0);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    int p = 1;
    for (int s = 0; s < f.n; ++s) {
        const int R = f.r[s], off = fast::stage_offset(f, s);
        for (int j = 1; j < R; ++j)
            for (int k = 0; k < p; ++k) {
                const long long e = ((long long)j * k) % ((long long)p * R);
                const long double ang = two_pi * (long double)e / (long double)(p * R);
                const size_t at = (size_t)off + (size_t)(j - 1) * p + k;
                t[2 * at] = (T)cosl(ang);
                t[2 * at + 1] = (T)(-sinl(ang));
            }
        p *= R;
    }
    return t;
}

template <typename T>
static int upload_stage_tables(Plan &P) {
    const int nx = (int)P.nx, ny = (int)P.ny, m = (int)(P.nz / 2);
    std::vector<T> tx, ty, tz;
    if (P.fb) tx = stage_table<T>(nx, P.fb->v);
    if (P.fa) {
        ty = stage_table<T>(ny, P.fa->vy);
        tz = stage_table<T>(m, P.fa->vz);
    }
    const size_t bx = tx.size() * sizeof(T), by = ty.size() * sizeof(T), bz = tz.size() * sizeof(T);
    if (P.stage_dev) {
        cudaFree(P.stage_dev);
        P.stage_dev = nullptr;
    }
    if (bx + by + bz == 0) return GPUFFT_SUCCESS;
    cudaError_t e = cudaMalloc(&P.stage_dev, bx + by + bz);
    if (e != cudaSuccess) return set_error(GPUFFT_ERR_OOM, "cudaMalloc stage tables: %s", cudaGetErrorString(e));
    char *b = (char *)P.stage_dev;
    if (bx) e = cudaMemcpy(b, tx.data(), bx, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && by) e = cudaMemcpy(b + bx, ty.data(), by, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && bz) e = cudaMemcpy(b + bx + by, tz.data(), bz, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_error(e, "cudaMemcpy stage tables");
    P.pb.stw = bx ? b : nullptr;
    P.pa.sty = by ? b + bx : nullptr;
    P.pa.stz = bz ? b + bx + by : nullptr;
    return GPUFFT_SUCCESS;
}

// ---------------------------------------------------------------------------
// plan
// ---------------------------------------------------------------------------
static int device_sms(int dev) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v > 0 ? v : 1;
}

// Cluster size for Pass A: enough CTAs per plane that the planes in flight
// fit in about half of L2, and enough clusters to fill the GPU; at most 8
// (the portable cluster limit) and at most one column tile per CTA.
static int choose_cluster(int dev, int nx, int ny, int m, int wy, size_t plane_bytes, int occ, int sms) {
    int l2 = 0;
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev);
    if (l2 <= 0) l2 = 96 << 20;
    const int resident = std::max(1, occ) * sms;
    const int tiles_y = (m + wy - 1) / wy;
    const int kcap = std::max(1, std::min({8, tiles_y, ny}));
    int K = 1;
    while (K < kcap && (long long)(resident / K) * (long long)plane_bytes > (long long)l2 / 2) K *= 2;
    while (K < kcap && (long long)nx * K < resident) K *= 2;
    return std::min(K, kcap);
}

static int max_clusters(const void *kernel, int K, int nx, size_t smem, int nt, int fallback) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim = dim3(K * std::max(1, nx), 1, 1);
    cfg.blockDim = dim3(nt, 1, 1);
    cfg.dynamicSmemBytes = smem;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = K;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kernel, &cfg) != cudaSuccess || n < 1) {
        cudaGetLastError();
        n = fallback;
    }
    return n;
}

// Every specialisation of a precision, in a fixed order (the main table,
// then the table of 3-smooth lengths); candidate indices refer to it.
static const std::vector<fast::VariantA> &variants_a(int dtype) {
    static const std::vector<fast::VariantA> f32 = [] {
        // the queue form first: the default where it exists (512^2 planes)
        std::vector<fast::VariantA> v(fast::kVariantsA_f32q, fast::kVariantsA_f32q + fast::kNumVariantsA_f32q);
        v.insert(v.end(), fast::kVariantsA_f32, fast::kVariantsA_f32 + fast::kNumVariantsA_f32);
        v.insert(v.end(), fast::kVariantsA_f32s, fast::kVariantsA_f32s + fast::kNumVariantsA_f32s);
        return v;
    }();
    static const std::vector<fast::VariantA> f64 = [] {
        std::vector<fast::VariantA> v(fast::kVariantsA_f64q, fast::kVariantsA_f64q + fast::kNumVariantsA_f64q);
        v.insert(v.end(), fast::kVariantsA_f64, fast::kVariantsA_f64 + fast::kNumVariantsA_f64);
        return v;
    }();
    return dtype == GPUFFT_FLOAT ? f32 : f64;
}

static const std::vector<fast::VariantB> &variants_b(int dtype) {
    static const std::vector<fast::VariantB> f32 = [] {
        // the tensor-copy form first: the default where it exists
        std::vector<fast::VariantB> v(fast::kVariantsB_f32q, fast::kVariantsB_f32q + fast::kNumVariantsB_f32q);
        v.insert(v.end(), fast::kVariantsB_f32, fast::kVariantsB_f32 + fast::kNumVariantsB_f32);
        v.insert(v.end(), fast::kVariantsB_f32s, fast::kVariantsB_f32s + fast::kNumVariantsB_f32s);
        return v;
    }();
    static const std::vector<fast::VariantB> f64 = [] {
        std::vector<fast::VariantB> v(fast::kVariantsB_f64q, fast::kVariantsB_f64q + fast::kNumVariantsB_f64q);
        v.insert(v.end(), fast::kVariantsB_f64, fast::kVariantsB_f64 + fast::kNumVariantsB_f64);
        return v;
    }();
    return dtype == GPUFFT_FLOAT ? f32 : f64;
}

// A Pass B entry serves this plan: its length, 16-byte tile rows for the
// cp.async and tensor-copy forms, and tensor-core stages (v = 2: mma.sync,
// v = 3: tcgen05) exactly when the plan asks for them.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();
static bool b_eligible(const Plan &P, const fast::VariantB &v) {
    const int m = (int)(P.nz / 2);
    const bool rows16 = ((long long)P.ny * (m + 1) * (P.dtype == GPUFFT_FLOAT ? 8 : 16)) % 16 == 0;
    return v.nx == (int)P.nx && (v.kind == 0 || rows16) && ((v.v >= 2) == P.tc_split) &&
           (v.kind != 3 || tensor_map_encoder());
}

// ---------------------------------------------------------------------------
// queue-scheduled Pass A (kind 2): item lists, counters, unpack table
// ---------------------------------------------------------------------------
static void free_queue(Plan &P) {
    if (P.q_dev) cudaFree(P.q_dev);
    P.q_dev = nullptr;
    P.q_items_f = P.q_items_i = nullptr;
    P.q_unp = nullptr;
    P.q_unp_i = nullptr;
    P.q_rtw = nullptr;
}

// Work list of one direction: block b holds the first-phase items of plane b
// (b < nx) interleaved with the second-phase items of plane b - depth
// (b >= depth), so a plane's second phase is claimed about `depth` planes of
// work after its first.
static std::vector<int> queue_items(int nx, int nfirst, int nsecond, int first_type, int depth) {
    std::vector<int> v;
    v.reserve((size_t)nx * (nfirst + nsecond));
    for (int b = 0; b < nx + depth; ++b) {
        const int a = b < nx ? nfirst : 0;
        const int c = b >= depth ? nsecond : 0;
        const int tot = a + c;
        int ia = 0, ic = 0;
        for (int i = 0; i < tot; ++i) {
            // spread the two kinds evenly through the block
            const bool take_a = ic >= c || (ia < a && (long long)ia * tot <= (long long)i * a);
            if (take_a)
                v.push_back(q::item_code(b, first_type, ia++));
            else
                v.push_back(q::item_code(b - depth, 1 - first_type, ic++));
        }
    }
    return v;
}

static int setup_queue(Plan &P) {
    free_queue(P);
    const int nx = (int)P.nx, ny = (int)P.ny, m = (int)(P.nz / 2);
    const int ri = (P.fa->nt - 32) / 16, wy = P.fa->wy;  // two rows per consumer warp
    const int nri = ny / ri, nci = m / wy;
    // default depth: about 1024 items between a plane's two phases (measured
    // best: 16-32 planes of 32 items at 512^3, 32 of 24 items at 512 x 128
    // planes, 32-48 of 30 items at 360 x 240 planes)
    int depth = P.kfix > 0 ? P.kfix : std::max(8, std::min(64, 1024 / std::max(1, nri + nci)));
    if (const char *ev = std::getenv("GPUFFT_QUEUE_DEPTH")) depth = std::atoi(ev);
    depth = std::max(1, std::min(nx, depth));
    const std::vector<int> fwd = queue_items(nx, nri, nci, q::ROW_ITEM, depth);
    const std::vector<int> inv = queue_items(nx, nci, nri, q::COL_ITEM, depth);
    // the unpack factors u_k = -i w^k / 2 (forward) and the pack factors
    // v_k = i conj(w^k) (inverse), w = exp(-2 pi i / Nz), k < M; then the row
    // FFT's step-1 twiddles exp(-2 pi i a f / M) at (f - 1) * 16 + a
    // (M = 16 * R2): long-double host values rounded once
    const int r2 = m / 16;
    std::vector<double> unp(4 * (size_t)m + 2 * 16 * (size_t)std::max(r2 - 1, 0));
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int k = 0; k < m; ++k) {
        const long double ang = two_pi * (long double)k / (long double)(2 * m);
        const long double c = cosl(ang), sn = sinl(ang);  // w^k = c - i sn
        unp[2 * k] = (double)(-sn / 2);                   // -i w^k / 2
        unp[2 * k + 1] = (double)(-c / 2);
        unp[2 * m + 2 * k] = (double)(-sn);               // i conj(w^k)
        unp[2 * m + 2 * k + 1] = (double)c;
    }
    for (int f = 1; f < r2; ++f)
        for (int a = 0; a < 16; ++a) {
            const size_t at = 4 * (size_t)m + 2 * ((size_t)(f - 1) * 16 + a);
            const long double ang = two_pi * (long double)((a * f) % m) / (long double)m;
            unp[at] = (double)cosl(ang);
            unp[at + 1] = (double)(-sinl(ang));
        }
    // rounded once to the plan's precision
    const size_t tsz = P.dtype == GPUFFT_FLOAT ? sizeof(float) : sizeof(double);
    std::vector<unsigned char> tab(unp.size() * tsz);
    for (size_t i = 0; i < unp.size(); ++i) {
        if (tsz == sizeof(float)) {
            const float v = (float)unp[i];
            std::memcpy(tab.data() + i * tsz, &v, tsz);
        } else {
            std::memcpy(tab.data() + i * tsz, &unp[i], tsz);
        }
    }
    const size_t cbytes = ((size_t)(4 + nx) * sizeof(int) + 255) / 256 * 256;
    const size_t lbytes = (fwd.size() * sizeof(int) + 255) / 256 * 256;
    const size_t ubytes = tab.size();
    cudaError_t e = cudaMalloc(&P.q_dev, cbytes + 2 * lbytes + ubytes);
    if (e != cudaSuccess) {
        P.q_dev = nullptr;
        return set_error(GPUFFT_ERR_OOM, "cudaMalloc Pass A queue state: %s", cudaGetErrorString(e));
    }
    char *b = (char *)P.q_dev;
    e = cudaMemset(b, 0, cbytes);
    if (e == cudaSuccess) e = cudaMemcpy(b + cbytes, fwd.data(), fwd.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b + cbytes + lbytes, inv.data(), inv.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b + cbytes + 2 * lbytes, tab.data(), ubytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        free_queue(P);
        return cuda_error(e, "upload Pass A queue state");
    }
    P.q_depth = depth;
    P.q_nitems = (int)fwd.size();
    P.q_need = nri;
    // test hook of the bounded dependency wait: with GPUFFT_QUEUE_UNREACHABLE=1
    // at plan creation every second-phase item waits for one first-phase item
    // more than exist, so the wait runs out (GPUFFT_QUEUE_WAIT_MS, read at
    // launch, sets the limit) and gpufft_plan_check reports it
    if (const char *ev = std::getenv("GPUFFT_QUEUE_UNREACHABLE")) P.q_extra = std::atoi(ev) == 1 ? 1 : 0;
    P.q_items_f = reinterpret_cast<const int *>(b + cbytes);
    P.q_items_i = reinterpret_cast<const int *>(b + cbytes + lbytes);
    P.q_unp = b + cbytes + 2 * lbytes;
    P.q_unp_i = b + cbytes + 2 * lbytes + 2 * (size_t)m * tsz;
    P.q_rtw = b + cbytes + 2 * lbytes + 4 * (size_t)m * tsz;
    return GPUFFT_SUCCESS;
}

// cuTensorMapEncodeTiled from the driver, found at run time (no libcuda link)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// A 2D view of the field in 8-byte elements: `width` elements per line,
// `lines` lines `pitch` bytes apart, boxes of box_w x box_h.
static bool encode_view(CUtensorMap *m, void *data, long long width, long long lines, long long pitch, int box_w,
                        int box_h) {
    const auto enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)width, (cuuint64_t)lines};
    const cuuint64_t strides[1] = {(cuuint64_t)pitch};
    const cuuint32_t box[2] = {(cuuint32_t)box_w, (cuuint32_t)box_h};
    const cuuint32_t es[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, data, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The row-pair view of an FP32 field with Nh odd: lines of 2*Nh 8-byte
// elements (rows 2r and 2r+1), Nx*Ny/2 lines, line pitch 16*Nh bytes.
static bool encode_pair_map(CUtensorMap *m, void *data, long long nh, long long lines, int box_w, int box_h) {
    return encode_view(m, data, 2 * nh, lines, 2 * nh * 8, box_w, box_h);
}

// Picks the specialised kernels for this plan's shape (first registry entry,
// or the entries named by the autotuner) and sizes their launches.
static int setup_fast(Plan &P, int idx_a, int idx_b) {
    const int vs = P.dtype == GPUFFT_FLOAT ? 8 : 16;
    const fast::VariantA *va = variants_a(P.dtype).data();
    const int na = (int)variants_a(P.dtype).size();
    const fast::VariantB *vb = variants_b(P.dtype).data();
    const int nb = (int)variants_b(P.dtype).size();
    const int nx = (int)P.nx, ny = (int)P.ny, m = (int)(P.nz / 2);
    const int sms = device_sms(P.device);
    P.fa = nullptr;
    P.fb = nullptr;
    P.idx_a = idx_a;
    P.idx_b = idx_b;
    int seen = 0;
    for (int i = 0; i < na && !P.fa; ++i)
        if (va[i].ny == ny && va[i].m == m && seen++ == idx_a) P.fa = &va[i];
    seen = 0;
    for (int i = 0; i < nb && !P.fb; ++i)
        if (b_eligible(P, vb[i]) && seen++ == idx_b) P.fb = &vb[i];
    if (P.fa) {
        for (const void *k : {P.fa->kfwd, P.fa->kinv, P.fa->kfwd_x, P.fa->kinv_x}) {
            if (!k) continue;
            cudaError_t e = raise_smem_limit(k, P.fa->smem);
            if (e != cudaSuccess) {
                cudaGetLastError();
                P.fa = nullptr;
                break;
            }
        }
    }
    if (P.fa && P.fa->kind == 2 && (!tensor_map_encoder() || P.nx > 32767)) P.fa = nullptr;
    free_queue(P);
    if (P.fa && P.fa->kind == 2) {
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, P.fa->kfwd, P.fa->nt, P.fa->smem);
        P.occ_fa = std::max(occ, 1);
        P.k_fa = 1;
        P.split_a = false;
        P.grid_fa = P.occ_fa * sms;
        const int rq = setup_queue(P);
        if (rq != GPUFFT_SUCCESS) return rq;
    } else if (P.fa) {
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, P.fa->kfwd, P.fa->nt, P.fa->smem);
        P.occ_fa = std::max(occ, 1);
        const size_t plane = (size_t)ny * (m + 1) * vs;
        int K = choose_cluster(P.device, nx, ny, m, P.fa->wy, plane, P.occ_fa, sms);
        // the autotuner may set the cluster size: smaller clusters put more
        // planes in flight with shorter barriers (512^3 FP32 takes 4 over 8),
        // 16-CTA clusters (non-portable) put fewer in flight when planes are
        // large (1024^2)
        if (P.kfix > 0 && P.kfix <= 16 && P.fa->kind == 0) {  // (a queue form's kfix is its depth)
            K = std::min(P.kfix, std::max(1, ny));
            if (K > 8) {
                for (const void *k : {P.fa->kfwd, P.fa->kinv, P.fa->kfwd_x, P.fa->kinv_x})
                    if (k) cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            }
        }
        // split Pass A: z rows and y columns as two plain launches (the plane
        // goes through DRAM between them); K CTAs still share each plane
        P.split_a = P.kfix == -1 && P.fa->kind == 0;
        if (P.split_a) {
            P.k_fa = K;
            P.grid_fa = K * std::max(1, std::min(nx, P.occ_fa * sms / K));
        } else {
            if (P.fa->kind == 1) {
                // the plane lives in the cluster's shared memory: the cluster size is fixed
                K = P.fa->k;
                if (K > 8) {
                    cudaFuncSetAttribute(P.fa->kfwd, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
                    cudaFuncSetAttribute(P.fa->kinv, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
                }
            }
            const int mc = max_clusters(P.fa->kfwd, K, nx, P.fa->smem, P.fa->nt, std::max(1, P.occ_fa * sms / K));
            P.k_fa = K;
            P.grid_fa = K * std::min(nx, mc);
            if (P.fa->kind == 1 && mc < 1) P.fa = nullptr;
        }
    }
    if (P.fb) {
        for (const void *k : {P.fb->kfwd, P.fb->kinv, P.fb->kfwd_epi, P.fb->kinv_epi}) {
            cudaError_t e = raise_smem_limit(k, P.fb->smem);
            if (e != cudaSuccess) {
                cudaGetLastError();
                P.fb = nullptr;
                break;
            }
        }
    }
    if (P.fb) {
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, P.fb->kfwd, P.fb->nt, P.fb->smem);
        P.occ_fb = std::max(occ, 1);
        const long long ncols = (long long)ny * (m + 1);
        const long long tiles = (ncols + P.fb->w - 1) / P.fb->w;
        P.grid_fb = (int)std::min<long long>(tiles, (long long)P.occ_fb * sms);
    }
    return P.dtype == GPUFFT_FLOAT ? upload_stage_tables<float>(P) : upload_stage_tables<double>(P);
}

// ---------------------------------------------------------------------------
// wisdom: (device, dtype, grid) -> chosen candidate per pass
// ---------------------------------------------------------------------------
namespace {
using WisdomKey = std::tuple<std::string, int, long long, long long, long long>;
std::mutex g_wisdom_mu;
struct WisdomEntry {
    int a, b, k;  // Pass A candidate, Pass B candidate, Pass A cluster size (0: chosen from L2)
};
std::map<WisdomKey, WisdomEntry> g_wisdom;
bool g_wisdom_env_loaded = false;
}  // namespace

static std::string device_tag(int dev) {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return "unknown";
    std::string name = prop.name;
    for (auto &c : name)
        if (c == ' ') c = '_';
    return name + "_sm" + std::to_string(prop.major * 10 + prop.minor);
}

// tensor-core plans are remembered apart from plain ones (dtype + 16)
static WisdomKey wisdom_key(const Plan &P) {
    return WisdomKey(device_tag(P.device), P.dtype + (P.tc_split ? 16 : 0), (long long)P.nx, (long long)P.ny,
                     (long long)P.nz);
}

static int wisdom_load_locked(const char *path) {
    std::ifstream in(path);
    if (!in) return set_error(GPUFFT_ERR_INVALID, "cannot read wisdom file %s", path);
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::istringstream ss(line);
        std::string dev;
        int dt, a, b, k = 0;
        long long nx, ny, nz;
        if (ss >> dev >> dt >> nx >> ny >> nz >> a >> b) {
            if (!(ss >> k) || k < -1 || k > 16 || (k > 0 && (k & (k - 1)))) k = 0;  // older files have none
            g_wisdom[WisdomKey(dev, dt, nx, ny, nz)] = {a, b, k};
        }
    }
    return GPUFFT_SUCCESS;
}

static int wisdom_save_locked(const char *path) {
    std::ofstream out(path);
    if (!out) return set_error(GPUFFT_ERR_INVALID, "cannot write wisdom file %s", path);
    out << "# gpufft_b200 wisdom: device dtype nx ny nz passA_candidate passB_candidate passA_cluster_size(0=auto,-1=split)\n";
    for (const auto &kv : g_wisdom)
        out << std::get<0>(kv.first) << " " << std::get<1>(kv.first) << " " << std::get<2>(kv.first) << " "
            << std::get<3>(kv.first) << " " << std::get<4>(kv.first) << " " << kv.second.a << " " << kv.second.b << " "
            << kv.second.k << "\n";
    return GPUFFT_SUCCESS;
}

int wisdom_save(const char *path) {
    std::lock_guard<std::mutex> lk(g_wisdom_mu);
    return wisdom_save_locked(path);
}

int wisdom_load(const char *path) {
    std::lock_guard<std::mutex> lk(g_wisdom_mu);
    return wisdom_load_locked(path);
}

static bool wisdom_lookup(const Plan &P, int &ia, int &ib, int &k) {
    std::lock_guard<std::mutex> lk(g_wisdom_mu);
    if (!g_wisdom_env_loaded) {
        g_wisdom_env_loaded = true;
        const char *path = std::getenv("GPUFFT_WISDOM");
        if (path) {
            std::ifstream probe(path);
            if (probe) wisdom_load_locked(path);
        }
    }
    auto it = g_wisdom.find(wisdom_key(P));
    if (it == g_wisdom.end()) return false;
    ia = it->second.a;
    ib = it->second.b;
    k = it->second.k;
    return true;
}

static void wisdom_store(const Plan &P) {
    std::lock_guard<std::mutex> lk(g_wisdom_mu);
    g_wisdom[wisdom_key(P)] = {P.idx_a, P.idx_b, P.kfix};
    const char *path = std::getenv("GPUFFT_WISDOM");
    if (path) wisdom_save_locked(path);
}

static int count_candidates(const Plan &P, int pass) {
    const int ny = (int)P.ny, m = (int)(P.nz / 2);
    int n = 0;
    if (pass == 0) {
        const fast::VariantA *va = variants_a(P.dtype).data();
        const int na = (int)variants_a(P.dtype).size();
        for (int i = 0; i < na; ++i) n += (va[i].ny == ny && va[i].m == m);
    } else {
        const fast::VariantB *vb = variants_b(P.dtype).data();
        const int nb = (int)variants_b(P.dtype).size();
        for (int i = 0; i < nb; ++i) n += b_eligible(P, vb[i]);
    }
    return n;
}

static int plan_exec_pass_impl(const Plan *P, void *data, void *stream, int pass, bool forward);

// mean ms of forward + inverse of one pass over `reps` repetitions
static float time_pass(const Plan &P, void *data, cudaStream_t s, int pass, int reps) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int w = 0; w < 2; ++w) {
        plan_exec_pass_impl(&P, data, s, pass, true);
        plan_exec_pass_impl(&P, data, s, pass, false);
    }
    cudaEventRecord(e0, s);
    int rc = GPUFFT_SUCCESS;
    for (int r = 0; r < reps && rc == GPUFFT_SUCCESS; ++r) {
        rc = plan_exec_pass_impl(&P, data, s, pass, true);
        if (rc == GPUFFT_SUCCESS) rc = plan_exec_pass_impl(&P, data, s, pass, false);
    }
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != GPUFFT_SUCCESS || cudaGetLastError() != cudaSuccess) return 1e30f;
    return ms / reps;
}

int plan_autotune(Plan *P, void *scratch, void *stream) {
    if (!P) return set_error(GPUFFT_ERR_NOT_INIT, "no plan");
    cudaStream_t s = (cudaStream_t)stream;
    const size_t bytes = (size_t)P->nx * P->ny * (P->nz / 2 + 1) * (P->dtype == GPUFFT_FLOAT ? 8 : 16);
    void *buf = scratch;
    if (!buf) {
        cudaError_t e = cudaMalloc(&buf, bytes);
        if (e != cudaSuccess)
            return set_error(GPUFFT_ERR_OOM, "autotune scratch (%zu bytes): %s", bytes, cudaGetErrorString(e));
    }
    cudaMemsetAsync(buf, 0, bytes, s);
    const int reps = bytes > (256u << 20) ? 3 : 10;
    int best[2] = {-1, -1}, best_k = 0;
    for (int pass = 0; pass < 2; ++pass) {
        const int n = count_candidates(*P, pass);
        float best_ms = 1e30f;
        // (a tensor-core plan's x pass is one of its v = 2 kernels, never generic)
        for (int c = (pass == 1 && P->tc_split) ? 0 : -1; c < n; ++c) {
            // Pass A candidates are timed at the cluster size chosen from the
            // L2 size (K), at K/2 and K/4, at 16 when K is 8, and split into
            // two launches
            int ks[5] = {0, 0, 0, 0, 0}, nk = 1;
            if (pass == 0 && c >= 0) {
                P->kfix = 0;
                setup_fast(*P, c, P->idx_b);
                if (P->fa && P->fa->kind == 0) {
                    const int k0 = P->k_fa;
                    for (int k : {k0 / 2, k0 / 4, k0 == 8 ? 16 : 0})
                        if (k >= 2) ks[nk++] = k;
                    ks[nk++] = -1;
                } else if (P->fa && P->fa->kind == 2) {
                    // the queue form: planes between a plane's two phases
                    ks[nk++] = 16;
                    ks[nk++] = 32;
                }
            }
            for (int ki = 0; ki < nk; ++ki) {
                P->kfix = pass == 0 ? ks[ki] : best_k;
                if (pass == 0)
                    setup_fast(*P, c, P->idx_b);
                else
                    setup_fast(*P, best[0], c);
                if ((pass == 0 && c >= 0 && !P->fa) || (pass == 1 && c >= 0 && !P->fb)) continue;
                if (pass == 0 && ks[ki] > 0 && P->fa && P->fa->kind != 2 && P->k_fa != ks[ki]) continue;
                if (pass == 0 && ks[ki] == -1 && !P->split_a) continue;
                const float ms = time_pass(*P, buf, s, pass, reps);
                if (ms < best_ms) {
                    best_ms = ms;
                    best[pass] = c;
                    if (pass == 0) best_k = ks[ki];
                }
            }
        }
    }
    if (!scratch) cudaFree(buf);
    P->kfix = best_k;
    const int rc = setup_fast(*P, best[0], best[1]);
    if (rc != GPUFFT_SUCCESS) return rc;
    P->tuned = true;
    wisdom_store(*P);
    return GPUFFT_SUCCESS;
}

template <typename T>
static int build_plan(Plan &P) {
    using V = cx_t<T>;
    const int vs = (int)sizeof(V);
    const int maxe = MaxE<T>::value;
    const int nx = (int)P.nx, ny = (int)P.ny, nz = (int)P.nz, m = nz / 2, nh = nz / 2 + 1;
    std::vector<int> rx, ry, rz;
    if (!factorize(nx, rx) || !factorize(ny, ry) || !factorize(m, rz))
        return set_error(GPUFFT_ERR_UNSUPPORTED,
                         "grid %dx%dx%d: Nx, Ny and Nz/2 must factor into 2,3,5,7,11,13", nx, ny, nz);

    int smem_optin = 0;
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, P.device);
    if (smem_optin <= 0) smem_optin = 227 * 1024;
    const int budget = smem_optin - 1024;

    // Tiles are sized so that both ping-pong tiles plus the twiddle tables
    // take about a third of the SM's shared memory (three CTAs per SM), with
    // rows of at most 128 bytes; long axes shrink the tile width down to 1.
    const long long target = std::min<long long>(budget, 75 * 1024);
    const int wmax = 128 / vs;

    // ---- Pass B (x axis): column tiles of wx columns, [nx][wx] in smem
    int wx = wmax;
    while (wx > 1 && (long long)(nx + 2LL * nx * wx) * vs > target) wx /= 2;
    if ((long long)(nx + 2LL * nx * wx) * vs > budget)
        return set_error(GPUFFT_ERR_UNSUPPORTED, "Nx=%d too long for one shared-memory tile", nx);

    // ---- Pass A phase 2 (y axis)
    int wy = wmax;
    while (wy > 1 && (long long)(nz + ny + 2LL * ny * wy) * vs > target) wy /= 2;
    if ((long long)(nz + ny + 2LL * ny * wy) * vs > budget)
        return set_error(GPUFFT_ERR_UNSUPPORTED, "Ny=%d too long for one shared-memory tile", ny);

    // ---- Pass A phase 1 (z rows): odd pitch >= m+1 keeps row accesses conflict-free
    const int pz = (m % 2 == 0) ? m + 1 : m + 2;
    int wz = 32;
    auto bytes_a = [&](int wzc) {
        return (long long)(nz + ny + 2LL * std::max<long long>((long long)wzc * pz, (long long)ny * wy)) * vs;
    };
    while (wz > 1 && bytes_a(wz) > target) wz = (wz > 16) ? wz - 8 : wz / 2;
    if (bytes_a(wz) > budget) return set_error(GPUFFT_ERR_UNSUPPORTED, "Nz=%d too long for one shared-memory tile", nz);
    (void)maxe;

    // ---- parameters
    PassAParams &A = P.pa;
    std::memset(&A, 0, sizeof(A));
    A.nx = nx; A.ny = ny; A.nz = nz; A.nh = nh; A.m = m;
    A.wz = wz; A.pz = pz; A.wzdiv = make_fastdiv(wz); A.nhdiv = make_fastdiv(nh);
    A.wy = wy; A.wydiv = make_fastdiv(wy);
    fill_axis(A.az, m, rz, 2);
    fill_axis(A.ay, ny, ry, 1);
    A.tile_elems = std::max(wz * pz, ny * wy);
    P.smem_a = (size_t)(nz + ny + 2 * (size_t)A.tile_elems) * vs;

    PassBParams &B = P.pb;
    std::memset(&B, 0, sizeof(B));
    B.nx = nx; B.ncols = (long long)ny * nh; B.wx = wx; B.wxdiv = make_fastdiv(wx);
    fill_axis(B.ax, nx, rx, 1);
    B.ntiles = (B.ncols + wx - 1) / wx;
    B.epi = 0;
    B.dealias = 0;
    B.scale = 1.0;
    B.ny = ny;
    B.nh = nh;
    B.nz = nz;
    P.smem_b = (size_t)(nx + 2 * (size_t)nx * wx) * vs;

    // ---- twiddle tables on the device
    const std::vector<T> hx = twiddle_table<T>(nx), hy = twiddle_table<T>(ny), hz = twiddle_table<T>(nz);
    const size_t bx = hx.size() * sizeof(T), by = hy.size() * sizeof(T), bz = hz.size() * sizeof(T);
    // (then 16 bytes of device flags: [0] a tensor-core x pass's bounded wait ran out)
    const size_t fl = (bx + by + bz + 15) / 16 * 16;
    cudaError_t e = cudaMalloc(&P.tw_dev, fl + 16);
    if (e != cudaSuccess) return set_error(GPUFFT_ERR_OOM, "cudaMalloc twiddles: %s", cudaGetErrorString(e));
    char *base = (char *)P.tw_dev;
    e = cudaMemset(base + fl, 0, 16);
    if (e == cudaSuccess) e = cudaMemcpy(base, hx.data(), bx, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(base + bx, hy.data(), by, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(base + bx + by, hz.data(), bz, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_error(e, "cudaMemcpy twiddles");
    B.twx = base;
    B.err = reinterpret_cast<int *>(base + fl);
    A.twy = base + bx;
    A.twz = base + bx + by;

    // ---- kernel attributes and launch geometry
    auto ka_f = pass_a_kernel<T, true>, ka_i = pass_a_kernel<T, false>;
    auto kb_f = pass_b_kernel<T, true>, kb_i = pass_b_kernel<T, false>;
    for (auto k : {ka_f, ka_i}) {
        e = raise_smem_limit((const void *)k, P.smem_a);
        if (e != cudaSuccess) return cuda_error(e, "cudaFuncSetAttribute(pass A smem)");
        cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    }
    for (auto k : {kb_f, kb_i}) {
        e = raise_smem_limit((const void *)k, P.smem_b);
        if (e != cudaSuccess) return cuda_error(e, "cudaFuncSetAttribute(pass B smem)");
    }
    const int sms = device_sms(P.device);
    int occ_a = 0, occ_b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_a, ka_f, kThreads, P.smem_a);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_b, kb_f, kThreads, P.smem_b);
    occ_a = std::max(occ_a, 1);
    occ_b = std::max(occ_b, 1);

    const size_t plane_bytes = (size_t)ny * nh * vs;
    const int K = choose_cluster(P.device, nx, ny, m, wy, plane_bytes, occ_a, sms);
    A.K = K;
    const int max_cl = max_clusters((const void *)ka_f, K, nx, P.smem_a, kThreads, std::max(1, occ_a * sms / K));
    P.grid_a = K * std::min(nx, max_cl);
    P.grid_b = (int)std::min<long long>(B.ntiles, (long long)occ_b * sms);
    P.occ_a = occ_a;
    P.occ_b = occ_b;
    if (std::getenv("GPUFFT_GENERIC_ONLY") && !P.tc_split) {
        P.idx_a = P.idx_b = -1;
        return GPUFFT_SUCCESS;
    }
    int ia = 0, ib = 0;
    if (wisdom_lookup(P, ia, ib, P.kfix)) P.tuned = true;
    const char *va = std::getenv("GPUFFT_VARIANT_A"), *vb = std::getenv("GPUFFT_VARIANT_B");
    if (va) ia = std::atoi(va);
    if (vb) ib = std::atoi(vb);
    const int rc = setup_fast(P, ia, ib);
    if (rc == GPUFFT_SUCCESS && P.tc_split && !P.fb)
        return set_error(GPUFFT_ERR_UNSUPPORTED,
                         "no tensor-core x-pass kernel for Nx=%lld (compiled: FP32, Nx = 512 and 1024)", (long long)nx);
    return rc;
}

int plan_create(Plan **out, int64_t nx, int64_t ny, int64_t nz, int dtype, int flags) {
    if (!out) return set_error(GPUFFT_ERR_INVALID, "plan pointer is NULL");
    *out = nullptr;
    if (nx < 1 || ny < 1 || nz < 1)
        return set_error(GPUFFT_ERR_INVALID, "grid %lldx%lldx%lld: every size must be >= 1", (long long)nx,
                         (long long)ny, (long long)nz);
    if (dtype != GPUFFT_FLOAT && dtype != GPUFFT_DOUBLE)
        return set_error(GPUFFT_ERR_INVALID, "dtype %d is neither GPUFFT_FLOAT nor GPUFFT_DOUBLE", dtype);
    if (nz % 2 != 0)
        return set_error(GPUFFT_ERR_UNSUPPORTED, "odd Nz=%lld is not supported", (long long)nz);
    if (nx > (1 << 24) || ny > (1 << 24) || nz > (1 << 24) || ny * (nz / 2 + 1) >= (1LL << 31))
        return set_error(GPUFFT_ERR_UNSUPPORTED, "grid too large for 32-bit in-plane indexing");
    Plan *P = new (std::nothrow) Plan();
    if (!P) return set_error(GPUFFT_ERR_OOM, "host allocation failed");
    P->nx = nx; P->ny = ny; P->nz = nz; P->dtype = dtype;
    P->tc_split = (flags & GPUFFT_PLAN_TC_SPLIT) != 0;
    if (P->tc_split && dtype != GPUFFT_FLOAT) {
        delete P;
        return set_error(GPUFFT_ERR_UNSUPPORTED, "GPUFFT_PLAN_TC_SPLIT is an FP32 form");
    }
    cudaError_t e = cudaGetDevice(&P->device);
    if (e != cudaSuccess) { delete P; return cuda_error(e, "cudaGetDevice"); }
    const int rc = dtype == GPUFFT_FLOAT ? build_plan<float>(*P) : build_plan<double>(*P);
    if (rc != GPUFFT_SUCCESS) { plan_destroy(P); return rc; }
    const char *env = std::getenv("GPUFFT_AUTOTUNE");
    if (((flags & GPUFFT_PLAN_AUTOTUNE) || (env && env[0] == '1')) && !P->tuned) {
        const int rt = plan_autotune(P, nullptr, nullptr);
        if (rt != GPUFFT_SUCCESS) { plan_destroy(P); return rt; }
    }
    *out = P;
    return GPUFFT_SUCCESS;
}

int plan_adopt(Plan *P, const Plan *Q) {
    if (!P || !Q) return set_error(GPUFFT_ERR_NOT_INIT, "no plan");
    if (P->nx != Q->nx || P->ny != Q->ny || P->nz != Q->nz || P->dtype != Q->dtype || P->tc_split != Q->tc_split)
        return set_error(GPUFFT_ERR_INVALID, "plan_adopt: the plans differ in grid or form");
    if (Q->idx_a < 0 && Q->idx_b < 0) return GPUFFT_SUCCESS;  // generic kernels: nothing to copy
    P->kfix = Q->kfix;
    const int rc = setup_fast(*P, Q->idx_a, Q->idx_b);
    if (rc == GPUFFT_SUCCESS) P->tuned = Q->tuned;
    return rc;
}

int plan_destroy(Plan *P) {
    if (!P) return GPUFFT_SUCCESS;
    if (P->tw_dev) {
        int cur = -1;
        cudaGetDevice(&cur);
        if (cur != P->device) cudaSetDevice(P->device);
        cudaFree(P->tw_dev);
        if (P->stage_dev) cudaFree(P->stage_dev);
        free_queue(*P);
        if (cur != P->device && cur >= 0) cudaSetDevice(cur);
    }
    delete P;
    return GPUFFT_SUCCESS;
}

// xch (optional, specialised kernels only): the y columns' global side in
// the slab decomposition's exchange layout (PassAParams::xch)
struct XchLayout {
    void *buf;
    int nyl;
    long long chunk;  // complex elements
};

template <typename T>
static int launch_pass_a(const Plan &P, void *data, cudaStream_t s, bool fwd, const XchLayout *xch = nullptr) {
    PassAParams prm = P.pa;
    prm.data = data;
    const void *kf = P.fa ? P.fa->kfwd : nullptr, *ki = P.fa ? P.fa->kinv : nullptr;
    if (xch) {
        if (!P.fa || !P.fa->kfwd_x) return set_error(GPUFFT_ERR_UNSUPPORTED, "no exchange-layout Pass A kernel");
        prm.xch = xch->buf;
        prm.xch_nyl = xch->nyl;
        prm.xch_chunk = xch->chunk;
        kf = P.fa->kfwd_x;
        ki = P.fa->kinv_x;
    }
    if (P.fa && P.fa->kind == 2 && !xch && ((uintptr_t)data) % 16 == 0) {
        // queue-scheduled Pass A: the tensor maps carry this call's field address
        const long long nh = P.nz / 2 + 1;
        const int wy = P.fa->wy;
        CUtensorMap tm[3];
        bool ok;
        if (P.dtype == GPUFFT_FLOAT) {
            // row pairs: lines of 2 Nh complex, boxes of Ny/2 lines
            const long long lines = P.nx * P.ny / 2;
            const int bh = (int)(P.ny / 2);
            ok = encode_pair_map(&tm[0], data, nh, lines, wy, bh) && encode_pair_map(&tm[1], data, nh, lines, wy + 2, bh) &&
                 encode_pair_map(&tm[2], data, nh, lines, 2, bh);
        } else {
            // single rows: 2 Nh 8-byte elements per row (16 Nh bytes), equal boxes of up to 256 rows
            const int bh = q::box_rows((int)P.ny);
            ok = encode_view(&tm[0], data, 2 * nh, P.nx * P.ny, 16 * nh, 2 * wy, bh) &&
                 encode_view(&tm[1], data, 2 * nh, P.nx * P.ny, 16 * nh, 2 * wy, bh) &&
                 encode_view(&tm[2], data, 2 * nh, P.nx * P.ny, 16 * nh, 2, bh);
        }
        if (!ok) return set_error(GPUFFT_ERR_CUDA, "cuTensorMapEncodeTiled failed for the Pass A field view");
        q::PassAQParams qp{};
        qp.data = data;
        qp.unp = fwd ? P.q_unp : P.q_unp_i;
        qp.rtw = P.q_rtw;
        qp.sty = P.pa.sty;
        qp.items = fwd ? P.q_items_f : P.q_items_i;
        qp.nitems = P.q_nitems;
        qp.ctr = reinterpret_cast<int *>(P.q_dev);
        qp.need = (fwd ? P.q_need : (int)((P.nz / 2) / wy)) + P.q_extra;
        qp.wait_ns = 2000000000LL;  // 2 s: far above any launch's length
        if (const char *ev = std::getenv("GPUFFT_QUEUE_WAIT_MS")) qp.wait_ns = 1000000LL * std::max(1, std::atoi(ev));
        void *args[] = {&qp, &tm[0], &tm[1], &tm[2]};
        const cudaError_t e =
            cudaLaunchKernel(fwd ? P.fa->kfwd : P.fa->kinv, dim3(P.grid_fa), dim3(P.fa->nt), args, P.fa->smem, s);
        return e == cudaSuccess ? GPUFFT_SUCCESS : cuda_error(e, "launch pass A (queue)");
    }
    if (P.fa && P.fa->kind == 2) {
        // (a field not 16-byte aligned: the generic kernels below)
        kf = ki = nullptr;
    }
    if (P.fa && P.split_a) {
        // forward: z rows then y columns; inverse: y columns then z rows
        prm.K = P.k_fa;
        void *args[] = {&prm};
        for (int half = 0; half < 2; ++half) {
            prm.phases = (fwd == (half == 0)) ? 1 : 2;
            const cudaError_t e = cudaLaunchKernel(fwd ? kf : ki, dim3(P.grid_fa), dim3(P.fa->nt), args, P.fa->smem, s);
            if (e != cudaSuccess) return cuda_error(e, "launch split pass A (specialised)");
        }
        return GPUFFT_SUCCESS;
    }
    if (P.fa && kf) {
        prm.K = P.k_fa;
        prm.phases = 0;
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        cfg.gridDim = dim3(P.grid_fa, 1, 1);
        cfg.blockDim = dim3(P.fa->nt, 1, 1);
        cfg.dynamicSmemBytes = P.fa->smem;
        cfg.stream = s;
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = prm.K;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        void *args[] = {&prm};
        const cudaError_t e = cudaLaunchKernelExC(&cfg, fwd ? kf : ki, args);
        return e == cudaSuccess ? GPUFFT_SUCCESS : cuda_error(e, "launch pass A (specialised)");
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim = dim3(P.grid_a, 1, 1);
    cfg.blockDim = dim3(kThreads, 1, 1);
    cfg.dynamicSmemBytes = P.smem_a;
    cfg.stream = s;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = prm.K;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = fwd ? cudaLaunchKernelEx(&cfg, pass_a_kernel<T, true>, prm)
                        : cudaLaunchKernelEx(&cfg, pass_a_kernel<T, false>, prm);
    return e == cudaSuccess ? GPUFFT_SUCCESS : cuda_error(e, "launch pass A");
}

template <typename T>
static int launch_pass_b(const Plan &P, void *data, cudaStream_t s, bool fwd, double scale = 1.0, int dealias = 0) {
    if (P.nx == 1) return GPUFFT_SUCCESS;  // a length-1 DFT is the identity
    PassBParams prm = P.pb;
    prm.data = data;
    prm.scale = scale;
    prm.dealias = dealias;
    prm.epi = (scale != 1.0 || dealias) ? 1 : 0;
    if (P.fb && P.fb->kind == 3 && ((uintptr_t)data) % 16 == 0) {
        // tensor-copy tiles: the map carries this call's field address
        prm.wx = P.fb->w;
        prm.ntiles = (prm.ncols + P.fb->w - 1) / P.fb->w;
        CUtensorMap tm;
        const int epc = (int)sizeof(cx_t<T>) / 8;  // 8-byte elements per complex
        if (!encode_view(&tm, data, prm.ncols * epc, P.nx, prm.ncols * (long long)sizeof(cx_t<T>), P.fb->w * epc,
                         q::box_rows((int)P.nx)))  // the kernel's rows per copy (BShape::BOXH)
            return set_error(GPUFFT_ERR_CUDA, "cuTensorMapEncodeTiled failed for the Pass B field view");
        void *args[] = {&prm, &tm};
        const void *k = prm.epi ? (fwd ? P.fb->kfwd_epi : P.fb->kinv_epi) : (fwd ? P.fb->kfwd : P.fb->kinv);
        const cudaError_t e = cudaLaunchKernel(k, dim3(P.grid_fb), dim3(P.fb->nt), args, P.fb->smem, s);
        return e == cudaSuccess ? GPUFFT_SUCCESS : cuda_error(e, "launch pass B (tensor copies)");
    }
    if (P.fb && P.fb->kind != 3 && !(P.fb->kind != 0 && ((uintptr_t)data) % 16 != 0)) {
        prm.wx = P.fb->w;
        prm.ntiles = (prm.ncols + P.fb->w - 1) / P.fb->w;
        void *args[] = {&prm};
        const void *k = prm.epi ? (fwd ? P.fb->kfwd_epi : P.fb->kinv_epi) : (fwd ? P.fb->kfwd : P.fb->kinv);
        const cudaError_t e = cudaLaunchKernel(k, dim3(P.grid_fb), dim3(P.fb->nt), args, P.fb->smem, s);
        return e == cudaSuccess ? GPUFFT_SUCCESS : cuda_error(e, "launch pass B (specialised)");
    }
    if (fwd)
        pass_b_kernel<T, true><<<P.grid_b, kThreads, P.smem_b, s>>>(prm);
    else
        pass_b_kernel<T, false><<<P.grid_b, kThreads, P.smem_b, s>>>(prm);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GPUFFT_SUCCESS : cuda_error(e, "launch pass B");
}

int plan_exec_ex(const Plan *P, void *data, void *stream, bool forward, double scale, int dealias) {
    if (!P) return set_error(GPUFFT_ERR_NOT_INIT, "no plan");
    if (!data) return set_error(GPUFFT_ERR_INVALID, "data pointer is NULL");
    if (((uintptr_t)data) % (P->dtype == GPUFFT_FLOAT ? 8 : 16) != 0)
        return set_error(GPUFFT_ERR_INVALID, "data pointer is not aligned to its complex type");
    if ((scale != 1.0 || dealias) && P->nx == 1)
        return set_error(GPUFFT_ERR_UNSUPPORTED, "Nx = 1 has no x pass to fuse the scale or dealiasing into");
    if (dealias && !forward) return set_error(GPUFFT_ERR_INVALID, "dealiasing is fused into R2C only");
    cudaStream_t s = (cudaStream_t)stream;
    int rc;
    if (P->dtype == GPUFFT_FLOAT) {
        if (forward) {
            rc = launch_pass_a<float>(*P, data, s, true);
            if (rc == GPUFFT_SUCCESS) rc = launch_pass_b<float>(*P, data, s, true, scale, dealias);
        } else {
            rc = launch_pass_b<float>(*P, data, s, false, scale);
            if (rc == GPUFFT_SUCCESS) rc = launch_pass_a<float>(*P, data, s, false);
        }
    } else {
        if (forward) {
            rc = launch_pass_a<double>(*P, data, s, true);
            if (rc == GPUFFT_SUCCESS) rc = launch_pass_b<double>(*P, data, s, true, scale, dealias);
        } else {
            rc = launch_pass_b<double>(*P, data, s, false, scale);
            if (rc == GPUFFT_SUCCESS) rc = launch_pass_a<double>(*P, data, s, false);
        }
    }
    return rc;
}

int plan_exec(const Plan *P, void *data, void *stream, bool forward) {
    return plan_exec_ex(P, data, stream, forward, 1.0, 0);
}

int plan_exec_pass(const Plan *P, void *data, void *stream, int pass, bool forward) {
    return plan_exec_pass_impl(P, data, stream, pass, forward);
}

static int plan_exec_pass_impl(const Plan *P, void *data, void *stream, int pass, bool forward) {
    if (!P) return set_error(GPUFFT_ERR_NOT_INIT, "no plan");
    if (!data) return set_error(GPUFFT_ERR_INVALID, "data pointer is NULL");
    if (((uintptr_t)data) % (P->dtype == GPUFFT_FLOAT ? 8 : 16) != 0)
        return set_error(GPUFFT_ERR_INVALID, "data pointer is not aligned to its complex type");
    if (pass != 0 && pass != 1) return set_error(GPUFFT_ERR_INVALID, "pass %d is neither 0 (A) nor 1 (B)", pass);
    cudaStream_t s = (cudaStream_t)stream;
    if (P->dtype == GPUFFT_FLOAT)
        return pass == 0 ? launch_pass_a<float>(*P, data, s, forward) : launch_pass_b<float>(*P, data, s, forward);
    return pass == 0 ? launch_pass_a<double>(*P, data, s, forward) : launch_pass_b<double>(*P, data, s, forward);
}

bool plan_has_xch(const Plan *P) { return P && P->fa && P->fa->kfwd_x && P->fa->kinv_x; }

int plan_exec_pass_a_xch(const Plan *P, void *data, void *xch, int nyl, long long chunk, void *stream, bool forward) {
    if (!P) return set_error(GPUFFT_ERR_NOT_INIT, "no plan");
    if (!data || !xch) return set_error(GPUFFT_ERR_INVALID, "data or exchange buffer is NULL");
    if (nyl < 1 || P->ny % nyl != 0) return set_error(GPUFFT_ERR_INVALID, "Ny = %lld is not a multiple of %d",
                                                      (long long)P->ny, nyl);
    const XchLayout x{xch, nyl, chunk};
    cudaStream_t s = (cudaStream_t)stream;
    return P->dtype == GPUFFT_FLOAT ? launch_pass_a<float>(*P, data, s, forward, &x)
                                    : launch_pass_a<double>(*P, data, s, forward, &x);
}

int plan_launches(const Plan *P) { return P ? (P->nx == 1 ? 1 : 2) + (P->fa && P->split_a ? 1 : 0) : 0; }

static void describe_axis(std::string &out, const char *name, const AxisPlan &ax) {
    char b[64];
    snprintf(b, sizeof(b), "%s=%d[", name, ax.n);
    out += b;
    for (int s = 0; s < ax.nst; ++s) {
        snprintf(b, sizeof(b), "%s%d", s ? "x" : "", ax.radix[s]);
        out += b;
    }
    out += "]";
}

int plan_describe(const Plan *P, char *buf, int len) {
    if (!P) return set_error(GPUFFT_ERR_NOT_INIT, "no plan");
    std::string s;
    char b[256];
    snprintf(b, sizeof(b), "grid=%lldx%lldx%lld dtype=%s tuned=%d candA=%d candB=%d ", (long long)P->nx,
             (long long)P->ny, (long long)P->nz, P->dtype == GPUFFT_FLOAT ? "f32" : "f64", P->tuned ? 1 : 0, P->idx_a,
             P->idx_b);
    s += b;
    describe_axis(s, "x", P->pb.ax);
    s += " ";
    describe_axis(s, "y", P->pa.ay);
    s += " ";
    describe_axis(s, "zhalf", P->pa.az);
    snprintf(b, sizeof(b),
             " passA{K=%d grid=%d occ=%d smem=%zu wz=%d pz=%d wy=%d} passB{grid=%d occ=%d smem=%zu wx=%d tiles=%lld}",
             P->pa.K, P->grid_a, P->occ_a, P->smem_a, P->pa.wz, P->pa.pz, P->pa.wy, P->grid_b, P->occ_b, P->smem_b,
             P->pb.wx, P->pb.ntiles);
    s += b;
    if (P->fa) {
        snprintf(b, sizeof(b),
                 " fastA{kind=%d ny=%d m=%d rw=%d wy=%d nt=%d K=%d grid=%d occ=%d smem=%zu depth=%d split=%d}",
                 P->fa->kind, P->fa->ny, P->fa->m, P->fa->rw, P->fa->wy, P->fa->nt, P->k_fa, P->grid_fa, P->occ_fa,
                 P->fa->smem, P->fa->kind == 2 ? P->q_depth : 0, P->split_a ? 1 : 0);
        s += b;
    }
    if (P->fb) {
        snprintf(b, sizeof(b), " fastB{kind=%d nx=%d w=%d nt=%d v=%d grid=%d occ=%d smem=%zu}", P->fb->kind, P->fb->nx, P->fb->w,
                 P->fb->nt, P->fb->v, P->grid_fb, P->occ_fb, P->fb->smem);
        s += b;
    }
    if (buf && len > 0) {
        strncpy(buf, s.c_str(), (size_t)len - 1);
        buf[len - 1] = 0;
    }
    return (int)s.size() + 1;
}

}  // namespace gpufft

// ===========================================================================
// C ABI
// ===========================================================================
using namespace gpufft;

namespace {
std::mutex g_mu;
// the reference-shaped process-wide plan, one per dtype: single-GPU or slab-decomposed
Plan *g_global[2] = {nullptr, nullptr};
DistPlan *g_dist[2] = {nullptr, nullptr};
}  // namespace

extern "C" int gpufft_init(int64_t nx, int64_t ny, int64_t nz, int dtype, int procs, int rank) {
    if (procs != 1 || rank != 0)
        return set_error(GPUFFT_ERR_UNSUPPORTED,
                         "procs=%d rank=%d: more than one rank needs the NCCL unique id (gpufft_init_dist)", procs,
                         rank);
    Plan *P = nullptr;
    const int rc = plan_create(&P, nx, ny, nz, dtype, 0);
    if (rc != GPUFFT_SUCCESS) return rc;
    std::lock_guard<std::mutex> lk(g_mu);
    plan_destroy(g_global[dtype]);
    g_global[dtype] = P;
    dist_free(g_dist[dtype]);
    g_dist[dtype] = nullptr;
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_init_dist(int64_t nx, int64_t ny, int64_t nz, int dtype, int procs, int rank, const void *id) {
    if (dtype != GPUFFT_FLOAT && dtype != GPUFFT_DOUBLE) return set_error(GPUFFT_ERR_INVALID, "bad dtype %d", dtype);
    gpufft_dplan D = nullptr;
    const int rc = gpufft_dplan_create(&D, nx, ny, nz, dtype, procs, rank, id);
    if (rc != GPUFFT_SUCCESS) return rc;
    std::lock_guard<std::mutex> lk(g_mu);
    dist_free(g_dist[dtype]);
    g_dist[dtype] = reinterpret_cast<DistPlan *>(D);
    plan_destroy(g_global[dtype]);
    g_global[dtype] = nullptr;
    return GPUFFT_SUCCESS;
}

static Plan *global_plan(int dtype) {
    if (dtype != GPUFFT_FLOAT && dtype != GPUFFT_DOUBLE) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    return g_global[dtype];
}

static DistPlan *global_dist(int dtype) {
    std::lock_guard<std::mutex> lk(g_mu);
    return g_dist[dtype];
}

extern "C" int gpufft_r2c(int dtype, void *data, void *stream) {
    if (dtype != GPUFFT_FLOAT && dtype != GPUFFT_DOUBLE) return set_error(GPUFFT_ERR_INVALID, "bad dtype %d", dtype);
    if (DistPlan *D = global_dist(dtype)) return dist_exec(D, data, (cudaStream_t)stream, true);
    Plan *P = global_plan(dtype);
    if (!P) return set_error(GPUFFT_ERR_NOT_INIT, "gpufft_r2c: no %s plan; call gpufft_init first",
                             dtype == GPUFFT_FLOAT ? "float" : "double");
    return plan_exec(P, data, stream, true);
}

extern "C" int gpufft_c2r(int dtype, void *data, void *stream) {
    if (dtype != GPUFFT_FLOAT && dtype != GPUFFT_DOUBLE) return set_error(GPUFFT_ERR_INVALID, "bad dtype %d", dtype);
    if (DistPlan *D = global_dist(dtype)) return dist_exec(D, data, (cudaStream_t)stream, false);
    Plan *P = global_plan(dtype);
    if (!P) return set_error(GPUFFT_ERR_NOT_INIT, "gpufft_c2r: no %s plan; call gpufft_init first",
                             dtype == GPUFFT_FLOAT ? "float" : "double");
    return plan_exec(P, data, stream, false);
}

extern "C" int gpufft_finalize(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto &p : g_global) {
        plan_destroy(p);
        p = nullptr;
    }
    for (auto &d : g_dist) {
        dist_free(d);
        d = nullptr;
    }
    return GPUFFT_SUCCESS;
}

extern "C" const char *gpufft_last_error(void) { return last_error(); }

extern "C" int gpufft_plan_create(gpufft_plan *plan, int64_t nx, int64_t ny, int64_t nz, int dtype) {
    return gpufft_plan_create_ex(plan, nx, ny, nz, dtype, 0);
}

extern "C" int gpufft_plan_create_ex(gpufft_plan *plan, int64_t nx, int64_t ny, int64_t nz, int dtype, int flags) {
    Plan *P = nullptr;
    const int rc = plan_create(&P, nx, ny, nz, dtype, flags);
    if (plan) *plan = reinterpret_cast<gpufft_plan>(P);
    return rc;
}

extern "C" int gpufft_plan_autotune(gpufft_plan plan, void *scratch, void *stream) {
    return plan_autotune(reinterpret_cast<Plan *>(plan), scratch, stream);
}

extern "C" int gpufft_wisdom_save(const char *path) {
    if (!path) return set_error(GPUFFT_ERR_INVALID, "wisdom path is NULL");
    return wisdom_save(path);
}

extern "C" int gpufft_wisdom_load(const char *path) {
    if (!path) return set_error(GPUFFT_ERR_INVALID, "wisdom path is NULL");
    return wisdom_load(path);
}

extern "C" int gpufft_plan_destroy(gpufft_plan plan) { return plan_destroy(reinterpret_cast<Plan *>(plan)); }

extern "C" int gpufft_plan_check(gpufft_plan plan) {
    Plan *P = reinterpret_cast<Plan *>(plan);
    if (!P || !P->tw_dev) return set_error(GPUFFT_ERR_NOT_INIT, "no plan");
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != P->device) cudaSetDevice(P->device);
    int tc = 0, qe = 0;
    cudaError_t e = cudaMemcpy(&tc, P->pb.err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && P->q_dev) e = cudaMemcpy(&qe, reinterpret_cast<int *>(P->q_dev) + 2, sizeof(int), cudaMemcpyDeviceToHost);
    if (cur != P->device && cur >= 0) cudaSetDevice(cur);
    if (e != cudaSuccess) return cuda_error(e, "read the plan's device flags");
    if (tc || qe)
        return set_error(GPUFFT_ERR_CUDA, "a bounded device-side wait of this plan's kernels ran out (%s%s%s)",
                         qe ? "queue Pass A" : "", qe && tc ? ", " : "", tc ? "tensor-core x pass" : "");
    return GPUFFT_SUCCESS;
}

extern "C" int gpufft_exec_r2c(gpufft_plan plan, void *data, void *stream) {
    return plan_exec(reinterpret_cast<Plan *>(plan), data, stream, true);
}

extern "C" int gpufft_exec_c2r(gpufft_plan plan, void *data, void *stream) {
    return plan_exec(reinterpret_cast<Plan *>(plan), data, stream, false);
}

extern "C" int gpufft_exec_r2c_ex(gpufft_plan plan, void *data, void *stream, double scale, int dealias) {
    return plan_exec_ex(reinterpret_cast<Plan *>(plan), data, stream, true, scale, dealias);
}

extern "C" int gpufft_exec_c2r_ex(gpufft_plan plan, void *data, void *stream, double scale) {
    return plan_exec_ex(reinterpret_cast<Plan *>(plan), data, stream, false, scale, 0);
}

extern "C" int gpufft_exec_pass(gpufft_plan plan, void *data, void *stream, int pass, int forward) {
    return plan_exec_pass(reinterpret_cast<Plan *>(plan), data, stream, pass, forward != 0);
}

extern "C" int64_t gpufft_field_bytes(int64_t nx, int64_t ny, int64_t nz, int dtype) {
    if (nx < 1 || ny < 1 || nz < 1 || (dtype != GPUFFT_FLOAT && dtype != GPUFFT_DOUBLE)) return -1;
    return nx * ny * (nz / 2 + 1) * (dtype == GPUFFT_FLOAT ? 8 : 16);
}

extern "C" int gpufft_plan_launches(gpufft_plan plan) { return plan_launches(reinterpret_cast<Plan *>(plan)); }

extern "C" int gpufft_plan_describe(gpufft_plan plan, char *buf, int len) {
    return plan_describe(reinterpret_cast<Plan *>(plan), buf, len);
}

// fft_queue.cuh — Pass A (z R2C/C2R + y C2C of every x-plane) as one
// persistent, queue-scheduled kernel whose inputs arrive by bulk and tensor
// copies (sm_100a: cp.async.bulk / cp.async.bulk.tensor completing on
// mbarriers).
//
// Replaces the reference's batched 2D cuFFT R2C/C2R over x-planes
// (GPU_FFT/src/initialize_GPU_FFT/GPU_FFT_init.cu:61-64,90-91, executed at
// GPU_FFT/src/FFT_implementation/FFT_R2C.cu:45 and FFT_C2R.cu:66).
//
// Work items.  A plane (Ny rows of Nh = M+1 complex, M = Nz/2) is cut into
//   * row items: RI consecutive z-rows (one contiguous span of the field,
//     fetched by ONE 1D bulk copy), each row's M-point FFT plus the
//     real-to-complex unpack (forward) or pack (inverse) done by half a warp
//     in shared memory;
//   * column items: WY consecutive kz columns of all Ny rows, the y FFT,
//     fetched by TWO 2D tensor copies over a "row pair" view of the field:
//     with Nh odd, two rows are 16*Nh bytes, so rows 2r and 2r+1 form one
//     16-byte-aligned line of 2*Nh complex.  Box E (WY wide at x = c0) holds
//     the even rows' columns; box O (WY+2 wide at x = Nh-1+c0, the odd row's
//     first column rounded down to 16 bytes) holds the odd rows' columns one
//     slot in.  Slots read beyond the tile are ignored (another item may be
//     writing them).  The inverse's tile 0 also needs bin M of every row:
//     even rows find it in box O's slot 0, odd rows in a third 2-wide box.
// The forward runs row items then column items of a plane (the intermediate
// plane stays in place, in L2), the inverse the reverse.
//
// Schedule.  The item list (built on the host) interleaves the first-phase
// items of plane b with the second-phase items of plane b - D, so that only
// about D planes are between their phases at any time (the intermediate
// stays in L2; one cluster per plane put 40-70 planes there).  CTAs claim
// items in list order from an atomic counter.  A second-phase item waits
// (acquire load of the plane's completion count, bounded by a time limit,
// then an error flag) until its plane's first phase is complete; first-
// phase items are published with a release add by the copy warp once their
// buffer is released (after the consumers' stores).
//
// CTA roles: NT/32 consumer warps transform items; one producer warp (lane
// 0) claims the next item, waits for its plane when needed and issues its
// copies into the next free buffer of an NBUF-deep ring (full/empty
// mbarrier pairs), so an item's loads are in flight while the consumers
// transform the previous one and no load occupies a register.
//
// Write-back.  Consumers store column items (and, unless FB says otherwise,
// the forward's row items) with their own stores.  The inverse's row items,
// and per FB the forward's row items and the column items' E boxes, are
// left in the buffer and written back by the producer with one bulk or
// tensor store per item; it waits for a store to have read the buffer before
// refilling it, for a first-phase item's store to complete before publishing
// the item, and for all its stores before the CTA exits.
//
// Deadlock freedom: a CTA waits for a plane only in its producer, while its
// consumers finish every item the CTA claimed earlier (they never wait on
// anything but copies already issued) and the producer keeps publishing them
// during the wait.  Items are claimed in list order, so the lowest-numbered
// unpublished item always belongs to a CTA that can finish and publish it:
// its dependencies have lower numbers and are published.  This holds however
// many CTAs are resident.
//
// Counters (plan-owned, int): [0] next item, [1] CTAs finished, [2] error
// flag, [3] spare, [4 + x] items finished of plane x.  The last CTA to finish
// zeroes [0], [1] and the plane counts for the next launch, so one plan's
// executions must not overlap on the GPU.
#pragma once
#include <cuda.h>

#include "fft_fast.cuh"

namespace gpufft {
namespace q {

using fast::TileFFT;
using fast::COLS;
using fast::GROUP;
using fast::FromSmem;
using fast::ToSmem;

struct PassAQParams {
    void *data;
    const void *unp;    // unpack / pack factors, k < M: forward -i w^k / 2, inverse i conj(w^k), w = exp(-2 pi i / Nz)
    const void *rtw;    // row FFT step-1 twiddles: exp(-2 pi i a f / M) at (f - 1) * 16 + a, f < M / 16
    const void *sty;    // per-stage table of the y FFT (fft_fast.cuh stage_offset)
    const int *items;   // work list: (plane << 16) | (type << 15) | sub
    int nitems;
    int *ctr;           // counters (header)
    int need;           // first-phase items per plane
    long long wait_ns;  // time limit of one dependency or copy wait
};

enum ItemType { ROW_ITEM = 0, COL_ITEM = 1 };
__host__ __device__ constexpr int item_code(int plane, int type, int sub) { return (plane << 16) | (type << 15) | sub; }

// ---------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// makes the initialised barriers visible to the copy engine
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}
// Waits for the phase of parity `parity` to complete; false once `limit_ns`
// has passed without it.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer();
    while (true) {
        for (int i = 0; i < 64; ++i)
            if (mbar_try_wait(bar, parity)) return true;
        if ((long long)(globaltimer() - t0) > limit_ns) return false;
    }
}
// generic-proxy accesses before this point are ordered before later copies
__device__ __forceinline__ void fence_proxy_async_shared() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;\n" ::: "memory"); }
// 1D bulk copy global -> shared (16-byte aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// 1D bulk copy shared -> global (same alignment rules), committed as one bulk group
__device__ __forceinline__ void bulk_store(void *dst, const void *src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(dst), "r"(smem_u32(src)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}
// this thread's bulk stores have read their shared-memory sources / have completed
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
// 2D tensor copy shared -> global of the box at (x, y) of `map`, committed as one bulk group
__device__ __forceinline__ void tensor_store_2d(const CUtensorMap *map, int x, int y, const void *src) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];\n" ::"l"(
                     reinterpret_cast<unsigned long long>(map)),
                 "r"(smem_u32(src)), "r"(x), "r"(y)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}
// 2D tensor copy global -> shared of the box at (x, y) of `map` (no multicast)
__device__ __forceinline__ void tensor_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add(int *p, int v) {
    asm volatile("red.release.gpu.global.add.s32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
template <int N>
__device__ __forceinline__ void group_sync() {
    asm volatile("bar.sync 1, %0;\n" ::"n"(N) : "memory");
}

// Rows per tensor copy of the single-row view: the plane's rows in the fewest
// equal boxes of at most 256 rows (a tensor-copy box dimension is <= 256).
__host__ __device__ constexpr int box_rows(int ny) {
    int k = 1;
    while (ny / k > 256 || ny % k != 0) ++k;
    return ny / k;
}

// ---------------------------------------------------------------------------
// shape of one instantiation
// ---------------------------------------------------------------------------
// FP32 (PAIR): the row-pair view above, boxes E and O of NY/2 lines each.
// FP64: rows are 16-byte aligned on their own; the view is [rows][2 Nh]
// 8-byte elements and box E is WY columns of every row (NBX boxes of BHT
// rows), box X the one column M of every row.
template <typename T, int NY, int M, int NT, int NBUF, int WY_>
struct QShape {
    using V = cx_t<T>;
    static constexpr bool PAIR = sizeof(V) == 8;
    static constexpr int NH = M + 1;
    static constexpr int WY = WY_;                   // columns per column item
    static constexpr int RI = NT / 16;               // rows per row item (two per consumer warp)
    static constexpr int BH = NY / 2;                // row pairs per box (PAIR)
    static constexpr int BHT = box_rows(NY);         // rows per box (FP64)
    static constexpr int NBX = NY / BHT;
    static constexpr int NRI = NY / RI;
    static constexpr int NCI = M / WY;
    static constexpr int E_BYTES = PAIR ? WY * BH * (int)sizeof(V) : WY * NY * (int)sizeof(V);
    static constexpr int O_BYTES = PAIR ? (WY + 2) * BH * (int)sizeof(V) : 0;
    static constexpr int X_BYTES = PAIR ? 2 * BH * (int)sizeof(V) : NY * (int)sizeof(V);
    static constexpr int ROW_BYTES = RI * NH * (int)sizeof(V);
    static constexpr int TILE_BYTES = NY * WY * (int)sizeof(V);
    static constexpr int rup(int v) { return (v + 127) / 128 * 128; }
    static constexpr int mx(int a, int b) { return a > b ? a : b; }
    static constexpr int O_OFF = rup(E_BYTES);
    static constexpr int X_OFF = O_OFF + rup(O_BYTES);
    // FP64: box X of every BHT rows lands at a 128-byte pitch (tensor-copy
    // destinations are 128-byte aligned); XP is that pitch in complex values
    static constexpr int XB = PAIR ? X_BYTES : rup(BHT * (int)sizeof(V));
    static constexpr int XP = XB / (int)sizeof(V);
    static constexpr int BUF = rup(mx(mx(ROW_BYTES, TILE_BYTES), X_OFF + (PAIR ? X_BYTES : NBX * XB)));
    static constexpr int R2 = M / 16;                // row FFT: M = 16 x R2
    static constexpr int TAB = rup((M + M + NY) * (int)sizeof(V));
    // tables, buffers, mbarriers, slot words, and slack for 128-byte alignment
    static constexpr size_t smem_bytes() { return (size_t)TAB + (size_t)NBUF * BUF + 2 * NBUF * 8 + NBUF * 4 + 128; }
    static_assert(!PAIR || NH % 2 == 1, "row-pair view needs Nh odd (Nz a multiple of 4)");
    static_assert(!PAIR || BH <= 256, "box height");
    static_assert(PAIR || NY % BHT == 0, "whole boxes");
    static_assert(NY % RI == 0 && NY % 2 == 0, "rows per item");
    static_assert(M % WY == 0, "whole column tiles");
    static_assert(M % 16 == 0 && (R2 == 8 || R2 == 15 || R2 == 16), "the row FFT is 16 x 8, 16 x 15 or 16 x 16");
    static_assert(NT % 32 == 0 && NT == 16 * RI, "two rows per consumer warp");
    static_assert(!PAIR || WY % 2 == 0, "16-byte box rows");
    // every tensor-copy destination is 128-byte aligned: the buffers, O_OFF,
    // X_OFF and XB by rounding; the FP64 E boxes of BHT rows by this
    static_assert(PAIR || (BHT * WY * (int)sizeof(V)) % 128 == 0, "128-byte aligned E boxes");
};

// ---------------------------------------------------------------------------
// one warp, two z-rows of M = 16 R2 complex (16 lanes per row), in place in
// the natural row layout.  Step 1: lane a transforms x[a + 16 n] over n < R2
// and twiddles by w_M^(a f); its outputs go to slot 16 f + (a ^ f) (an XOR
// swizzle: the writes of step 1 and the reads of step 2 are both
// conflict-free).  Step 2: lane b < R2 transforms those of frequency b over
// a, giving X[b + R2 j], j < 16, in registers.  The twiddle table holds
// w_M^(a f) at (f - 1) 16 + a: lanes read consecutive entries.
// ---------------------------------------------------------------------------
template <bool FWD, int R2, typename V>
__device__ __forceinline__ void row_step1(V (&x)[R2], V *row, const V *rtw, int a) {
    Dft<R2, FWD, V>::run(x);
#pragma unroll
    for (int f = 1; f < R2; ++f) x[f] = c_tw<FWD>(x[f], rtw[(f - 1) * 16 + a]);
    __syncwarp();  // every lane has read its inputs before the row is overwritten
#pragma unroll
    for (int f = 0; f < R2; ++f) row[16 * f + (a ^ f)] = x[f];
    __syncwarp();
}
template <bool FWD, typename V>
__device__ __forceinline__ void row_step2(V (&y)[16], const V *row, int b) {
#pragma unroll
    for (int a = 0; a < 16; ++a) y[a] = row[16 * b + (a ^ b)];
    Dft<16, FWD, V>::run(y);
}

// ---------------------------------------------------------------------------
// the kernel
// ---------------------------------------------------------------------------
// FB bit 0: the forward's row items are also written back by bulk stores
// (the inverse's always are); the copy warp then waits for each store before
// it publishes the item.  FB bits 1 (inverse) and 2 (forward): a column
// item's results go back by tensor stores of its E boxes from the copy warp
// -- with the row-pair view (FP32) only the even rows (the odd ones start 8
// bytes off a 16-byte boundary and are stored by the consumers), with the
// single-row view (FP64) every row; it needs one more barrier per item.
template <typename T, int NY, int M, int NT, bool FWD, int VY, int NBUF, int WY_ = 16, int FB = 0>
__global__ void __launch_bounds__(NT + 32, 1)
    pass_a_queue(const PassAQParams P, const __grid_constant__ CUtensorMap tm_e, const __grid_constant__ CUtensorMap tm_o,
                 const __grid_constant__ CUtensorMap tm_x) {
    using S = QShape<T, NY, M, NT, NBUF, WY_>;
    using V = cx_t<T>;
    using ColFFT = TileFFT<T, NY, S::WY, NT, FWD, COLS, VY, GROUP>;
    using ColL = typename ColFFT::L;
    constexpr int NH = S::NH, WY = S::WY, RI = S::RI, BH = S::BH, R2 = S::R2;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // copy destinations are 128-byte aligned (smem_bytes() reserves the slack)
    unsigned char *smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
    V *unp = reinterpret_cast<V *>(smem);
    V *rtw = unp + M;
    V *sty = rtw + M;
    unsigned char *bufs = smem + S::TAB;
    uint64_t *full = reinterpret_cast<uint64_t *>(bufs + (size_t)NBUF * S::BUF);
    uint64_t *empty = full + NBUF;
    int *info = reinterpret_cast<int *>(empty + NBUF);

    for (int q = threadIdx.x; q < M; q += blockDim.x) unp[q] = reinterpret_cast<const V *>(P.unp)[q];
    for (int q = threadIdx.x; q < 16 * (R2 - 1); q += blockDim.x) rtw[q] = reinterpret_cast<const V *>(P.rtw)[q];
    for (int q = threadIdx.x; q < NY - 1; q += blockDim.x) sty[q] = reinterpret_cast<const V *>(P.sty)[q];
    if (threadIdx.x == 0) {
        for (int s = 0; s < NBUF; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        fence_mbar_init();
    }
    __syncthreads();

    V *field = reinterpret_cast<V *>(P.data);
    int *ctr = P.ctr;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int first_type = FWD ? ROW_ITEM : COL_ITEM;  // the phase that publishes
    constexpr bool CT = (FB & (FWD ? 4 : 2)) != 0;

    if (warp == NT / 32) {
        // ------------------------------ producer ------------------------------
        if (lane == 0) {
            bool err = false;
            // A first-phase item is published here, once the consumers have
            // released its buffer: their stores precede their arrival on the
            // empty barrier (block barrier, then arrive), which precedes this
            // release at GPU scope.  The release waits for those stores to
            // reach L2 -- on this otherwise idle warp, not on a consumer.
            // Items are published in claim order; `pub` is the next one.  The
            // dependency wait below keeps publishing the CTA's own finished
            // items, so it never waits on an item of its own CTA.
            // Row items leave their rows in the buffer; this warp writes the
            // span back with one bulk store, and waits for it to have read the
            // buffer before the buffer is refilled (stores_out).  A forward
            // row item is a first-phase item: its store completes, and is
            // ordered before the release, before the item is published.
            // The wait for a forward row store's completion is deferred to the
            // end of the loop iteration, so that it overlaps the next claim and
            // loads (0.369 -> 0.364 ms at 512^3; the inverse's column stores
            // were slower that way and wait at once).
            // (Publishing such items one whole item late instead measured
            // slower: 0.406 / 0.374 against 0.369 / 0.354 ms at 512^3 --
            // waiting planes wait longer.)
            int pub = 0;
            bool stores_out = false;
            // first-phase items whose store is in flight: published at the end
            // of the loop iteration (after the next item's loads are issued) or
            // before any dependency wait
            int npend = 0, pend[NBUF];
            auto release_pending = [&]() {
                if (npend == 0) return;
                bulk_wait_all();
                fence_proxy_async_global();  // the stores' writes precede the releases
                for (int q = 0; q < npend; ++q) red_release_add(&ctr[4 + (pend[q] >> 16)], 1);
                npend = 0;
            };
            auto publish = [&](int j) {
                const int code = info[j % NBUF];
                if (code < 0) return;
                const int type = (code >> 15) & 1;
                if (type == ROW_ITEM && (!FWD || (FB & 1))) {
                    const long long row0 = (long long)(code >> 16) * NY + (long long)(code & 0x7fff) * RI;
                    bulk_store(field + row0 * NH, bufs + (size_t)(j % NBUF) * S::BUF, (uint32_t)S::ROW_BYTES);
                    stores_out = true;
                    if (FWD) {
                        pend[npend++] = code;
                        return;
                    }
                } else if (type == COL_ITEM && CT && !(FWD && (code & 0x7fff) == 0)) {
                    unsigned char *src = bufs + (size_t)(j % NBUF) * S::BUF;
                    if constexpr (S::PAIR) {
                        tensor_store_2d(&tm_e, (code & 0x7fff) * WY, (code >> 16) * BH, src);
                    } else {
                        constexpr int EPC = (int)sizeof(V) / 8;
#pragma unroll
                        for (int q = 0; q < S::NBX; ++q)
                            tensor_store_2d(&tm_e, EPC * (code & 0x7fff) * WY, (code >> 16) * NY + q * S::BHT,
                                            src + (size_t)q * S::BHT * WY * sizeof(V));
                    }
                    stores_out = true;
                    if (!FWD) {  // (deferring this wait too measured slower)
                        bulk_wait_all();
                        fence_proxy_async_global();
                    }
                }
                if (type == first_type) red_release_add(&ctr[4 + (code >> 16)], 1);
            };
            // publish items < upto that are finished, without waiting
            auto try_publish = [&](int upto) {
                while (pub < upto && mbar_try_wait(&empty[pub % NBUF], (uint32_t)((pub / NBUF) & 1))) publish(pub++);
            };
            int k = 0;
            for (;; ++k) {
                const int s = k % NBUF;
                const uint32_t ph = (uint32_t)((k / NBUF) & 1);
                if (!mbar_wait(&empty[s], ph ^ 1u, P.wait_ns)) {
                    err = true;
                    info[s] = -1;
                    mbar_arrive(&full[s]);  // consumers may be waiting for this slot
                    break;
                }
                // items up to k - NBUF are finished (in order): publish them
                // before slot s is reused
                while (pub <= k - NBUF) publish(pub++);
                const int g = atomicAdd(&ctr[0], 1);
                const int it = g < P.nitems ? P.items[g] : -1;
                info[s] = it;
                if (it < 0) {
                    mbar_arrive(&full[s]);
                    // publish the items still in the ring as they finish
                    while (pub < k && !err) {
                        if (!mbar_wait(&empty[pub % NBUF], (uint32_t)((pub / NBUF) & 1), P.wait_ns))
                            err = true;
                        else
                            publish(pub++);
                    }
                    break;
                }
                const int plane = it >> 16, type = (it >> 15) & 1, sub = it & 0x7fff;
                if (type != first_type) {
                    const int *cnt = &ctr[4 + plane];
                    if (ld_acquire(cnt) < P.need) {
                        release_pending();  // never wait on this CTA's own item
                        const unsigned long long t0 = globaltimer();
                        while (ld_acquire(cnt) < P.need) {
                            try_publish(k);
                            release_pending();
                            __nanosleep(200);
                            // once any CTA has given up, the others stop waiting too
                            if ((long long)(globaltimer() - t0) > P.wait_ns || ld_acquire(&ctr[2]) != 0) {
                                err = true;  // go on: wrong results, no hang
                                atomicExch(&ctr[2], 1);  // every other wait gives up at once
                                break;
                            }
                        }
                    }
                    fence_proxy_async_global();
                }
                fence_proxy_async_shared();  // the consumers' accesses to buffer s come first
                if (stores_out) {
                    bulk_wait_read();  // a bulk store from buffer s has read it
                    stores_out = false;
                }
                unsigned char *b = bufs + (size_t)s * S::BUF;
                if (type == ROW_ITEM) {
                    mbar_arrive_expect_tx(&full[s], (uint32_t)S::ROW_BYTES);
                    bulk_load(b, field + ((long long)plane * NY + (long long)sub * RI) * NH, (uint32_t)S::ROW_BYTES,
                              &full[s]);
                } else {
                    const int c0 = sub * WY;
                    const bool xtra = !FWD && sub == 0;
                    mbar_arrive_expect_tx(&full[s], (uint32_t)(S::E_BYTES + S::O_BYTES + (xtra ? S::X_BYTES : 0)));
                    if constexpr (S::PAIR) {
                        const int y = plane * BH;
                        tensor_load_2d(b, &tm_e, c0, y, &full[s]);
                        tensor_load_2d(b + S::O_OFF, &tm_o, NH - 1 + c0, y, &full[s]);
                        if (xtra) tensor_load_2d(b + S::X_OFF, &tm_x, 2 * NH - 2, y, &full[s]);
                    } else {
                        constexpr int EPC = (int)sizeof(V) / 8;  // 8-byte elements per complex
#pragma unroll
                        for (int q = 0; q < S::NBX; ++q) {
                            const int y = plane * NY + q * S::BHT;
                            tensor_load_2d(b + (size_t)q * S::BHT * WY * sizeof(V), &tm_e, EPC * c0, y, &full[s]);
                            if (xtra)
                                tensor_load_2d(b + S::X_OFF + (size_t)q * S::XB, &tm_x, EPC * M, y,
                                               &full[s]);
                        }
                    }
                }
                release_pending();  // the stores issued this iteration, overlapped with the claim and loads
            }
            release_pending();
            bulk_wait_all();  // every row this CTA stored is in global memory before it exits
            if (err) atomicExch(&ctr[2], 1);
        }
    } else {
        // ------------------------------ consumers ------------------------------
        const int tid = threadIdx.x;
        for (int k = 0;; ++k) {
            const int s = k % NBUF;
            const uint32_t ph = (uint32_t)((k / NBUF) & 1);
            if (!mbar_wait(&full[s], ph, P.wait_ns)) {
                // a copy that never completed: flag it, give it one more time
                // limit so that no copy is left in flight at exit, and stop
                if (tid == 0) atomicExch(&ctr[2], 1);
                mbar_wait(&full[s], ph, P.wait_ns);
                break;
            }
            const int it = info[s];
            if (it < 0) break;
            const int plane = it >> 16, type = (it >> 15) & 1, sub = it & 0x7fff;
            unsigned char *b = bufs + (size_t)s * S::BUF;
            V *gplane = field + (long long)plane * NY * NH;
            if (type == ROW_ITEM) {
                // two rows per warp: lanes 0-15 row 2w, lanes 16-31 row 2w+1
                const int h = lane >> 4, a = lane & 15;
                const int r = 2 * warp + h;
                V *row = reinterpret_cast<V *>(b) + r * NH;
                V *grow = gplane + ((long long)sub * RI + r) * NH;
                V x[R2];
                if constexpr (FWD) {
#pragma unroll
                    for (int n = 0; n < R2; ++n) x[n] = row[a + 16 * n];
                    row_step1<true, R2>(x, row, rtw, a);
                    {
                        V y[16];
                        if (R2 == 16 || a < R2) row_step2<true>(y, row, a);
                        __syncwarp();  // step 2's reads are done before X is stored
                        if (R2 == 16 || a < R2) {
#pragma unroll
                            for (int j = 0; j < 16; ++j) row[a + R2 * j] = y[j];
                        }
                        if constexpr (R2 == 16) {
#pragma unroll
                            for (int j = 0; j < 16; ++j) x[j] = y[j];  // X[a + 16 j] stays in registers
                        }
                    }
                    __syncwarp();
                    // unpack: X[k] = E + O, E = (Z[k] + conj Z[M-k]) / 2,
                    // O = -i w^k (Z[k] - conj Z[M-k]) / 2 = (Z[k] - conj Z[M-k]) u_k with
                    // the table u_k = -i w^k / 2; bins 0 and M packed in slot 0
                    // (with FB every bin goes into x[] first: the row is
                    // overwritten in place after the warp's partner reads, and the
                    // copy warp writes the span back with one bulk store)
                    const T hf = (T)0.5;
#pragma unroll
                    for (int j = 0; j < R2; ++j) {
                        const int kk = a + 16 * j;
                        const V za = R2 == 16 ? x[j] : row[kk];
                        const V zb = c_conj(row[(kk == 0 ? 0 : M - kk)]);
                        const V e2 = c_add(za, zb);
                        const V o = c_mul(c_sub(za, zb), unp[kk]);
                        const V xa = V{fma(hf, e2.x, o.x), fma(hf, e2.y, o.y)};
                        const V xs = kk == 0 ? V{xa.x, fma(hf, e2.x, -o.x)} : xa;  // slot 0: (Re X0, Re XM)
                        if constexpr ((FB & 1) != 0)
                            x[j] = xs;
                        else
                            st_g(grow + kk, xs);
                    }
                    if constexpr ((FB & 1) != 0) {
                        __syncwarp();
#pragma unroll
                        for (int j = 0; j < R2; ++j) row[a + 16 * j] = x[j];
                        fence_proxy_async_shared();  // the copy warp's bulk store reads the row
                    }
                } else {
                    // pack: Z[k] = S + Pk, S = X[k] + conj X[M-k], Pk = i conj(w^k) (X[k] - conj X[M-k]);
                    // slot 0 holds (Re X0, Re XM)
#pragma unroll
                    for (int j = 0; j < R2; ++j) {
                        const int kk = a + 16 * j;
                        V xa = row[kk], xb = row[(kk == 0 ? 0 : M - kk)];
                        if (kk == 0) {
                            xb = V{xa.y, (T)0};
                            xa = V{xa.x, (T)0};
                        }
                        // (the table holds i conj(w^k))
                        const V cm = c_conj(xb);
                        x[j] = c_add(c_add(xa, cm), c_mul(c_sub(xa, cm), unp[kk]));
                    }
                    row_step1<false, R2>(x, row, rtw, a);
                    V y[16];
                    if (R2 == 16 || a < R2) row_step2<false>(y, row, a);
                    __syncwarp();  // step 2's reads are done before the real row is stored in place
                    if (R2 == 16 || a < R2) {
#pragma unroll
                        for (int j = 0; j < 16; ++j) row[a + R2 * j] = y[j];
                    }
                    if (a == 0) row[M] = V{(T)0, (T)0};  // padding cells of the real row
                    fence_proxy_async_shared();  // the copy warp's bulk store reads the row
                }
            } else {
                // column item: y FFT of columns c0 .. c0 + WY - 1 of all NY rows
                const int c0 = sub * WY;
                const V *be = reinterpret_cast<const V *>(b);
                const V *bo = reinterpret_cast<const V *>(b + S::O_OFF);
                const V *bx = reinterpret_cast<const V *>(b + S::X_OFF);
                V *tile = reinterpret_cast<V *>(b);
                auto at = [&](int n, int w) -> V {
                    if constexpr (S::PAIR) {
                        // one load path for both parities (an integer select, no
                        // branch): half-warps hold rows of opposite parity
                        const int h = n >> 1;
                        const int off = (n & 1) ? S::O_OFF / (int)sizeof(V) + h * (WY + 2) + 1 : h * WY;
                        return be[off + w];
                    } else {
                        return be[n * WY + w];
                    }
                };
                auto dst = [&](int n, int w, V v) { st_g(gplane + (long long)n * NH + c0 + w, v); };
                // CT: rows into the E boxes' place at the start of the buffer, once a
                // barrier (the hook's) has ended the last stage's reads of the tile
                V *ew = reinterpret_cast<V *>(b);
                auto dst_ct = [&](int n, int w, V v) {
                    if constexpr (S::PAIR) {
                        if (n & 1)
                            st_g(gplane + (long long)n * NH + c0 + w, v);
                        else
                            ew[(n >> 1) * WY + w] = v;
                    } else {
                        ew[n * WY + w] = v;
                    }
                };
                auto after_reads = [] {};
                // the y FFT in place in the buffer; returns where a ToSmem result lies
                auto colfft = [&](auto &src_, auto &dst_) -> V * {
                    ColFFT::run(src_, dst_, tile, sty);
                    return tile;
                };
                if constexpr (FWD) {
                    auto src = [&](int n, int w) -> V { return at(n, w); };
                    if (sub != 0) {
                        if constexpr (CT) {
                            ColFFT::run(src, dst_ct, tile, sty, after_reads);
                            fence_proxy_async_shared();  // the copy warp's tensor store reads box E
                        } else {
                            colfft(src, dst);
                        }
                    } else {
                        // column 0 carries (bin 0) + i (bin M); split after the FFT
                        ToSmem ts;
                        const V *res = colfft(src, ts);
                        group_sync<NT>();
                        const T hf = (T)0.5;
                        for (int qq = tid; qq < NY * WY; qq += NT) {
                            const int n = qq / WY, w = qq % WY;
                            const V c1 = res[ColL::idx(n, w)];
                            V *orow = gplane + (long long)n * NH;
                            if (w == 0) {
                                const V c2 = c_conj(res[ColL::idx((NY - n) % NY, 0)]);
                                st_g(orow, c_scale(c_add(c1, c2), hf));
                                st_g(orow + M, c_rot<true>(c_scale(c_sub(c1, c2), hf)));
                            } else {
                                st_g(orow + w, c1);
                            }
                        }
                    }
                } else {
                    // inverse, tile 0: the Hermitian projection of bins 0 (a) and M (b)
                    // along y, packed as a' + i b' into column 0
                    const T hf = (T)0.5;
                    auto binm = [&](int n) -> V {
                        if constexpr (S::PAIR)
                            return (n & 1) ? bx[(n >> 1) * 2 + 1] : bo[(n >> 1) * (WY + 2)];
                        else
                            return bx[(n / S::BHT) * S::XP + n % S::BHT];
                    };
                    auto src = [&](int n, int w) -> V {
                        if (sub == 0 && w == 0) {
                            const int n2 = (NY - n) % NY;
                            const V ha = c_scale(c_add(at(n, 0), c_conj(at(n2, 0))), hf);
                            const V hb = c_scale(c_add(binm(n), c_conj(binm(n2))), hf);
                            return V{ha.x - hb.y, ha.y + hb.x};
                        }
                        return at(n, w);
                    };
                    if constexpr (CT) {
                        ColFFT::run(src, dst_ct, tile, sty, after_reads);
                        fence_proxy_async_shared();  // the copy warp's tensor store reads box E
                    } else {
                        colfft(src, dst);
                    }
                }
            }
            group_sync<NT>();  // stores issued, buffer reads done
            if (tid == 0) mbar_arrive(&empty[s]);  // the copy warp publishes the item
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&ctr[1], 1) == (int)gridDim.x - 1) {
            // last CTA out: every other CTA is done with the counters
            const int nx = P.nitems / (S::NRI + S::NCI);
            for (int p = 0; p < nx; ++p) ctr[4 + p] = 0;
            atomicExch(&ctr[0], 0);
            atomicExch(&ctr[1], 0);
            __threadfence();
        }
    }
}

// ---------------------------------------------------------------------------
// Pass B (x C2C over column tiles) fed by tensor copies.
//
// Replaces the reference's strided 1D cuFFT C2C along x
// (GPU_FFT/src/initialize_GPU_FFT/GPU_FFT_init.cu:66-73,89).  A tile is the
// NX x W block of W consecutive columns c = ky*Nh + kz (W*8 = 128 bytes per
// row) of all NX rows: a 2D box of the view [NX][Ny*Nh] (row pitch Ny*Nh*8
// bytes, a multiple of 16; tile starts are 128-byte aligned), landing in the
// COLS layout the tile FFT reads.  Tiles have no dependencies: CTA b takes
// tiles b, b + grid, ...; NBUF tiles are in flight, and thread 0 issues the
// copies of tile k + NBUF as soon as the barrier after tile k's FFT has freed
// its buffer (no copy-issuing warp, so every warp's registers go to the FFT).
// NBUF = 1 (tiles too large for two buffers: Nx = 1024) refills the one
// buffer as soon as the last FFT stage has read it (TileFFT::run's hook),
// so the next tile streams in while that stage computes and stores.
// VARIANT 3 runs the radix-16 stages but the last on tcgen05 (fft_tc5.cuh):
// the CTA holds the whole tensor memory; if a wait for the MMAs runs out
// (2 s), the CTA stops, waits for its copies still in flight (bounded),
// frees the tensor memory and raises P.err.
// ---------------------------------------------------------------------------
template <typename T, int NX, int NT, int NBUF, int WW = 0>
struct BShape {
    using V = cx_t<T>;
    static constexpr int W = WW > 0 ? WW : 128 / (int)sizeof(V);  // columns per tile (128-byte rows by default)
    static constexpr int BOXH = box_rows(NX);         // rows per tensor copy
    static constexpr int NBOX = (NX + BOXH - 1) / BOXH;
    static constexpr int TILE_BYTES = NX * W * (int)sizeof(V);
    static constexpr int BUF = (TILE_BYTES + 127) / 128 * 128;
    static constexpr int TAB = ((NX * (int)sizeof(V)) + 127) / 128 * 128;
    static constexpr size_t smem_bytes() { return (size_t)TAB + (size_t)NBUF * BUF + NBUF * 8 + 128; }
    static constexpr int EPC = (int)sizeof(V) / 8;   // 8-byte elements per complex
    static_assert(NX % BOXH == 0, "whole boxes");
    static_assert((BOXH * W * (int)sizeof(V)) % 128 == 0, "128-byte aligned box destinations");
};

template <typename T, int NX, int NT, bool FWD, int VARIANT, int NBUF, bool EPI, int WW = 0>
__global__ void __launch_bounds__(NT, 1) pass_b_tma(const PassBParams P, const __grid_constant__ CUtensorMap tm) {
    using S = BShape<T, NX, NT, NBUF, WW>;
    using V = cx_t<T>;
    using FFT = TileFFT<T, NX, S::W, NT, FWD, COLS, VARIANT, fast::BLOCK>;
    static_assert(!FFT::kTcStage, "the tensor-core stage uses its own swizzled layout");
    constexpr int W = S::W;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char *smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
    V *tw = reinterpret_cast<V *>(smem);
    unsigned char *bufs = smem + S::TAB;
    uint64_t *full = reinterpret_cast<uint64_t *>(bufs + (size_t)NBUF * S::BUF);
    for (int q = threadIdx.x; q < NX - 1; q += NT) tw[q] = reinterpret_cast<const V *>(P.stw)[q];
    constexpr bool TC5 = FFT::kTc5Stage;
    if constexpr (TC5) tc5::setup<FWD>();
    auto issue = [&](long long t, int s) {
        unsigned char *b = bufs + (size_t)s * S::BUF;
        mbar_arrive_expect_tx(&full[s], (uint32_t)S::TILE_BYTES);
#pragma unroll
        for (int bx = 0; bx < S::NBOX; ++bx)
            tensor_load_2d(b + (size_t)bx * S::BOXH * W * sizeof(V), &tm, (int)(t * W * S::EPC), bx * S::BOXH, &full[s]);
    };
    if (threadIdx.x == 0) {
        for (int s = 0; s < NBUF; ++s) mbar_init(&full[s], 1);
        fence_mbar_init();
        for (int s = 0; s < NBUF; ++s) {
            const long long t = blockIdx.x + (long long)s * gridDim.x;
            if (t < P.ntiles) issue(t, s);
        }
    }
    __syncthreads();
    const long long ncols = P.ncols;
    V *base = reinterpret_cast<V *>(P.data);
    int k = 0;
    for (long long t = blockIdx.x; t < P.ntiles; t += gridDim.x, ++k) {
        const int s = k % NBUF;
        const uint32_t ph = (uint32_t)((k / NBUF) & 1);
        if (!mbar_wait(&full[s], ph, 2000000000LL)) {
            mbar_wait(&full[s], ph, 2000000000LL);  // nothing is left in flight at exit
            break;
        }
        V *tile = reinterpret_cast<V *>(bufs + (size_t)s * S::BUF);
        const long long c0 = t * W;
        const int wv = (int)min((long long)W, ncols - c0);
        V *g = base + c0;
        auto dst = [&](int n, int w, V v) {
            if (w < wv) {
                if constexpr (EPI)
                    st_g(g + (long long)n * ncols + w, pass_b_epilogue(P, v, n, c0 + w));
                else
                    st_g(g + (long long)n * ncols + w, v);
            }
        };
        FromSmem fs;
        const long long tn = t + (long long)NBUF * gridDim.x;
        if constexpr (NBUF == 1) {
            static_assert(FFT::NS >= 2, "the first stage must read the tile from shared memory");
            auto refill = [&]() {  // (called by every thread after the last stage's reads and a barrier)
                if (threadIdx.x == 0 && tn < P.ntiles) {
                    fence_proxy_async_shared();
                    issue(tn, s);
                }
            };
            FFT::run(fs, dst, tile, tw, refill);
            if constexpr (TC5) __syncthreads();
        } else {
            FFT::run(fs, dst, tile, tw);
            __syncthreads();  // every read of the tile is done: refill its buffer
            if (threadIdx.x == 0 && tn < P.ntiles) {
                fence_proxy_async_shared();
                issue(tn, s);
            }
        }
        if constexpr (TC5) {
            if (tc5::state().err) {
                // copies of the next NBUF tiles may be in flight: wait for them
                if (threadIdx.x == 0) {
                    for (int e = 1; e <= NBUF; ++e) {
                        if (t + (long long)e * gridDim.x >= P.ntiles) break;
                        const int k2 = k + e;
                        mbar_wait(&full[k2 % NBUF], (uint32_t)((k2 / NBUF) & 1), 2000000000LL);
                    }
                    if (P.err) atomicExch(P.err, 1);
                }
                break;
            }
        }
    }
    if constexpr (TC5) tc5::teardown();
}

}  // namespace q
}  // namespace gpufft

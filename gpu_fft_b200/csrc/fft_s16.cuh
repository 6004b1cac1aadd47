// fft_s16.cuh — the precision form: fields stored in BF16 or FP16 with one
// FP32 scale per pencil, butterflies in FP32 registers.
//
// Storage (in place, half the bytes of the FP32 form):
//   real space  [Nx][Ny][2*Nh] 16-bit reals, scale per z-row      rs[x*Ny + y]
//   spectrum    [Nx][Ny][Nh]   16-bit complex, scale per x-pencil ks[ky*Nh + kz]
// A stored pencil holds value/scale with scale = max(|re|, |im|) over the
// pencil (so every stored magnitude is <= 1, which keeps FP16 in range at any
// grid size; an all-zero pencil has scale 0).  Between the passes the data is
// stored the same way with plan-owned FP32 scale arrays: after Pass A (fwd)
// one scale per y-pencil ms[x*Nh + kz]; after Pass B (inv) one per x-pencil
// ms2[ky*Nh + kz].  Inside Pass A the z rows are exchanged through L2 in
// 16-bit with a per-row scale (written over rs).  A forward transform rounds
// to 16 bits three times (row exchange, after Pass A, after Pass B); so does
// the inverse.
//
// The kernels are the compile-time specialised passes of fft_fast.cuh with
// 16-bit sources and sinks: a load converts to FP32 and multiplies by its
// pencil's scale; the last FFT stage writes the shared tile, the per-column
// (or per-row) max is reduced, then the scaled values and the scale are stored.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "fft_fast.cuh"

namespace gpufft {
namespace s16 {

using fast::COLS;
using fast::FromSmem;
using fast::ROWS;
using fast::TileFFT;
using fast::TileLayout;
using fast::ToSmem;
using fast::WARP;
using fast::BLOCK;
using fast::cp_async16;
using fast::cp_async_commit;
using fast::cp_async_wait;

// storage formats: 0 = bf16, 1 = fp16; a complex (or a pair of reals) is 32 bits
template <int FMT> struct Fmt;
template <> struct Fmt<0> {
    static __device__ __forceinline__ float2 load(const uint32_t *p) {
        const uint32_t u = __ldcg(p);
        __nv_bfloat162 h;
        memcpy(&h, &u, 4);
        return __bfloat1622float2(h);
    }
    static __device__ __forceinline__ void store(uint32_t *p, float2 v) {
        const __nv_bfloat162 h = __float22bfloat162_rn(v);
        uint32_t u;
        memcpy(&u, &h, 4);
        __stcg(p, u);
    }
};
template <> struct Fmt<1> {
    static __device__ __forceinline__ float2 load(const uint32_t *p) {
        const uint32_t u = __ldcg(p);
        __half2 h;
        memcpy(&h, &u, 4);
        return __half22float2(h);
    }
    static __device__ __forceinline__ void store(uint32_t *p, float2 v) {
        const __half2 h = __float22half2_rn(v);
        uint32_t u;
        memcpy(&u, &h, 4);
        __stcg(p, u);
    }
};

__device__ __forceinline__ float amax(float2 v) { return fmaxf(fabsf(v.x), fabsf(v.y)); }
__device__ __forceinline__ float inv_of(float s) { return s > 0.f ? 1.f / s : 0.f; }
__device__ __forceinline__ float2 mulf(float2 v, float s) { return make_float2(v.x * s, v.y * s); }
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

struct PassA16Params {
    uint32_t *data;       // 16-bit field (32 bits per complex)
    float *rs;            // per z-row scales (user buffer)
    float *ms;            // per y-pencil scales [Nx][Nh] (plan scratch)
    const float *ms2;     // per x-pencil scales [Ny][Nh] after Pass B inverse (plan scratch)
    const float2 *twz;    // exp(-2 pi i e / Nz)
    const float2 *stz;    // stage tables of the z half length and of Ny
    const float2 *sty;
    int nx;
    int K;
};

struct PassB16Params {
    uint32_t *data;
    float *ks;            // per x-pencil scales of the spectrum (user buffer)
    float *ms;            // per y-pencil scales [Nx][Nh] (Pass A fwd output / Pass B fwd input)
    float *ms2;           // per x-pencil scales [Ny][Nh] (Pass B inv output)
    const float2 *stw;
    long long ncols;      // Ny*Nh
    int nh;
    long long ntiles;
};

// per-column max of a COLS tile [N][W] into cmax[W] (shared), block-wide
template <int N, int W, int NT>
__device__ __forceinline__ void col_max(const float2 *tile, unsigned *cmax) {
    using L = TileLayout<float, N, W, COLS>;
    for (int q = threadIdx.x; q < W; q += NT) cmax[q] = 0u;
    __syncthreads();
    constexpr int ROWS_PER = NT / W > 0 ? NT / W : 1;
    const int w = threadIdx.x % W, r0 = threadIdx.x / W;
    if (threadIdx.x < ROWS_PER * W) {
        float m = 0.f;
        for (int n = r0; n < N; n += ROWS_PER) m = fmaxf(m, amax(tile[L::idx(n, w)]));
        atomicMax(&cmax[w], __float_as_uint(m));  // non-negative floats order as their bits
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Pass B (x axis), 16-bit storage
// ---------------------------------------------------------------------------
template <int FMT, int NX, int W, int NT, bool FWD, int VARIANT, int MINB>
__global__ void __launch_bounds__(NT, MINB) pass_b_s16(PassB16Params P) {
    using V = float2;
    using F = Fmt<FMT>;
    using FFT = TileFFT<float, NX, W, NT, FWD, COLS, VARIANT, BLOCK>;
    using L = typename FFT::L;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tw = reinterpret_cast<V *>(smem_raw);
    V *tile = tw + NX;
    float *tscale = reinterpret_cast<float *>(tile + NX * W);  // forward: the tile's input scales
    __shared__ unsigned cmax[W];
    for (int q = threadIdx.x; q < NX - 1; q += NT) tw[q] = P.stw[q];
    const long long ncols = P.ncols;
    const int nh = P.nh;
    for (long long t = blockIdx.x; t < P.ntiles; t += gridDim.x) {
        const long long c0 = t * W;
        const int wv = (int)min((long long)W, ncols - c0);
        uint32_t *g = P.data + c0;
        const int kz0 = (int)(c0 % nh);
        if (FWD) {
            // The forward input has one scale per (x, kz): gather the tile's
            // NX x W scales into shared memory first, in one batch of loads.
            // (Loaded inside the first FFT stage beside each value, they left
            // the pass waiting on one load after another: 2.6x slower at 512^3.)
            __syncthreads();  // the previous tile's readers of tscale are done
            for (int q = threadIdx.x; q < NX * W; q += NT) {
                const int n = q / W, w = q % W;
                int kz = kz0 + w;
                if (kz >= nh) kz %= nh;
                tscale[q] = w < wv ? __ldg(&P.ms[(long long)n * nh + kz]) : 0.f;
            }
            __syncthreads();
        }
        auto src = [&](int n, int w) -> V {
            if (w >= wv) return V{0.f, 0.f};
            // forward input: y-pencil scale of (x = n, kz); inverse input: x-pencil scale of column c0+w
            float sc;
            if (FWD) {
                sc = tscale[n * W + w];
            } else {
                sc = __ldg(&P.ks[c0 + w]);
            }
            return mulf(F::load(g + (long long)n * ncols + w), sc);
        };
        ToSmem ts;
        FFT::run(src, ts, tile, tw);
        __syncthreads();
        col_max<NX, W, NT>(tile, cmax);
        float *oscale = FWD ? P.ks : P.ms2;
        for (int q = threadIdx.x; q < wv; q += NT) oscale[c0 + q] = __uint_as_float(cmax[q]);
        for (int q = threadIdx.x; q < NX * W; q += NT) {
            const int n = q / W, w = q % W;
            if (w < wv) F::store(g + (long long)n * ncols + w, mulf(tile[L::idx(n, w)], inv_of(__uint_as_float(cmax[w]))));
        }
    }
}

// ---------------------------------------------------------------------------
// Pass B, 16-bit storage, tiles double-buffered by cp.async.  While a tile is
// transformed, the next one's 16-bit values (and, forward, its per-(x, kz)
// input scales) stream into the other buffers.  The last FFT stage keeps its
// values in registers: each thread's values all belong to one column, so the
// column max is a register max, one shuffle and a shared-memory atomic, and
// the scaled 16-bit values are stored straight from registers — no extra
// passes over the tile.  Requires NT % W == 0, rows of the 16-bit field
// 16-byte aligned (Ny*Nh a multiple of 4) and W a multiple of 4.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}

template <int NX, int W>
struct PassB16PipeShape {
    // stage tables | 2 x 16-bit tiles | 2 x input scales (forward) | FP32 tile
    static constexpr size_t raw_bytes = (size_t)NX * W * 4;
    static constexpr size_t smem_bytes() {
        return (size_t)NX * 8 + 2 * raw_bytes + 2 * (size_t)NX * W * 4 + (size_t)NX * W * 8;
    }
};

template <int FMT, int NX, int W, int NT, bool FWD, int VARIANT, int MINB>
__global__ void __launch_bounds__(NT, MINB) pass_b_s16_pipe(PassB16Params P) {
    using V = float2;
    using F = Fmt<FMT>;
    using FFT = TileFFT<float, NX, W, NT, FWD, COLS, VARIANT, BLOCK>;
    static_assert(NT % W == 0 && W % 4 == 0, "a thread's values share one column; 16-byte row chunks");
    static_assert(((NX / FFT::F.r[FFT::NS - 1]) * W) % NT == 0, "every thread holds the same number of outputs");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tw = reinterpret_cast<V *>(smem_raw);
    uint32_t *raw0 = reinterpret_cast<uint32_t *>(tw + NX);
    uint32_t *raw1 = raw0 + NX * W;
    float *sc0 = reinterpret_cast<float *>(raw1 + NX * W);
    float *sc1 = sc0 + NX * W;
    V *tile = reinterpret_cast<V *>(sc1 + NX * W);
    __shared__ unsigned cmax[W];
    __shared__ float colsc[W];
    for (int q = threadIdx.x; q < NX - 1; q += NT) tw[q] = P.stw[q];
    const long long ncols = P.ncols;
    const int nh = P.nh;
    const int w_me = (int)threadIdx.x % W;  // the column of every value this thread holds
    auto prefetch = [&](long long t, uint32_t *raw, float *sc) {
        const long long c0 = t * W;
        const int wv = (int)min((long long)W, ncols - c0);
        for (int q = threadIdx.x; q < NX * (W / 4); q += NT) {
            const int n = q / (W / 4), ch = q % (W / 4);
            const int valid = max(0, min(4, wv - ch * 4));
            const uint32_t *src = P.data + (long long)n * ncols + c0 + (valid > 0 ? ch * 4 : 0);
            cp_async16(raw + n * W + ch * 4, src, valid * 4);
        }
        if (FWD) {
            const int kz0 = (int)(c0 % nh);
            for (int q = threadIdx.x; q < NX * W; q += NT) {
                const int n = q / W, w = q % W;
                if (w < wv) {
                    int kz = kz0 + w;
                    if (kz >= nh) kz %= nh;
                    cp_async4(sc + q, P.ms + (long long)n * nh + kz);
                }
            }
        }
        cp_async_commit();
    };
    long long t = blockIdx.x;
    if (t < P.ntiles) prefetch(t, raw0, sc0);
    int k = 0;
    for (; t < P.ntiles; t += gridDim.x, k ^= 1) {
        uint32_t *raw = k ? raw1 : raw0;
        float *sc = k ? sc1 : sc0;
        const long long tn = t + gridDim.x;
        if (tn < P.ntiles) {
            prefetch(tn, k ? raw0 : raw1, k ? sc0 : sc1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        const long long c0 = t * W;
        const int wv = (int)min((long long)W, ncols - c0);
        if (threadIdx.x < W) {
            cmax[threadIdx.x] = 0u;
            if (!FWD) colsc[threadIdx.x] = (int)threadIdx.x < wv ? __ldg(&P.ks[c0 + threadIdx.x]) : 0.f;
        }
        __syncthreads();  // the tile's copies (every thread's), cmax and colsc are in place
        auto src = [&](int n, int w) -> V {
            if (w >= wv) return V{0.f, 0.f};
            const int q = n * W + w;
            uint32_t u = raw[q];
            float2 v;
            if constexpr (FMT == 0) {
                __nv_bfloat162 h;
                memcpy(&h, &u, 4);
                v = __bfloat1622float2(h);
            } else {
                __half2 h;
                memcpy(&h, &u, 4);
                v = __half22float2(h);
            }
            return mulf(v, FWD ? sc[q] : colsc[w]);
        };
        // the last stage's values go to registers, in call order
        constexpr int NOUT = NX * W / NT;
        V out[NOUT];
        int orow[NOUT];
        int slot = 0;
        auto dst = [&](int n, int w, V v) {
            out[slot] = v;
            orow[slot] = n;
            ++slot;
        };
        FFT::run(src, dst, tile, tw);
        float m = 0.f;
#pragma unroll
        for (int i = 0; i < NOUT; ++i) m = fmaxf(m, amax(out[i]));
        // lanes w, w+W, w+2W, ... of a warp hold the same column
#pragma unroll
        for (int o = W; o < 32; o <<= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) < W) atomicMax(&cmax[w_me], __float_as_uint(m));
        __syncthreads();
        const float cm = __uint_as_float(cmax[w_me]);
        const float inv = inv_of(cm);
        if (w_me < wv) {
            uint32_t *g = P.data + c0 + w_me;
#pragma unroll
            for (int i = 0; i < NOUT; ++i) F::store(g + (long long)orow[i] * ncols, mulf(out[i], inv));
            if ((int)threadIdx.x < W) (FWD ? P.ks : P.ms2)[c0 + w_me] = cm;
        }
        __syncthreads();  // buffers, cmax and colsc are free for the next tile
    }
}

// ---------------------------------------------------------------------------
// Pass A (z and y), 16-bit storage; plane exchanged through L2 in a cluster
// ---------------------------------------------------------------------------
template <int NY, int M, int RW, int WY, int NT>
struct PassA16Shape {
    using RowL = TileLayout<float, M, RW, ROWS>;
    using ColL = TileLayout<float, NY, WY, COLS>;
    static constexpr int NWARP = NT / 32;
    static constexpr int ROWS_ELEMS = NWARP * RowL::ELEMS;
    static constexpr int TILE = ROWS_ELEMS > ColL::ELEMS ? ROWS_ELEMS : ColL::ELEMS;
    static constexpr int UNP = M / 2 + 1;
    // unpack roots, z and y stage tables, tile, extra column (bin m), plane row scales
    static constexpr size_t smem_bytes() { return (size_t)(UNP + M + NY + TILE + NY) * 8 + (size_t)NY * 4; }
};

template <int FMT, int NY, int M, int RW, int WY, int NT, bool FWD, int VY, int VZ, int MINB>
__global__ void __launch_bounds__(NT, MINB) pass_a_s16(PassA16Params P) {
    using V = float2;
    using F = Fmt<FMT>;
    using Shape = PassA16Shape<NY, M, RW, WY, NT>;
    using RowFFT = TileFFT<float, M, RW, 32, FWD, ROWS, VZ, WARP>;
    using ColFFT = TileFFT<float, NY, WY, NT, FWD, COLS, VY, BLOCK>;
    using RowL = typename RowFFT::L;
    using ColL = typename ColFFT::L;
    constexpr int NH = M + 1;
    constexpr int UNP = Shape::UNP;
    constexpr int HALF = M / 2 + 1;
    constexpr int PER_LANE = (HALF + 31) / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *unp = reinterpret_cast<V *>(smem_raw);
    V *stz = unp + UNP;
    V *sty = stz + M;
    V *tile = sty + NY;
    V *extra = tile + Shape::TILE;                       // bin m of tile 0 (forward split / inverse projection)
    float *rowsc = reinterpret_cast<float *>(extra + NY);  // this plane's row scales
    __shared__ unsigned cmax[WY + 1];
    for (int q = threadIdx.x; q < UNP; q += NT) unp[q] = P.twz[q];
    for (int q = threadIdx.x; q < M - 1; q += NT) stz[q] = P.stz[q];
    for (int q = threadIdx.x; q < NY - 1; q += NT) sty[q] = P.sty[q];
    __syncthreads();

    const int K = P.K;
    const int crank = blockIdx.x % K;
    const int cid = blockIdx.x / K;
    const int ncl = gridDim.x / K;
    const int rows_per = (NY + K - 1) / K;
    const int rb = min(NY, crank * rows_per), re = min(NY, rb + rows_per);
    constexpr int ntiles_y = (M + WY - 1) / WY;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    V *wtile = tile + wid * RowL::ELEMS;

    for (int plane = cid; plane < P.nx; plane += ncl) {
        uint32_t *g = P.data + (long long)plane * NY * NH;
        float *rsp = P.rs + (long long)plane * NY;     // row scales of this plane
        float *msp = P.ms + (long long)plane * NH;     // y-pencil scales of this plane
        if (FWD) {
            // ---- z rows: 16-bit rows (scale rs) -> R2C -> unpack -> 16-bit rows (new scale rs)
            for (int r0 = rb + wid * RW; r0 < re; r0 += (NT / 32) * RW) {
                const int wv = min(RW, re - r0);
                uint32_t *gr = g + (long long)r0 * NH;
                float sc_in[RW];
#pragma unroll
                for (int w = 0; w < RW; ++w) sc_in[w] = (w < wv) ? rsp[r0 + w] : 0.f;
                auto src = [&](int n, int w) -> V {
                    float sc = 0.f;
#pragma unroll
                    for (int u = 0; u < RW; ++u)
                        if (u == w) sc = sc_in[u];
                    return (w < wv) ? mulf(F::load(gr + (long long)w * NH + n), sc) : V{0.f, 0.f};
                };
                ToSmem ts;
                RowFFT::run(src, ts, wtile, stz);
                __syncwarp();
                for (int w = 0; w < wv; ++w) {
                    V xa[PER_LANE], xb[PER_LANE];
                    float m = 0.f;
#pragma unroll
                    for (int u = 0; u < PER_LANE; ++u) {
                        const int k = lane + 32 * u;
                        xa[u] = xb[u] = V{0.f, 0.f};
                        if (k < HALF) {
                            const V a = wtile[RowL::idx(k, w)];
                            const V b = c_conj(wtile[RowL::idx(k == 0 ? 0 : M - k, w)]);
                            const V e = c_scale(c_add(a, b), 0.5f);
                            const V d = c_scale(c_sub(a, b), 0.5f);
                            const V o = c_rot<true>(c_mul(d, unp[k]));
                            xa[u] = c_add(e, o);
                            xb[u] = c_conj(c_sub(e, o));
                            if (k == 0) xa[u] = V{xa[u].x, xb[u].x};  // packed (X0, Xm)
                            m = fmaxf(m, fmaxf(amax(xa[u]), k == 0 ? 0.f : amax(xb[u])));
                        }
                    }
                    m = warp_max(m);
                    const float inv = inv_of(m);
                    uint32_t *row = gr + (long long)w * NH;
#pragma unroll
                    for (int u = 0; u < PER_LANE; ++u) {
                        const int k = lane + 32 * u;
                        if (k < HALF) {
                            F::store(row + k, mulf(xa[u], inv));
                            if (k != 0 && M - k != k) F::store(row + M - k, mulf(xb[u], inv));
                        }
                    }
                    if (lane == 0) rsp[r0 + w] = m;
                }
            }
            __syncthreads();
            if (K > 1) {
                fast::cluster_arrive();
                fast::cluster_wait();
            }
            // ---- y columns: 16-bit rows (scale rs) -> y FFT -> 16-bit, scale per y-pencil ms
            for (int q = threadIdx.x; q < NY; q += NT) rowsc[q] = __ldcg(&rsp[q]);
            __syncthreads();
            for (int t = crank; t < ntiles_y; t += K) {
                const int c0 = t * WY;
                const int wv = min(WY, M - c0);
                uint32_t *gc = g + c0;
                auto src = [&](int n, int w) -> V {
                    return (w < wv) ? mulf(F::load(gc + (long long)n * NH + w), rowsc[n]) : V{0.f, 0.f};
                };
                ToSmem ts;
                ColFFT::run(src, ts, tile, sty);
                __syncthreads();
                if (c0 == 0) {
                    // column 0 carried (bin 0) + i (bin m): split into column 0 and `extra`
                    for (int n = threadIdx.x; n <= NY / 2; n += NT) {
                        const int n2 = (NY - n) % NY;
                        const V c1 = tile[ColL::idx(n, 0)], c1b = tile[ColL::idx(n2, 0)];
                        const V A1 = c_scale(c_add(c1, c_conj(c1b)), 0.5f);
                        const V B1 = c_rot<true>(c_scale(c_sub(c1, c_conj(c1b)), 0.5f));
                        const V A2 = c_conj(A1), B2 = c_conj(B1);  // the -ky partners
                        tile[ColL::idx(n, 0)] = A1;
                        extra[n] = B1;
                        if (n2 != n) {
                            tile[ColL::idx(n2, 0)] = A2;
                            extra[n2] = B2;
                        }
                    }
                    __syncthreads();
                }
                col_max<NY, WY, NT>(tile, cmax);
                if (c0 == 0) {
                    // max of the extra column (bin m)
                    if (threadIdx.x == 0) cmax[WY] = 0u;
                    __syncthreads();
                    float m = 0.f;
                    for (int n = threadIdx.x; n < NY; n += NT) m = fmaxf(m, amax(extra[n]));
                    m = warp_max(m);
                    if (lane == 0) atomicMax(&cmax[WY], __float_as_uint(m));
                    __syncthreads();
                    const float sm = __uint_as_float(cmax[WY]);
                    if (threadIdx.x == 0) msp[M] = sm;
                    const float inv = inv_of(sm);
                    for (int n = threadIdx.x; n < NY; n += NT) F::store(g + (long long)n * NH + M, mulf(extra[n], inv));
                }
                for (int q = threadIdx.x; q < wv; q += NT) msp[c0 + q] = __uint_as_float(cmax[q]);
                for (int q = threadIdx.x; q < NY * WY; q += NT) {
                    const int n = q / WY, w = q % WY;
                    if (w < wv) F::store(gc + (long long)n * NH + w, mulf(tile[ColL::idx(n, w)], inv_of(__uint_as_float(cmax[w]))));
                }
                __syncthreads();
            }
        } else {
            // ---- y columns (inverse): 16-bit, x-pencil scales ms2 -> y inverse -> 16-bit, y-pencil scales ms
            for (int t = crank; t < ntiles_y; t += K) {
                const int c0 = t * WY;
                const int wv = min(WY, M - c0);
                uint32_t *gc = g + c0;
                if (c0 == 0) {
                    // tile 0 through shared memory: Hermitian projection of bins 0 and m
                    __syncthreads();
                    for (int q = threadIdx.x; q < NY * WY; q += NT) {
                        const int n = q / WY, w = q % WY;
                        tile[ColL::idx(n, w)] =
                            (w < wv) ? mulf(F::load(gc + (long long)n * NH + w), __ldg(&P.ms2[(long long)n * NH + c0 + w]))
                                     : V{0.f, 0.f};
                    }
                    for (int n = threadIdx.x; n < NY; n += NT)
                        extra[n] = mulf(F::load(g + (long long)n * NH + M), __ldg(&P.ms2[(long long)n * NH + M]));
                    __syncthreads();
                    for (int n = threadIdx.x; n <= NY / 2; n += NT) {
                        const int n2 = (NY - n) % NY;
                        const V a1 = tile[ColL::idx(n, 0)], a2 = tile[ColL::idx(n2, 0)];
                        const V b1 = extra[n], b2 = extra[n2];
                        const V ha = c_scale(c_add(a1, c_conj(a2)), 0.5f);
                        const V hb = c_scale(c_add(b1, c_conj(b2)), 0.5f);
                        tile[ColL::idx(n, 0)] = V{ha.x - hb.y, ha.y + hb.x};
                        if (n2 != n) tile[ColL::idx(n2, 0)] = V{ha.x + hb.y, -ha.y + hb.x};
                    }
                    FromSmem fs;
                    ToSmem ts;
                    ColFFT::run(fs, ts, tile, sty);
                } else {
                    auto src = [&](int n, int w) -> V {
                        return (w < wv) ? mulf(F::load(gc + (long long)n * NH + w), __ldg(&P.ms2[(long long)n * NH + c0 + w]))
                                        : V{0.f, 0.f};
                    };
                    ToSmem ts;
                    ColFFT::run(src, ts, tile, sty);
                }
                __syncthreads();
                col_max<NY, WY, NT>(tile, cmax);
                for (int q = threadIdx.x; q < wv; q += NT) msp[c0 + q] = __uint_as_float(cmax[q]);
                for (int q = threadIdx.x; q < NY * WY; q += NT) {
                    const int n = q / WY, w = q % WY;
                    if (w < wv) F::store(gc + (long long)n * NH + w, mulf(tile[ColL::idx(n, w)], inv_of(__uint_as_float(cmax[w]))));
                }
                __syncthreads();
            }
            __syncthreads();
            if (K > 1) {
                fast::cluster_arrive();
                fast::cluster_wait();
            }
            // ---- z rows (inverse): 16-bit rows (y-pencil scales ms) -> C2R -> 16-bit real rows (scale rs)
            for (int r0 = rb + wid * RW; r0 < re; r0 += (NT / 32) * RW) {
                const int wv = min(RW, re - r0);
                uint32_t *gr = g + (long long)r0 * NH;
                __syncwarp();
                for (int w = 0; w < RW; ++w) {
                    const uint32_t *row = gr + (long long)w * NH;
                    for (int k = lane; k < HALF; k += 32) {
                        V za = V{0.f, 0.f}, zb = V{0.f, 0.f};
                        if (w < wv) {
                            V xk, xmk;
                            if (k == 0) {
                                const V pk = mulf(F::load(row), __ldcg(&msp[0]));
                                xk = V{pk.x, 0.f};
                                xmk = V{pk.y, 0.f};
                            } else {
                                xk = mulf(F::load(row + k), __ldcg(&msp[k]));
                                xmk = mulf(F::load(row + M - k), __ldcg(&msp[M - k]));
                            }
                            const V cm = c_conj(xmk);
                            const V s = c_add(xk, cm);
                            const V pk = c_rot<false>(c_mulc(c_sub(xk, cm), unp[k]));
                            za = c_add(s, pk);
                            zb = c_conj(c_sub(s, pk));
                        }
                        wtile[RowL::idx(k, w)] = za;
                        if (k != 0 && M - k != k) wtile[RowL::idx(M - k, w)] = zb;
                    }
                }
                FromSmem fs;
                ToSmem ts;
                RowFFT::run(fs, ts, wtile, stz);
                __syncwarp();
                for (int w = 0; w < wv; ++w) {
                    float m = 0.f;
                    for (int n = lane; n < M; n += 32) m = fmaxf(m, amax(wtile[RowL::idx(n, w)]));
                    m = warp_max(m);
                    const float inv = inv_of(m);
                    uint32_t *row = gr + (long long)w * NH;
                    for (int n = lane; n < M; n += 32) F::store(row + n, mulf(wtile[RowL::idx(n, w)], inv));
                    if (lane == 0) {
                        F::store(row + M, V{0.f, 0.f});  // padding cells of the real row
                        rsp[r0 + w] = m;
                    }
                }
            }
        }
        __syncthreads();
    }
}

}  // namespace s16
}  // namespace gpufft

// fft_fast.cuh — compile-time specialised passes for the common axis lengths.
//
// Same algorithm, layout and packing as fft_kernels.cuh (read that file's
// header first); what changes is how each 1D FFT of a tile runs:
//  * the length, its radix list, the tile width and the thread count are
//    template parameters, so every index, stride and twiddle position is a
//    compile-time expression except the thread's own (butterfly, column);
//  * a stage keeps its butterflies in registers (load all, barrier, store
//    all), so the tile is transformed in place in one shared buffer;
//  * the first stage reads global memory directly and the last stage writes
//    global memory directly (the Stockham input and output positions of the
//    first and last stage are both i + j*N/R, which keeps those accesses
//    coalesced), so a 3-stage FFT touches shared memory 4 times per element
//    instead of 8.
#pragma once
#include <cooperative_groups.h>
#include <cuda_bf16.h>

#include <type_traits>

#include "fft_kernels.cuh"
#include "fft_radix.cuh"
#include "fft_tc5.cuh"

namespace gpufft {
namespace fast {

// ---------------------------------------------------------------------------
// compile-time radix lists (same rule as the host factorize(): the power of
// two split into balanced stages of at most 16, then pairs of 3s as radix 9,
// then odd primes 3..13).
// VARIANT 1 prefers radix-16 stages for the power-of-two part; VARIANT 2 has
// the same radix list and runs the radix-16 stages of FP32 column tiles on
// the tensor cores (split BF16, TileFFT::stage_tc16).
// ---------------------------------------------------------------------------
struct Fac {
    int n;
    int r[16];
};

__host__ __device__ constexpr Fac factor(int N, int variant) {
    Fac f{0, {0}};
    int a = 0, m = N;
    while (m % 2 == 0) {
        m /= 2;
        ++a;
    }
    if (a > 0) {
        if (variant >= 1) {
            int left = a;
            while (left >= 4) {
                f.r[f.n++] = 16;
                left -= 4;
            }
            if (left > 0) f.r[f.n++] = 1 << left;
        } else {
            const int k = (a + 3) / 4;
            for (int s = 0; s < k; ++s) f.r[f.n++] = 1 << (a / k + (s < a % k ? 1 : 0));
        }
    }
    // pairs of 3s as radix-9 stages (3x3 in registers): fewer passes over the tile
    while (m % 9 == 0) {
        f.r[f.n++] = 9;
        m /= 9;
    }
    const int primes[5] = {3, 5, 7, 11, 13};
    for (int pi = 0; pi < 5; ++pi)
        while (m % primes[pi] == 0) {
            f.r[f.n++] = primes[pi];
            m /= primes[pi];
        }
    if (m != 1) f.n = -1;
    return f;
}

__host__ __device__ constexpr int fac_prod(const Fac &f, int upto) {
    int p = 1;
    for (int s = 0; s < upto; ++s) p *= f.r[s];
    return p;
}

// Per-stage twiddle tables.  Stage s (radix R, sub-length p) uses
// w_{pR}^{j*k} for j = 1..R-1, k = 0..p-1, stored at stage_offset(s) +
// (j-1)*p + k: threads that hold consecutive k read consecutive entries
// (conflict-free), and the stages together take sum (R_s - 1) p_s = N - 1
// entries.  The host computes them in FP64 and rounds once.
__host__ __device__ constexpr int stage_offset(const Fac &f, int s) {
    int off = 0, p = 1;
    for (int t = 0; t < s; ++t) {
        off += (f.r[t] - 1) * p;
        p *= f.r[t];
    }
    return off;
}

// which threads cooperate on a tile: the whole CTA, one warp, or the first
// NT threads of the CTA (GROUP: named barrier 1, so a CTA can run other warps
// -- a copy-issuing warp -- beside the ones that transform the tile)
enum Scope { BLOCK = 0, WARP = 1, GROUP = 2 };

// shared-memory layouts of a tile of W sequences of length N
//  COLS: element (n, w) at n*W + w             (columns contiguous in w)
//  ROWS: element (n, w) at w*PITCH + n + n/G   (one pad slot per G elements,
//        G = 128 bytes / sizeof(complex), so strided stage writes stay
//        conflict-free); PITCH keeps rows apart by an odd number of slots
enum Layout { COLS = 0, ROWS = 1 };

//  TC (COLS, W = 16, FP32, tensor-core radix-16 stages): column pairs are
//        XOR-swizzled by row bits, w ^ sw(n), so the fragment-shaped loads
//        and stores of TileFFT::stage_tc16 are conflict-free (a whole row is
//        still a permutation of its 16 columns, and a 16-byte pair stays
//        together):
//          sw bit 2 = n bit B, sw bit 3 = n bit B+1 ^ n bits log2(p_s),
//        with 2^B = 2 N/16 (the loads of a radix-16 stage touch rows
//        i + (2t + c) N/16, t = lane % 4) and p_s the sub-length of each
//        tensor-core stage s (its stores touch rows o + g p_s, g = lane / 4).
template <typename T, int N, int W, int LAYOUT, bool TC = false>
struct TileLayout {
    using V = cx_t<T>;
    static constexpr int G = 128 / (int)sizeof(V);
    static constexpr int ROWLEN = N + (N + G - 1) / G;
    static constexpr int PITCH = (ROWLEN % 2 == 0) ? ROWLEN + 1 : ROWLEN;
    static constexpr int ELEMS = LAYOUT == COLS ? N * W : W * PITCH;
    static constexpr int ilog2(int v) { return v <= 1 ? 0 : 1 + ilog2(v / 2); }
    static constexpr int SWB = ilog2(N / 8);
    // rows whose bit log2(p_s) feeds sw bit 3: the radix-16 stages but the last
    static constexpr unsigned pmask() {
        const Fac f = factor(N, 2);
        unsigned m = 0;
        int p = 1;
        for (int s = 0; s + 1 < f.n; ++s) {
            if (f.r[s] == 16) m |= (unsigned)p;
            p *= f.r[s];
        }
        return m;
    }
    static constexpr unsigned PMASK = pmask();
    static constexpr bool kSw = LAYOUT == COLS && TC;
    static __host__ __device__ constexpr int parity(unsigned v) {
        v ^= v >> 16;
        v ^= v >> 8;
        v ^= v >> 4;
        v ^= v >> 2;
        v ^= v >> 1;
        return (int)(v & 1u);
    }
    static __host__ __device__ constexpr int swz(int n) {
        const int b3 = (parity((unsigned)n & PMASK) ^ (n >> (SWB + 1))) & 1;
        return (((n >> SWB) & 1) << 2) | (b3 << 3);
    }
    static __device__ __forceinline__ int idx(int n, int w) {
        if constexpr (LAYOUT == COLS && TC)
            return n * W + (w ^ swz(n));
        else if constexpr (LAYOUT == COLS)
            return n * W + w;
        else
            return w * PITCH + n + n / G;
    }
    // idx(a + b, w) for a and b without common set bits (a stage's row
    // i + j*nb with i < nb, or o + j*p, for power-of-two lengths): the
    // swizzle is XOR-linear in the row bits, so sw(a + b) = sw(a) ^ sw(b),
    // and with b a compile-time multiple after unrolling, sw(b) folds away
    static __device__ __forceinline__ int idx_sum(int a, int b, int w) {
        if constexpr (LAYOUT == COLS && TC)
            return (a + b) * W + (w ^ swz(a) ^ swz(b));
        else
            return idx(a + b, w);
    }
};

// Sources / sinks of a tile FFT.  A Global functor is called as v = src(n, w)
// and dst(n, w, v); FromSmem / ToSmem mean the first stage reads, or the last
// stage writes, the shared tile itself (natural order).
struct FromSmem {};
struct ToSmem {};
struct NoHook {
    __device__ __forceinline__ void operator()() const {}
};

template <typename T, int N, int W, int NT, bool FWD, int LAYOUT, int VARIANT = 0, int SCOPE = BLOCK>
struct TileFFT {
    using V = cx_t<T>;
    static constexpr bool kTcStage = VARIANT == 2 && std::is_same<T, float>::value && LAYOUT == COLS &&
                                     SCOPE == BLOCK && W == 16 && NT >= 64 && (N & (N - 1)) == 0 &&
                                     (NT & (NT - 1)) == 0;
    // VARIANT 3: the radix-16 stages but the last on tcgen05 (fft_tc5.cuh):
    // FP32 column tiles of width 16 read from shared memory, whole CTA, one
    // butterfly per thread, NT / 128 blocks of 128 butterflies
    static constexpr bool kTc5Stage = VARIANT == 3 && std::is_same<T, float>::value && LAYOUT == COLS &&
                                      SCOPE == BLOCK && W == 16 && NT % 128 == 0 && NT / 128 <= tc5::kMaxBlocks;
    using L = TileLayout<T, N, W, LAYOUT, kTcStage>;
    static constexpr Fac F = factor(N, VARIANT);
    static constexpr int NS = F.n;
    static_assert(NS >= 0, "length must factor into 2,3,5,7,11,13");
    static_assert(SCOPE != WARP || NT == 32, "a warp-scope tile has 32 threads");
    static_assert(SCOPE != GROUP || NT % 32 == 0, "a group-scope tile has whole warps");

    static __device__ __forceinline__ void sync() {
        if constexpr (SCOPE == WARP)
            __syncwarp();
        else if constexpr (SCOPE == GROUP)
            asm volatile("bar.sync 1, %0;\n" ::"n"(NT) : "memory");
        else
            __syncthreads();
    }
    static __device__ __forceinline__ int tid() {
        if constexpr (SCOPE == WARP)
            return (int)(threadIdx.x & 31);
        else
            return (int)threadIdx.x;
    }

    // ---- radix-16 stage on the tensor cores (VARIANT 2: FP32 column tiles
    // of width 16, whole CTA; every radix-16 stage but the last).
    // The 16-point DFTs of 8 butterflies (same i, 8 adjacent columns) are one
    // 16x16 by 16x8 product Y = F X, done by mma.sync.m16n8k16 with BF16
    // operands and FP32 accumulation.  Each FP32 value (the DFT entries, and
    // the inputs after their twiddle) is split into three BF16 terms
    // h + m + l (8 significant bits each, 24 together); the six products
    // with term orders adding up to at most 2 are kept (hh; hm, mh; hl, mm,
    // lh), smallest first, so the result carries about FP32's precision.
    // Complex arithmetic as real products: Yr = Fr Xr + Fi (-Xi),
    // Yi = Fr Xi + Fi Xr (24 MMAs per 8 butterflies).
    // Fragment layouts (PTX ISA, m16n8k16 .row.col), with g = lane/4 and
    // t = lane%4: A[g(+8)][2t(+1)(+8)], B[2t(+1)(+8)][g], D[g(+8)][2t(+1)].
    struct Split3 {
        uint32_t h, m, l;  // packed BF16 pairs (low half = first value)
    };
    static __device__ __forceinline__ uint32_t bf16x2(float a, float b) {
        const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
        uint32_t u;
        memcpy(&u, &v, 4);
        return u;
    }
    // the BF16 pair u widened back to two FP32 values (exact)
    static __device__ __forceinline__ float lo_f(uint32_t u) { return __uint_as_float(u << 16); }
    static __device__ __forceinline__ float hi_f(uint32_t u) { return __uint_as_float(u & 0xffff0000u); }
    static __device__ __forceinline__ Split3 split3(float a, float b) {
        Split3 s;
        s.h = bf16x2(a, b);
        const float ra = a - lo_f(s.h), rb = b - hi_f(s.h);  // exact remainders
        s.m = bf16x2(ra, rb);
        s.l = bf16x2(ra - lo_f(s.m), rb - hi_f(s.m));
        return s;
    }
    static __device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
    }
    // cos(2 pi m / 16), m = 0..15, from the exact values of cos(k pi / 8)
    static __device__ __forceinline__ float cos16(int m) {
        const float c1 = 0.92387953251128675613f, c2 = 0.70710678118654752440f, c3 = 0.38268343236508977173f;
        const int q = m & 7;  // cos(x + pi) = -cos(x)
        const int r = q <= 4 ? q : 8 - q;
        const float v = r == 0 ? 1.f : r == 1 ? c1 : r == 2 ? c2 : r == 3 ? c3 : 0.f;
        return ((m & 8) != 0) != (q > 4) ? -v : v;
    }
    // A fragments of the DFT-16 matrix F[r][c] = exp(-+ 2 pi i r c / 16),
    // real and imaginary parts, three BF16 terms each.  Only a0 (F[g][2t],
    // F[g][2t+1]) is kept: F[r+8][c] = (-1)^c F[r][c] and F[r][c+8] =
    // (-1)^r F[r][c], so a1..a3 are a0 with sign bits flipped (exact, as
    // the split of -x is minus the split of x).
    struct DftFrag {
        uint32_t re[3], im[3];
    };
    static __device__ __forceinline__ DftFrag dft16_fragments() {
        DftFrag f;
        const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
        const int m0 = (g * 2 * t) & 15, m1 = (g * (2 * t + 1)) & 15;
        // sin(x) = cos(x - pi/2); forward transform: exp(-i x)
        const float s0 = cos16((m0 + 12) & 15), s1 = cos16((m1 + 12) & 15);
        const Split3 re = split3(cos16(m0), cos16(m1));
        const Split3 im = FWD ? split3(-s0, -s1) : split3(s0, s1);
        f.re[0] = re.h;
        f.re[1] = re.m;
        f.re[2] = re.l;
        f.im[0] = im.h;
        f.im[1] = im.m;
        f.im[2] = im.l;
        return f;
    }
    // D += A(a0) B, with A's other three registers derived from a0
    static __device__ __forceinline__ void mma_dft(float (&d)[4], uint32_t a0, uint32_t sg, uint32_t b0, uint32_t b1) {
        const uint32_t a[4] = {a0, a0 ^ 0x80000000u, a0 ^ sg, a0 ^ sg ^ 0x80000000u};
        mma_bf16(d, a, b0, b1);
    }

    // Work split: warp wp takes butterflies i = wp/2 + u*NWARP/2 (u = 0, 1,
    // ...) in columns (wp%2)*8 .. +7.  Every tile row index below is a sum of
    // parts without common bits -- a per-thread part (wp/2, t or g) and a
    // compile-time part (u, the input or output slot) -- so the swizzle of
    // a row is the XOR of per-thread constants and folded constants.
    template <int S, class Src, class Dst>
    static __device__ __forceinline__ void stage_tc16(Src &src, Dst &dst, V *sm, const V *tw) {
        constexpr int R = 16;
        constexpr int p = fac_prod(F, S);
        constexpr int nb = N / R;
        constexpr bool src_smem = S != 0 || std::is_same<Src, FromSmem>::value;
        constexpr int NWARP = NT / 32;
        constexpr int HB = NWARP / 2;  // butterfly rows i per u step
        constexpr int GPW = (nb + HB - 1) / HB;
        static_assert(S < NS - 1, "the last stage runs on the FP32 pipes");
        static_assert(p == 1 || p >= HB, "k = i mod p splits into per-thread and compile-time parts");
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
        const int a = warp >> 1;           // per-thread part of i (< HB)
        const int w0 = (warp & 1) * 8;     // first column of the warp's butterflies
        const DftFrag fr = dft16_fragments();
        const uint32_t sg = (g & 1) ? 0x80008000u : 0u;  // (-1)^g on both halves
        V x[GPW][4];
        if (src_smem) sync();
        {
            // input rows i + j*nb, j = 2t + c (c = 0, 1, 8, 9)
            const int sw_ld = L::swz(a) ^ L::swz(2 * t * nb);
#pragma unroll
            for (int u = 0; u < GPW; ++u) {
                if ((u + 1) * HB <= nb || a + u * HB < nb) {
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const int c = (e & 1) + ((e & 2) ? 8 : 0);
                        const int row = a + u * HB + (2 * t + c) * nb;
                        if constexpr (src_smem)
                            x[u][e] = sm[row * W + ((w0 + g) ^ sw_ld ^ L::swz(u * HB + c * nb))];
                        else
                            x[u][e] = src(row, w0 + g);
                    }
                }
            }
        }
        sync();  // every reader of the tile is done before it is overwritten
        // output rows o + jout*p, o = (i - k)*R + k, k = i mod p
        constexpr int ao_mul = p == 1 ? R : 1;  // per-thread part of o: a*R (p = 1) or a
        const int sw_st = L::swz(a * ao_mul) ^ L::swz(g * p);
#pragma unroll
        for (int u = 0; u < GPW; ++u) {
            if ((u + 1) * HB <= nb || a + u * HB < nb) {
                const int b = u * HB;                           // compile-time part of i
                const int bk = p == 1 ? 0 : b % p;              // compile-time part of k
                const int k = p == 1 ? 0 : a + bk;
                const int oc = p == 1 ? b * R : (b - bk) * R + bk;  // compile-time part of o
                if constexpr (p > 1) {
                    constexpr int off = stage_offset(F, S);
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const int j = 2 * t + (e & 1) + ((e & 2) ? 8 : 0);
                        if (j > 0) x[u][e] = c_tw<FWD>(x[u][e], tw[off + (j - 1) * p + k]);
                    }
                }
                // B fragments: b0 = rows 2t, 2t+1; b1 = rows 2t+8, 2t+9 (column g)
                const Split3 r0 = split3(x[u][0].x, x[u][1].x), r1 = split3(x[u][2].x, x[u][3].x);
                const Split3 i0 = split3(x[u][0].y, x[u][1].y), i1 = split3(x[u][2].y, x[u][3].y);
                const uint32_t xr[3][2] = {{r0.h, r1.h}, {r0.m, r1.m}, {r0.l, r1.l}};
                const uint32_t xi[3][2] = {{i0.h, i1.h}, {i0.m, i1.m}, {i0.l, i1.l}};
                constexpr uint32_t NEG = 0x80008000u;
                float yr[4] = {0.f, 0.f, 0.f, 0.f}, yi[4] = {0.f, 0.f, 0.f, 0.f};
                // term pairs (F term, X term), smallest first
                constexpr int ta[6] = {0, 1, 2, 0, 1, 0}, tb[6] = {2, 1, 0, 1, 0, 0};
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    const int fa = ta[q], xb = tb[q];
                    mma_dft(yr, fr.re[fa], sg, xr[xb][0], xr[xb][1]);
                    mma_dft(yr, fr.im[fa], sg, xi[xb][0] ^ NEG, xi[xb][1] ^ NEG);
                    mma_dft(yi, fr.re[fa], sg, xi[xb][0], xi[xb][1]);
                    mma_dft(yi, fr.im[fa], sg, xr[xb][0], xr[xb][1]);
                }
                // D: outputs jout = g (d0, d1) and g + 8 (d2, d3) of the
                // butterflies in columns w0 + 2t and w0 + 2t + 1, stored as
                // one 16-byte pair per output row
                const int row = a * ao_mul + oc + g * p;
                const int col = (w0 + 2 * t) ^ sw_st ^ L::swz(oc);
                st_pair(sm, row * W + col, V{yr[0], yi[0]}, V{yr[1], yi[1]});
                st_pair(sm, (row + 8 * p) * W + (col ^ L::swz(8 * p)), V{yr[2], yi[2]}, V{yr[3], yi[3]});
            }
        }
    }
    // ---- radix-16 stage on tcgen05 (VARIANT 3).  Thread t takes butterfly
    // (i, w) = (t / W, t % W): it reads its 16 inputs, applies the stage's
    // twiddles, writes the TF32 split operands to its tensor-memory lane,
    // and after the block barrier and the MMAs (issued by thread 0) reads
    // its 16 outputs back and stores them to the tile.
    template <int S>
    static __device__ __forceinline__ void stage_tc5(V *sm, const V *tw) {
        constexpr int R = 16;
        constexpr int p = fac_prod(F, S);
        constexpr int nb = N / R;
        static_assert(nb * W == NT, "one butterfly per thread");
        static_assert(S < NS - 1, "the last stage runs on the FP32 pipes");
        tc5::State &ts = tc5::state();
        const int tid = threadIdx.x, warp = tid >> 5;
        const int w = tid % W, i = tid / W, k = i % p;
        V v[R];
        sync();  // the previous writer of the tile is done
        const uint32_t par = ts.phase & 1u;  // (advanced by thread 0 after the next barrier)
#pragma unroll
        for (int j = 0; j < R; ++j) v[j] = sm[L::idx_sum(i, j * nb, w)];
        if constexpr (p > 1) {
            constexpr int off = stage_offset(F, S);
#pragma unroll
            for (int j = 1; j < R; ++j) v[j] = c_tw<FWD>(v[j], tw[off + (j - 1) * p + k]);
        }
        // this thread's lane of its block's columns: Xh = [Re | Im] at 0-31, Xl at 32-63, Y at 64-95
        const uint32_t taddr = ts.tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)((warp >> 2) * tc5::kColsPerBlock);
        {
            uint32_t h[16], l[16];
#pragma unroll
            for (int j = 0; j < R; ++j) {
                h[j] = tc5::rna_tf32(v[j].x);
                l[j] = __float_as_uint(v[j].x - __uint_as_float(h[j]));
            }
            tc5::st16(taddr, h);
            tc5::st16(taddr + 32, l);
#pragma unroll
            for (int j = 0; j < R; ++j) {
                h[j] = tc5::rna_tf32(v[j].y);
                l[j] = __float_as_uint(v[j].y - __uint_as_float(h[j]));
            }
            tc5::st16(taddr + 16, h);
            tc5::st16(taddr + 48, l);
        }
        tc5::wait_st();
        tc5::fence_before();
        sync();  // every operand is in tensor memory and every input of the tile has been read
        if (tid == 0) {
            tc5::issue(NT / 128);
            ts.phase += 1;
        }
        if (!tc5::bar_wait(&ts.bar, par)) ts.err = 1;
        tc5::fence_after();
        uint32_t d[32];
        tc5::ld32(taddr + 64, d);
        tc5::wait_ld();
        tc5::fence_before();  // these reads precede the next MMAs (after a barrier)
        // outputs at rows o + j p, o = (i - k) R + k
        const int o = (i - k) * R + k;
#pragma unroll
        for (int j = 0; j < R; ++j) sm[L::idx_sum(o, j * p, w)] = V{__uint_as_float(d[j]), __uint_as_float(d[16 + j])};
    }

    // two adjacent complex values at an even tile index (16-byte aligned)
    static __device__ __forceinline__ void st_pair(V *sm, int idx, V a, V b) {
        *reinterpret_cast<float4 *>(sm + idx) = make_float4(a.x, a.y, b.x, b.y);
    }

    template <int S, class Src, class Dst, class Hook>
    static __device__ __forceinline__ void stage(Src &src, Dst &dst, V *sm, const V *tw, Hook &hook) {
        if constexpr (kTcStage && F.r[S] == 16 && S < NS - 1) {
            stage_tc16<S>(src, dst, sm, tw);
            return;
        } else if constexpr (kTc5Stage && F.r[S] == 16 && S < NS - 1) {
            static_assert(S != 0 || std::is_same<Src, FromSmem>::value,
                          "the tcgen05 stages read the tile from shared memory");
            stage_tc5<S>(sm, tw);
            return;
        } else {
            stage_scalar<S>(src, dst, sm, tw, hook);
        }
    }

    // Hook: called by every thread once the last stage has read the whole
    // tile from shared memory (after a barrier) when the last stage writes
    // global memory -- the tile buffer is free from then on.  NoHook: none.
    template <int S, class Src, class Dst, class Hook>
    static __device__ __forceinline__ void stage_scalar(Src &src, Dst &dst, V *sm, const V *tw, Hook &hook) {
        constexpr int R = F.r[S];
        constexpr int p = fac_prod(F, S);
        constexpr int nb = N / R;
        constexpr int items = nb * W;
        constexpr int C = (items + NT - 1) / NT;
        constexpr bool first = (S == 0);
        constexpr bool last = (S == NS - 1);
        constexpr bool src_smem = !first || std::is_same<Src, FromSmem>::value;
        constexpr bool dst_smem = !last || std::is_same<Dst, ToSmem>::value;
        const int tid = TileFFT::tid();
        V v[C][R];
        int ii[C], ww[C];
        if (src_smem) sync();  // the previous writer of the tile is done
#pragma unroll
        for (int m = 0; m < C; ++m) {
            const int q = tid + m * NT;
            if ((m + 1) * NT <= items || q < items) {
                int i, w;
                if constexpr (LAYOUT == COLS) {
                    w = q % W;
                    i = q / W;
                } else {
                    i = q % nb;
                    w = q / nb;
                }
                ii[m] = i;
                ww[m] = w;
#pragma unroll
                for (int j = 0; j < R; ++j) {
                    if constexpr (src_smem && L::kSw)  // i = tid/W + m*NT/W (disjoint bits)
                        v[m][j] = sm[L::idx_sum(tid / W, m * (NT / W) + j * nb, w)];
                    else if constexpr (src_smem)
                        v[m][j] = sm[L::idx_sum(i, j * nb, w)];
                    else
                        v[m][j] = src(i + j * nb, w);
                }
            }
        }
        if (dst_smem) sync();  // every reader of the tile is done before it is overwritten
        if constexpr (last && !dst_smem && src_smem && !std::is_same<Hook, NoHook>::value) {
            sync();
            hook();
        }
        // In the COLS layout a thread's butterflies are NT/W apart in i; when
        // that is a multiple of p they share k = i mod p, so their twiddles
        // are read from shared memory once.
        constexpr bool shared_k = LAYOUT == COLS && p > 1 && C > 1 && (NT / W) % p == 0 && NT % W == 0;
        V tws[shared_k ? R : 1];
        if constexpr (shared_k) {
            constexpr int off = stage_offset(F, S);
            const int k0 = ii[0] % p;
#pragma unroll
            for (int j = 1; j < R; ++j) tws[j] = tw[off + (j - 1) * p + k0];
        }
#pragma unroll
        for (int m = 0; m < C; ++m) {
            const int q = tid + m * NT;
            if ((m + 1) * NT <= items || q < items) {
                const int i = ii[m], w = ww[m];
                const int k = i % p;
                if constexpr (shared_k) {
#pragma unroll
                    for (int j = 1; j < R; ++j) v[m][j] = c_tw<FWD>(v[m][j], tws[j]);
                } else if constexpr (p > 1) {
                    constexpr int off = stage_offset(F, S);
#pragma unroll
                    for (int j = 1; j < R; ++j) v[m][j] = c_tw<FWD>(v[m][j], tw[off + (j - 1) * p + k]);
                }
                Dft<R, FWD, V>::run(v[m]);
                if constexpr (last) {
                    // last stage: p = nb, k = i, output positions i + j*nb
#pragma unroll
                    for (int j = 0; j < R; ++j) {
                        if constexpr (dst_smem && L::kSw)
                            sm[L::idx_sum(tid / W, m * (NT / W) + j * nb, w)] = v[m][j];
                        else if constexpr (dst_smem)
                            sm[L::idx_sum(i, j * nb, w)] = v[m][j];
                        else
                            dst(i + j * nb, w, v[m][j]);
                    }
                } else {
                    const int o = (i - k) * R + k;
#pragma unroll
                    for (int j = 0; j < R; ++j) sm[L::idx_sum(o, j * p, w)] = v[m][j];
                }
            }
        }
    }

    template <int S, class Src, class Dst, class Hook>
    static __device__ __forceinline__ void stages(Src &src, Dst &dst, V *sm, const V *tw, Hook &hook) {
        if constexpr (S < NS) {
            stage<S>(src, dst, sm, tw, hook);
            stages<S + 1>(src, dst, sm, tw, hook);
        }
    }

    // Runs the whole FFT.  With a Global source the tile buffer must be free
    // (the first stage synchronises before writing it); a ToSmem result is
    // complete only after the caller's next __syncthreads().
    template <class Src, class Dst>
    static __device__ __forceinline__ void run(Src &src, Dst &dst, V *sm, const V *tw) {
        NoHook none;
        run(src, dst, sm, tw, none);
    }
    template <class Src, class Dst, class Hook>
    static __device__ __forceinline__ void run(Src &src, Dst &dst, V *sm, const V *tw, Hook &hook) {
        if constexpr (NS == 0) {
            // length 1: identity (copy)
            if constexpr (std::is_same<Src, FromSmem>::value) sync();
            for (int q = tid(); q < W; q += NT) {
                V x;
                if constexpr (std::is_same<Src, FromSmem>::value) {
                    x = sm[L::idx(0, q)];
                } else {
                    x = src(0, q);
                }
                if constexpr (std::is_same<Dst, ToSmem>::value)
                    sm[L::idx(0, q)] = x;
                else
                    dst(0, q, x);
            }
        } else {
            stages<0>(src, dst, sm, tw, hook);
        }
    }
};

// ---------------------------------------------------------------------------
// Pass B: x-axis FFT over column tiles (stride Ny*Nh), compile-time Nx
// ---------------------------------------------------------------------------
// Tiles first_tile, first_tile + tile_step, ... of Pass B (the kernel below
// runs it over the grid; the batched form runs single tiles).  EPI: the
// x-pass epilogue (scale, dealiasing; PassBParams) is compiled in.
template <typename T, int NX, int W, int NT, bool FWD, int VARIANT, bool EPI>
__device__ __forceinline__ void pass_b_fast_run(const PassBParams &P, unsigned char *smem_raw, long long first_tile,
                                                long long tile_step) {
    using V = cx_t<T>;
    using FFT = TileFFT<T, NX, W, NT, FWD, COLS, VARIANT, BLOCK>;
    V *tw = reinterpret_cast<V *>(smem_raw);
    V *tile = tw + NX;
    for (int q = threadIdx.x; q < NX - 1; q += NT) tw[q] = reinterpret_cast<const V *>(P.stw)[q];
    // (the first stage's barrier orders these writes before any twiddle read)
    V *base = reinterpret_cast<V *>(P.data);
    const long long ncols = P.ncols;
    for (long long t = first_tile; t < P.ntiles; t += tile_step) {
        const long long c0 = t * W;
        const int wv = (int)min((long long)W, ncols - c0);
        V *g = base + c0;
        auto src = [&](int n, int w) -> V {
            return (w < wv) ? ld_g(g + (long long)n * ncols + w) : V{(T)0, (T)0};
        };
        auto dst = [&](int n, int w, V v) {
            if (w < wv) {
                if constexpr (EPI)
                    st_g(g + (long long)n * ncols + w, pass_b_epilogue(P, v, n, c0 + w));
                else
                    st_g(g + (long long)n * ncols + w, v);
            }
        };
        FFT::run(src, dst, tile, tw);
    }
}

template <typename T, int NX, int W, int NT, bool FWD, int VARIANT, int MINB, bool EPI = false>
__global__ void __launch_bounds__(NT, MINB) pass_b_fast(PassBParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pass_b_fast_run<T, NX, W, NT, FWD, VARIANT, EPI>(P, smem_raw, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// Pass B with the tiles double-buffered by cp.async: while a tile is being
// transformed (in place in shared memory, last stage written to global
// memory), the next tile streams from global memory into the other buffer.
// 16-byte copies; requires Ny*Nh even (row starts 16-byte aligned) and W even.
// Columns of a ragged last tile past ncols are zero-filled by the copy.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// one complex element (8 or 16 bytes, both addresses aligned to its size);
// zero-filled when `valid` is false
template <typename V>
__device__ __forceinline__ void cp_async_elem(V *smem, const V *gmem, bool valid) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? (int)sizeof(V) : 0;
    if constexpr (sizeof(V) == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(n) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(n) : "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <typename T, int NX, int W, int NT, bool FWD, int VARIANT, int MINB, bool EPI = false>
__global__ void __launch_bounds__(NT, MINB) pass_b_pipe(PassBParams P) {
    using V = cx_t<T>;
    using FFT = TileFFT<T, NX, W, NT, FWD, COLS, VARIANT, BLOCK>;
    constexpr int PER16 = 16 / (int)sizeof(V);  // complex per 16-byte chunk
    constexpr int CH = W / PER16;                // chunks per tile row
    static_assert(W % PER16 == 0, "tile rows must be whole 16-byte chunks");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tw = reinterpret_cast<V *>(smem_raw);
    V *buf0 = tw + ((NX + PER16 - 1) / PER16) * PER16;
    V *buf1 = buf0 + NX * W;
    for (int q = threadIdx.x; q < NX - 1; q += NT) tw[q] = reinterpret_cast<const V *>(P.stw)[q];
    const V *base = reinterpret_cast<const V *>(P.data);
    V *obase = reinterpret_cast<V *>(P.data);
    const long long ncols = P.ncols;
    auto prefetch = [&](long long t, V *buf) {
        const long long c0 = t * W;
        const int wv = (int)min((long long)W, ncols - c0);
        for (int q = threadIdx.x; q < NX * CH; q += NT) {
            const int n = q / CH, ch = q % CH;
            const int w = ch * PER16;
            const int valid = max(0, min(PER16, wv - w));
            const V *src = base + (long long)n * ncols + c0 + (valid > 0 ? w : 0);
            cp_async16(buf + FFT::L::idx(n, w), src, valid * (int)sizeof(V));
        }
        cp_async_commit();
    };
    long long t = blockIdx.x;
    if (t < P.ntiles) prefetch(t, buf0);
    int k = 0;
    for (; t < P.ntiles; t += gridDim.x, k ^= 1) {
        V *cur = k ? buf1 : buf0;
        V *nxt = k ? buf0 : buf1;
        const long long tn = t + gridDim.x;
        if (tn < P.ntiles) {
            prefetch(tn, nxt);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        // (the FFT's first stage begins with a block barrier: the copies of
        // every thread have landed before any thread reads the tile)
        const long long c0 = t * W;
        const int wv = (int)min((long long)W, ncols - c0);
        V *g = obase + c0;
        auto dst = [&](int n, int w, V v) {
            if (w < wv) {
                if constexpr (EPI)
                    st_g(g + (long long)n * ncols + w, pass_b_epilogue(P, v, n, c0 + w));
                else
                    st_g(g + (long long)n * ncols + w, v);
            }
        };
        FromSmem fs;
        FFT::run(fs, dst, cur, tw);
        __syncthreads();  // the tile is free for the copy issued next iteration
    }
}

// ---------------------------------------------------------------------------
// Pass B with ONE tile buffer refilled early: the next tile's cp.async copies
// are issued as soon as the last FFT stage has read the current tile from
// shared memory, so they stream in while that stage computes and writes its
// results to global memory.  For tiles too large to double-buffer
// (Nx = 1024 with 16-column tiles: 128 KB).  Same alignment rules as
// pass_b_pipe.
// ---------------------------------------------------------------------------
template <typename T, int NX, int W, int NT, bool FWD, int VARIANT, int MINB, bool EPI = false>
__global__ void __launch_bounds__(NT, MINB) pass_b_pipe1(PassBParams P) {
    using V = cx_t<T>;
    using FFT = TileFFT<T, NX, W, NT, FWD, COLS, VARIANT, BLOCK>;
    constexpr int PER16 = 16 / (int)sizeof(V);
    constexpr int CH = W / PER16;
    static_assert(W % PER16 == 0, "tile rows must be whole 16-byte chunks");
    static_assert(FFT::NS >= 2, "the first stage must read the tile from shared memory");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tw = reinterpret_cast<V *>(smem_raw);
    V *buf = tw + ((NX + PER16 - 1) / PER16) * PER16;
    for (int q = threadIdx.x; q < NX - 1; q += NT) tw[q] = reinterpret_cast<const V *>(P.stw)[q];
    const V *base = reinterpret_cast<const V *>(P.data);
    V *obase = reinterpret_cast<V *>(P.data);
    const long long ncols = P.ncols;
    auto prefetch = [&](long long t) {
        const long long c0 = t * W;
        const int wv = (int)min((long long)W, ncols - c0);
        for (int q = threadIdx.x; q < NX * CH; q += NT) {
            const int n = q / CH, ch = q % CH;
            const int w = ch * PER16;
            const int valid = max(0, min(PER16, wv - w));
            const V *src = base + (long long)n * ncols + c0 + (valid > 0 ? w : 0);
            cp_async16(buf + FFT::L::idx(n, w), src, valid * (int)sizeof(V));
        }
        cp_async_commit();
    };
    long long t = blockIdx.x;
    if (t < P.ntiles) prefetch(t);
    for (; t < P.ntiles; t += gridDim.x) {
        cp_async_wait<0>();
        // (the first stage begins with a block barrier: every thread's copies
        // have landed before any thread reads the tile)
        const long long c0 = t * W;
        const int wv = (int)min((long long)W, ncols - c0);
        V *g = obase + c0;
        auto dst = [&](int n, int w, V v) {
            if (w < wv) {
                if constexpr (EPI)
                    st_g(g + (long long)n * ncols + w, pass_b_epilogue(P, v, n, c0 + w));
                else
                    st_g(g + (long long)n * ncols + w, v);
            }
        };
        const long long tn = t + gridDim.x;
        auto refill = [&]() {
            if (tn < P.ntiles) prefetch(tn);
        };
        FromSmem fs;
        FFT::run(fs, dst, buf, tw, refill);
    }
}

// ---------------------------------------------------------------------------
// Pass A: per x-plane z-axis R2C/C2R (rows, one warp per group of RW rows,
// no CTA barrier) and y-axis C2C (column tiles of WY, whole CTA)
// ---------------------------------------------------------------------------
template <typename T, int NY, int M, int RW, int WY, int NT, int VY, int VZ>
struct PassAShape {
    using V = cx_t<T>;
    using RowL = TileLayout<T, M, RW, ROWS>;
    using ColL = TileLayout<T, NY, WY, COLS>;
    static constexpr int NWARP = NT / 32;
    static constexpr int ROWS_ELEMS = NWARP * RowL::ELEMS;
    static constexpr int TILE = ROWS_ELEMS > ColL::ELEMS ? ROWS_ELEMS : ColL::ELEMS;
    // unpack roots w_Nz^k (k <= M/2), z and y stage tables, tile
    static constexpr int UNP = M / 2 + 1;
    static constexpr size_t smem_bytes() { return (size_t)(UNP + M + NY + TILE) * sizeof(V); }
};

// Split cluster barrier: arrive (release) after a phase, wait (acquire)
// before the dependent phase; the CTA may do independent work in between.
__device__ __forceinline__ void cluster_arrive() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// One CTA's part of Pass A: CTA `crank` of the K that share each x-plane
// (rows [crank*NY/K, ...), column tiles crank, crank+K, ...), for planes
// first_plane, first_plane + plane_step, ...  The kernel below runs it over
// the grid; the batched form runs it for one whole plane (K = 1).
// CP = 1: column tiles after the first are copied into the tile buffer by
// cp.async, the next one issued as soon as the last FFT stage of the current
// one has read the buffer (TileFFT::run's hook), so its loads overlap that
// stage's arithmetic and stores.  Column tile 0 (the packed bins 0 and Nz/2)
// keeps its own path.
// XCH: the y columns' global side (the forward's output, the inverse's
// input) is the slab decomposition's exchange layout (PassAParams::xch).
template <typename T, int NY, int M, int RW, int WY, int NT, bool FWD, int VY, int VZ, int CP = 0, bool XCH = false>
__device__ __forceinline__ void pass_a_fast_run(const PassAParams &P, unsigned char *smem_raw, const int crank,
                                                const int K, const int first_plane, const int plane_step) {
    using V = cx_t<T>;
    using Shape = PassAShape<T, NY, M, RW, WY, NT, VY, VZ>;
    using RowFFT = TileFFT<T, M, RW, 32, FWD, ROWS, VZ, WARP>;
    using ColFFT = TileFFT<T, NY, WY, NT, FWD, COLS, VY, BLOCK>;
    using RowL = typename RowFFT::L;
    using ColL = typename ColFFT::L;
    constexpr int NH = M + 1;
    constexpr int UNP = Shape::UNP;
    constexpr int HALF = M / 2 + 1;
    V *unp = reinterpret_cast<V *>(smem_raw);
    V *stz = unp + UNP;
    V *sty = stz + M;
    V *tile = sty + NY;
    for (int q = threadIdx.x; q < UNP; q += NT) unp[q] = reinterpret_cast<const V *>(P.twz)[q];
    for (int q = threadIdx.x; q < M - 1; q += NT) stz[q] = reinterpret_cast<const V *>(P.stz)[q];
    for (int q = threadIdx.x; q < NY - 1; q += NT) sty[q] = reinterpret_cast<const V *>(P.sty)[q];
    __syncthreads();

    const int cid = first_plane, ncl = plane_step;
    const int rows_per = (NY + K - 1) / K;
    const int rb = min(NY, crank * rows_per), re = min(NY, rb + rows_per);
    constexpr int ntiles_y = (M + WY - 1) / WY;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    V *wtile = tile + wid * RowL::ELEMS;  // this warp's rows (overlaps the column tile)
    V *base = reinterpret_cast<V *>(P.data);
    const T hf = (T)0.5;

    // ---------------- y columns of plane g (whole CTA) ----------------
    // CP: copies of column tile t (t >= 1) of plane g into the tile buffer
    // row n of plane g on the columns' global side: the exchange layout
    // (XCH) or the field itself
    auto xrow = [&](V *g, int plane, int n) -> V * {
        if constexpr (XCH) {
            const int s = n / P.xch_nyl;
            return reinterpret_cast<V *>(P.xch) + s * P.xch_chunk +
                   ((long long)plane * P.xch_nyl + (n - s * P.xch_nyl)) * NH;
        } else {
            return g + (long long)n * NH;
        }
    };
    // where the columns read from and write to
    auto in_row = [&](V *g, int plane, int n) -> V * { return FWD ? g + (long long)n * NH : xrow(g, plane, n); };
    auto out_row = [&](V *g, int plane, int n) -> V * { return FWD ? xrow(g, plane, n) : g + (long long)n * NH; };
    auto prefetch_cols = [&](V *g, int plane, int t) {
        const int c0 = t * WY;
        const int wv = min(WY, M - c0);
        for (int q = threadIdx.x; q < NY * WY; q += NT) {
            const int n = q / WY, w = q % WY;
            cp_async_elem(tile + ColL::idx(n, w), in_row(g, plane, n) + c0 + (w < wv ? w : 0), w < wv);
        }
        cp_async_commit();
    };
    auto cols = [&](V *g, int plane) {
        if constexpr (CP) {
            if (crank != 0 && crank < ntiles_y) prefetch_cols(g, plane, crank);
        }
        for (int t = crank; t < ntiles_y; t += K) {
            const int c0 = t * WY;
            const int wv = min(WY, M - c0);
            auto src = [&](int n, int w) -> V {
                return (w < wv) ? ld_g(in_row(g, plane, n) + c0 + w) : V{(T)0, (T)0};
            };
            auto dst = [&](int n, int w, V v) {
                if (w < wv) st_g(out_row(g, plane, n) + c0 + w, v);
            };
            if (CP && c0 != 0) {
                cp_async_wait<0>();
                // (the first stage begins with a block barrier)
                const int tn = t + K;
                auto refill = [&]() {
                    if (tn < ntiles_y) prefetch_cols(g, plane, tn);
                };
                FromSmem fs;
                ColFFT::run(fs, dst, tile, sty, refill);
            } else if (c0 != 0) {
                ColFFT::run(src, dst, tile, sty);
            } else if (FWD) {
                // column 0 carries (bin 0) + i (bin m); split after the FFT
                ToSmem ts;
                ColFFT::run(src, ts, tile, sty);
                __syncthreads();
                for (int q = threadIdx.x; q < NY * WY; q += NT) {
                    const int n = q / WY, w = q % WY;
                    if (w >= wv) continue;
                    const V c1 = tile[ColL::idx(n, w)];
                    V *orow = out_row(g, plane, n);
                    if (w == 0) {
                        const V c2 = c_conj(tile[ColL::idx((NY - n) % NY, 0)]);
                        st_g(orow, c_scale(c_add(c1, c2), hf));
                        st_g(orow + M, c_rot<true>(c_scale(c_sub(c1, c2), hf)));
                    } else {
                        st_g(orow + c0 + w, c1);
                    }
                }
            } else {
                // inverse: Hermitian projection of bins kz=0 (a) and kz=m (b) along y,
                // packed as a' + i b' into column 0 in place (each thread owns the
                // pair of rows n, -n), then the plain column FFT
                __syncthreads();
                for (int n = threadIdx.x; n <= NY / 2; n += NT) {
                    const int n2 = (NY - n) % NY;
                    V *r1 = in_row(g, plane, n), *r2 = in_row(g, plane, n2);
                    const V a1 = ld_g(r1), a2 = ld_g(r2);
                    const V b1 = ld_g(r1 + M), b2 = ld_g(r2 + M);
                    const V ha = c_scale(c_add(a1, c_conj(a2)), hf);
                    const V hb = c_scale(c_add(b1, c_conj(b2)), hf);
                    st_g(r1, V{ha.x - hb.y, ha.y + hb.x});
                    if (n2 != n) st_g(r2, V{ha.x + hb.y, -ha.y + hb.x});
                }
                __syncthreads();
                ColFFT::run(src, dst, tile, sty);
            }
            if constexpr (CP) {
                if (c0 == 0 && t + K < ntiles_y) {
                    __syncthreads();  // tile 0's last reads of the buffer are done
                    prefetch_cols(g, plane, t + K);
                }
            }
        }
    };
    // ---------------- z rows of plane g: each warp takes RW rows at a time ----------------
    auto rows = [&](V *g) {
        for (int r0 = rb + wid * RW; r0 < re; r0 += (NT / 32) * RW) {
            const int wv = min(RW, re - r0);
            V *gr = g + (long long)r0 * NH;
            if (FWD) {
                auto src = [&](int n, int w) -> V {
                    return (w < wv) ? ld_g(gr + (long long)w * NH + n) : V{(T)0, (T)0};
                };
                ToSmem ts;
                RowFFT::run(src, ts, wtile, stz);
                __syncwarp();
                // unpack: X[k] = E + O, X[m-k] = conj(E - O), E = (Z[k] + conj Z[m-k])/2,
                // O = -i w^k (Z[k] - conj Z[m-k])/2, w = exp(-2 pi i/Nz); bins 0 and m packed in slot 0
                for (int w = 0; w < wv; ++w) {
                    V *row = gr + (long long)w * NH;
                    for (int k = lane; k < HALF; k += 32) {
                        const V a = wtile[RowL::idx(k, w)];
                        const V b = c_conj(wtile[RowL::idx(k == 0 ? 0 : M - k, w)]);
                        const V e = c_scale(c_add(a, b), hf);
                        const V d = c_scale(c_sub(a, b), hf);
                        const V o = c_rot<true>(c_mul(d, unp[k]));
                        const V xa = c_add(e, o), xb = c_conj(c_sub(e, o));
                        if (k == 0) {
                            st_g(row, V{xa.x, xb.x});
                        } else {
                            st_g(row + k, xa);
                            if (M - k != k) st_g(row + M - k, xb);
                        }
                    }
                }
            } else {
                // pre-process: Z[k] = S + Pk, Z[m-k] = conj(S - Pk), S = X[k] + conj X[m-k],
                // Pk = i conj(w^k)(X[k] - conj X[m-k]); slot 0 holds (Re X0, Re Xm).
                // All loads of the warp's rows are issued before any use, so their
                // latencies overlap instead of adding up.
                constexpr int KPL = (HALF + 31) / 32;
                V xk[RW][KPL], xm[RW][KPL];
#pragma unroll
                for (int w = 0; w < RW; ++w) {
                    const V *row = gr + (long long)w * NH;
#pragma unroll
                    for (int u = 0; u < KPL; ++u) {
                        const int k = lane + 32 * u;
                        xk[w][u] = V{(T)0, (T)0};
                        xm[w][u] = V{(T)0, (T)0};
                        if (w < wv && k < HALF) {
                            xk[w][u] = ld_g(row + k);
                            if (k != 0) xm[w][u] = ld_g(row + M - k);
                        }
                    }
                }
                __syncwarp();
#pragma unroll
                for (int w = 0; w < RW; ++w) {
#pragma unroll
                    for (int u = 0; u < KPL; ++u) {
                        const int k = lane + 32 * u;
                        if (k < HALF) {
                            V a = xk[w][u], b = xm[w][u];
                            if (k == 0) {
                                b = V{a.y, (T)0};
                                a = V{a.x, (T)0};
                            }
                            const V cm = c_conj(b);
                            const V s = c_add(a, cm);
                            const V pk = c_rot<false>(c_mulc(c_sub(a, cm), unp[k]));
                            wtile[RowL::idx(k, w)] = c_add(s, pk);
                            if (k != 0 && M - k != k) wtile[RowL::idx(M - k, w)] = c_conj(c_sub(s, pk));
                        }
                    }
                }
                auto dst = [&](int n, int w, V v) {
                    if (w < wv) st_g(gr + (long long)w * NH + n, v);
                };
                FromSmem fs;
                RowFFT::run(fs, dst, wtile, stz);
                // slot m = padding cells of the real row: zero
                if (lane < wv) st_g(gr + (long long)lane * NH + M, V{(T)0, (T)0});
            }
        }
    };

    // Schedule: forward runs rows then columns of each plane, inverse the
    // reverse, with the cluster barrier (release/acquire, so the plane's
    // rows written by every CTA of the cluster are visible) in between.
    // Running the next plane's first phase before the barrier wait was
    // measured slower at 512^3: two planes per cluster in flight overflow L2.
    // Block barriers separate the warp-private row tiles from the shared
    // column tile, which overlap in shared memory.
    // A split Pass A (P.phases 1 or 2, for planes too large to stay in L2
    // while a cluster works on them) runs one of the two phases per launch.
    const bool do_rows = P.phases != 2, do_cols = P.phases != 1;
    for (int plane = cid; plane < P.nx; plane += ncl) {
        V *g = base + (long long)plane * NY * NH;
        if (FWD) {
            if (do_rows) rows(g);
        } else if (do_cols) {
            cols(g, plane);
        }
        __syncthreads();
        if (K > 1 && P.phases == 0) {
            cluster_arrive();
            cluster_wait();
        }
        if (FWD) {
            if (do_cols) cols(g, plane);
        } else if (do_rows) {
            rows(g);
        }
        __syncthreads();
    }
}

template <typename T, int NY, int M, int RW, int WY, int NT, bool FWD, int VY, int VZ, int MINB, int CP = 0,
          bool XCH = false>
__global__ void __launch_bounds__(NT, MINB) pass_a_fast(PassAParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int K = P.K;
    pass_a_fast_run<T, NY, M, RW, WY, NT, FWD, VY, VZ, CP, XCH>(P, smem_raw, (int)blockIdx.x % K, K,
                                                                (int)blockIdx.x / K, (int)gridDim.x / K);
}

// ---------------------------------------------------------------------------
// Pass A, distributed-shared-memory form.  A cluster of K CTAs holds one
// x-plane in shared memory: CTA r owns rows [r*NY/K, (r+1)*NY/K) of the
// plane (ROWS layout, its "slice").  Forward: every warp transforms its rows
// from global memory in place in the slice (z R2C + unpack); cluster barrier;
// the column tiles read the slices of all CTAs of the cluster over DSMEM, run
// the y FFT and write the result to global memory; cluster barrier before the
// next plane overwrites the slices.  Inverse: the y inverse writes its output
// into the owners' slices over DSMEM, then each warp runs the z C2R of its
// rows from the slice to global memory.  Global memory sees one read and one
// write of the field; no L2 round trip between the axes.
// ---------------------------------------------------------------------------
template <typename T, int NY, int M, int RW, int WY, int NT, int K, int VY, int VZ>
struct PassADsmemShape {
    using V = cx_t<T>;
    using SliceL = TileLayout<T, M, NY / K, ROWS>;
    using ColL = TileLayout<T, NY, WY, COLS>;
    static constexpr int UNP = M / 2 + 1;
    static constexpr size_t smem_bytes() {
        return (size_t)(UNP + M + NY + SliceL::ELEMS + ColL::ELEMS) * sizeof(V);
    }
};

template <typename T, int NY, int M, int RW, int WY, int NT, int K, bool FWD, int VY, int VZ, int MINB>
__global__ void __launch_bounds__(NT, MINB) pass_a_dsmem(PassAParams P) {
    using V = cx_t<T>;
    using Shape = PassADsmemShape<T, NY, M, RW, WY, NT, K, VY, VZ>;
    constexpr int SLICE = NY / K;
    static_assert(NY % K == 0, "rows must split evenly over the cluster");
    static_assert(SLICE % RW == 0, "warp row groups must tile the slice");
    using RowFFT = TileFFT<T, M, RW, 32, FWD, ROWS, VZ, WARP>;
    using ColFFT = TileFFT<T, NY, WY, NT, FWD, COLS, VY, BLOCK>;
    using SliceL = typename Shape::SliceL;
    using ColL = typename ColFFT::L;
    static_assert(SliceL::PITCH == RowFFT::L::PITCH, "row tiles live inside the slice");
    constexpr int NH = M + 1;
    constexpr int UNP = Shape::UNP;
    constexpr int HALF = M / 2 + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *unp = reinterpret_cast<V *>(smem_raw);
    V *stz = unp + UNP;
    V *sty = stz + M;
    V *slice = sty + NY;
    V *ctile = slice + SliceL::ELEMS;
    for (int q = threadIdx.x; q < UNP; q += NT) unp[q] = reinterpret_cast<const V *>(P.twz)[q];
    for (int q = threadIdx.x; q < M - 1; q += NT) stz[q] = reinterpret_cast<const V *>(P.stz)[q];
    for (int q = threadIdx.x; q < NY - 1; q += NT) sty[q] = reinterpret_cast<const V *>(P.sty)[q];
    __syncthreads();

    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const int crank = (int)cluster.block_rank();
    const int cid = blockIdx.x / K;
    const int ncl = gridDim.x / K;
    constexpr int ntiles_y = (M + WY - 1) / WY;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    V *base = reinterpret_cast<V *>(P.data);
    const T hf = (T)0.5;
    // element (row n, column c) of the plane in the owner's slice (DSMEM address)
    auto at = [&](int n, int c) -> V * {
        return cluster.map_shared_rank(slice + SliceL::idx(c, n % SLICE), n / SLICE);
    };

    for (int plane = cid; plane < P.nx; plane += ncl) {
        V *g = base + (long long)plane * NY * NH;
        V *gs = g + (long long)crank * SLICE * NH;  // this CTA's rows in global memory
        if (FWD) {
            // ---- z rows: global -> slice, R2C, unpack in place ----
            for (int lr = wid * RW; lr < SLICE; lr += (NT / 32) * RW) {
                V *gr = gs + (long long)lr * NH;
                V *wt = slice + lr * SliceL::PITCH;
                auto src = [&](int n, int w) -> V { return ld_g(gr + (long long)w * NH + n); };
                ToSmem ts;
                RowFFT::run(src, ts, wt, stz);
                __syncwarp();
                for (int w = 0; w < RW; ++w) {
                    for (int k = lane; k < HALF; k += 32) {
                        const int km = (k == 0) ? 0 : M - k;
                        const V a = wt[SliceL::idx(k, w)];
                        const V b = c_conj(wt[SliceL::idx(km, w)]);
                        const V e = c_scale(c_add(a, b), hf);
                        const V d = c_scale(c_sub(a, b), hf);
                        const V o = c_rot<true>(c_mul(d, unp[k]));
                        const V xa = c_add(e, o), xb = c_conj(c_sub(e, o));
                        if (k == 0) {
                            wt[SliceL::idx(0, w)] = V{xa.x, xb.x};
                        } else {
                            wt[SliceL::idx(k, w)] = xa;
                            if (km != k) wt[SliceL::idx(km, w)] = xb;
                        }
                    }
                }
            }
            cluster.sync();
            // ---- y columns: slices (DSMEM) -> y FFT -> global ----
            for (int t = crank; t < ntiles_y; t += K) {
                const int c0 = t * WY;
                const int wv = min(WY, M - c0);
                V *gc = g + c0;
                auto src = [&](int n, int w) -> V { return (w < wv) ? *at(n, c0 + w) : V{(T)0, (T)0}; };
                auto dst = [&](int n, int w, V v) {
                    if (w < wv) st_g(gc + (long long)n * NH + w, v);
                };
                if (c0 != 0) {
                    ColFFT::run(src, dst, ctile, sty);
                } else {
                    ToSmem ts;
                    ColFFT::run(src, ts, ctile, sty);
                    __syncthreads();
                    for (int q = threadIdx.x; q < NY * WY; q += NT) {
                        const int n = q / WY, w = q % WY;
                        if (w >= wv) continue;
                        const V c1 = ctile[ColL::idx(n, w)];
                        if (w == 0) {
                            const V c2 = c_conj(ctile[ColL::idx((NY - n) % NY, 0)]);
                            st_g(g + (long long)n * NH, c_scale(c_add(c1, c2), hf));
                            st_g(g + (long long)n * NH + M, c_rot<true>(c_scale(c_sub(c1, c2), hf)));
                        } else {
                            st_g(gc + (long long)n * NH + w, c1);
                        }
                    }
                }
            }
            cluster.sync();  // every peer is done reading the slices
        } else {
            // ---- y columns: global -> y inverse FFT -> owners' slices (DSMEM) ----
            for (int t = crank; t < ntiles_y; t += K) {
                const int c0 = t * WY;
                const int wv = min(WY, M - c0);
                V *gc = g + c0;
                auto src = [&](int n, int w) -> V {
                    return (w < wv) ? ld_g(gc + (long long)n * NH + w) : V{(T)0, (T)0};
                };
                auto dst = [&](int n, int w, V v) {
                    if (w < wv) *at(n, c0 + w) = v;
                };
                if (c0 == 0) {
                    // Hermitian projection of bins kz=0 and kz=m along y, packed into column 0
                    __syncthreads();
                    for (int n = threadIdx.x; n <= NY / 2; n += NT) {
                        const int n2 = (NY - n) % NY;
                        const V a1 = ld_g(g + (long long)n * NH), a2 = ld_g(g + (long long)n2 * NH);
                        const V b1 = ld_g(g + (long long)n * NH + M), b2 = ld_g(g + (long long)n2 * NH + M);
                        const V ha = c_scale(c_add(a1, c_conj(a2)), hf);
                        const V hb = c_scale(c_add(b1, c_conj(b2)), hf);
                        st_g(g + (long long)n * NH, V{ha.x - hb.y, ha.y + hb.x});
                        if (n2 != n) st_g(g + (long long)n2 * NH, V{ha.x + hb.y, -ha.y + hb.x});
                    }
                    __syncthreads();
                }
                ColFFT::run(src, dst, ctile, sty);
            }
            cluster.sync();
            // ---- z rows: slice -> pre-process -> C2R -> global ----
            for (int lr = wid * RW; lr < SLICE; lr += (NT / 32) * RW) {
                V *gr = gs + (long long)lr * NH;
                V *wt = slice + lr * SliceL::PITCH;
                for (int w = 0; w < RW; ++w) {
                    for (int k = lane; k < HALF; k += 32) {
                        const int km = M - k;
                        V xk, xmk;
                        if (k == 0) {
                            const V pk = wt[SliceL::idx(0, w)];
                            xk = V{pk.x, (T)0};
                            xmk = V{pk.y, (T)0};
                        } else {
                            xk = wt[SliceL::idx(k, w)];
                            xmk = wt[SliceL::idx(km, w)];
                        }
                        const V cm = c_conj(xmk);
                        const V sv = c_add(xk, cm);
                        const V pk = c_rot<false>(c_mulc(c_sub(xk, cm), unp[k]));
                        wt[SliceL::idx(k, w)] = c_add(sv, pk);
                        if (k != 0 && km != k) wt[SliceL::idx(km, w)] = c_conj(c_sub(sv, pk));
                    }
                }
                auto dst = [&](int n, int w, V v) { st_g(gr + (long long)w * NH + n, v); };
                FromSmem fs;
                RowFFT::run(fs, dst, wt, stz);
                if (lane < RW) st_g(gr + (long long)lane * NH + M, V{(T)0, (T)0});
            }
            cluster.sync();  // slices free for the next plane's columns
        }
    }
}

}  // namespace fast
}  // namespace gpufft

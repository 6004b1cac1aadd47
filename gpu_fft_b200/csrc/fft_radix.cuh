// fft_radix.cuh — complex arithmetic and register-resident small DFTs.
//
// Every length-R DFT here computes y[k] = sum_j x[j] * exp(s*2*pi*i*j*k/R)
// with s = -1 (FWD) or +1 (inverse), unscaled — the convention of the
// transforms GPU_FFT calls (cuFFT FORWARD/INVERSE, FFT_R2C.cu:69, FFT_C2R.cu:45).
// Radix 2, 4, 8, 9 and 16 are hand-factored (4 = 2x2, 8 = 2x4, 9 = 3x3,
// 16 = 4x4 with constant twiddles); odd primes 3..13 use the symmetric pair form
//   y[k] = x0 + sum_{j<=(R-1)/2} cos(2pi jk/R)(x_j + x_{R-j})  -/+  i sin(2pi jk/R)(x_j - x_{R-j}).
// The trigonometric constants are the mathematical values written out to
// 25 significant digits and rounded by the compiler to the storage type.
#pragma once
#include <type_traits>
#include <cuda_runtime.h>
#include <stdint.h>

namespace gpufft {

template <typename T> struct CxOf;
template <> struct CxOf<float> { using type = float2; };
template <> struct CxOf<double> { using type = double2; };
template <typename T> using cx_t = typename CxOf<T>::type;

template <typename V> __device__ __forceinline__ V c_add(V a, V b) { return V{a.x + b.x, a.y + b.y}; }
template <typename V> __device__ __forceinline__ V c_sub(V a, V b) { return V{a.x - b.x, a.y - b.y}; }
// FP32 complex add / subtract as one packed f32x2 operation (sm_100): the
// same IEEE sums as the two scalar ones, half the instructions
__device__ __forceinline__ unsigned long long f2_bits(float2 v) {
    unsigned long long u;
    asm("mov.b64 %0, {%1, %2};" : "=l"(u) : "f"(v.x), "f"(v.y));
    return u;
}
__device__ __forceinline__ float2 bits_f2(unsigned long long u) {
    float2 v;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(u));
    return v;
}
__device__ __forceinline__ float2 c_add(float2 a, float2 b) {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)));
    return bits_f2(d);
}
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)));
    return bits_f2(d);
}
template <typename V> __device__ __forceinline__ V c_mul(V a, V b) {
    return V{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// a * conj(b)
template <typename V> __device__ __forceinline__ V c_mulc(V a, V b) {
    return V{a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
template <typename V> __device__ __forceinline__ V c_conj(V a) { return V{a.x, -a.y}; }
template <typename V, typename T> __device__ __forceinline__ V c_scale(V a, T s) { return V{a.x * s, a.y * s}; }
// multiply by -i (forward) or +i (inverse)
template <bool FWD, typename V> __device__ __forceinline__ V c_rot(V a) {
    return FWD ? V{a.y, -a.x} : V{-a.y, a.x};
}
// twiddle multiply by table entry w = exp(-2 pi i e/N): forward uses w, inverse conj(w)
template <bool FWD, typename V> __device__ __forceinline__ V c_tw(V a, V w) {
    return FWD ? c_mul(a, w) : c_mulc(a, w);
}

// ---------------------------------------------------------------------------
// trigonometric constants cos/sin(2*pi*m/R)
// ---------------------------------------------------------------------------
template <int R> struct Trig;
template <> struct Trig<3> {
    static __host__ __device__ constexpr double c(int i) {
        constexpr double t[3] = {1.0, -0.5, -0.5};
        return t[i];
    }
    static __host__ __device__ constexpr double s(int i) {
        constexpr double t[3] = {0.0, 0.8660254037844386467637232, -0.8660254037844386467637232};
        return t[i];
    }
};
template <> struct Trig<5> {
    static __host__ __device__ constexpr double c(int i) {
        constexpr double t[5] = {1.0, 0.3090169943749474241022934, -0.8090169943749474241022934,
                                    -0.8090169943749474241022934, 0.3090169943749474241022934};
        return t[i];
    }
    static __host__ __device__ constexpr double s(int i) {
        constexpr double t[5] = {0.0, 0.9510565162951535721164393, 0.587785252292473129168706,
                                    -0.587785252292473129168706, -0.9510565162951535721164393};
        return t[i];
    }
};
template <> struct Trig<7> {
    static __host__ __device__ constexpr double c(int i) {
        constexpr double t[7] = {1.0, 0.6234898018587335305250049, -0.2225209339563144042889026,
                                    -0.9009688679024191262361023, -0.9009688679024191262361023,
                                    -0.2225209339563144042889026, 0.6234898018587335305250049};
        return t[i];
    }
    static __host__ __device__ constexpr double s(int i) {
        constexpr double t[7] = {0.0, 0.7818314824680298087084445, 0.9749279121818236070181317,
                                    0.4338837391175581204757683, -0.4338837391175581204757683,
                                    -0.9749279121818236070181317, -0.7818314824680298087084445};
        return t[i];
    }
};
template <> struct Trig<11> {
    static __host__ __device__ constexpr double c(int i) {
        constexpr double t[11] = {1.0, 0.8412535328311811688618116, 0.4154150130018864255292741,
                                     -0.1423148382732851404437927, -0.6548607339452850640569251,
                                     -0.9594929736144973898903681, -0.9594929736144973898903681,
                                     -0.6548607339452850640569251, -0.1423148382732851404437927,
                                     0.4154150130018864255292741, 0.8412535328311811688618116};
        return t[i];
    }
    static __host__ __device__ constexpr double s(int i) {
        constexpr double t[11] = {0.0, 0.540640817455597582107636, 0.9096319953545183714117154,
                                     0.989821441880932732376092, 0.7557495743542582837740358,
                                     0.2817325568414296977114179, -0.2817325568414296977114179,
                                     -0.7557495743542582837740358, -0.989821441880932732376092,
                                     -0.9096319953545183714117154, -0.540640817455597582107636};
        return t[i];
    }
};
template <> struct Trig<13> {
    static __host__ __device__ constexpr double c(int i) {
        constexpr double t[13] = {1.0, 0.8854560256532098959003755, 0.5680647467311558025118076,
                                     0.1205366802553230533490677, -0.3546048870425356259696379,
                                     -0.7485107481711010986346306, -0.9709418174260520271569823,
                                     -0.9709418174260520271569823, -0.7485107481711010986346306,
                                     -0.3546048870425356259696379, 0.1205366802553230533490677,
                                     0.5680647467311558025118076, 0.8854560256532098959003755};
        return t[i];
    }
    static __host__ __device__ constexpr double s(int i) {
        constexpr double t[13] = {0.0, 0.4647231720437685456560153, 0.8229838658936563945796174,
                                     0.9927088740980539928007516, 0.9350162426854148234397846,
                                     0.6631226582407952023767855, 0.2393156642875577671487537,
                                     -0.2393156642875577671487537, -0.6631226582407952023767855,
                                     -0.9350162426854148234397846, -0.9927088740980539928007516,
                                     -0.8229838658936563945796174, -0.4647231720437685456560153};
        return t[i];
    }
};

// cos/sin(2*pi*m/9), m = 0..8 (twiddles inside the radix-9 DFT)
struct Trig9 {
    static __host__ __device__ constexpr double c(int i) {
        constexpr double t[9] = {1.0, 0.7660444431189780352023927, 0.1736481776669303488517166, -0.5,
                                 -0.9396926207859083840541093, -0.9396926207859083840541093, -0.5,
                                 0.1736481776669303488517166, 0.7660444431189780352023927};
        return t[i];
    }
    static __host__ __device__ constexpr double s(int i) {
        constexpr double t[9] = {0.0, 0.6427876096865393263226434, 0.984807753012208059366743,
                                 0.8660254037844386467637232, 0.3420201433256687330440996,
                                 -0.3420201433256687330440996, -0.8660254037844386467637232,
                                 -0.984807753012208059366743, -0.6427876096865393263226434};
        return t[i];
    }
};

// cos/sin(2*pi*m/16), m = 0..15
struct Trig16 {
    static __host__ __device__ constexpr double c(int i) {
        constexpr double t[16] = {1.0, 0.9238795325112867561281832, 0.7071067811865475244008444,
                                     0.38268343236508977172846, 0.0, -0.38268343236508977172846,
                                     -0.7071067811865475244008444, -0.9238795325112867561281832, -1.0,
                                     -0.9238795325112867561281832, -0.7071067811865475244008444,
                                     -0.38268343236508977172846, 0.0, 0.38268343236508977172846,
                                     0.7071067811865475244008444, 0.9238795325112867561281832};
        return t[i];
    }
    static __host__ __device__ constexpr double s(int i) {
        constexpr double t[16] = {0.0, 0.38268343236508977172846, 0.7071067811865475244008444,
                                     0.9238795325112867561281832, 1.0, 0.9238795325112867561281832,
                                     0.7071067811865475244008444, 0.38268343236508977172846, 0.0,
                                     -0.38268343236508977172846, -0.7071067811865475244008444,
                                     -0.9238795325112867561281832, -1.0, -0.9238795325112867561281832,
                                     -0.7071067811865475244008444, -0.38268343236508977172846};
        return t[i];
    }
};

// x * exp(s*2*pi*i*m/16) for compile-time m
template <bool FWD, int M, typename V> __device__ __forceinline__ V tw16(V a) {
    using T = decltype(a.x);
    constexpr int m = M & 15;
    if constexpr (m == 0) return a;
    else if constexpr (m == 4) return c_rot<FWD>(a);
    else if constexpr (m == 8) return V{-a.x, -a.y};
    else if constexpr (m == 12) return c_rot<!FWD>(a);
    else {
        const T c = (T)Trig16::c(m);
        const T s = FWD ? -(T)Trig16::s(m) : (T)Trig16::s(m);
        return V{a.x * c - a.y * s, a.x * s + a.y * c};
    }
}

// ---------------------------------------------------------------------------
// DFTs in registers, in place on x[0..R)
// ---------------------------------------------------------------------------
template <bool FWD, typename V> __device__ __forceinline__ void dft2(V &a, V &b) {
    V t = a;
    a = c_add(t, b);
    b = c_sub(t, b);
}

template <bool FWD, typename V> __device__ __forceinline__ void dft4(V &x0, V &x1, V &x2, V &x3) {
    V t0 = c_add(x0, x2), t1 = c_sub(x0, x2), t2 = c_add(x1, x3);
    x0 = c_add(t0, t2);
    x2 = c_sub(t0, t2);
    if constexpr (std::is_same<V, float2>::value) {
        // t1 -/+ i d with the rotation folded into scalar adds (a packed add
        // would first have to build the swapped pair)
        const V d = c_sub(x1, x3);
        x1 = FWD ? V{t1.x + d.y, t1.y - d.x} : V{t1.x - d.y, t1.y + d.x};
        x3 = FWD ? V{t1.x - d.y, t1.y + d.x} : V{t1.x + d.y, t1.y - d.x};
    } else {
        const V t3 = c_rot<FWD>(c_sub(x1, x3));
        x1 = c_add(t1, t3);
        x3 = c_sub(t1, t3);
    }
}

// length-3 DFT in place: y0 = a+b+c, y1,2 = a - (b+c)/2 -/+ i (sqrt3/2)(b-c) (forward)
template <bool FWD, typename V> __device__ __forceinline__ void dft3(V &a, V &b, V &c) {
    using T = decltype(a.x);
    const T h = (T)0.5, s3 = (T)0.8660254037844386467637232;
    const V sp = c_add(b, c), sm = c_sub(b, c);
    const V m = V{a.x - h * sp.x, a.y - h * sp.y};
    const V r = V{s3 * sm.x, s3 * sm.y};  // multiplied by -i (forward) or +i below
    a = c_add(a, sp);
    const V ir = c_rot<FWD>(r);
    b = c_add(m, ir);
    c = c_sub(m, ir);
}

// x * exp(s*2*pi*i*m/9) for compile-time m (s = -1 forward, +1 inverse)
template <bool FWD, int M, typename V> __device__ __forceinline__ V tw9(V a) {
    using T = decltype(a.x);
    constexpr int m = M % 9;
    if constexpr (m == 0) return a;
    else {
        const T c = (T)Trig9::c(m);
        const T s = FWD ? -(T)Trig9::s(m) : (T)Trig9::s(m);
        return V{a.x * c - a.y * s, a.x * s + a.y * c};
    }
}

template <int R, bool FWD, typename V> struct Dft;

template <bool FWD, typename V> struct Dft<2, FWD, V> {
    static __device__ __forceinline__ void run(V *x) { dft2<FWD>(x[0], x[1]); }
};
template <bool FWD, typename V> struct Dft<4, FWD, V> {
    static __device__ __forceinline__ void run(V *x) { dft4<FWD>(x[0], x[1], x[2], x[3]); }
};
template <bool FWD, typename V> struct Dft<8, FWD, V> {
    static __device__ __forceinline__ void run(V *x) {
        // even/odd split: E = DFT4(x0,x2,x4,x6), O = DFT4(x1,x3,x5,x7); y[k] = E[k] + w8^k O[k]
        dft4<FWD>(x[0], x[2], x[4], x[6]);
        dft4<FWD>(x[1], x[3], x[5], x[7]);
        V o1 = tw16<FWD, 2>(x[3]), o2 = tw16<FWD, 4>(x[5]), o3 = tw16<FWD, 6>(x[7]);
        V e0 = x[0], e1 = x[2], e2 = x[4], e3 = x[6], o0 = x[1];
        x[0] = c_add(e0, o0);
        x[4] = c_sub(e0, o0);
        x[1] = c_add(e1, o1);
        x[5] = c_sub(e1, o1);
        x[2] = c_add(e2, o2);
        x[6] = c_sub(e2, o2);
        x[3] = c_add(e3, o3);
        x[7] = c_sub(e3, o3);
    }
};
template <bool FWD, typename V> struct Dft<16, FWD, V> {
    static __device__ __forceinline__ void run(V *x) {
        // F_j = DFT4 over x[j + 4m]; twiddle w16^(j*k1); DFT4 over j -> y[k1 + 4*k2]
        dft4<FWD>(x[0], x[4], x[8], x[12]);
        dft4<FWD>(x[1], x[5], x[9], x[13]);
        dft4<FWD>(x[2], x[6], x[10], x[14]);
        dft4<FWD>(x[3], x[7], x[11], x[15]);
        x[5] = tw16<FWD, 1>(x[5]);
        x[9] = tw16<FWD, 2>(x[9]);
        x[13] = tw16<FWD, 3>(x[13]);
        x[6] = tw16<FWD, 2>(x[6]);
        x[10] = tw16<FWD, 4>(x[10]);
        x[14] = tw16<FWD, 6>(x[14]);
        x[7] = tw16<FWD, 3>(x[7]);
        x[11] = tw16<FWD, 6>(x[11]);
        x[15] = tw16<FWD, 9>(x[15]);
        // now F_j[k1] sits at x[j + 4*k1]; DFT4 over j for each k1
        dft4<FWD>(x[0], x[1], x[2], x[3]);
        dft4<FWD>(x[4], x[5], x[6], x[7]);
        dft4<FWD>(x[8], x[9], x[10], x[11]);
        dft4<FWD>(x[12], x[13], x[14], x[15]);
        // y[k1 + 4*k2] is at x[4*k1 + k2]: transpose the 4x4 index
        V t;
        t = x[1]; x[1] = x[4]; x[4] = t;
        t = x[2]; x[2] = x[8]; x[8] = t;
        t = x[3]; x[3] = x[12]; x[12] = t;
        t = x[6]; x[6] = x[9]; x[9] = t;
        t = x[7]; x[7] = x[13]; x[13] = t;
        t = x[11]; x[11] = x[14]; x[14] = t;
    }
};

// radix 9 = 3 x 3: DFT3 over x[j + 3m] for j = 0..2, twiddle w9^(j*k1),
// DFT3 over j, then the 3x3 index transpose (as radix 16 = 4 x 4)
template <bool FWD, typename V> struct Dft<9, FWD, V> {
    static __device__ __forceinline__ void run(V *x) {
        dft3<FWD>(x[0], x[3], x[6]);
        dft3<FWD>(x[1], x[4], x[7]);
        dft3<FWD>(x[2], x[5], x[8]);
        // F_j[k1] sits at x[j + 3*k1]
        x[4] = tw9<FWD, 1>(x[4]);
        x[7] = tw9<FWD, 2>(x[7]);
        x[5] = tw9<FWD, 2>(x[5]);
        x[8] = tw9<FWD, 4>(x[8]);
        dft3<FWD>(x[0], x[1], x[2]);
        dft3<FWD>(x[3], x[4], x[5]);
        dft3<FWD>(x[6], x[7], x[8]);
        // y[k1 + 3*k2] is at x[3*k1 + k2]: transpose the 3x3 index
        V t;
        t = x[1]; x[1] = x[3]; x[3] = t;
        t = x[2]; x[2] = x[6]; x[6] = t;
        t = x[5]; x[5] = x[7]; x[7] = t;
    }
};

// odd prime R: pair form
template <int R, bool FWD, typename V> struct DftOdd {
    static __device__ __forceinline__ void run(V *x) {
        using T = decltype(x[0].x);
        constexpr int H = (R - 1) / 2;
        V sp[H + 1], sm[H + 1];
#pragma unroll
        for (int j = 1; j <= H; ++j) {
            sp[j] = c_add(x[j], x[R - j]);
            sm[j] = c_sub(x[j], x[R - j]);
        }
        V y0 = x[0];
#pragma unroll
        for (int j = 1; j <= H; ++j) y0 = c_add(y0, sp[j]);
        V out[R];
        out[0] = y0;
#pragma unroll
        for (int k = 1; k <= H; ++k) {
            V a = x[0], b = V{(T)0, (T)0};
#pragma unroll
            for (int j = 1; j <= H; ++j) {
                const T c = (T)Trig<R>::c((j * k) % R);
                const T s = (T)Trig<R>::s((j * k) % R);
                a.x += c * sp[j].x;
                a.y += c * sp[j].y;
                b.x += s * sm[j].x;
                b.y += s * sm[j].y;
            }
            // forward: y_k = a - i b, y_{R-k} = a + i b ; inverse swaps the signs
            V mib = V{b.y, -b.x};
            out[k] = FWD ? c_add(a, mib) : c_sub(a, mib);
            out[R - k] = FWD ? c_sub(a, mib) : c_add(a, mib);
        }
#pragma unroll
        for (int k = 0; k < R; ++k) x[k] = out[k];
    }
};
template <bool FWD, typename V> struct Dft<3, FWD, V> : DftOdd<3, FWD, V> {};
// radix 15 = 3 x 5 by the prime-factor (Good-Thomas) map, no twiddles:
// input n = (5 n1 + 3 n2) mod 15, output k = (10 k1 + 6 k2) mod 15; DFT3 over
// n1 for each n2, then DFT5 over n2 for each k1
template <bool FWD, typename V> struct Dft<15, FWD, V> {
    static __device__ __forceinline__ void run(V *x) {
        V y[5][3];
#pragma unroll
        for (int n2 = 0; n2 < 5; ++n2) {
            V a = x[(3 * n2) % 15], b = x[(5 + 3 * n2) % 15], c = x[(10 + 3 * n2) % 15];
            dft3<FWD>(a, b, c);
            y[n2][0] = a;
            y[n2][1] = b;
            y[n2][2] = c;
        }
#pragma unroll
        for (int k1 = 0; k1 < 3; ++k1) {
            V b[5];
#pragma unroll
            for (int n2 = 0; n2 < 5; ++n2) b[n2] = y[n2][k1];
            DftOdd<5, FWD, V>::run(b);
#pragma unroll
            for (int k2 = 0; k2 < 5; ++k2) x[(10 * k1 + 6 * k2) % 15] = b[k2];
        }
    }
};
template <bool FWD, typename V> struct Dft<5, FWD, V> : DftOdd<5, FWD, V> {};
template <bool FWD, typename V> struct Dft<7, FWD, V> : DftOdd<7, FWD, V> {};
template <bool FWD, typename V> struct Dft<11, FWD, V> : DftOdd<11, FWD, V> {};
template <bool FWD, typename V> struct Dft<13, FWD, V> : DftOdd<13, FWD, V> {};

// ---------------------------------------------------------------------------
// Division by a runtime-invariant divisor: q = (umulhi(n, m) + n) >> s for
// 0 <= n < 2^31 (Granlund & Montgomery, "Division by invariant integers
// using multiplication", PLDI 1994, round-up variant).
// ---------------------------------------------------------------------------
struct FastDiv {
    uint32_t d, m, s;
};

__host__ __device__ inline FastDiv make_fastdiv(uint32_t d) {
    FastDiv f;
    f.d = d;
    if (d <= 1) {
        f.m = 0;
        f.s = 0;
        return f;
    }
    uint32_t s = 0;
    while ((1ull << s) < d) ++s;
    f.s = s;
    f.m = (uint32_t)(((1ull << 32) * ((1ull << s) - d)) / d + 1);
    return f;
}

__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv &f) {
    return f.d <= 1 ? n : ((__umulhi(n, f.m) + n) >> f.s);
}

}  // namespace gpufft

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

#include <type_traits>

#include "fft_kernels.cuh"
#include "fft_radix.cuh"

namespace gpufft {
namespace fast {

// ---------------------------------------------------------------------------
// compile-time radix lists (same rule as the host factorize(): the power of
// two split into balanced stages of at most 16, then odd primes 3..13).
// VARIANT 1 prefers radix-16 stages for the power-of-two part.
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
        if (variant == 1) {
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

// shared-memory layouts of a tile of W sequences of length N
//  COLS: element (n, w) at n*W + w             (columns contiguous in w)
//  ROWS: element (n, w) at w*PITCH + n + n/G   (one pad slot per G elements,
//        G = 128 bytes / sizeof(complex), so strided stage writes stay
//        conflict-free); PITCH keeps rows apart by an odd number of slots
enum Layout { COLS = 0, ROWS = 1 };

template <typename T, int N, int W, int LAYOUT>
struct TileLayout {
    using V = cx_t<T>;
    static constexpr int G = 128 / (int)sizeof(V);
    static constexpr int ROWLEN = N + (N + G - 1) / G;
    static constexpr int PITCH = (ROWLEN % 2 == 0) ? ROWLEN + 1 : ROWLEN;
    static constexpr int ELEMS = LAYOUT == COLS ? N * W : W * PITCH;
    static __device__ __forceinline__ int idx(int n, int w) {
        if constexpr (LAYOUT == COLS)
            return n * W + w;
        else
            return w * PITCH + n + n / G;
    }
};

// Sources / sinks of a tile FFT.  A Global functor is called as v = src(n, w)
// and dst(n, w, v); FromSmem / ToSmem mean the first stage reads, or the last
// stage writes, the shared tile itself (natural order).
struct FromSmem {};
struct ToSmem {};

template <typename T, int N, int W, int NT, bool FWD, int LAYOUT, int TABMUL = 1, int VARIANT = 0>
struct TileFFT {
    using V = cx_t<T>;
    using L = TileLayout<T, N, W, LAYOUT>;
    static constexpr Fac F = factor(N, VARIANT);
    static constexpr int NS = F.n;
    static_assert(NS >= 0, "length must factor into 2,3,5,7,11,13");

    template <int S, class Src, class Dst>
    static __device__ __forceinline__ void stage(Src &src, Dst &dst, V *sm, const V *tw) {
        constexpr int R = F.r[S];
        constexpr int p = fac_prod(F, S);
        constexpr int nb = N / R;
        constexpr int items = nb * W;
        constexpr int C = (items + NT - 1) / NT;
        constexpr bool first = (S == 0);
        constexpr bool last = (S == NS - 1);
        constexpr bool src_smem = !first || std::is_same<Src, FromSmem>::value;
        constexpr bool dst_smem = !last || std::is_same<Dst, ToSmem>::value;
        const int tid = threadIdx.x;
        V v[C][R];
        int ii[C], ww[C];
        if (src_smem) __syncthreads();  // the previous writer of the tile is done
#pragma unroll
        for (int m = 0; m < C; ++m) {
            const int q = tid + m * NT;
            if (items % NT == 0 || q < items) {
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
                    if constexpr (src_smem)
                        v[m][j] = sm[L::idx(i + j * nb, w)];
                    else
                        v[m][j] = src(i + j * nb, w);
                }
            }
        }
        if (dst_smem) __syncthreads();  // every reader of the tile is done before it is overwritten
#pragma unroll
        for (int m = 0; m < C; ++m) {
            const int q = tid + m * NT;
            if (items % NT == 0 || q < items) {
                const int i = ii[m], w = ww[m];
                const int k = i % p;
                if constexpr (p > 1) {
                    constexpr int step = TABMUL * (N / (p * R));
#pragma unroll
                    for (int j = 1; j < R; ++j) v[m][j] = c_tw<FWD>(v[m][j], tw[j * k * step]);
                }
                Dft<R, FWD, V>::run(v[m]);
                if constexpr (last) {
                    // last stage: p = nb, k = i, output positions i + j*nb
#pragma unroll
                    for (int j = 0; j < R; ++j) {
                        if constexpr (dst_smem)
                            sm[L::idx(i + j * nb, w)] = v[m][j];
                        else
                            dst(i + j * nb, w, v[m][j]);
                    }
                } else {
                    const int o = (i - k) * R + k;
#pragma unroll
                    for (int j = 0; j < R; ++j) sm[L::idx(o + j * p, w)] = v[m][j];
                }
            }
        }
    }

    template <int S, class Src, class Dst>
    static __device__ __forceinline__ void stages(Src &src, Dst &dst, V *sm, const V *tw) {
        if constexpr (S < NS) {
            stage<S>(src, dst, sm, tw);
            stages<S + 1>(src, dst, sm, tw);
        }
    }

    // Runs the whole FFT.  With a Global source the tile buffer must be free
    // (the first stage synchronises before writing it); a ToSmem result is
    // complete only after the caller's next __syncthreads().
    template <class Src, class Dst>
    static __device__ __forceinline__ void run(Src &src, Dst &dst, V *sm, const V *tw) {
        if constexpr (NS == 0) {
            // length 1: identity (copy)
            if constexpr (std::is_same<Src, FromSmem>::value) __syncthreads();
            for (int q = threadIdx.x; q < W; q += NT) {
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
            stages<0>(src, dst, sm, tw);
        }
    }
};

// ---------------------------------------------------------------------------
// Pass B: x-axis FFT over column tiles (stride Ny*Nh), compile-time Nx
// ---------------------------------------------------------------------------
template <typename T, int NX, int W, int NT, bool FWD, int VARIANT, int MINB>
__global__ void __launch_bounds__(NT, MINB) pass_b_fast(PassBParams P) {
    using V = cx_t<T>;
    using FFT = TileFFT<T, NX, W, NT, FWD, COLS, 1, VARIANT>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tw = reinterpret_cast<V *>(smem_raw);
    V *tile = tw + NX;
    for (int q = threadIdx.x; q < NX; q += NT) tw[q] = reinterpret_cast<const V *>(P.twx)[q];
    // (the first stage's barrier orders these writes before any twiddle read)
    V *base = reinterpret_cast<V *>(P.data);
    const long long ncols = P.ncols;
    for (long long t = blockIdx.x; t < P.ntiles; t += gridDim.x) {
        const long long c0 = t * W;
        const int wv = (int)min((long long)W, ncols - c0);
        V *g = base + c0;
        auto src = [&](int n, int w) -> V {
            return (w < wv) ? ld_g(g + (long long)n * ncols + w) : V{(T)0, (T)0};
        };
        auto dst = [&](int n, int w, V v) {
            if (w < wv) st_g(g + (long long)n * ncols + w, v);
        };
        FFT::run(src, dst, tile, tw);
    }
}

// ---------------------------------------------------------------------------
// Pass A: per x-plane z-axis R2C/C2R (rows) and y-axis C2C (columns)
// ---------------------------------------------------------------------------
template <typename T, int NY, int M, int WZ, int WY, int NT, int VY, int VZ>
struct PassAShape {
    using V = cx_t<T>;
    using RowL = TileLayout<T, M, WZ, ROWS>;
    using ColL = TileLayout<T, NY, WY, COLS>;
    static constexpr int TILE = RowL::ELEMS > ColL::ELEMS ? RowL::ELEMS : ColL::ELEMS;
    static constexpr size_t smem_bytes() { return (size_t)(2 * M + NY + TILE) * sizeof(V); }
};

template <typename T, int NY, int M, int WZ, int WY, int NT, bool FWD, int VY, int VZ, int MINB>
__global__ void __launch_bounds__(NT, MINB) pass_a_fast(PassAParams P) {
    using V = cx_t<T>;
    using Shape = PassAShape<T, NY, M, WZ, WY, NT, VY, VZ>;
    using RowFFT = TileFFT<T, M, WZ, NT, FWD, ROWS, 2, VZ>;
    using ColFFT = TileFFT<T, NY, WY, NT, FWD, COLS, 1, VY>;
    using RowL = typename RowFFT::L;
    using ColL = typename ColFFT::L;
    constexpr int NZ = 2 * M, NH = M + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *twz = reinterpret_cast<V *>(smem_raw);
    V *twy = twz + NZ;
    V *tile = twy + NY;
    for (int q = threadIdx.x; q < NZ; q += NT) twz[q] = reinterpret_cast<const V *>(P.twz)[q];
    for (int q = threadIdx.x; q < NY; q += NT) twy[q] = reinterpret_cast<const V *>(P.twy)[q];
    __syncthreads();

    const int K = P.K;
    const int crank = blockIdx.x % K;
    const int cid = blockIdx.x / K;
    const int ncl = gridDim.x / K;
    const int rows_per = (NY + K - 1) / K;
    const int rb = min(NY, crank * rows_per), re = min(NY, rb + rows_per);
    constexpr int ntiles_y = (M + WY - 1) / WY;
    V *base = reinterpret_cast<V *>(P.data);
    const T hf = (T)0.5;

    for (int plane = cid; plane < P.nx; plane += ncl) {
        V *g = base + (long long)plane * NY * NH;
        // ---------------- y columns (inverse: first) ----------------
        auto cols = [&](auto fwd_tag) {
            constexpr bool F = decltype(fwd_tag)::value;
            for (int t = crank; t < ntiles_y; t += K) {
                const int c0 = t * WY;
                const int wv = min(WY, M - c0);
                V *gc = g + c0;
                auto dst = [&](int n, int w, V v) {
                    if (w < wv) st_g(gc + (long long)n * NH + w, v);
                };
                if (c0 != 0) {
                    auto src = [&](int n, int w) -> V {
                        return (w < wv) ? ld_g(gc + (long long)n * NH + w) : V{(T)0, (T)0};
                    };
                    ColFFT::run(src, dst, tile, twy);
                } else if (F) {
                    // column 0 carries (bin 0) + i (bin m); split after the FFT
                    auto src = [&](int n, int w) -> V {
                        return (w < wv) ? ld_g(gc + (long long)n * NH + w) : V{(T)0, (T)0};
                    };
                    ToSmem ts;
                    ColFFT::run(src, ts, tile, twy);
                    __syncthreads();
                    for (int q = threadIdx.x; q < NY * WY; q += NT) {
                        const int n = q / WY, w = q % WY;
                        if (w >= wv) continue;
                        const V c1 = tile[ColL::idx(n, w)];
                        if (w == 0) {
                            const V c2 = c_conj(tile[ColL::idx((NY - n) % NY, 0)]);
                            st_g(g + (long long)n * NH, c_scale(c_add(c1, c2), hf));
                            st_g(g + (long long)n * NH + M, c_rot<true>(c_scale(c_sub(c1, c2), hf)));
                        } else {
                            st_g(gc + (long long)n * NH + w, c1);
                        }
                    }
                } else {
                    // inverse: Hermitian projection of bins kz=0 (a) and kz=m (b) along y,
                    // packed as a' + i b' into column 0 in place (each thread owns the
                    // pair of rows n, -n), then the plain column FFT
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
                    auto src = [&](int n, int w) -> V {
                        return (w < wv) ? ld_g(gc + (long long)n * NH + w) : V{(T)0, (T)0};
                    };
                    ColFFT::run(src, dst, tile, twy);
                }
            }
        };
        // ---------------- z rows ----------------
        auto rows_fwd = [&]() {
            for (int r0 = rb; r0 < re; r0 += WZ) {
                const int wv = min(WZ, re - r0);
                V *gr = g + (long long)r0 * NH;
                auto src = [&](int n, int w) -> V {
                    return (w < wv) ? ld_g(gr + (long long)w * NH + n) : V{(T)0, (T)0};
                };
                ToSmem ts;
                RowFFT::run(src, ts, tile, twz);
                __syncthreads();
                // unpack: X[k] = E + O, X[m-k] = conj(E - O), E = (Z[k] + conj Z[m-k])/2,
                // O = -i w^k (Z[k] - conj Z[m-k])/2, w = exp(-2 pi i/Nz); bins 0 and m packed in slot 0
                constexpr int HALF = M / 2 + 1;
                for (int q = threadIdx.x; q < HALF * WZ; q += NT) {
                    const int k = q % HALF, w = q / HALF;
                    if (w >= wv) continue;
                    const V a = tile[RowL::idx(k, w)];
                    const V b = c_conj(tile[RowL::idx(k == 0 ? 0 : M - k, w)]);
                    const V e = c_scale(c_add(a, b), hf);
                    const V d = c_scale(c_sub(a, b), hf);
                    const V o = c_rot<true>(c_mul(d, twz[k]));
                    const V xa = c_add(e, o), xb = c_conj(c_sub(e, o));
                    V *row = gr + (long long)w * NH;
                    if (k == 0) {
                        st_g(row, V{xa.x, xb.x});
                    } else {
                        st_g(row + k, xa);
                        if (M - k != k) st_g(row + M - k, xb);
                    }
                }
            }
        };
        auto rows_inv = [&]() {
            for (int r0 = rb; r0 < re; r0 += WZ) {
                const int wv = min(WZ, re - r0);
                V *gr = g + (long long)r0 * NH;
                // pre-process: Z[k] = S + Pk, Z[m-k] = conj(S - Pk), S = X[k] + conj X[m-k],
                // Pk = i conj(w^k)(X[k] - conj X[m-k]); slot 0 holds (Re X0, Re Xm)
                constexpr int HALF = M / 2 + 1;
                __syncthreads();
                for (int q = threadIdx.x; q < HALF * WZ; q += NT) {
                    const int k = q % HALF, w = q / HALF;
                    V za = V{(T)0, (T)0}, zb = V{(T)0, (T)0};
                    if (w < wv) {
                        const V *row = gr + (long long)w * NH;
                        V xk, xmk;
                        if (k == 0) {
                            const V pk = ld_g(row);
                            xk = V{pk.x, (T)0};
                            xmk = V{pk.y, (T)0};
                        } else {
                            xk = ld_g(row + k);
                            xmk = ld_g(row + M - k);
                        }
                        const V cm = c_conj(xmk);
                        const V s = c_add(xk, cm);
                        const V pk = c_rot<false>(c_mulc(c_sub(xk, cm), twz[k]));
                        za = c_add(s, pk);
                        zb = c_conj(c_sub(s, pk));
                    }
                    tile[RowL::idx(k, w)] = za;
                    if (k != 0 && M - k != k) tile[RowL::idx(M - k, w)] = zb;
                }
                auto dst = [&](int n, int w, V v) {
                    if (w < wv) st_g(gr + (long long)w * NH + n, v);
                };
                FromSmem fs;
                RowFFT::run(fs, dst, tile, twz);
                // slot m = padding cells of the real row: zero
                for (int q = threadIdx.x; q < wv; q += NT) st_g(gr + (long long)q * NH + M, V{(T)0, (T)0});
            }
        };
        if (FWD) {
            rows_fwd();
            cluster_barrier(K);
            cols(std::integral_constant<bool, true>{});
        } else {
            cols(std::integral_constant<bool, false>{});
            cluster_barrier(K);
            rows_inv();
        }
    }
}

}  // namespace fast
}  // namespace gpufft

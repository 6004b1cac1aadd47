// fft_kernels.cuh — the two passes of the in-place 3D R2C / C2R transform.
//
// Data layout (the reference's, GPU_FFT_TEST_SCRIPT/test.cu:110-135 and
// Readme.md:47-52 at procs=1): the real field is [Nx][Ny][2*Nh] reals with
// Nh = Nz/2+1 (row pitch Nz+2 for even Nz); the spectrum occupies the same
// bytes as [Nx][Ny][Nh] complex, kz fastest — exactly numpy.fft.rfftn's order.
//
// Forward (replaces GPU_FFT_R2C, FFT_R2C.cu:41-70):
//   Pass A, one cluster of K CTAs per x-plane:
//     phase 1  every row: Nz reals viewed as Nz/2 complex, Nz/2-point FFT, then
//              the real-to-complex unpack to Nh bins; rows written back in place.
//              Bins 0 and Nz/2 are real here; they are stored packed as one
//              complex value (Re X0, Re X_{Nz/2}) in slot 0.
//     cluster barrier (release/acquire): the plane now sits in L2.
//     phase 2  y-axis FFT of the Nz/2 columns 0..Nz/2-1 (column 0 packed);
//              column 0's result is split back into bins 0 and Nz/2.
//   Pass B: x-axis FFT of the Ny*Nh columns (stride Ny*Nh), in place.
// Inverse (replaces GPU_FFT_C2R, FFT_C2R.cu:41-70) runs the mirror image;
// the imaginary parts of bins kz=0 and kz=Nz/2 are dropped as numpy's irfftn
// drops them (a Hermitian projection of those two y-columns before the
// y-axis inverse, which packs them into one complex column).
//
// The reference's three permutation kernels (transpose.cu:41-91) and its
// self-copy (FFT_R2C.cu:62) compose to the identity at procs=1, so nothing
// here performs them.  HBM traffic: 2 reads + 2 writes of the field per
// transform, provided Pass A's in-flight planes stay resident in L2.
//
// Each 1D FFT is a self-sorting (Stockham) sequence of radix-R stages run on
// a shared-memory tile: stage with radix R after sub-length p reads butterfly
// i's inputs x[i + j*N/R], twiddles them by w_{pR}^{j*k} (k = i mod p),
// applies the register DFT_R and writes y_j to (i-k)*R + k + j*p.
#pragma once
#include <cooperative_groups.h>

#include "fft_radix.cuh"

namespace gpufft {

constexpr int kMaxStages = 24;
constexpr int kThreads = 256;  // threads per CTA for every pass

// One 1D FFT length as its stage list.  Twiddles come from a table of the
// roots exp(-2 pi i e / L) with L = n * tabmul; stage s uses table index
// j*k*twstep[s], twstep = tabmul * n / (p*R).
struct AxisPlan {
    int n;
    int nst;
    int radix[kMaxStages];
    int p[kMaxStages];
    int twstep[kMaxStages];
    FastDiv pdiv[kMaxStages];
};

struct PassAParams {
    void *data;          // field base (complex view)
    const void *twz;     // exp(-2 pi i e / Nz), e < Nz
    const void *twy;     // exp(-2 pi i e / Ny), e < Ny
    const void *stz;     // per-stage tables of the specialised kernels (fft_fast.cuh)
    const void *sty;
    int nx, ny, nz, nh, m;  // m = Nz/2
    int K;               // CTAs per cluster (per x-plane)
    // phase with rows (z axis): tile of wz rows, smem row pitch pz (odd)
    int wz, pz;
    FastDiv wzdiv, nhdiv;
    // phase with columns (y axis): tile of wy columns
    int wy;
    FastDiv wydiv;
    AxisPlan az;  // n = Nz/2, tabmul 2
    AxisPlan ay;  // n = Ny, tabmul 1
    int tile_elems;  // complex elements reserved for the tile
    // specialised kernels: 0 = both axes per plane (cluster barrier between),
    // 1 = z rows only, 2 = y columns only (the two halves of a split Pass A,
    // launched one after the other without clusters; K then only splits the
    // work of a plane between CTAs)
    int phases;
    // slab decomposition, exchange layout (the XCH kernels): the forward's
    // y-column results go to, and the inverse's y-column inputs come from,
    // chunk y / xch_nyl of xch at element (plane * xch_nyl + y % xch_nyl) * Nh
    // + kz -- the all-to-all's send/receive layout, so no pack or unpack copy
    void *xch;
    int xch_nyl;
    long long xch_chunk;  // complex elements per chunk
};

struct PassBParams {
    void *data;
    const void *twx;
    const void *stw;     // per-stage table of the specialised kernel (fft_fast.cuh)
    int nx;
    long long ncols;   // Ny * Nh
    int wx;
    FastDiv wxdiv;
    AxisPlan ax;
    long long ntiles;
    // Epilogue fused into the x pass (the last pass of R2C, the first of
    // C2R), on when epi != 0: every stored value times `scale`; with
    // `dealias` (R2C) modes outside the 2/3-rule box |kx| <= Nx/3,
    // |ky| <= Ny/3, kz <= Nz/3 are stored as zero.  ny, nh, nz decode a
    // column c = ky*Nh + kz.
    int epi, dealias;
    double scale;
    int ny, nh, nz;
    int *err;  // device flag raised by a kernel whose bounded wait ran out (or null)
};

// the x pass's store of value v at (kx, column), with the epilogue applied
template <typename V>
__device__ __forceinline__ V pass_b_epilogue(const PassBParams &P, V v, int kx, long long col) {
    using T = decltype(v.x);
    if (P.dealias) {
        const int c = (int)col;  // Ny*Nh < 2^31 (checked at plan time)
        const int ky = c / P.nh, kz = c - ky * P.nh;
        const int fx = min(kx, P.nx - kx), fy = min(ky, P.ny - ky);
        if (3 * fx > P.nx || 3 * fy > P.ny || 3 * kz > P.nz) return V{(T)0, (T)0};
    }
    const T s = (T)P.scale;
    return V{v.x * s, v.y * s};
}

// ---------------------------------------------------------------------------
// global memory access: L2-only loads (the plane written in phase 1 is read
// by other CTAs of the cluster in phase 2; bypassing L1 keeps that coherent)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 ld_g(const float2 *p) { return __ldcg(p); }
__device__ __forceinline__ double2 ld_g(const double2 *p) { return __ldcg(p); }
__device__ __forceinline__ void st_g(float2 *p, float2 v) { __stcg(p, v); }
__device__ __forceinline__ void st_g(double2 *p, double2 v) { __stcg(p, v); }

template <typename T> struct MaxE;
template <> struct MaxE<float> { static constexpr int value = 32; };
template <> struct MaxE<double> { static constexpr int value = 16; };

// ---------------------------------------------------------------------------
// one out-of-place Stockham stage between shared tiles; element (n, w) of a
// tile at s[n*sn + w*sw].  Each thread walks its butterflies one at a time,
// so only R complex values are live per thread whatever the radix.
// ---------------------------------------------------------------------------
template <typename T, int R, bool FWD>
__device__ __forceinline__ void stage(const cx_t<T> *__restrict__ src, cx_t<T> *__restrict__ dst, int sn, int sw,
                                      int W, const FastDiv &wdiv, int n, int p, const FastDiv &pdiv, int twstep,
                                      const cx_t<T> *tw) {
    using V = cx_t<T>;
    const int nb = n / R;
    const int items = nb * W;
    const int jstride = nb * sn, ostride = p * sn;
    for (int q = threadIdx.x; q < items; q += kThreads) {
        const int i = (int)fdiv((uint32_t)q, wdiv);
        const int w = q - i * W;
        const int ip = (int)fdiv((uint32_t)i, pdiv);
        const int k = i - ip * p;
        const V *in = src + i * sn + w * sw;
        V v[R];
#pragma unroll
        for (int j = 0; j < R; ++j) v[j] = in[j * jstride];
        if (p > 1) {
            const int e = k * twstep;
#pragma unroll
            for (int j = 1; j < R; ++j) v[j] = c_tw<FWD>(v[j], tw[j * e]);
        }
        Dft<R, FWD, V>::run(v);
        V *out = dst + (ip * p * R + k) * sn + w * sw;
#pragma unroll
        for (int j = 0; j < R; ++j) out[j * ostride] = v[j];
    }
}

// Runs all stages of `ax`, ping-ponging between a and b; returns the tile
// that holds the result.  Ends with a block barrier.
template <typename T, bool FWD>
__device__ __forceinline__ cx_t<T> *fft_tile(cx_t<T> *a, cx_t<T> *b, int sn, int sw, int W, const FastDiv &wdiv,
                                             const AxisPlan &ax, const cx_t<T> *tw) {
    for (int st = 0; st < ax.nst; ++st) {
        const int p = ax.p[st], tws = ax.twstep[st];
        const FastDiv pd = ax.pdiv[st];
        switch (ax.radix[st]) {
            case 2: stage<T, 2, FWD>(a, b, sn, sw, W, wdiv, ax.n, p, pd, tws, tw); break;
            case 3: stage<T, 3, FWD>(a, b, sn, sw, W, wdiv, ax.n, p, pd, tws, tw); break;
            case 4: stage<T, 4, FWD>(a, b, sn, sw, W, wdiv, ax.n, p, pd, tws, tw); break;
            case 5: stage<T, 5, FWD>(a, b, sn, sw, W, wdiv, ax.n, p, pd, tws, tw); break;
            case 7: stage<T, 7, FWD>(a, b, sn, sw, W, wdiv, ax.n, p, pd, tws, tw); break;
            case 8: stage<T, 8, FWD>(a, b, sn, sw, W, wdiv, ax.n, p, pd, tws, tw); break;
            case 9: stage<T, 9, FWD>(a, b, sn, sw, W, wdiv, ax.n, p, pd, tws, tw); break;
            case 11: stage<T, 11, FWD>(a, b, sn, sw, W, wdiv, ax.n, p, pd, tws, tw); break;
            case 13: stage<T, 13, FWD>(a, b, sn, sw, W, wdiv, ax.n, p, pd, tws, tw); break;
            case 16: stage<T, 16, FWD>(a, b, sn, sw, W, wdiv, ax.n, p, pd, tws, tw); break;
            default: break;  // the plan only emits the radices above
        }
        __syncthreads();
        cx_t<T> *t = a;
        a = b;
        b = t;
    }
    return a;
}

// ---------------------------------------------------------------------------
// column tiles: ncol columns starting at g, element (n, c) at g[n*gsn + c];
// tile columns [0, wv) valid; smem layout [n][W]
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void load_cols(cx_t<T> *s, const cx_t<T> *g, long long gsn, int n, int W,
                                          const FastDiv &wdiv, int wv) {
    using V = cx_t<T>;
    const int total = n * W;
    for (int q = threadIdx.x; q < total; q += kThreads) {
        const int r = (int)fdiv((uint32_t)q, wdiv);
        const int w = q - r * W;
        s[q] = (w < wv) ? ld_g(g + (long long)r * gsn + w) : V{(T)0, (T)0};
    }
}

template <typename T>
__device__ __forceinline__ void store_cols(const cx_t<T> *s, cx_t<T> *g, long long gsn, int n, int W,
                                           const FastDiv &wdiv, int wfirst, int wv) {
    const int total = n * W;
    for (int q = threadIdx.x; q < total; q += kThreads) {
        const int r = (int)fdiv((uint32_t)q, wdiv);
        const int w = q - r * W;
        if (w >= wfirst && w < wv) st_g(g + (long long)r * gsn + w, s[q]);
    }
}

// ---------------------------------------------------------------------------
// Pass A phases.  `ta` and `tb` are the two shared tiles.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void load_rows(const PassAParams &P, const cx_t<T> *src, cx_t<T> *tile, int wv) {
    using V = cx_t<T>;
    const int nh = P.nh, pz = P.pz;
    const int total = wv * nh;
    for (int q = threadIdx.x; q < total; q += kThreads) {
        const int r = (int)fdiv((uint32_t)q, P.nhdiv);
        tile[r * pz + (q - r * nh)] = ld_g(src + q);
    }
    for (int q = threadIdx.x + wv * pz; q < P.wz * pz; q += kThreads) tile[q] = V{(T)0, (T)0};
}

template <typename T>
__device__ __forceinline__ void store_rows(const PassAParams &P, cx_t<T> *dst, const cx_t<T> *tile, int wv) {
    const int nh = P.nh, pz = P.pz;
    const int total = wv * nh;
    for (int q = threadIdx.x; q < total; q += kThreads) {
        const int r = (int)fdiv((uint32_t)q, P.nhdiv);
        st_g(dst + q, tile[r * pz + (q - r * nh)]);
    }
}

// Forward rows [r0, r0+wv) of plane g: z-axis R2C.
template <typename T>
__device__ void rows_r2c(const PassAParams &P, cx_t<T> *g, cx_t<T> *ta, cx_t<T> *tb, const cx_t<T> *twz, int r0,
                         int wv) {
    using V = cx_t<T>;
    const int m = P.m, pz = P.pz, W = P.wz;
    load_rows<T>(P, g + (long long)r0 * P.nh, ta, wv);
    __syncthreads();
    // m-point complex FFT of every row: z[n] = x[2n] + i x[2n+1]
    V *res = fft_tile<T, true>(ta, tb, 1, pz, W, P.wzdiv, P.az, twz);
    V *out = (res == ta) ? tb : ta;
    // unpack: X[k] = E + O, X[m-k] = conj(E - O),  E = (Z[k] + conj Z[m-k])/2,
    // O = -i w^k (Z[k] - conj Z[m-k])/2,  w = exp(-2 pi i / Nz); k = 0..m/2.
    // Bins 0 and m are real: they go packed into slot 0 as (X0, Xm).
    const int items = (m / 2 + 1) * W;
    for (int q = threadIdx.x; q < items; q += kThreads) {
        const int k = (int)fdiv((uint32_t)q, P.wzdiv);
        const int w = q - k * W;
        const V a = res[w * pz + k];
        const V b = c_conj(res[w * pz + (k == 0 ? 0 : m - k)]);
        const T hf = (T)0.5;
        const V e = c_scale(c_add(a, b), hf);
        const V d = c_scale(c_sub(a, b), hf);
        const V o = c_rot<true>(c_mul(d, twz[k]));
        const V xa = c_add(e, o), xb = c_conj(c_sub(e, o));
        if (k == 0) {
            out[w * pz] = V{xa.x, xb.x};
            out[w * pz + m] = V{xb.x, (T)0};
        } else {
            out[w * pz + k] = xa;
            if (m - k != k) out[w * pz + m - k] = xb;
        }
    }
    __syncthreads();
    store_rows<T>(P, g + (long long)r0 * P.nh, out, wv);
    __syncthreads();
}

// Inverse rows: z-axis C2R.  Slot 0 holds (Re X0, Re X_m) packed by cols_y<inverse>.
template <typename T>
__device__ void rows_c2r(const PassAParams &P, cx_t<T> *g, cx_t<T> *ta, cx_t<T> *tb, const cx_t<T> *twz, int r0,
                         int wv) {
    using V = cx_t<T>;
    const int m = P.m, pz = P.pz, W = P.wz;
    load_rows<T>(P, g + (long long)r0 * P.nh, ta, wv);
    __syncthreads();
    // pre-process: Z[k] = S + Pk, Z[m-k] = conj(S - Pk), S = X[k] + conj X[m-k],
    // Pk = i conj(w^k) (X[k] - conj X[m-k]); k = 0..m/2 (Z[m] is not formed)
    const int items = (m / 2 + 1) * W;
    for (int q = threadIdx.x; q < items; q += kThreads) {
        const int k = (int)fdiv((uint32_t)q, P.wzdiv);
        const int w = q - k * W;
        V xk, xmk;
        if (k == 0) {
            const V pk = ta[w * pz];
            xk = V{pk.x, (T)0};
            xmk = V{pk.y, (T)0};
        } else {
            xk = ta[w * pz + k];
            xmk = ta[w * pz + m - k];
        }
        const V cm = c_conj(xmk);
        const V s = c_add(xk, cm);
        const V pk = c_rot<false>(c_mulc(c_sub(xk, cm), twz[k]));
        tb[w * pz + k] = c_add(s, pk);
        if (k != 0 && m - k != k) tb[w * pz + m - k] = c_conj(c_sub(s, pk));
    }
    __syncthreads();
    V *res = fft_tile<T, false>(tb, ta, 1, pz, W, P.wzdiv, P.az, twz);
    // slot m is padding of the real row (cells Nz, Nz+1): written as zero
    for (int q = threadIdx.x; q < W; q += kThreads) res[q * pz + m] = V{(T)0, (T)0};
    __syncthreads();
    store_rows<T>(P, g + (long long)r0 * P.nh, res, wv);
    __syncthreads();
}

// y-axis FFT of columns [c0, c0+wv) of plane g (columns 0..m-1; column 0 packed).
template <typename T, bool FWD>
__device__ void cols_y(const PassAParams &P, cx_t<T> *g, cx_t<T> *ta, cx_t<T> *tb, const cx_t<T> *twy, int c0,
                       int wv) {
    using V = cx_t<T>;
    const int ny = P.ny, nh = P.nh, W = P.wy, m = P.m;
    load_cols<T>(ta, g + c0, nh, ny, W, P.wydiv, wv);
    __syncthreads();
    if (!FWD && c0 == 0) {
        // Hermitian projection of bins kz=0 (a) and kz=m (b) along y, packed:
        // c[ky] = h(a)[ky] + i h(b)[ky], h(v)[ky] = (v[ky] + conj v[-ky]) / 2
        const int npair = ny / 2 + 1;
        for (int q = threadIdx.x; q < npair; q += kThreads) {
            const int k1 = q, k2 = (ny - q) % ny;
            const V a1 = ta[k1 * W], a2 = ta[k2 * W];
            const V b1 = ld_g(g + (long long)k1 * nh + m), b2 = ld_g(g + (long long)k2 * nh + m);
            const T hf = (T)0.5;
            const V ha = c_scale(c_add(a1, c_conj(a2)), hf);
            const V hb = c_scale(c_add(b1, c_conj(b2)), hf);
            // c[k1] = ha + i hb ; c[k2] = conj(ha) + i conj(hb)
            ta[k1 * W] = V{ha.x - hb.y, ha.y + hb.x};
            if (k2 != k1) ta[k2 * W] = V{ha.x + hb.y, -ha.y + hb.x};
        }
        __syncthreads();
    }
    V *res = fft_tile<T, FWD>(ta, tb, W, 1, W, P.wydiv, P.ay, twy);
    if (FWD && c0 == 0) {
        // column 0 carried a (bin 0) + i b (bin m), both real along y:
        // A[ky] = (C[ky] + conj C[-ky]) / 2,  B[ky] = -i (C[ky] - conj C[-ky]) / 2
        for (int q = threadIdx.x; q < ny; q += kThreads) {
            const V c1 = res[q * W], c2 = c_conj(res[((ny - q) % ny) * W]);
            const T hf = (T)0.5;
            const V A = c_scale(c_add(c1, c2), hf);
            const V B = c_rot<true>(c_scale(c_sub(c1, c2), hf));
            st_g(g + (long long)q * nh, A);
            st_g(g + (long long)q * nh + m, B);
        }
        store_cols<T>(res, g + c0, nh, ny, W, P.wydiv, 1, wv);
    } else {
        store_cols<T>(res, g + c0, nh, ny, W, P.wydiv, 0, wv);
    }
    __syncthreads();
}

__device__ __forceinline__ void cluster_barrier(int K) {
    if (K > 1) {
        cooperative_groups::this_cluster().sync();
    } else {
        __syncthreads();
    }
}

template <typename T, bool FWD>
__global__ void __launch_bounds__(kThreads) pass_a_kernel(PassAParams P) {
    using V = cx_t<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *twz = reinterpret_cast<V *>(smem_raw);
    V *twy = twz + P.nz;
    V *ta = twy + P.ny;
    V *tb = ta + P.tile_elems;
    for (int q = threadIdx.x; q < P.nz; q += kThreads) twz[q] = reinterpret_cast<const V *>(P.twz)[q];
    for (int q = threadIdx.x; q < P.ny; q += kThreads) twy[q] = reinterpret_cast<const V *>(P.twy)[q];
    __syncthreads();

    const int K = P.K;
    const int crank = blockIdx.x % K;
    const int cid = blockIdx.x / K;
    const int ncl = gridDim.x / K;
    const int rows_per = (P.ny + K - 1) / K;
    const int rb = min(P.ny, crank * rows_per), re = min(P.ny, rb + rows_per);
    const int ntiles_y = (P.m + P.wy - 1) / P.wy;
    V *base = reinterpret_cast<V *>(P.data);

    for (int plane = cid; plane < P.nx; plane += ncl) {
        V *g = base + (long long)plane * P.ny * P.nh;
        if (FWD) {
            for (int r0 = rb; r0 < re; r0 += P.wz) rows_r2c<T>(P, g, ta, tb, twz, r0, min(P.wz, re - r0));
            cluster_barrier(K);
            for (int t = crank; t < ntiles_y; t += K) {
                const int c0 = t * P.wy;
                cols_y<T, true>(P, g, ta, tb, twy, c0, min(P.wy, P.m - c0));
            }
        } else {
            for (int t = crank; t < ntiles_y; t += K) {
                const int c0 = t * P.wy;
                cols_y<T, false>(P, g, ta, tb, twy, c0, min(P.wy, P.m - c0));
            }
            cluster_barrier(K);
            for (int r0 = rb; r0 < re; r0 += P.wz) rows_c2r<T>(P, g, ta, tb, twz, r0, min(P.wz, re - r0));
        }
    }
}

template <typename T, bool FWD>
__global__ void __launch_bounds__(kThreads) pass_b_kernel(PassBParams P) {
    using V = cx_t<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *twx = reinterpret_cast<V *>(smem_raw);
    V *ta = twx + P.nx;
    V *tb = ta + (size_t)P.nx * P.wx;
    for (int q = threadIdx.x; q < P.nx; q += kThreads) twx[q] = reinterpret_cast<const V *>(P.twx)[q];
    __syncthreads();
    V *base = reinterpret_cast<V *>(P.data);
    for (long long t = blockIdx.x; t < P.ntiles; t += gridDim.x) {
        const long long c0 = t * P.wx;
        const int wv = (int)min((long long)P.wx, P.ncols - c0);
        load_cols<T>(ta, base + c0, P.ncols, P.nx, P.wx, P.wxdiv, wv);
        __syncthreads();
        V *res = fft_tile<T, FWD>(ta, tb, P.wx, 1, P.wx, P.wxdiv, P.ax, twx);
        if (P.epi) {
            for (int q = threadIdx.x; q < P.nx * P.wx; q += kThreads) {
                const int r = (int)fdiv((uint32_t)q, P.wxdiv);
                const int w = q - r * P.wx;
                if (w < wv) st_g(base + c0 + (long long)r * P.ncols + w, pass_b_epilogue(P, res[q], r, c0 + w));
            }
        } else {
            store_cols<T>(res, base + c0, P.ncols, P.nx, P.wx, P.wxdiv, 0, wv);
        }
        __syncthreads();
    }
}

}  // namespace gpufft

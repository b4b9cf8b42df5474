// Register-resident FFT kernels for power-of-two line lengths N in [8, 1024] (included by fft.cu).
//
// A line of N points is handled by T = N / 8 threads; thread t holds the 8 points t + i T
// (i = 0..7) in registers.  Every Stockham pass (radix 8, the last one possibly 4 or 2) reads
// exactly those 8 points, so a pass is: butterflies in registers, write the outputs to shared
// memory at their Stockham destinations, barrier, read back the thread's 8 points, barrier.  The
// first pass reads its points straight from global memory and the last pass leaves the outputs
// in registers at the same positions t + i T, so they are stored straight to global memory.
// Shared memory only carries the (passes - 1) exchanges.  All sizes are compile-time, so index
// arithmetic is shifts and masks.
//
// Layouts in shared memory:
//   strided tiles (y and x passes): B lines = B adjacent z-columns, point k of column c at
//   k * B + c (B complex per row = 128 bytes in FP32, so a warp's accesses never conflict);
//   row tiles (z passes): R rows, point k of row r at r * RS + k + k / 8 (one pad per 8 points).
#pragma once

namespace fast {

constexpr int ilog8(int n) { return n >= 8 ? 1 + ilog8(n / 8) : 0; }
constexpr int ipow8(int p) { return p == 0 ? 1 : 8 * ipow8(p - 1); }

template <int N> struct Plan {
    static_assert(N >= 8 && (N & (N - 1)) == 0, "power of two >= 8");
    static constexpr int T = N / 8;                   // threads per line
    static constexpr int P8 = ilog8(N);               // radix-8 passes
    static constexpr int REM = N / ipow8(P8);         // radix of the last pass when > 1 (2 or 4)
    static constexpr int NPASS = P8 + (REM > 1 ? 1 : 0);
};

template <typename C, int DIR, int R> __device__ __forceinline__ void dftR(C* u) {
    if constexpr (R == 8) dft8<C, DIR>(u);
    else if constexpr (R == 4) dft4<C, DIR>(u);
    else dft2<C, DIR>(u);
}

// One radix-R pass on the thread's 8 points (8 / R butterflies).  tw[m * TWS] = w_N^m.
template <typename C, int N, int R, int NS, int DIR, int TWS>
__device__ __forceinline__ void pass_regs(C (&v)[8], int t, const C* __restrict__ tw) {
    constexpr int T = N / 8, NB = 8 / R, TWSTEP = N / (NS * R);
#pragma unroll
    for (int b = 0; b < NB; b++) {
        C u[R];
#pragma unroll
        for (int r = 0; r < R; r++) u[r] = v[b + r * NB];
        if constexpr (NS > 1) {
            const int k = (t + b * T) & (NS - 1);
#pragma unroll
            for (int r = 1; r < R; r++) {
                C w = tw[((r * k * TWSTEP) & (N - 1)) * TWS];
                if (DIR > 0) w = cconj(w);
                u[r] = cmul(u[r], w);
            }
        }
        dftR<C, DIR, R>(u);
#pragma unroll
        for (int r = 0; r < R; r++) v[b + r * NB] = u[r];
    }
}

// Write the pass outputs to their Stockham destinations, then read back points t + i T.
template <typename C, int N, int R, int NS, class Addr>
__device__ __forceinline__ void exchange(C (&v)[8], int t, C* s, const Addr& addr) {
    constexpr int T = N / 8, NB = 8 / R;
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = t + b * T;
        const int k = j & (NS - 1);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) s[addr(base + r * NS)] = v[b + r * NB];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = s[addr(t + i * T)];
    __syncthreads();
}

template <typename C, int N, int DIR, int TWS, int P> struct Passes {
    template <class Addr>
    static __device__ __forceinline__ void run(C (&v)[8], int t, C* s, const Addr& addr, const C* tw) {
        constexpr int R = (P < Plan<N>::P8) ? 8 : Plan<N>::REM;
        constexpr int NS = ipow8(P);
        pass_regs<C, N, R, NS, DIR, TWS>(v, t, tw);
        if constexpr (P + 1 < Plan<N>::NPASS) {
            exchange<C, N, R, NS>(v, t, s, addr);
            Passes<C, N, DIR, TWS, P + 1>::run(v, t, s, addr, tw);
        }
    }
};

// In: v[i] = x[t + i T].  Out: v[i] = X[t + i T] (unnormalised DFT, sign DIR).
template <typename C, int N, int DIR, int TWS = 1, class Addr>
__device__ __forceinline__ void fft_regs(C (&v)[8], int t, C* s, const Addr& addr, const C* tw) {
    Passes<C, N, DIR, TWS, 0>::run(v, t, s, addr, tw);
}

struct ColAddr {
    int B, col;
    __device__ __forceinline__ int operator()(int k) const { return k * B + col; }
};

struct RowAddr {
    int base;
    __device__ __forceinline__ int operator()(int k) const { return base + k + (k >> 3); }
};

__host__ __device__ constexpr int row_stride(int n) { return n + 1 + ((n + 1) >> 3) + 1; }

// ---------------------------------------------------------------------------------------------
// Strided pass (y or x axis), in place: CTA = T x B threads, tile = B adjacent columns.
// ---------------------------------------------------------------------------------------------
template <typename T, int N, int B, int DIR>
__global__ void __launch_bounds__(N / 8 * B) strided(Specs<cplx_t<T>> data, int nbatch, Strided s) {
    typedef cplx_t<T> C;
    constexpr int TL = N / 8;
    extern __shared__ unsigned char smem_raw[];
    C* tw = (C*)smem_raw;
    C* buf = tw + N;
    fill_twiddles(tw, N);
    __syncthreads();
    const int col = threadIdx.x % B, t = threadIdx.x / B;
    const ColAddr addr{B, col};
    const int ctiles = (s.ncols + B - 1) / B;
    const int64_t tiles_per = (int64_t)s.outer * ctiles;
    const int64_t ntiles = tiles_per * nbatch;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int bi = (int)(tile / tiles_per);
        const int64_t r = tile % tiles_per;
        const int o = (int)(r / ctiles), c0 = (int)(r % ctiles) * B;
        const bool ok = c0 + col < s.ncols;
        C* g = data.p[bi] + (int64_t)o * s.os + c0 + col;
        C v[8];
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = ok ? g[(int64_t)(t + i * TL) * s.ls] : cmake<C>(0, 0);
        fft_regs<C, N, DIR>(v, t, buf, addr, tw);
        if (ok) {
#pragma unroll
            for (int i = 0; i < 8; i++) g[(int64_t)(t + i * TL) * s.ls] = v[i];
        }
    }
}

// ---------------------------------------------------------------------------------------------
// x pass with the k-space step: forward x, multiply by each output's multiplier, inverse x.
// The forward spectrum stays in registers across outputs.
// ---------------------------------------------------------------------------------------------
template <typename T> struct KGeom {
    T k0, k1, k2;    // wavenumbers at the point
    T t0, t1, t2;    // wavenumbers at the reflected index
};

template <typename T>
__device__ __forceinline__ T kval(int i, int n, T fscale) {
    const int s = i < (n + 1) / 2 ? i : i - n;
    return (T)6.283185307179586 * ((T)s * fscale);
}

// Symmetrised multiplier (re, im) of output o (see kmultiplier in fft.cu), in precision T,
// for the compile-time operator KT.
template <typename T, int KT>
__device__ __forceinline__ void kmult(const KOp& op, int o, int ix, int iy, int iz, T& re, T& im) {
    const int idx[3] = {ix, iy, iz};
    T k[3], kt[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        k[a] = kval<T>(idx[a], op.n[a], (T)op.fscale[a]);
        kt[a] = nyquist(idx[a], op.n[a]) ? k[a] : -k[a];
    }
    const T k2 = (k[1] * k[1] + k[0] * k[0]) + k[2] * k[2];
    const bool zero = (ix == 0 && iy == 0 && iz == 0);
    const T norm = (T)op.norm;
    re = 0;
    im = 0;
    if constexpr (KT == KOP_GAUSS) {
        T e = 0;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const T rk = (T)op.radius[a] * k[a];
            e += (T)-0.5 * (rk * rk);
        }
        re = exp(e) * norm;
    } else if constexpr (KT == KOP_PP) {
        if (zero) return;
        const T l0 = (T)op.los[0], l1 = (T)op.los[1], l2 = (T)op.los[2];
        const T kl = k[0] * l0 + k[1] * l1 + k[2] * l2;
        const T klt = kt[0] * l0 + kt[1] * l1 + kt[2] * l2;
        const T m = k[o] / (k2 * ((T)1 + (T)op.beta * (kl * kl / k2)));
        const T mt = kt[o] / (k2 * ((T)1 + (T)op.beta * (klt * klt / k2)));
        im = (T)0.5 * (m - mt) * norm;
    } else if constexpr (KT == KOP_ITER_GLOBAL) {
        if (zero) return;
        const T l0 = (T)op.los[0], l1 = (T)op.los[1], l2 = (T)op.los[2];
        const T kl = k[0] * l0 + k[1] * l1 + k[2] * l2;
        const T klt = kt[0] * l0 + kt[1] * l1 + kt[2] * l2;
        re = (T)0.5 * (kl * kl + klt * klt) / k2 * norm;
    } else if constexpr (KT == KOP_ITER_LOCAL) {
        if (zero) return;
        const int i = o < 3 ? 0 : (o < 5 ? 1 : 2);
        const int j = o < 3 ? o : (o < 5 ? o - 2 : 2);
        re = (T)0.5 * (k[i] * k[j] + kt[i] * kt[j]) / k2 * norm;
    } else if constexpr (KT == KOP_PSI) {
        if (zero) return;
        im = (T)0.5 * (k[o] - kt[o]) / k2 * norm;
    } else {
        re = norm;
    }
}

template <typename T, int N, int B, int KT>
__global__ void __launch_bounds__(N / 8 * B) x_kspace(Specs<cplx_t<T>> in, int nin, Specs<cplx_t<T>> out, Dims dims,
                                                      KOp op) {
    typedef cplx_t<T> C;
    constexpr int TL = N / 8;
    extern __shared__ unsigned char smem_raw[];
    C* tw = (C*)smem_raw;
    C* buf = tw + N;
    fill_twiddles(tw, N);
    __syncthreads();
    const int n1 = dims.n[1], nh = dims.n[2] / 2 + 1;
    const int64_t ls = (int64_t)n1 * nh;
    const int col = threadIdx.x % B, t = threadIdx.x / B;
    const ColAddr addr{B, col};
    const int ctiles = (nh + B - 1) / B;
    const int64_t tiles_per = (int64_t)n1 * ctiles;
    const int64_t ntiles = tiles_per * nin;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int bi = (int)(tile / tiles_per);
        const int64_t r = tile % tiles_per;
        const int iy = (int)(r / ctiles), c0 = (int)(r % ctiles) * B;
        const int iz = c0 + col;
        const bool ok = iz < nh;
        const int64_t off = (int64_t)iy * nh + iz;
        const C* g = in.p[bi] + off;
        C v[8];
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = ok ? g[(int64_t)(t + i * TL) * ls] : cmake<C>(0, 0);
        fft_regs<C, N, -1>(v, t, buf, addr, tw);
        for (int o = 0; o < op.nper; o++) {
            C u[8];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                T re, im;
                kmult<T, KT>(op, o, t + i * TL, iy, iz, re, im);
                u[i] = cmake<C>(re * v[i].x - im * v[i].y, re * v[i].y + im * v[i].x);
            }
            fft_regs<C, N, +1>(u, t, buf, addr, tw);
            C* go = out.p[bi * op.nper + o] + off;
            if (ok) {
#pragma unroll
                for (int i = 0; i < 8; i++) go[(int64_t)(t + i * TL) * ls] = u[i];
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// z pass, forward r2c: rows of n2 = 2M reals, M-point FFT of the packed pairs, then unpack.
// CTA = (M / 8) x ROWS threads.
// ---------------------------------------------------------------------------------------------
template <typename T, typename TIN, int M, int ROWS>
__global__ void __launch_bounds__(M / 8 * ROWS) z_r2c(RealsIn in, Specs<cplx_t<T>> out, int nbatch, int64_t rows) {
    typedef cplx_t<T> C;
    constexpr int TL = M / 8, N2 = 2 * M, NH = M + 1, RS = row_stride(M);
    extern __shared__ unsigned char smem_raw[];
    C* tw = (C*)smem_raw;                 // N2 entries: w_{n2}^m
    C* buf = tw + N2;                     // ROWS * RS
    fill_twiddles(tw, N2);
    __syncthreads();
    const int line = threadIdx.x / TL, t = threadIdx.x % TL;
    const RowAddr addr{line * RS};
    const int64_t tiles_per = (rows + ROWS - 1) / ROWS;
    const int64_t ntiles = tiles_per * nbatch;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int bi = (int)(tile / tiles_per);
        const int64_t row = (tile % tiles_per) * ROWS + line;
        const bool ok = row < rows;
        C v[8];
        if (sizeof(TIN) == sizeof(T)) {
            const C* src = (const C*)((const TIN*)in.p[bi] + row * N2);
#pragma unroll
            for (int i = 0; i < 8; i++) v[i] = ok ? src[t + i * TL] : cmake<C>(0, 0);
        } else {
            typedef cplx_t<TIN> CI;
            const CI* src = (const CI*)((const TIN*)in.p[bi] + row * N2);
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const CI x = ok ? src[t + i * TL] : cmake<CI>(0, 0);
                v[i] = cmake<C>((T)x.x, (T)x.y);
            }
        }
        fft_regs<C, M, -1, 2>(v, t, buf, addr, tw);
        // unpack needs Z[M - k]: publish Z, then combine
#pragma unroll
        for (int i = 0; i < 8; i++) buf[addr(t + i * TL)] = v[i];
        __syncthreads();
        C* dst = out.p[bi] + row * NH;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int k = t + i * TL;
            const C zk = v[i];
            const C zc = cconj(buf[addr(k == 0 ? 0 : M - k)]);
            const C e = cscale(cadd(zk, zc), (T)0.5);
            const C o = cmul_i(cscale(csub(zk, zc), (T)0.5), -1);
            const C x = cadd(e, cmul(tw[k], o));
            if (ok) dst[k] = x;
        }
        if (t == 0 && ok) {
            const C z0 = v[0];
            dst[M] = cmake<C>(z0.x - z0.y, (T)0);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// z pass, inverse c2r over nin inputs with a register-resident real-space epilogue.
// The input loop is unrolled at compile time (at most NMAX inputs for epilogue ET), so every
// input pointer and every per-input register array is indexed statically.
// ---------------------------------------------------------------------------------------------
template <int ET> struct EpiInputs {
    static constexpr int NMAX = ET == EPI_ITER_LOCAL ? 6 : (ET == EPI_DENSITY ? 2 : (ET == EPI_STORE ? 3 : 1));
};

// Inverse z transform of one row: returns v[i] = (x[2k], x[2k+1]), k = t + i TL, unscaled.
template <typename T, int M, class Addr>
__device__ __forceinline__ void row_c2r(const cplx_t<T>* __restrict__ src, bool ok, int t, cplx_t<T>* buf,
                                        const Addr& addr, const cplx_t<T>* tw, cplx_t<T> (&v)[8]) {
    typedef cplx_t<T> C;
    constexpr int TL = M / 8;
    // stage X (M + 1 points) in shared memory for the X[M - k] partner reads
#pragma unroll
    for (int i = 0; i < 8; i++) buf[addr(t + i * TL)] = ok ? src[t + i * TL] : cmake<C>(0, 0);
    if (t == 0) buf[addr(M)] = ok ? src[M] : cmake<C>(0, 0);
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int k = t + i * TL;
        const C xk = buf[addr(k)];
        const C xc = cconj(buf[addr(M - k)]);
        const C ev = cadd(xk, xc);
        const C od = cmul(cconj(tw[k]), csub(xk, xc));
        v[i] = cadd(ev, cmul_i(od, +1));
    }
    __syncthreads();
    fft_regs<C, M, +1, 2>(v, t, buf, addr, tw);
}

template <typename T, int M, int ROWS, int ET>
__global__ void __launch_bounds__(M / 8 * ROWS) z_c2r(Specs<cplx_t<T>> in, int nin, Dims dims, Epi<T> e) {
    typedef cplx_t<T> C;
    constexpr int TL = M / 8, N2 = 2 * M, NH = M + 1, RS = row_stride(M);
    constexpr int NMAX = EpiInputs<ET>::NMAX;
    extern __shared__ unsigned char smem_raw[];
    C* tw = (C*)smem_raw;
    C* buf = tw + N2;
    fill_twiddles(tw, N2);
    __syncthreads();
    const int line = threadIdx.x / TL, t = threadIdx.x % TL;
    const RowAddr addr{line * RS};
    const int64_t rows = (int64_t)dims.n[0] * dims.n[1];
    const int64_t ntiles = (rows + ROWS - 1) / ROWS;
    const T sc = (T)e.scale;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t row = tile * ROWS + line;
        const bool ok = row < rows;
        const int ix = ok ? (int)(row / dims.n[1]) : 0, iy = ok ? (int)(row % dims.n[1]) : 0;
        C* out0 = (C*)(e.out[0] + (ok ? row : 0) * N2);
        if constexpr (ET == EPI_STORE) {
#pragma unroll
            for (int c = 0; c < NMAX; c++) {
                if (c < nin) {
                    C v[8];
                    row_c2r<T, M>(in.p[c] + row * NH, ok, t, buf, addr, tw, v);
                    C* o = (C*)(e.out[c] + (ok ? row : 0) * N2);
                    if (ok) {
#pragma unroll
                        for (int i = 0; i < 8; i++) o[t + i * TL] = cmake<C>(v[i].x * sc, v[i].y * sc);
                    }
                }
            }
        } else if constexpr (ET == EPI_DENSITY) {
            C d[8], r[8];
            row_c2r<T, M>(in.p[0] + row * NH, ok, t, buf, addr, tw, d);
            row_c2r<T, M>(in.p[1] + row * NH, ok, t, buf, addr, tw, r);
            const double sd = e.sums[0], sr = e.sums[1];
            const double alpha = sd * 1. / sr;
            const double threshold = e.ran_min * sr / e.size_randoms;
            if (ok) {
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const double d0 = (double)(d[i].x * sc), d1 = (double)(d[i].y * sc);
                    const double r0 = (double)(r[i].x * sc), r1 = (double)(r[i].y * sc);
                    const double o0 = r0 > threshold ? (d0 - alpha * r0) / (e.bias * alpha * r0) : 0.;
                    const double o1 = r1 > threshold ? (d1 - alpha * r1) / (e.bias * alpha * r1) : 0.;
                    out0[t + i * TL] = cmake<C>((T)o0, (T)o1);
                }
            }
        } else if constexpr (ET == EPI_DENSITY_NORANDOMS) {
            C d[8];
            row_c2r<T, M>(in.p[0] + row * NH, ok, t, buf, addr, tw, d);
            const double mean = e.sums[0] / e.ncells;
            if (ok) {
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const double o0 = ((double)(d[i].x * sc) / mean - 1.) / e.bias;
                    const double o1 = ((double)(d[i].y * sc) / mean - 1.) / e.bias;
                    out0[t + i * TL] = cmake<C>((T)o0, (T)o1);
                }
            }
        } else {
            // RSD removal: delta_real = delta - sum_c factor_c w_c(x) IFFT_c, accumulated in registers
            const C* dl = (const C*)(e.delta + (ok ? row : 0) * N2);
            T acc[8][2];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const C d0 = ok ? dl[t + i * TL] : cmake<C>(0, 0);
                acc[i][0] = d0.x;
                acc[i][1] = d0.y;
            }
#pragma unroll
            for (int c = 0; c < NMAX; c++) {
                C v[8];
                row_c2r<T, M>(in.p[c] + row * NH, ok, t, buf, addr, tw, v);
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const int k = t + i * TL;
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const double val = (double)((h ? v[i].y : v[i].x) * sc);
                        if constexpr (ET == EPI_ITER_GLOBAL) {
                            acc[i][h] = (T)((double)acc[i][h] - e.factor[0] * val);
                        } else {
                            // component c = (pi, pj) in the order (0,0) (0,1) (0,2) (1,1) (1,2) (2,2)
                            const int pi = c < 3 ? 0 : (c < 5 ? 1 : 2);
                            const int pj = c < 3 ? c : (c < 5 ? c - 2 : 2);
                            const int iz = 2 * k + h;
                            const double x[3] = {e.offset[0] + e.cell[0] * ix, e.offset[1] + e.cell[1] * iy,
                                                 e.offset[2] + e.cell[2] * iz};
                            const double x2 = (x[0] * x[0] + x[1] * x[1]) + x[2] * x[2];
                            acc[i][h] = (T)((double)acc[i][h] - e.factor[c] * ((x[pi] * x[pj] * val) / x2));
                        }
                    }
                }
            }
            if (ok) {
#pragma unroll
                for (int i = 0; i < 8; i++) out0[t + i * TL] = cmake<C>(acc[i][0], acc[i][1]);
            }
        }
    }
}

}  // namespace fast

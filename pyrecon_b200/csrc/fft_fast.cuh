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

// PRC_PREFETCH=1: strided and k-space kernels issue the next tile's loads before computing the
// current one (register double buffering).
#ifndef PRC_PREFETCH
#define PRC_PREFETCH 1
#endif

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

// Twiddles of every pass in one table: pass P (radix R_P, sub-transform size NS_P = 8^P) owns
// NS_P (R_P - 1) entries laid out [k][r - 1] = w_{NS_P R_P}^{r k}, so the lanes of a warp, which
// differ in k, read addresses R_P - 1 complex apart (an odd pitch: no bank conflicts).  The sizes
// telescope: the table has exactly N - 1 entries.
template <int N> struct TwLayout {
    static constexpr int radix(int P) { return P < Plan<N>::P8 ? 8 : Plan<N>::REM; }
    static constexpr int offset(int P) {
        int o = 0, ns = 1;
        for (int q = 0; q < P; q++) {
            o += ns * (radix(q) - 1);
            ns *= radix(q);
        }
        return o;
    }
    static constexpr int SIZE = N - 1;
};

// tw[m] = w_n^m = exp(-2 pi i m / n) for m < count.
template <typename C> __device__ void fill_roots(C* tw, int count, int n) {
    typedef decltype(C().x) T;
    for (int m = threadIdx.x; m < count; m += blockDim.x) {
        double sn, cs;
        sincospi(-2.0 * (double)m / (double)n, &sn, &cs);
        tw[m] = cmake<C>((T)cs, (T)sn);
    }
}

// Twiddle table of an N-point transform (fft_regs).  Powers of two: the pass table (N - 1 entries).  N = 3 M:
// the pass table of the M-point sub-transforms, then w_N^k for k < M at tw + M (2 M <= N entries).
template <typename C, int N> __device__ void fill_pass_twiddles(C* tw) {
    if constexpr (N % 3 == 0) {
        fill_pass_twiddles<C, N / 3>(tw);
        fill_roots(tw + N / 3, N / 3, N);
    } else {
    typedef decltype(C().x) T;
    for (int idx = threadIdx.x; idx < TwLayout<N>::SIZE; idx += blockDim.x) {
        int off = 0, ns = 1, R = 8;
        for (int q = 0; q < Plan<N>::NPASS; q++) {
            R = TwLayout<N>::radix(q);
            if (idx < off + ns * (R - 1)) break;
            off += ns * (R - 1);
            ns *= R;
        }
        const int local = idx - off, k = local / (R - 1), r = local % (R - 1) + 1;
        const int m = (r * k * (N / (ns * R))) & (N - 1);
        double sn, cs;
        sincospi(-2.0 * (double)m / (double)N, &sn, &cs);
        tw[idx] = cmake<C>((T)cs, (T)sn);
    }
    }
}


template <typename C, int DIR, int R> __device__ __forceinline__ void dftR(C* u) {
    if constexpr (R == 8) dft8<C, DIR>(u);
    else if constexpr (R == 4) dft4<C, DIR>(u);
    else dft2<C, DIR>(u);
}

// PRC_TW_RECUR=1: a radix-8 butterfly reads w, w^2 and w^4 from the pass table and forms w^3, w^5, w^6,
// w^7 as products (at most two roundings deep), so it issues 3 shared-memory loads instead of 7; the
// passes are bound by shared-memory instruction traffic (exchanges and twiddles), not by arithmetic.
#ifndef PRC_TW_RECUR
#define PRC_TW_RECUR 1
#endif

// One radix-R pass on the thread's 8 points (8 / R butterflies); tw = this pass's table.
template <typename C, int N, int R, int NS, int DIR>
__device__ __forceinline__ void pass_regs(C (&v)[8], int t, const C* __restrict__ tw) {
    constexpr int T = N / 8, NB = 8 / R;
#pragma unroll
    for (int b = 0; b < NB; b++) {
        C u[R];
#pragma unroll
        for (int r = 0; r < R; r++) u[r] = v[b + r * NB];
        if constexpr (NS > 1) {
            const int k = (t + b * T) & (NS - 1);
            const C* row = tw + k * (R - 1);
            if constexpr (R == 8 && PRC_TW_RECUR) {
                C w[8];
                w[1] = row[0];
                w[2] = row[1];
                w[4] = row[3];
                if (DIR > 0) {
                    w[1] = cconj(w[1]);
                    w[2] = cconj(w[2]);
                    w[4] = cconj(w[4]);
                }
                w[3] = cmul(w[1], w[2]);
                w[5] = cmul(w[1], w[4]);
                w[6] = cmul(w[2], w[4]);
                w[7] = cmul(w[3], w[4]);
#pragma unroll
                for (int r = 1; r < 8; r++) u[r] = cmul(u[r], w[r]);
            } else {
#pragma unroll
                for (int r = 1; r < R; r++) {
                    C w = row[r - 1];
                    if (DIR > 0) w = cconj(w);
                    u[r] = cmul(u[r], w);
                }
            }
        }
        dftR<C, DIR, R>(u);
#pragma unroll
        for (int r = 0; r < R; r++) v[b + r * NB] = u[r];
    }
}

// The barrier of an exchange: the block's, or the warp's (WS) when every line the exchange buffer serves
// lies within one warp (rows of at most 32 threads in whole warps: RowWarp).
template <bool WS> __device__ __forceinline__ void xsync() {
    if constexpr (WS) __syncwarp();
    else __syncthreads();
}

// PRC_ROW_WARP_SYNC=1: the z passes of power-of-two rows of at most 256 complex points (one warp or less a
// row, rows in whole warps) synchronise their row-private exchanges per warp instead of per block.
#ifndef PRC_ROW_WARP_SYNC
#define PRC_ROW_WARP_SYNC 1
#endif
template <int M, int ROWS> struct RowWarp {
    static constexpr bool value =
        PRC_ROW_WARP_SYNC && (M & (M - 1)) == 0 && M / 8 <= 32 && (M / 8 * ROWS) % 32 == 0;
};

// Write the pass outputs to their Stockham destinations, then read back points t + i T.
template <typename C, int N, int R, int NS, class Addr, bool WS = false>
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
    xsync<WS>();
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = s[addr(t + i * T)];
    xsync<WS>();
}

template <typename C, int N, int DIR, int P, bool WS = false> struct Passes {
    template <class Addr>
    static __device__ __forceinline__ void run(C (&v)[8], int t, C* s, const Addr& addr, const C* tw) {
        constexpr int R = TwLayout<N>::radix(P);
        constexpr int NS = ipow8(P);
        pass_regs<C, N, R, NS, DIR>(v, t, tw + TwLayout<N>::offset(P));
        if constexpr (P + 1 < Plan<N>::NPASS) {
            exchange<C, N, R, NS, Addr, WS>(v, t, s, addr);
            Passes<C, N, DIR, P + 1, WS>::run(v, t, s, addr, tw);
        }
    }
};

// Same passes with the exchanges alternating between two buffers (s0 first) and no barrier after an
// exchange's reads: the next write to a buffer comes one exchange later, behind that exchange's
// barrier.  The caller orders its own accesses to s0 / s1 around the call: s0 must not be read by
// anyone once the call starts, and neither buffer may be written after it before a barrier.
template <typename C, int N, int R, int NS, class Addr, bool WS = false>
__device__ __forceinline__ void exchange_pp(C (&v)[8], int t, C* s, const Addr& addr) {
    constexpr int T = N / 8, NB = 8 / R;
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = t + b * T;
        const int k = j & (NS - 1);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) s[addr(base + r * NS)] = v[b + r * NB];
    }
    xsync<WS>();
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = s[addr(t + i * T)];
}

template <typename C, int N, int DIR, int P, bool WS = false> struct PassesPP {
    template <class Addr0, class Addr1>
    static __device__ __forceinline__ void run(C (&v)[8], int t, C* s0, const Addr0& addr0, C* s1, const Addr1& addr1,
                                               const C* tw) {
        constexpr int R = TwLayout<N>::radix(P);
        constexpr int NS = ipow8(P);
        pass_regs<C, N, R, NS, DIR>(v, t, tw + TwLayout<N>::offset(P));
        if constexpr (P + 1 < Plan<N>::NPASS) {
            if constexpr (P % 2 == 0) exchange_pp<C, N, R, NS, Addr0, WS>(v, t, s0, addr0);
            else exchange_pp<C, N, R, NS, Addr1, WS>(v, t, s1, addr1);
            PassesPP<C, N, DIR, P + 1, WS>::run(v, t, s0, addr0, s1, addr1, tw);
        }
    }
};

// ---- lines of N = 3 M points (M a power of two) ----
// The transform is three M-point transforms of the points decimated by 3 (sub-line r holds x[3 m + r] at
// position m) followed by one radix-3 step, X[k + j M] = sum_r w_N^(r k) w_3^(r j) X_r[k]: an exchange
// that decimates, the sub-transforms (threads t = r M/8 + t' work on sub-line r, in its own region
// r M .. r M + M - 1 of the exchange buffer), an exchange that makes X_0..2[k] readable by the thread of
// each output, and the radix-3 step in registers.  Points in and out stay t + i T, T = N / 8.
template <int N> struct Shape {
    static constexpr bool R3 = N % 3 == 0;
    static constexpr int M = R3 ? N / 3 : N;                          // the power-of-two part
    static constexpr int NX = Plan<M>::NPASS - 1 + (R3 ? 2 : 0);      // shared-memory exchanges of a transform
};

template <class Addr> struct SubAddr {
    Addr a;
    int off;
    __device__ __forceinline__ int operator()(int k) const { return a(off + k); }
};

// Output p of the radix-3 step from the sub-transforms in s (sub-line r at r M): with b = w^k X_1[k],
// c = w^(2k) X_2[k], X[k] = a + b + c, X[k + M] = a - (b + c) / 2 + i s (b - c), X[k + 2M] = a - (b + c) / 2
// - i s (b - c), s = DIR sqrt(3) / 2.
template <typename C, int N, int DIR, class Addr>
__device__ __forceinline__ C combine3(const C* s, const Addr& addr, const C* tw, int p) {
    typedef decltype(C().x) T;
    constexpr int M = N / 3;
    const int k = p & (M - 1), j = p / M;
    C w1 = tw[M + k];
    if (DIR > 0) w1 = cconj(w1);
    const C w2 = cmul(w1, w1);
    const C a = s[addr(k)];
    const C b = cmul(s[addr(M + k)], w1);
    const C c = cmul(s[addr(2 * M + k)], w2);
    const C sum = cadd(b, c), dif = csub(b, c);
    const C h = csub(a, cscale(sum, (T)0.5));
    const T sg = (T)(DIR * 0.86602540378443864676);
    const C rot = cmake<C>(-sg * dif.y, sg * dif.x);
    return j == 0 ? cadd(a, sum) : (j == 1 ? cadd(h, rot) : csub(h, rot));
}

template <typename C, int N, int DIR, class Addr>
__device__ __forceinline__ void fft_regs3(C (&v)[8], int t, C* s, const Addr& addr, const C* tw) {
    constexpr int M = N / 3, T = N / 8, TM = M / 8;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int p = t + i * T;
        s[addr((p % 3) * M + p / 3)] = v[i];
    }
    __syncthreads();
    const int r = t / TM, tm = t - r * TM;
    const SubAddr<Addr> sa{addr, r * M};
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = s[sa(tm + i * TM)];
    __syncthreads();
    Passes<C, M, DIR, 0>::run(v, tm, s, sa, tw);
#pragma unroll
    for (int i = 0; i < 8; i++) s[sa(tm + i * TM)] = v[i];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = combine3<C, N, DIR>(s, addr, tw, t + i * T);
    __syncthreads();
}

// The same with the exchanges alternating between s0 and s1 (the fft_regs_pp contract): decimation in s0,
// the sub-transforms' exchanges from s1 on, the radix-3 exchange in the buffer the last one did not use.
template <typename C, int N, int DIR, class Addr0, class Addr1>
__device__ __forceinline__ void fft_regs3_pp(C (&v)[8], int t, C* s0, const Addr0& addr0, C* s1, const Addr1& addr1,
                                             const C* tw) {
    constexpr int M = N / 3, T = N / 8, TM = M / 8, NXM = Plan<M>::NPASS - 1;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int p = t + i * T;
        s0[addr0((p % 3) * M + p / 3)] = v[i];
    }
    __syncthreads();
    const int r = t / TM, tm = t - r * TM;
    const SubAddr<Addr0> sa0{addr0, r * M};
    const SubAddr<Addr1> sa1{addr1, r * M};
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = s0[sa0(tm + i * TM)];
    PassesPP<C, M, DIR, 0>::run(v, tm, s1, sa1, s0, sa0, tw);
    if constexpr ((NXM + 1) % 2 == 0) {
#pragma unroll
        for (int i = 0; i < 8; i++) s0[sa0(tm + i * TM)] = v[i];
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = combine3<C, N, DIR>(s0, addr0, tw, t + i * T);
    } else {
#pragma unroll
        for (int i = 0; i < 8; i++) s1[sa1(tm + i * TM)] = v[i];
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = combine3<C, N, DIR>(s1, addr1, tw, t + i * T);
    }
}

// In: v[i] = x[t + i T].  Out: v[i] = X[t + i T] (unnormalised DFT, sign DIR).  tw: the table filled by
// fill_pass_twiddles<C, N>.  N a power of two, or 3 times one.
// WS: warp barriers (RowWarp; powers of two only).
template <typename C, int N, int DIR, bool WS = false, class Addr>
__device__ __forceinline__ void fft_regs(C (&v)[8], int t, C* s, const Addr& addr, const C* tw) {
    static_assert(!WS || N % 3 != 0, "warp barriers need power-of-two lines");
    if constexpr (N % 3 == 0) fft_regs3<C, N, DIR>(v, t, s, addr, tw);
    else Passes<C, N, DIR, 0, WS>::run(v, t, s, addr, tw);
}

template <typename C, int N, int DIR, bool WS = false, class Addr>
__device__ __forceinline__ void fft_regs_pp(C (&v)[8], int t, C* s0, C* s1, const Addr& addr, const C* tw) {
    static_assert(!WS || N % 3 != 0, "warp barriers need power-of-two lines");
    if constexpr (N % 3 == 0) fft_regs3_pp<C, N, DIR>(v, t, s0, addr, s1, addr, tw);
    else PassesPP<C, N, DIR, 0, WS>::run(v, t, s0, addr, s1, addr, tw);
}

// The same with a separate layout for s0, the buffer of the first (and every even) exchange.
template <typename C, int N, int DIR, class Addr0, class Addr1>
__device__ __forceinline__ void fft_regs_pp(C (&v)[8], int t, C* s0, const Addr0& addr0, C* s1, const Addr1& addr1,
                                            const C* tw) {
    if constexpr (N % 3 == 0) fft_regs3_pp<C, N, DIR>(v, t, s0, addr0, s1, addr1, tw);
    else PassesPP<C, N, DIR, 0>::run(v, t, s0, addr0, s1, addr1, tw);
}

struct ColAddr {
    int B, col;
    __device__ __forceinline__ int operator()(int k) const { return k * B + col; }
};

// ColAddr with one row of padding after every 8 rows, for the exchange buffer of the first Stockham pass
// of a tile with B = 8 FP32 columns: that pass writes the rows 8 t + r of the four lines t a warp holds,
// which in the dense layout all start on the same bank (a row is 16 banks wide), two-way conflicting;
// padded, they alternate between the two halves of the banks.  Reads of consecutive rows stay
// conflict-free.  The buffer holds (N + N / 8) B values.
struct PadAddr {
    int B, col;
    __device__ __forceinline__ int operator()(int k) const { return (k + (k >> 3)) * B + col; }
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
    fill_pass_twiddles<C, N>(tw);
    __syncthreads();
    const int col = threadIdx.x % B, t = threadIdx.x / B;
    const ColAddr addr{B, col};
    const int ctiles = (s.ncols + B - 1) / B;
    const int64_t tiles_per = (int64_t)s.outer * ctiles;
    const int64_t ntiles = tiles_per * nbatch;
    auto locate = [&](int64_t tile, bool& ok) {
        const int bi = (int)(tile / tiles_per);
        const int64_t r = tile % tiles_per;
        const int o = (int)(r / ctiles), c0 = (int)(r % ctiles) * B;
        ok = c0 + col < s.ncols;
        return data.p[bi] + (int64_t)o * s.os + c0 + col;
    };
    C v[8];
    bool ok = false;
    C* g = nullptr;
    if (blockIdx.x < ntiles) {
        g = locate(blockIdx.x, ok);
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = ok ? g[(int64_t)(t + i * TL) * s.ls] : cmake<C>(0, 0);
    }
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t next = tile + gridDim.x;
        bool nok = false;
        C* ng = nullptr;
        C nv[8];
        if (PRC_PREFETCH && next < ntiles) {
            ng = locate(next, nok);
#pragma unroll
            for (int i = 0; i < 8; i++) nv[i] = nok ? ng[(int64_t)(t + i * TL) * s.ls] : cmake<C>(0, 0);
        }
        fft_regs<C, N, DIR>(v, t, buf, addr, tw);
        if (ok) {
#pragma unroll
            for (int i = 0; i < 8; i++) g[(int64_t)(t + i * TL) * s.ls] = v[i];
        }
        if (next < ntiles) {
            if (PRC_PREFETCH) {
#pragma unroll
                for (int i = 0; i < 8; i++) v[i] = nv[i];
                g = ng;
                ok = nok;
            } else {
                g = locate(next, ok);
#pragma unroll
                for (int i = 0; i < 8; i++) v[i] = ok ? g[(int64_t)(t + i * TL) * s.ls] : cmake<C>(0, 0);
            }
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

// Per-point quantities of the multiplier that do not depend on the output: computed once after the
// forward x transform and reused by every output (one division per point instead of one per
// point and output).
template <typename T, int KT> struct KPoint {
    T a, b;        // GAUSS: a = exp(...) * norm; PP: a = 1/(k^2 + beta (k.l)^2), b = same at k~;
                   // ITER_*, PSI: a = norm / k^2 (0 at k = 0)
};

// The k-space step on one x-line held as 8 points per thread (points t + i N/8) at fixed (iy, iz):
// `setup` computes what does not depend on the output once, `apply` multiplies the forward
// spectrum v by output o's symmetrised multiplier into u.
template <typename T, int N, int KT> struct KLine {
    typedef cplx_t<T> C;
    static constexpr int TL = N / 8;
    T ky, kz, ty, tz;
    KPoint<T, KT> kp[8];

    __device__ __forceinline__ void setup(const KOp& op, const Dims& dims, int t, int iy, int iz) {
        const T norm = (T)op.norm, beta = (T)op.beta;
        const T l0 = (T)op.los[0], l1 = (T)op.los[1], l2 = (T)op.los[2];
        ky = kval<T>(iy, dims.n[1], (T)op.fscale[1]);
        kz = kval<T>(iz, dims.n[2], (T)op.fscale[2]);
        ty = nyquist(iy, dims.n[1]) ? ky : -ky;
        tz = nyquist(iz, dims.n[2]) ? kz : -kz;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int ix = t + i * TL;
            const T kx = kval<T>(ix, dims.n[0], (T)op.fscale[0]);
            const T tx = nyquist(ix, dims.n[0]) ? kx : -kx;
            const T k2 = (ky * ky + kx * kx) + kz * kz;
            const bool zero = (ix == 0 && iy == 0 && iz == 0);
            if constexpr (KT == KOP_GAUSS) {
                const T rx = (T)op.radius[0] * kx, ry = (T)op.radius[1] * ky, rz = (T)op.radius[2] * kz;
                kp[i].a = exp((T)-0.5 * (rx * rx) + (T)-0.5 * (ry * ry) + (T)-0.5 * (rz * rz)) * norm;
            } else if constexpr (KT == KOP_PP) {
                const T kl = kx * l0 + ky * l1 + kz * l2, klt = tx * l0 + ty * l1 + tz * l2;
                kp[i].a = zero ? (T)0 : (T)1 / (k2 + beta * (kl * kl));
                kp[i].b = zero ? (T)0 : (T)1 / (k2 + beta * (klt * klt));
            } else {
                kp[i].a = zero ? (T)0 : norm / k2;
            }
        }
    }

    __device__ __forceinline__ void apply(const KOp& op, const Dims& dims, int t, int o, const C (&v)[8],
                                          C (&u)[8]) const {
        const T norm = (T)op.norm;
        const T l0 = (T)op.los[0], l1 = (T)op.los[1], l2 = (T)op.los[2];
        if constexpr (KT == KOP_HESS3) {
            // E, s_x E, k_x^2 E with E = norm delta / k^2 (s_x = k_x, 0 on the Nyquist index); o is the
            // same for the whole CTA, so each output is one uniform branch
            if (o == 0) {
#pragma unroll
                for (int i = 0; i < 8; i++) u[i] = cscale(v[i], kp[i].a);
            } else {
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const int ix = t + i * TL;
                    const T kx = kval<T>(ix, dims.n[0], (T)op.fscale[0]);
                    const T tx = nyquist(ix, dims.n[0]) ? kx : -kx;
                    u[i] = cscale(v[i], (o == 1 ? (T)0.5 * (kx - tx) : kx * kx) * kp[i].a);
                }
            }
        } else {
#pragma unroll
            for (int i = 0; i < 8; i++) {
                T re = 0, im = 0;
                const int ix = t + i * TL;
                const T kx = kval<T>(ix, dims.n[0], (T)op.fscale[0]);
                const T tx = nyquist(ix, dims.n[0]) ? kx : -kx;
                if constexpr (KT == KOP_GAUSS) {
                    re = kp[i].a;
                } else if constexpr (KT == KOP_PP) {
                    // (i m(k) + conj(i m(k~))) / 2 with m = k_o / (k^2 (1 + beta mu^2))
                    const T ko = o == 0 ? kx : (o == 1 ? ky : kz), to = o == 0 ? tx : (o == 1 ? ty : tz);
                    im = (T)0.5 * (ko * kp[i].a - to * kp[i].b) * norm;
                } else if constexpr (KT == KOP_ITER_GLOBAL) {
                    const T kl = kx * l0 + ky * l1 + kz * l2, klt = tx * l0 + ty * l1 + tz * l2;
                    re = (T)0.5 * (kl * kl + klt * klt) * kp[i].a;
                } else if constexpr (KT == KOP_ITER_LOCAL) {
                    const int ci = o < 3 ? 0 : (o < 5 ? 1 : 2);
                    const int cj = o < 3 ? o : (o < 5 ? o - 2 : 2);
                    const T ki = ci == 0 ? kx : (ci == 1 ? ky : kz), ti = ci == 0 ? tx : (ci == 1 ? ty : tz);
                    const T kj = cj == 0 ? kx : (cj == 1 ? ky : kz), tj = cj == 0 ? tx : (cj == 1 ? ty : tz);
                    re = (T)0.5 * (ki * kj + ti * tj) * kp[i].a;
                } else if constexpr (KT == KOP_PSI) {
                    const T ko = o == 0 ? kx : (o == 1 ? ky : kz), to = o == 0 ? tx : (o == 1 ? ty : tz);
                    im = (T)0.5 * (ko - to) * kp[i].a;
                } else {
                    re = norm;
                }
                // the multiplier is real or imaginary: one product per component
                if constexpr (KT == KOP_PP || KT == KOP_PSI) u[i] = cmake<C>(-(im * v[i].y), im * v[i].x);
                else u[i] = cmake<C>(re * v[i].x, re * v[i].y);
            }
        }
    }

    // KOP_HESS3: the line's point at the x Nyquist index (held by thread 0 as its point 4, since
    // N / 2 = 4 N / 8) feeds the y pass's Nyquist terms: q01[iz] = k_x k_y E on the y Nyquist index,
    // l02[iy] = k_x k_z E on the z Nyquist index (op.side = q01, then l02 after nh values).
    __device__ __forceinline__ void nyquist_lines(const KOp& op, const Dims& dims, int t, int iy, int iz,
                                                  const C (&v)[8]) const {
        if (t != 0 || op.side == nullptr) return;
        const int n1 = dims.n[1], n2 = dims.n[2], nh = n2 / 2 + 1;
        if (iz >= nh) return;
        const T kx = kval<T>(N / 2, N, (T)op.fscale[0]);
        const C e = cmake<C>(kp[4].a * v[4].x, kp[4].a * v[4].y);
        C* side = (C*)op.side;
        if (n1 % 2 == 0 && iy == n1 / 2) side[iz] = cmake<C>(kx * ky * e.x, kx * ky * e.y);
        if (n2 % 2 == 0 && iz == n2 / 2) side[nh + iy] = cmake<C>(kx * kz * e.x, kx * kz * e.y);
    }
};

// Blocks per SM requested from the register allocator for the FP32 k-space and c2r kernels
// (tuning knobs PRC_KSPACE_MINB / PRC_C2R_MINB; 1 leaves the allocator free).
#ifndef PRC_KSPACE_MINB
#define PRC_KSPACE_MINB 1
#endif
#ifndef PRC_C2R_MINB
#define PRC_C2R_MINB 2
#endif
template <typename T, int THREADS, int MINB> struct MinBlocks {
    static constexpr int value = (sizeof(T) == 4 && THREADS * MINB <= 2048) ? MINB : 1;
};

template <typename T, int N, int B, int KT>
__global__ void __launch_bounds__(N / 8 * B, (MinBlocks<T, N / 8 * B, PRC_KSPACE_MINB>::value)) x_kspace(Specs<cplx_t<T>> in, int nin, Specs<cplx_t<T>> out, Dims dims,
                                                      int pitch, KOp op) {
    typedef cplx_t<T> C;
    constexpr int TL = N / 8;
    extern __shared__ unsigned char smem_raw[];
    C* tw = (C*)smem_raw;
    C* buf = tw + N;
    fill_pass_twiddles<C, N>(tw);
    __syncthreads();
    const int n1 = dims.n[1], nh = dims.n[2] / 2 + 1;
    const int64_t ls = (int64_t)n1 * pitch;
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
        const int64_t off = (int64_t)iy * pitch + iz;
        const C* g = in.p[bi] + off;
        C v[8];
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = ok ? g[(int64_t)(t + i * TL) * ls] : cmake<C>(0, 0);
        fft_regs<C, N, -1>(v, t, buf, addr, tw);
        KLine<T, N, KT> kl;
        kl.setup(op, dims, t, iy, iz);
        for (int o = 0; o < op.nper; o++) {
            C u[8];
            kl.apply(op, dims, t, o, v, u);
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
// Forward real transform of one row held as packed pairs, v[i] = (x[2k], x[2k+1]) for k = t + i TL:
// the M-point transform Z, then X[k] = (Z[k] + conj Z[M-k]) / 2 - i w^k (Z[k] - conj Z[M-k]) / 2 for
// k < M and X[M] = Re Z[0] - Im Z[0], stored at dst when ok.  buf (the row's exchange buffer, addr) is
// written from the start: the caller's earlier reads of it must be behind a barrier.  Ends with a barrier.
template <typename T, int M, bool WS = false, class Addr>
__device__ __forceinline__ void row_r2c(cplx_t<T> (&v)[8], bool ok, int t, cplx_t<T>* buf, const Addr& addr,
                                        const cplx_t<T>* tw, const cplx_t<T>* wk, cplx_t<T>* dst) {
    typedef cplx_t<T> C;
    constexpr int TL = M / 8;
    fft_regs<C, M, -1, WS>(v, t, buf, addr, tw);
    // unpack needs Z[M - k]: publish Z, then combine
#pragma unroll
    for (int i = 0; i < 8; i++) buf[addr(t + i * TL)] = v[i];
    xsync<WS>();
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int k = t + i * TL;
        const C zk = v[i];
        const C zc = cconj(buf[addr(k == 0 ? 0 : M - k)]);
        const C e = cscale(cadd(zk, zc), (T)0.5);
        const C o = cmul_i(cscale(csub(zk, zc), (T)0.5), -1);
        const C x = cadd(e, cmul(wk[k], o));
        if (ok) dst[k] = x;
    }
    if (t == 0 && ok) {
        const C z0 = v[0];
        dst[M] = cmake<C>(z0.x - z0.y, (T)0);
    }
    xsync<WS>();
}

// row_r2c with the transform's exchanges alternating between s0 and s1 (fft_regs_pp) and Z published in
// the buffer the last exchange did not use, which every thread has finished reading by that exchange's
// barrier: a barrier per exchange plus one.  On entry s0 must be free (not read by anyone after the
// caller's last barrier) and s1 free once the first exchange's barrier is reached; on return the
// partner reads of Z are not fenced: the caller puts a barrier before the next write to either buffer.
template <typename T, int M, bool WS = false, class Addr>
__device__ __forceinline__ void row_r2c_pp(cplx_t<T> (&v)[8], bool ok, int t, cplx_t<T>* s0, cplx_t<T>* s1,
                                           const Addr& addr, const cplx_t<T>* tw, const cplx_t<T>* wk,
                                           cplx_t<T>* dst) {
    typedef cplx_t<T> C;
    constexpr int TL = M / 8, NX = Shape<M>::NX;   // exchanges: s0, s1, s0, ...
    fft_regs_pp<C, M, -1, WS>(v, t, s0, s1, addr, tw);
    C* zb = NX == 0 ? s0 : ((NX - 1) % 2 == 0 ? s1 : s0);
#pragma unroll
    for (int i = 0; i < 8; i++) zb[addr(t + i * TL)] = v[i];
    xsync<WS>();
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int k = t + i * TL;
        const C zk = v[i];
        const C zc = cconj(zb[addr(k == 0 ? 0 : M - k)]);
        const C e = cscale(cadd(zk, zc), (T)0.5);
        const C o = cmul_i(cscale(csub(zk, zc), (T)0.5), -1);
        const C x = cadd(e, cmul(wk[k], o));
        if (ok) dst[k] = x;
    }
    if (t == 0 && ok) {
        const C z0 = v[0];
        dst[M] = cmake<C>(z0.x - z0.y, (T)0);
    }
}

template <typename T, typename TIN, int M, int ROWS>
__global__ void __launch_bounds__(M / 8 * ROWS) z_r2c(RealsIn in, Specs<cplx_t<T>> out, int nbatch, int64_t rows, int pitch) {
    typedef cplx_t<T> C;
    constexpr int TL = M / 8, N2 = 2 * M, RS = row_stride(M);
    extern __shared__ unsigned char smem_raw[];
    C* tw = (C*)smem_raw;                 // pass table of the M-point transform (M entries)
    C* wk = tw + M;                       // w_{n2}^k, k < M + 1, for the real-FFT unpack
    C* buf = wk + M + 1;                  // ROWS * RS
    fill_pass_twiddles<C, M>(tw);
    fill_roots(wk, M + 1, N2);
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
        row_r2c<T, M, RowWarp<M, ROWS>::value>(v, ok, t, buf, addr, tw, wk, out.p[bi] + (ok ? row : 0) * pitch);
    }
}

// ---------------------------------------------------------------------------------------------
// z pass, inverse c2r over nin inputs with a register-resident real-space epilogue.
// The input loop is unrolled at compile time (at most NMAX inputs for epilogue ET), so every
// input pointer and every per-input register array is indexed statically.
// ---------------------------------------------------------------------------------------------
// p[c] for a rolled loop index c, written as selects so no parameter array is indexed at run time.
template <typename C> __device__ __forceinline__ const C* select6(const Specs<C>& s, int c) {
    return c == 0 ? s.p[0] : c == 1 ? s.p[1] : c == 2 ? s.p[2] : c == 3 ? s.p[3] : c == 4 ? s.p[4] : s.p[5];
}
__device__ __forceinline__ double select6(const double (&f)[6], int c) {
    return c == 0 ? f[0] : c == 1 ? f[1] : c == 2 ? f[2] : c == 3 ? f[3] : c == 4 ? f[4] : f[5];
}

template <int ET> struct EpiInputs {
    static constexpr int NMAX =
        ET == EPI_ITER_LOCAL ? 6
                             : (ET == EPI_DENSITY ? 2
                                                  : ((ET == EPI_STORE || ET == EPI_STORE4 || ET == EPI_ITER_POLY ||
                                                      ET == EPI_ITER_POLY_R2C) ? 3 : 1));
};

// Inverse z transform of one row: returns v[i] = (x[2k], x[2k+1]), k = t + i TL, unscaled.
template <typename T, int M, bool WS = false, class Addr>
__device__ __forceinline__ void row_c2r(const cplx_t<T>* __restrict__ src, bool ok, int t, cplx_t<T>* buf,
                                        const Addr& addr, const cplx_t<T>* tw, const cplx_t<T>* wk,
                                        cplx_t<T> (&v)[8]) {
    typedef cplx_t<T> C;
    constexpr int TL = M / 8;
    // stage X (M + 1 points) in shared memory for the X[M - k] partner reads
#pragma unroll
    for (int i = 0; i < 8; i++) buf[addr(t + i * TL)] = ok ? src[t + i * TL] : cmake<C>(0, 0);
    if (t == 0) buf[addr(M)] = ok ? src[M] : cmake<C>(0, 0);
    xsync<WS>();
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int k = t + i * TL;
        const C xk = buf[addr(k)];
        const C xc = cconj(buf[addr(M - k)]);
        const C ev = cadd(xk, xc);
        const C od = cmul(cconj(wk[k]), csub(xk, xc));
        v[i] = cadd(ev, cmul_i(od, +1));
    }
    xsync<WS>();
    fft_regs<C, M, +1, WS>(v, t, buf, addr, tw);
}

// Input rows read straight from global memory into the row buffer (register kernels).
template <typename T, int M> struct GlobalRows {
    typedef cplx_t<T> C;
    static constexpr bool PP = false;   // one exchange buffer (row_c2r uses fft_regs)
    const Specs<C>& in;
    int pitch;
    template <bool WS>
    __device__ __forceinline__ void row(int c, int64_t row, bool ok, int t, C* buf, const RowAddr& addr, const C* tw,
                                        const C* wk, C (&v)[8]) {
        row_c2r<T, M, WS>(select6(in, c) + row * pitch, ok, t, buf, addr, tw, wk, v);
    }
    __device__ __forceinline__ bool stop() { return false; }
};

// Inverse z pass over the tiles of ROWS rows, inputs fetched through `src` (GlobalRows, or the
// TMA-staged rows of fft_tma.cuh), epilogue ET.  tw, wk, buf: pass twiddles, real-FFT roots, the
// exchange buffer, filled by the caller.
template <typename T, int M, int ROWS, int ET, class Src>
__device__ __forceinline__ void z_c2r_body(Src& src, int nin, const Dims& dims, const Epi<T>& e,
                                           const cplx_t<T>* tw, const cplx_t<T>* wk, cplx_t<T>* buf) {
    typedef cplx_t<T> C;
    constexpr int TL = M / 8, N2 = 2 * M, RS = row_stride(M);
    constexpr int NMAX = EpiInputs<ET>::NMAX;
    constexpr bool WS = RowWarp<M, ROWS>::value;   // row-private exchanges synchronised per warp
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
                    src.template row<WS>(c, row, ok, t, buf, addr, tw, wk, v);
                    C* o = (C*)(e.out[c] + (ok ? row : 0) * N2);
                    if (ok) {
#pragma unroll
                        for (int i = 0; i < 8; i++) o[t + i * TL] = cmake<C>(v[i].x * sc, v[i].y * sc);
                    }
                }
            }
        } else if constexpr (ET == EPI_STORE4) {
            // three inputs -> one interleaved (x, y, z, 0) quadruple per cell
            C v0[8], v1[8], v2[8];
            src.template row<WS>(0, row, ok, t, buf, addr, tw, wk, v0);
            src.template row<WS>(1, row, ok, t, buf, addr, tw, wk, v1);
            src.template row<WS>(2, row, ok, t, buf, addr, tw, wk, v2);
            if (ok) {
                typedef typename vec4_of<T>::type V4;
                V4* o = (V4*)(e.out[0] + row * N2 * 4);
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const int k = t + i * TL;
                    o[2 * k] = make_vec4<T>(v0[i].x * sc, v1[i].x * sc, v2[i].x * sc);
                    o[2 * k + 1] = make_vec4<T>(v0[i].y * sc, v1[i].y * sc, v2[i].y * sc);
                }
            }
        } else if constexpr (ET == EPI_DENSITY) {
            C d[8], r[8];
            src.template row<WS>(0, row, ok, t, buf, addr, tw, wk, d);
            src.template row<WS>(1, row, ok, t, buf, addr, tw, wk, r);
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
            src.template row<WS>(0, row, ok, t, buf, addr, tw, wk, d);
            const double mean = e.sums[0] / e.ncells;
            if (ok) {
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const double o0 = ((double)(d[i].x * sc) / mean - 1.) / e.bias;
                    const double o1 = ((double)(d[i].y * sc) / mean - 1.) / e.bias;
                    out0[t + i * TL] = cmake<C>((T)o0, (T)o1);
                }
            }
        } else if constexpr (ET == EPI_ITER_POLY || ET == EPI_ITER_POLY_R2C) {
            // RSD removal from the quadratic in x2 formed by the Hessian y pass: inputs C, B, A, so
            // sum_ij f_ij x_i x_j d_ij = (C x2 + B) x2 + A, evaluated by Horner as the rows arrive.
            // EPI_ITER_POLY_R2C: the new real row goes straight into the next iteration's forward z
            // transform (row_r2c, the arithmetic of the r2c pass) instead of to memory.
            const T x0 = (T)(e.offset[0] + e.cell[0] * ix), x1 = (T)(e.offset[1] + e.cell[1] * iy);
            const T oz = (T)e.offset[2], cz = (T)e.cell[2];
            // the original density contrast is fetched first, so its latency hides behind the transforms
            const C* dl = (const C*)(e.delta + (ok ? row : 0) * N2);
            C dv[8];
#pragma unroll
            for (int i = 0; i < 8; i++) dv[i] = ok ? dl[t + i * TL] : cmake<C>(0, 0);
            T r[8][2];
#pragma unroll 1
            for (int c = 0; c < 3; c++) {
                C v[8];
                src.template row<WS>(c, row, ok, t, buf, addr, tw, wk, v);
#pragma unroll
                for (int i = 0; i < 8; i++) {
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const T val = (h ? v[i].y : v[i].x) * sc;
                        const T xz = oz + cz * (T)(2 * (t + i * TL) + h);
                        r[i][h] = c == 0 ? val : r[i][h] * xz + val;
                    }
                }
            }
            C z[8];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const C d0 = dv[i];
                T o[2];
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const T xz = oz + cz * (T)(2 * (t + i * TL) + h);
                    const T x2 = (x0 * x0 + x1 * x1) + xz * xz;
                    // FP32: fast reciprocal (2 ulp, far inside the FP32 mode's tolerance); FP64: exact
                    const T ix2 = sizeof(T) == 4 ? (T)__fdividef(1.f, (float)x2) : (T)1 / x2;
                    o[h] = (h ? d0.y : d0.x) - r[i][h] * ix2;
                }
                z[i] = ok ? cmake<C>(o[0], o[1]) : cmake<C>(0, 0);
            }
            if constexpr (ET == EPI_ITER_POLY_R2C) {
                C* dst = (C*)e.spec + (ok ? row : 0) * e.spec_pitch;
                if constexpr (Src::PP) {
                    // the inverse transforms exchanged through buf, buf2, buf, ...: the first buffer
                    // the forward one writes must not be the one their last exchange read
                    constexpr int NX = Shape<M>::NX;
                    if constexpr (NX == 0 || (NX - 1) % 2 == 0) xsync<WS>();
                    row_r2c_pp<T, M, WS>(z, ok, t, buf, src.buf2, addr, tw, wk, dst);
                    xsync<WS>();
                } else {
                    xsync<WS>();   // every thread of the row is past its reads of the exchange buffer
                    row_r2c<T, M, WS>(z, ok, t, buf, addr, tw, wk, dst);
                }
            } else if (ok) {
#pragma unroll
                for (int i = 0; i < 8; i++) out0[t + i * TL] = z[i];
            }
        } else {
            // RSD removal: delta_real = delta - sum_c factor_c w_c(x) IFFT_c, accumulated in registers;
            // w_c = x_i x_j / |x|^2 with 1/|x|^2 computed once per point, all in the mesh precision.
            const C* dl = (const C*)(e.delta + (ok ? row : 0) * N2);
            const T x0 = (T)(e.offset[0] + e.cell[0] * ix), x1 = (T)(e.offset[1] + e.cell[1] * iy);
            const T oz = (T)e.offset[2], cz = (T)e.cell[2];
            T acc[8][2], ix2[8][2];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const C d0 = ok ? dl[t + i * TL] : cmake<C>(0, 0);
                acc[i][0] = d0.x;
                acc[i][1] = d0.y;
                if constexpr (ET == EPI_ITER_LOCAL) {
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const T xz = oz + cz * (T)(2 * (t + i * TL) + h);
                        ix2[i][h] = (T)1 / ((x0 * x0 + x1 * x1) + xz * xz);
                    }
                }
            }
#pragma unroll 1
            for (int c = 0; c < NMAX; c++) {
                C v[8];
                src.template row<WS>(c, row, ok, t, buf, addr, tw, wk, v);
                const T fc = (T)select6(e.factor, c) * sc;
#pragma unroll
                for (int i = 0; i < 8; i++) {
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const T val = h ? v[i].y : v[i].x;
                        if constexpr (ET == EPI_ITER_GLOBAL) {
                            acc[i][h] -= fc * val;
                        } else {
                            // component c = (ci, cj) in the order (0,0) (0,1) (0,2) (1,1) (1,2) (2,2)
                            const int ci = c < 3 ? 0 : (c < 5 ? 1 : 2);
                            const int cj = c < 3 ? c : (c < 5 ? c - 2 : 2);
                            const T xz = oz + cz * (T)(2 * (t + i * TL) + h);
                            const T xi = ci == 0 ? x0 : (ci == 1 ? x1 : xz);
                            const T xj = cj == 0 ? x0 : (cj == 1 ? x1 : xz);
                            acc[i][h] -= fc * (xi * xj * val) * ix2[i][h];
                        }
                    }
                }
            }
            if (ok) {
#pragma unroll
                for (int i = 0; i < 8; i++) out0[t + i * TL] = cmake<C>(acc[i][0], acc[i][1]);
            }
        }
        if (src.stop()) return;
    }
}

template <typename T, int M, int ROWS, int ET>
__global__ void __launch_bounds__(M / 8 * ROWS, (MinBlocks<T, M / 8 * ROWS, PRC_C2R_MINB>::value))
    z_c2r(Specs<cplx_t<T>> in, int nin, Dims dims, int pitch, Epi<T> e) {
    typedef cplx_t<T> C;
    extern __shared__ unsigned char smem_raw[];
    C* tw = (C*)smem_raw;
    C* wk = tw + M;
    C* buf = wk + M + 1;
    fill_pass_twiddles<C, M>(tw);
    fill_roots(wk, M + 1, 2 * M);
    __syncthreads();
    GlobalRows<T, M> src{in, pitch};
    z_c2r_body<T, M, ROWS, ET>(src, nin, dims, e, tw, wk, buf);
}

}  // namespace fast

// Batched 3D real FFTs with fused k-space multipliers and real-space epilogues.
//
// A forward 3D r2c transform of an (n0, n1, n2) real mesh is three passes over the
// (n0, n1, nh = n2/2 + 1) half spectrum:
//   z: each row of n2 reals is read as n2/2 complex pairs, transformed (n2/2-point FFT) and
//      unpacked to nh complex (the standard real-FFT packing);
//   y, x: strided lines, a tile of B adjacent z-columns loaded per CTA so global accesses are
//      coalesced, transformed in shared memory.
// The k-space step of every algorithm sits between the forward and the inverse x transform,
// so one kernel does forward x, multiply (one or several outputs), inverse x.  The inverse z
// pass (c2r) ends with the real-space epilogue of the step (store, density contrast, or the
// Burden et al. RSD-removal update), so no intermediate real mesh is written.
//
// FFT core: Stockham autosort with mixed radices 8/4/2/3/5/7 (Govindaraju et al., SC08:
// pass with radix R and sub-transform size Ns reads x[j + r n/R], twiddles by w_{Ns R}^{r (j mod Ns)},
// does an R-point DFT and writes y[(j - j mod Ns) R + (j mod Ns) + r Ns]), ping-ponging between two
// shared-memory buffers laid out (k, line) with the line index fastest.
//
// Multipliers are applied Hermitian-symmetrised, M_h(k) = (M(k) + conj M(k~)) / 2 with
// k~ the wavevector of the reflected index (-k except on a Nyquist plane, where k~ = k), which
// is exactly what the reference's full complex transform followed by .real computes
// (pyrecon/mesh.py:842, recon.py:117).
#include "common.cuh"
#include "tma.cuh"

#include <algorithm>
#include <map>
#include <mutex>
#include <math.h>
#include <string.h>
#include <stdlib.h>

namespace prc {

constexpr int FFT_THREADS = 256;
constexpr int MAX_RADICES = 16;
constexpr int MAX_FFT_N = 2048;       // any length up to this on the shared-memory (generic) kernels
constexpr int MAX_FAST_N = 1024;      // register-resident power-of-two kernels
constexpr int MAX_BATCH = 6;

struct Radices {
    int n;
    int count;
    int r[MAX_RADICES];
};

static bool factorize(int n, Radices* out) {
    Radices rd;
    rd.n = n;
    rd.count = 0;
    int m = n;
    while (m % 8 == 0 && m > 0) { rd.r[rd.count++] = 8; m /= 8; }
    if (m % 4 == 0) { rd.r[rd.count++] = 4; m /= 4; }
    if (m % 2 == 0) { rd.r[rd.count++] = 2; m /= 2; }
    // odd primes in increasing order: 3, 5, 7 have their own butterflies, larger ones (11, 13, ...,
    // up to a prime length itself) run the direct-summation pass
    for (int f = 3; m > 1; f += 2) {
        if (f * f > m) f = m;
        while (m % f == 0) {
            if (rd.count >= MAX_RADICES) return false;
            rd.r[rd.count++] = f;
            m /= f;
        }
    }
    *out = rd;
    return true;
}

// ---------------------------------------------------------------------------------------------
// Small DFTs (DIR = -1 forward, +1 inverse)
// ---------------------------------------------------------------------------------------------
template <typename C, int DIR> __device__ __forceinline__ void dft2(C* v) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}

template <typename C, int DIR> __device__ __forceinline__ void dft4(C* v) {
    C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    C t2 = cadd(v[1], v[3]), t3 = cmul_i(csub(v[1], v[3]), DIR);
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
}

template <typename C, int DIR> __device__ __forceinline__ void dft8(C* v) {
    typedef decltype(C().x) T;
    const T h = (T)0.70710678118654752440;   // 1/sqrt(2)
    C e[4] = {v[0], v[2], v[4], v[6]};
    C o[4] = {v[1], v[3], v[5], v[7]};
    dft4<C, DIR>(e);
    dft4<C, DIR>(o);
    // o_k *= w8^k, w8 = exp(DIR i pi / 4)
    C o1 = o[1];
    o[1] = cmake<C>(h * (o1.x - DIR * o1.y), h * (o1.y + DIR * o1.x));
    o[2] = cmul_i(o[2], DIR);
    C o3 = o[3];
    o[3] = cmake<C>(h * (-o3.x - DIR * o3.y), h * (-o3.y + DIR * o3.x));
#pragma unroll
    for (int k = 0; k < 4; k++) {
        v[k] = cadd(e[k], o[k]);
        v[k + 4] = csub(e[k], o[k]);
    }
}

template <typename C, int DIR> __device__ __forceinline__ void dft3(C* v) {
    typedef decltype(C().x) T;
    const T s = (T)0.86602540378443864676;   // sin(2 pi / 3)
    C a = v[0], b = v[1], c = v[2];
    C sum = cadd(b, c), dif = csub(b, c);
    C t = cmake<C>(a.x - (T)0.5 * sum.x, a.y - (T)0.5 * sum.y);
    C u = cmul_i(cscale(dif, s), DIR);   // DIR i s (b - c)
    v[0] = cadd(a, sum);
    v[1] = cadd(t, u);
    v[2] = csub(t, u);
}

template <typename C, int DIR> __device__ __forceinline__ void dft5(C* v) {
    typedef decltype(C().x) T;
    const T c1 = (T)0.30901699437494742410;   // cos(2 pi / 5)
    const T c2 = (T)-0.80901699437494742410;  // cos(4 pi / 5)
    const T s1 = (T)0.95105651629515357212;   // sin(2 pi / 5)
    const T s2 = (T)0.58778525229247312917;   // sin(4 pi / 5)
    C a = v[0];
    C b1 = cadd(v[1], v[4]), d1 = csub(v[1], v[4]);
    C b2 = cadd(v[2], v[3]), d2 = csub(v[2], v[3]);
    C t1 = cmake<C>(a.x + c1 * b1.x + c2 * b2.x, a.y + c1 * b1.y + c2 * b2.y);
    C t2 = cmake<C>(a.x + c2 * b1.x + c1 * b2.x, a.y + c2 * b1.y + c1 * b2.y);
    C u1 = cmul_i(cmake<C>(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y), DIR);
    C u2 = cmul_i(cmake<C>(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y), DIR);
    v[0] = cadd(a, cadd(b1, b2));
    v[1] = cadd(t1, u1);
    v[4] = csub(t1, u1);
    v[2] = cadd(t2, u2);
    v[3] = csub(t2, u2);
}

// Generic R-point DFT from the twiddle table (w_n^m, n a multiple of R): used for R = 7.
template <typename C, int DIR, int R>
__device__ __forceinline__ void dft_generic(C* v, const C* __restrict__ tw, int n, int tws) {
    C out[R];
    const int step = n / R;
#pragma unroll
    for (int m = 0; m < R; m++) {
        C acc = v[0];
#pragma unroll
        for (int r = 1; r < R; r++) {
            C w = tw[(((r * m) % R) * step) * tws];
            if (DIR > 0) w = cconj(w);
            acc = cadd(acc, cmul(v[r], w));
        }
        out[m] = acc;
    }
#pragma unroll
    for (int m = 0; m < R; m++) v[m] = out[m];
}

// One Stockham pass of radix R over B lines of length n stored (k, line) at k * bp + line.
template <typename C, int DIR, int R>
__device__ __forceinline__ void stockham_pass(const C* __restrict__ src, C* __restrict__ dst, int n, int B, int bp,
                                              int Ns, const C* __restrict__ tw, int tws) {
    const int nb = n / R;
    const int twstep = n / (Ns * R);
    for (int q = threadIdx.x; q < nb * B; q += blockDim.x) {
        const int line = q % B, j = q / B;
        const int k = j % Ns;
        C v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = src[(j + r * nb) * bp + line];
        if (k > 0) {
#pragma unroll
            for (int r = 1; r < R; r++) {
                C w = tw[((r * k * twstep) % n) * tws];
                if (DIR > 0) w = cconj(w);
                v[r] = cmul(v[r], w);
            }
        }
        if (R == 2) dft2<C, DIR>(v);
        else if (R == 4) dft4<C, DIR>(v);
        else if (R == 8) dft8<C, DIR>(v);
        else if (R == 3) dft3<C, DIR>(v);
        else if (R == 5) dft5<C, DIR>(v);
        else dft_generic<C, DIR, R>(v, tw, n, tws);
        const int d = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) dst[(d + r * Ns) * bp + line] = v[r];
    }
}

// One Stockham pass of any radix R (the primes above 7) by direct summation: a thread makes one output
// m of one R-point sub-transform, y_m = sum_r x_r w_{Ns R}^{r k} w_R^{r m} = sum_r x_r w_n^{r E},
// E = k twstep + m nb (input twiddle and DFT kernel in one table lookup, exponent kept mod n by
// addition); O(R) operations per output.
template <typename C, int DIR>
__device__ __forceinline__ void stockham_pass_any(const C* __restrict__ src, C* __restrict__ dst, int n, int B, int bp,
                                                  int Ns, int R, const C* __restrict__ tw, int tws) {
    const int nb = n / R;
    const int twstep = n / (Ns * R);
    for (int q = threadIdx.x; q < n * B; q += blockDim.x) {
        const int line = q % B, rest = q / B;
        const int j = rest % nb, m = rest / nb;
        const int k = j % Ns;
        const int E = (k * twstep + m * nb) % n;
        C acc = src[j * bp + line];
        int ex = 0;
        for (int r = 1; r < R; r++) {
            ex += E;
            if (ex >= n) ex -= n;
            C w = tw[ex * tws];
            if (DIR > 0) w = cconj(w);
            acc = cadd(acc, cmul(src[(j + r * nb) * bp + line], w));
        }
        dst[((j - k) * R + k + m * Ns) * bp + line] = acc;
    }
}

// Transforms B lines in place-ish: data in `a`, scratch `b`; returns the buffer with the result.
// tw holds w_{n*tws}^m (so entry m*tws is w_n^m).
template <typename C, int DIR>
__device__ C* fft_lines(C* a, C* b, int n, int B, int bp, const Radices& rd, const C* __restrict__ tw, int tws) {
    int Ns = 1;
    for (int p = 0; p < rd.count; p++) {
        const int R = rd.r[p];
        switch (R) {
            case 8: stockham_pass<C, DIR, 8>(a, b, n, B, bp, Ns, tw, tws); break;
            case 4: stockham_pass<C, DIR, 4>(a, b, n, B, bp, Ns, tw, tws); break;
            case 2: stockham_pass<C, DIR, 2>(a, b, n, B, bp, Ns, tw, tws); break;
            case 3: stockham_pass<C, DIR, 3>(a, b, n, B, bp, Ns, tw, tws); break;
            case 5: stockham_pass<C, DIR, 5>(a, b, n, B, bp, Ns, tw, tws); break;
            case 7: stockham_pass<C, DIR, 7>(a, b, n, B, bp, Ns, tw, tws); break;
            default: stockham_pass_any<C, DIR>(a, b, n, B, bp, Ns, R, tw, tws); break;
        }
        __syncthreads();
        C* t = a;
        a = b;
        b = t;
        Ns *= R;
    }
    return a;
}

// Twiddle table w_n^m = exp(-2 pi i m / n), m in [0, n), computed in double then rounded.
template <typename C> __device__ void fill_twiddles(C* tw, int n) {
    for (int m = threadIdx.x; m < n; m += blockDim.x) {
        double s, c;
        sincospi(-2.0 * (double)m / (double)n, &s, &c);
        tw[m] = cmake<C>((decltype(C().x))c, (decltype(C().x))s);
    }
}

// ---------------------------------------------------------------------------------------------
// Pointer packs
// ---------------------------------------------------------------------------------------------
template <typename C> struct Specs { C* p[MAX_BATCH]; };
struct RealsIn { const void* p[MAX_BATCH]; };

// ---------------------------------------------------------------------------------------------
// z pass, forward r2c.  Tile = B rows (lines along z) of one mesh of the batch.
// Even n2: each row of n2 reals is read as n2/2 complex pairs (the packed real-FFT).  Odd n2: each row
// is transformed as n2 complex values with zero imaginary parts and the first nh = (n2 + 1)/2
// outputs are kept.  Buffers hold (k, line) at k * bp + line (bp = B + 1, or 1 for one row).
// ---------------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ int row_pitch(int B) { return B > 1 ? B + 1 : 1; }

template <typename T, typename TIN>
__global__ void __launch_bounds__(FFT_THREADS) fft_z_r2c(RealsIn in, Specs<cplx_t<T>> out, int nbatch, Dims dims,
                                                          int pitch, Radices rd, int B) {
    typedef cplx_t<T> C;
    extern __shared__ unsigned char smem_raw[];
    const int n2 = dims.n[2], nh = n2 / 2 + 1;
    const bool full = (n2 & 1) != 0;
    const int M = full ? n2 : n2 / 2;              // transform length
    const int L = full ? n2 : M + 1;               // buffer rows
    const int bp = row_pitch(B);
    C* tw = (C*)smem_raw;                          // n2 entries
    C* bufa = tw + n2;                             // L * bp
    C* bufb = bufa + L * bp;
    fill_twiddles(tw, n2);
    __syncthreads();
    const int64_t rows = (int64_t)dims.n[0] * dims.n[1];
    const int64_t tiles_per = (rows + B - 1) / B;
    const int64_t ntiles = tiles_per * nbatch;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int bi = (int)(t / tiles_per);
        const int64_t row0 = (t % tiles_per) * B;
        const int nrow = (int)min((int64_t)B, rows - row0);
        const TIN* src = (const TIN*)in.p[bi] + row0 * n2;
        if (full) {
            for (int q = threadIdx.x; q < B * n2; q += blockDim.x) {
                const int line = q / n2, m = q % n2;
                bufa[m * bp + line] = cmake<C>(line < nrow ? (T)src[(int64_t)line * n2 + m] : (T)0, (T)0);
            }
        } else {
            // load rows as complex pairs (x[2m], x[2m+1])
            for (int q = threadIdx.x; q < B * M; q += blockDim.x) {
                const int line = q / M, m = q % M;
                C v = cmake<C>((T)0, (T)0);
                if (line < nrow) {
                    const TIN* r = src + (int64_t)line * n2 + 2 * m;
                    v = cmake<C>((T)r[0], (T)r[1]);
                }
                bufa[m * bp + line] = v;
            }
        }
        __syncthreads();
        C* z = fft_lines<C, -1>(bufa, bufb, M, B, bp, rd, tw, full ? 1 : 2);
        C* x = z;
        if (!full) {
            x = z == bufa ? bufb : bufa;
            // unpack: X[k] = (Z[k] + conj Z[M-k]) / 2 - i w^k (Z[k] - conj Z[M-k]) / 2
            for (int q = threadIdx.x; q < B * nh; q += blockDim.x) {
                const int line = q % B, k = q / B;
                const C zk = z[(k == M ? 0 : k) * bp + line];
                const C zc = cconj(z[(k == 0 ? 0 : M - k) * bp + line]);
                const C e = cscale(cadd(zk, zc), (T)0.5);
                const C o = cmul_i(cscale(csub(zk, zc), (T)0.5), -1);   // -i (Zk - Zc*) / 2
                x[k * bp + line] = cadd(e, cmul(tw[k == M ? M : k], o));
            }
            __syncthreads();
        }
        C* dst = out.p[bi] + row0 * pitch;
        for (int q = threadIdx.x; q < B * nh; q += blockDim.x) {
            const int line = q / nh, k = q % nh;
            if (line < nrow) dst[(int64_t)line * pitch + k] = x[k * bp + line];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Strided pass (y or x axis), in place.  Element (k, col) of a tile at
// base + k * ls + col, base = outer * os + c0.
// ---------------------------------------------------------------------------------------------
struct Strided {
    int n;          // line length
    int64_t ls;     // stride between line elements
    int outer;      // number of outer positions
    int64_t os;     // outer stride
    int ncols;      // columns (z extent nh)
};

template <typename C>
__device__ __forceinline__ void load_tile(C* buf, const C* __restrict__ g, const Strided& s, int B, int cols) {
    for (int q = threadIdx.x; q < s.n * B; q += blockDim.x) {
        const int k = q / B, col = q % B;
        buf[k * B + col] = col < cols ? g[(int64_t)k * s.ls + col] : cmake<C>(0, 0);
    }
}

template <typename C>
__device__ __forceinline__ void store_tile(C* __restrict__ g, const C* buf, const Strided& s, int B, int cols) {
    for (int q = threadIdx.x; q < s.n * B; q += blockDim.x) {
        const int k = q / B, col = q % B;
        if (col < cols) g[(int64_t)k * s.ls + col] = buf[k * B + col];
    }
}

template <typename T, int DIR>
__global__ void __launch_bounds__(FFT_THREADS) fft_strided(Specs<cplx_t<T>> data, int nbatch, Strided s, Radices rd,
                                                            int B) {
    typedef cplx_t<T> C;
    extern __shared__ unsigned char smem_raw[];
    C* tw = (C*)smem_raw;
    C* bufa = tw + s.n;
    C* bufb = bufa + s.n * B;
    fill_twiddles(tw, s.n);
    __syncthreads();
    const int ctiles = (s.ncols + B - 1) / B;
    const int64_t tiles_per = (int64_t)s.outer * ctiles;
    const int64_t ntiles = tiles_per * nbatch;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int bi = (int)(t / tiles_per);
        const int64_t r = t % tiles_per;
        const int o = (int)(r / ctiles), c0 = (int)(r % ctiles) * B;
        const int cols = min(B, s.ncols - c0);
        C* g = data.p[bi] + (int64_t)o * s.os + c0;
        load_tile(bufa, g, s, B, cols);
        __syncthreads();
        C* res = fft_lines<C, DIR>(bufa, bufb, s.n, B, B, rd, tw, 1);
        store_tile(g, res, s, B, cols);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// k-space operators (applied between forward and inverse x transforms)
// ---------------------------------------------------------------------------------------------
// KOP_HESS3 (TMA passes only): the three x-transformed spectra of the local-line-of-sight iteration,
// E, s_x E and k_x^2 E with E = delta / k^2, plus the two Nyquist lines written to `side` (see
// fast::y_hessian_tma).
enum KOpType { KOP_IDENTITY = 0, KOP_GAUSS = 1, KOP_PP = 2, KOP_ITER_GLOBAL = 3, KOP_ITER_LOCAL = 4, KOP_PSI = 5,
               KOP_HESS3 = 6 };

struct KOp {
    int type;
    int nper;            // outputs per input
    int n[3];
    double fscale[3];    // numpy fftfreq spacing 1 / (n d), d = boxsize / n
    double radius[3];
    double los[3];
    double beta;
    double norm;         // overall scale (1 / (n0 n1 n2) when the inverse follows)
    void* side;          // KOP_HESS3: nh + n1 complex values (the Nyquist lines Q01, L02)
};

__device__ __forceinline__ double kvalue(int i, int n, double fscale) {
    const int s = i < (n + 1) / 2 ? i : i - n;
    return 6.283185307179586 * ((double)s * fscale);   // 2 * np.pi * fftfreq(n, d)
}

__device__ __forceinline__ bool nyquist(int i, int n) { return (n % 2 == 0) && i == n / 2; }

// Complex multiplier (re, im) of output `o` at grid point (ix, iy, iz), symmetrised.
__device__ __forceinline__ double2 kmultiplier(const KOp& op, int o, int ix, int iy, int iz) {
    const int idx[3] = {ix, iy, iz};
    double k[3], kt[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        k[a] = kvalue(idx[a], op.n[a], op.fscale[a]);
        kt[a] = nyquist(idx[a], op.n[a]) ? k[a] : -k[a];
    }
    const double k2 = (k[1] * k[1] + k[0] * k[0]) + k[2] * k[2];   // prod_sum order (mesh.c:335-337)
    const bool zero = (ix == 0 && iy == 0 && iz == 0);
    double re = 0., im = 0.;
    switch (op.type) {
        case KOP_GAUSS: {
            double e = 0.;
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const double rk = op.radius[a] * k[a];
                e += -0.5 * (rk * rk);
            }
            re = exp(e);
            break;
        }
        case KOP_PP: {
            if (zero) break;
            const double kl = k[0] * op.los[0] + k[1] * op.los[1] + k[2] * op.los[2];
            const double klt = kt[0] * op.los[0] + kt[1] * op.los[1] + kt[2] * op.los[2];
            const double m = k[o] / (k2 * (1. + op.beta * (kl * kl / k2)));
            const double mt = kt[o] / (k2 * (1. + op.beta * (klt * klt / k2)));
            im = 0.5 * (m - mt);   // (i m + conj(i mt)) / 2
            break;
        }
        case KOP_ITER_GLOBAL: {
            if (zero) break;
            const double kl = k[0] * op.los[0] + k[1] * op.los[1] + k[2] * op.los[2];
            const double klt = kt[0] * op.los[0] + kt[1] * op.los[1] + kt[2] * op.los[2];
            re = 0.5 * (kl * kl + klt * klt) / k2;
            break;
        }
        case KOP_ITER_LOCAL: {
            if (zero) break;
            const int pi[6] = {0, 0, 0, 1, 1, 2}, pj[6] = {0, 1, 2, 1, 2, 2};
            const int i = pi[o], j = pj[o];
            re = 0.5 * (k[i] * k[j] + kt[i] * kt[j]) / k2;
            break;
        }
        case KOP_PSI: {
            if (zero) break;
            im = 0.5 * (k[o] - kt[o]) / k2;
            break;
        }
        default:
            re = 1.;
    }
    return make_double2(re * op.norm, im * op.norm);
}

template <typename T>
__global__ void __launch_bounds__(FFT_THREADS) fft_x_fused(Specs<cplx_t<T>> in, int nin, Specs<cplx_t<T>> out,
                                                            Dims dims, int pitch, Radices rd, int B, KOp op) {
    typedef cplx_t<T> C;
    extern __shared__ unsigned char smem_raw[];
    const int n0 = dims.n[0], n1 = dims.n[1], nh = dims.n[2] / 2 + 1;
    C* tw = (C*)smem_raw;
    C* spec = tw + n0;
    C* bufa = spec + n0 * B;
    C* bufb = bufa + n0 * B;
    fill_twiddles(tw, n0);
    __syncthreads();
    Strided s;
    s.n = n0;
    s.ls = (int64_t)n1 * pitch;
    s.outer = n1;
    s.os = pitch;
    s.ncols = nh;
    const int ctiles = (nh + B - 1) / B;
    const int64_t tiles_per = (int64_t)n1 * ctiles;
    const int64_t ntiles = tiles_per * nin;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int bi = (int)(t / tiles_per);
        const int64_t r = t % tiles_per;
        const int iy = (int)(r / ctiles), c0 = (int)(r % ctiles) * B;
        const int cols = min(B, nh - c0);
        const int64_t off = (int64_t)iy * pitch + c0;
        load_tile(bufa, in.p[bi] + off, s, B, cols);
        __syncthreads();
        C* fwd = fft_lines<C, -1>(bufa, bufb, n0, B, B, rd, tw, 1);
        // keep the spectrum: copy to `spec` (the other buffer becomes free)
        for (int q = threadIdx.x; q < n0 * B; q += blockDim.x) spec[q] = fwd[q];
        __syncthreads();
        for (int o = 0; o < op.nper; o++) {
            for (int q = threadIdx.x; q < n0 * B; q += blockDim.x) {
                const int ix = q / B, col = q % B;
                const double2 m = kmultiplier(op, o, ix, iy, c0 + col);
                const C v = spec[q];
                bufa[q] = cmake<C>((T)(m.x * (double)v.x - m.y * (double)v.y), (T)(m.x * (double)v.y + m.y * (double)v.x));
            }
            __syncthreads();
            C* res = fft_lines<C, +1>(bufa, bufb, n0, B, B, rd, tw, 1);
            store_tile(out.p[bi * op.nper + o] + off, res, s, B, cols);
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------------------------
// z pass, inverse c2r, with real-space epilogues
// ---------------------------------------------------------------------------------------------
// EPI_ITER_POLY_R2C: EPI_ITER_POLY whose real row is not stored but transformed forward at once (the
// next iteration's r2c z pass, same arithmetic) into the spectrum rows at `spec`.
enum EpiType { EPI_STORE = 0, EPI_DENSITY = 1, EPI_DENSITY_NORANDOMS = 2, EPI_ITER_GLOBAL = 3, EPI_ITER_LOCAL = 4,
               EPI_STORE4 = 5, EPI_ITER_POLY = 6, EPI_ITER_POLY_R2C = 7 };

template <typename T> struct Epi {
    int type;
    T* out[3];             // EPI_STORE: one output per input; EPI_STORE4: out[0] = (N, 4) interleaved
    const T* delta;        // original density contrast (EPI_ITER_*)
    const double* sums;    // device {sum data, sum randoms} (EPI_DENSITY*)
    double scale;          // applied to every inverse-transformed value
    double bias, ran_min, size_randoms, ncells;
    double factor[6];      // RSD-removal factors (EPI_ITER_*)
    double offset[3], cell[3];   // node coordinates x_a = offset_a + cell_a * i (EPI_ITER_LOCAL)
    void* spec;            // EPI_ITER_POLY_R2C: the z-transformed rows (complex T, spec_pitch values a row)
    int spec_pitch;
};

// Epilogue of one cell (row, iz): vals[c * stride] is the inverse transform of input c there.
template <typename T>
__device__ __forceinline__ T epilogue_value(const Epi<T>& e, const T* vals, int stride, int64_t row, int iz,
                                            const Dims& dims) {
    const int64_t cell = row * dims.n[2] + iz;
    double res = 0.;
    switch (e.type) {
        case EPI_DENSITY: {
            const double d = (double)vals[0], r = (double)vals[stride];
            const double sd = e.sums[0], sr = e.sums[1];
            const double alpha = sd * 1. / sr;
            const double threshold = e.ran_min * sr / e.size_randoms;
            res = r > threshold ? (d - alpha * r) / (e.bias * alpha * r) : 0.;
            break;
        }
        case EPI_DENSITY_NORANDOMS: {
            const double mean = e.sums[0] / e.ncells;
            res = ((double)vals[0] / mean - 1.) / e.bias;
            break;
        }
        case EPI_ITER_GLOBAL: {
            res = (double)e.delta[cell] - e.factor[0] * (double)vals[0];
            break;
        }
        case EPI_ITER_LOCAL: {
            const int ix = (int)(row / dims.n[1]), iy = (int)(row % dims.n[1]);
            const double x[3] = {e.offset[0] + e.cell[0] * ix, e.offset[1] + e.cell[1] * iy,
                                 e.offset[2] + e.cell[2] * iz};
            const double x2 = (x[0] * x[0] + x[1] * x[1]) + x[2] * x[2];
            const int pi[6] = {0, 0, 0, 1, 1, 2}, pj[6] = {0, 1, 2, 1, 2, 2};
            double v = (double)e.delta[cell];
            for (int c = 0; c < 6; c++)
                v -= e.factor[c] * ((x[pi[c]] * x[pj[c]] * (double)vals[c * stride]) / x2);
            res = v;
            break;
        }
        case EPI_ITER_POLY: {
            // inputs C, B, A of the quadratic in x2 formed by the Hessian y pass: the RSD term is
            // ((C x2 + B) x2 + A) / |x|^2
            const int ix = (int)(row / dims.n[1]), iy = (int)(row % dims.n[1]);
            const double x0 = e.offset[0] + e.cell[0] * ix, x1 = e.offset[1] + e.cell[1] * iy;
            const double xz = e.offset[2] + e.cell[2] * iz;
            const double x2 = (x0 * x0 + x1 * x1) + xz * xz;
            const double poly = ((double)vals[0] * xz + (double)vals[stride]) * xz + (double)vals[2 * stride];
            res = (double)e.delta[cell] - poly / x2;
            break;
        }
        default:
            res = (double)vals[0];
    }
    return (T)res;
}

// Stores the inverse-transformed values of one cell: one output per input (EPI_STORE), the (N, 4)
// interleaved displacement (EPI_STORE4) or the epilogue's single output.
template <typename T>
__device__ __forceinline__ void epilogue_store(const Epi<T>& e, int nin, const T* vals, int stride, int64_t row, int iz,
                                               const Dims& dims) {
    const int64_t cell = row * dims.n[2] + iz;
    if (e.type == EPI_STORE) {
        for (int i = 0; i < nin; i++) e.out[i][cell] = vals[i * stride];
    } else if (e.type == EPI_STORE4) {
        T* o = e.out[0] + cell * 4;
        for (int i = 0; i < 3; i++) o[i] = vals[i * stride];
        o[3] = 0;
    } else {
        e.out[0][cell] = epilogue_value(e, vals, stride, row, iz, dims);
    }
}

// Inverse z pass.  Even n2: the nh = n2/2 + 1 Hermitian-half values are packed into n2/2 complex
// values whose inverse transform holds (x[2m], x[2m+1]).  Odd n2: the half is completed to all n2
// values by Hermitian symmetry (X[n2 - k] = conj X[k]) and the real part of its n2-point inverse kept,
// which is the reference's full complex inverse followed by .real.
template <typename T>
__global__ void __launch_bounds__(FFT_THREADS) fft_z_c2r(Specs<cplx_t<T>> in, int nin, Dims dims, int pitch,
                                                          Radices rd, int B, Epi<T> e) {
    typedef cplx_t<T> C;
    extern __shared__ unsigned char smem_raw[];
    const int n2 = dims.n[2], nh = n2 / 2 + 1;
    const bool full = (n2 & 1) != 0;
    const int M = full ? n2 : n2 / 2;          // transform length
    const int L = full ? n2 : nh;              // buffer rows
    const int bp = row_pitch(B);
    C* tw = (C*)smem_raw;                    // n2
    C* bufa = tw + n2;                       // L * bp
    C* bufb = bufa + L * bp;                 // L * bp
    T* acc = (T*)(bufb + L * bp);            // nin * B * n2 reals kept for the epilogue, row-major per input
    fill_twiddles(tw, n2);
    __syncthreads();
    const int64_t rows = (int64_t)dims.n[0] * dims.n[1];
    const int64_t ntiles = (rows + B - 1) / B;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int64_t row0 = t * B;
        const int nrow = (int)min((int64_t)B, rows - row0);
        for (int i = 0; i < nin; i++) {
            const C* src = in.p[i] + row0 * pitch;
            for (int q = threadIdx.x; q < B * nh; q += blockDim.x) {
                const int line = q / nh, k = q % nh;
                bufa[k * bp + line] = line < nrow ? src[(int64_t)line * pitch + k] : cmake<C>(0, 0);
            }
            __syncthreads();
            C* z;
            if (full) {
                for (int q = threadIdx.x; q < B * (n2 - nh); q += blockDim.x) {
                    const int line = q % B, k = nh + q / B;
                    bufa[k * bp + line] = cconj(bufa[(n2 - k) * bp + line]);
                }
                __syncthreads();
                z = fft_lines<C, +1>(bufa, bufb, n2, B, bp, rd, tw, 1);
                for (int q = threadIdx.x; q < B * n2; q += blockDim.x) {
                    const int line = q / n2, m = q % n2;
                    acc[((int64_t)i * B + line) * n2 + m] = (T)(z[m * bp + line].x * e.scale);
                }
            } else {
                // pack: Z[k] = (X[k] + conj X[M-k]) + i w^-k (X[k] - conj X[M-k]), k < M
                for (int q = threadIdx.x; q < B * M; q += blockDim.x) {
                    const int line = q % B, k = q / B;
                    const C xk = bufa[k * bp + line];
                    const C xc = cconj(bufa[(M - k) * bp + line]);
                    const C ev = cadd(xk, xc);
                    const C od = cmul(cconj(tw[k]), csub(xk, xc));
                    bufb[k * bp + line] = cadd(ev, cmul_i(od, +1));
                }
                __syncthreads();
                z = fft_lines<C, +1>(bufb, bufa, M, B, bp, rd, tw, 2);
                // (x[2m], x[2m+1]) * scale
                for (int q = threadIdx.x; q < B * M; q += blockDim.x) {
                    const int line = q / M, m = q % M;
                    const C v = z[m * bp + line];
                    T* a = acc + ((int64_t)i * B + line) * n2 + 2 * m;
                    a[0] = (T)(v.x * e.scale);
                    a[1] = (T)(v.y * e.scale);
                }
            }
            __syncthreads();
        }
        for (int q = threadIdx.x; q < B * n2; q += blockDim.x) {
            const int line = q / n2, iz = q % n2;
            if (line >= nrow) continue;
            epilogue_store(e, nin, acc + (int64_t)line * n2 + iz, B * n2, row0 + line, iz, dims);
        }
        __syncthreads();
    }
}

// Device fault word of the FFT kernels (bits prc::tma::FAULT_*), read by prc_device_fault_flags.
__device__ unsigned int g_fault;

// Failure path of the bounded waits, on purpose: thread 0 arms the CTA's transaction barrier for
// `bytes` that no copy will ever deliver (no copy is issued, so nothing is in flight), every thread
// waits on it for at most `limit_ns`, the wait runs out, the fault bit is set and the kernel returns
// with the barrier invalidated.  `out[0]` = 1 when the wait gave up, 0 if it (impossibly) completed.
__global__ void debug_wait_timeout(uint64_t limit_ns, uint32_t bytes, int* out) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        tma::barrier_init(&bar, 1);
        tma::fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) tma::arrive_expect_tx(&bar, bytes);
    const bool done = tma::wait_for(&bar, 0, limit_ns);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (!done) atomicOr(&g_fault, tma::FAULT_WAIT_TIMEOUT);
        out[0] = done ? 0 : 1;
        tma::barrier_inval(&bar);
    }
}

#include "fft_fast.cuh"
#include "fft_tma.cuh"

// ---------------------------------------------------------------------------------------------
// Host-side planning and launches
// ---------------------------------------------------------------------------------------------
struct Plan3 {
    Dims dims;
    int nh;
    int pitch;            // row stride of the half spectra in complex elements (>= nh)
    Radices rz, ry, rx;   // rz: the n2/2-point packed transform (even n2) or the n2-point one (odd n2)
};

// Any axis length in [2, MAX_FFT_N]: powers of two up to MAX_FAST_N and 96, 192, 384 run the
// register-resident kernels (fast_len), every other length (radices 8, 4, 2, 3, 5, 7 and any larger
// prime; an odd last axis unpacked) the shared-memory kernels.
static int make_plan(const int32_t nmesh[3], Plan3* p) {
    for (int d = 0; d < 3; d++)
        if (nmesh[d] < 2 || nmesh[d] > MAX_FFT_N) return PRC_ERR_UNSUPPORTED;
    for (int d = 0; d < 3; d++) p->dims.n[d] = nmesh[d];
    p->nh = nmesh[2] / 2 + 1;
    p->pitch = p->nh;
    const int zlen = nmesh[2] % 2 ? nmesh[2] : nmesh[2] / 2;
    if (!factorize(zlen, &p->rz) || !factorize(nmesh[1], &p->ry) || !factorize(nmesh[0], &p->rx))
        return PRC_ERR_UNSUPPORTED;
    return PRC_OK;
}

static size_t spectrum_elems(const Plan3& p) { return (size_t)p.dims.n[0] * p.dims.n[1] * p.pitch; }
// Complex values of one half spectrum, without the row padding (the compulsory bytes of a pass).
static double spectrum_values(const Plan3& p) { return (double)p.dims.n[0] * p.dims.n[1] * p.nh; }

// Spectra inside the library's own workspaces get rows padded to a multiple of 32 bytes, so every
// row and every tile of adjacent z-columns starts on a sector boundary (and the row stride meets the
// 16-byte rule of the tensor-memory-access copies).
template <typename T> static void pad_pitch(Plan3* p) {
    const int q = (int)(32 / sizeof(cplx_t<T>));
    p->pitch = (p->nh + q - 1) / q * q;
}

// Lines per tile B (power of two) so that `nbuf` buffers of n * B complex fit the budget.
static int choose_B(int n, int nbuf, size_t csize, size_t budget, int bmax) {
    int B = bmax;
    while (B > 1 && (size_t)nbuf * n * B * csize > budget) B >>= 1;
    return B;
}

static int fft_grid(int64_t ntiles, int ctas_per_sm) {
    int64_t cap = (int64_t)device_sm_count() * ctas_per_sm;
    return (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, cap));
}

// Lengths of the register-resident kernels: powers of two from 8 to MAX_FAST_N, and 96, 192, 384 (three
// times a power of two: three sub-transforms and a radix-3 step, fft_fast.cuh).
static bool fast_len(int n) {
    return (n >= 8 && n <= MAX_FAST_N && (n & (n - 1)) == 0) || n == 96 || n == 192 || n == 384;
}

// PRC_FFT_GENERIC=1 in the environment routes every size through the mixed-radix kernels
// (the tests use it to keep that path checked on power-of-two sizes too).
static bool getenv_generic() {
    static int cached = -1;
    if (cached < 0) {
        const char* v = getenv("PRC_FFT_GENERIC");
        cached = (v != nullptr && v[0] == '1') ? 1 : 0;
    }
    return cached == 1;
}

// Compile-time dispatch of a runtime length (fast_len) onto F<N>::run(args...).
template <template <int> class F, typename... A> static int dispatch_pow2(int n, A... a) {
    switch (n) {
        case 96: return F<96>::run(a...);
        case 192: return F<192>::run(a...);
        case 384: return F<384>::run(a...);
        case 8: return F<8>::run(a...);
        case 16: return F<16>::run(a...);
        case 32: return F<32>::run(a...);
        case 64: return F<64>::run(a...);
        case 128: return F<128>::run(a...);
        case 256: return F<256>::run(a...);
        case 512: return F<512>::run(a...);
        case 1024: return F<1024>::run(a...);
        default: return PRC_ERR_UNSUPPORTED;
    }
}

// Tile shapes (tuning knobs, overridable at build time):
//   PRC_STRIDED_B  columns per strided-pass tile in FP32 (FP64 uses half as many bytes' worth)
//   PRC_KSPACE_B   columns per k-space tile in FP32
//   PRC_ROW_THREADS target threads per z-pass CTA
#ifndef PRC_STRIDED_B
#define PRC_STRIDED_B 8
#endif
#ifndef PRC_KSPACE_B
#define PRC_KSPACE_B 8
#endif
#ifndef PRC_ROW_THREADS
#define PRC_ROW_THREADS 256
#endif

// Lines per strided tile: 64-byte rows (8 FP32 / 4 FP64 complex), at most 1024 threads.
template <typename T, int N> struct StridedCfg {
    static constexpr int B0 = sizeof(T) == 4 ? PRC_STRIDED_B : PRC_STRIDED_B / 2;
    static constexpr int B = (N / 8) * B0 <= 1024 ? B0 : 1024 / (N / 8);
    static constexpr int THREADS = (N / 8) * B;
    static constexpr size_t SMEM = (size_t)(N + N * B) * sizeof(cplx_t<T>);
};

// Rows per z tile: about 256 threads.
template <typename T, int M> struct RowCfg {
    static constexpr int TL = M / 8;
    static constexpr int ROWS = TL >= PRC_ROW_THREADS ? 1 : PRC_ROW_THREADS / TL;
    static constexpr int THREADS = TL * ROWS;
    static constexpr size_t SMEM = (size_t)(2 * M + 1 + ROWS * fast::row_stride(M)) * sizeof(cplx_t<T>);
};

static int fast_grid(int64_t ntiles, int threads) {
    int per_sm = std::max(1, 2048 / threads);
    int64_t cap = (int64_t)device_sm_count() * per_sm;
    return (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, cap));
}

template <typename T, int DIR> struct FastStrided {
    template <int N> struct K {
        static int run(Specs<cplx_t<T>> sp, int nb, Strided s, const char* name, double bytes, cudaStream_t st) {
            typedef StridedCfg<T, N> cfg;
            auto kern = fast::strided<T, N, cfg::B, DIR>;
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg::SMEM);
            int64_t ntiles = (int64_t)s.outer * ((s.ncols + cfg::B - 1) / cfg::B) * nb;
            PRC_LAUNCH_B(name, st, bytes, kern<<<fast_grid(ntiles, cfg::THREADS), cfg::THREADS, cfg::SMEM, st>>>(sp, nb, s));
            PRC_CHECK_LAUNCH();
            return PRC_OK;
        }
    };
};

// The k-space kernel keeps two 8-point sets per thread (the spectrum and one output).
template <typename T, int N> struct KSpaceCfg {
    static constexpr int B0 = sizeof(T) == 4 ? PRC_KSPACE_B : 4;
    static constexpr int B = (N / 8) * B0 <= 1024 ? B0 : 1024 / (N / 8);
    static constexpr int THREADS = (N / 8) * B;
    static constexpr size_t SMEM = (size_t)(N + N * B) * sizeof(cplx_t<T>);
};

template <typename T> struct FastX {
    template <int N> struct K {
        template <int KT>
        static int go(Specs<cplx_t<T>> si, int nin, Specs<cplx_t<T>> so, Dims dims, int pitch, KOp op, double bytes,
                      cudaStream_t st) {
            typedef KSpaceCfg<T, N> cfg;
            auto kern = fast::x_kspace<T, N, cfg::B, KT>;
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg::SMEM);
            const int nh = dims.n[2] / 2 + 1;
            int64_t ntiles = (int64_t)dims.n[1] * ((nh + cfg::B - 1) / cfg::B) * nin;
            PRC_LAUNCH_B("fft_x_kspace", st, bytes,
                         kern<<<fast_grid(ntiles, cfg::THREADS), cfg::THREADS, cfg::SMEM, st>>>(si, nin, so, dims, pitch, op));
            PRC_CHECK_LAUNCH();
            return PRC_OK;
        }
        static int run(Specs<cplx_t<T>> si, int nin, Specs<cplx_t<T>> so, Dims dims, int pitch, KOp op, double bytes,
                       cudaStream_t st) {
            switch (op.type) {
                case KOP_GAUSS: return go<KOP_GAUSS>(si, nin, so, dims, pitch, op, bytes, st);
                case KOP_PP: return go<KOP_PP>(si, nin, so, dims, pitch, op, bytes, st);
                case KOP_ITER_GLOBAL: return go<KOP_ITER_GLOBAL>(si, nin, so, dims, pitch, op, bytes, st);
                case KOP_ITER_LOCAL: return go<KOP_ITER_LOCAL>(si, nin, so, dims, pitch, op, bytes, st);
                case KOP_PSI: return go<KOP_PSI>(si, nin, so, dims, pitch, op, bytes, st);
                default: return go<KOP_IDENTITY>(si, nin, so, dims, pitch, op, bytes, st);
            }
        }
    };
};

template <typename T, typename TIN> struct FastZR2C {
    template <int M> struct K {
        static int run(RealsIn ri, Specs<cplx_t<T>> so, int nb, int64_t rows, int pitch, double bytes, cudaStream_t st) {
            typedef RowCfg<T, M> cfg;
            auto kern = fast::z_r2c<T, TIN, M, cfg::ROWS>;
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg::SMEM);
            int64_t ntiles = ((rows + cfg::ROWS - 1) / cfg::ROWS) * nb;
            PRC_LAUNCH_B("fft_z_r2c", st, bytes,
                         kern<<<fast_grid(ntiles, cfg::THREADS), cfg::THREADS, cfg::SMEM, st>>>(ri, so, nb, rows, pitch));
            PRC_CHECK_LAUNCH();
            return PRC_OK;
        }
    };
};

template <typename T> struct FastZC2R {
    template <int M> struct K {
        static int run(Specs<cplx_t<T>> si, int nin, Dims dims, int pitch, Epi<T> e, double bytes, cudaStream_t st) {
            switch (e.type) {
                case EPI_DENSITY: return go<EPI_DENSITY>(si, nin, dims, pitch, e, bytes, st);
                case EPI_DENSITY_NORANDOMS: return go<EPI_DENSITY_NORANDOMS>(si, nin, dims, pitch, e, bytes, st);
                case EPI_ITER_GLOBAL: return go<EPI_ITER_GLOBAL>(si, nin, dims, pitch, e, bytes, st);
                case EPI_ITER_LOCAL: return go<EPI_ITER_LOCAL>(si, nin, dims, pitch, e, bytes, st);
                case EPI_STORE4: return go<EPI_STORE4>(si, nin, dims, pitch, e, bytes, st);
                case EPI_ITER_POLY: return go<EPI_ITER_POLY>(si, nin, dims, pitch, e, bytes, st);
                case EPI_ITER_POLY_R2C: return go<EPI_ITER_POLY_R2C>(si, nin, dims, pitch, e, bytes, st);
                default: return go<EPI_STORE>(si, nin, dims, pitch, e, bytes, st);
            }
        }
        template <int ET>
        static int go(Specs<cplx_t<T>> si, int nin, Dims dims, int pitch, Epi<T> e, double bytes, cudaStream_t st) {
            typedef RowCfg<T, M> cfg;
            auto kern = fast::z_c2r<T, M, cfg::ROWS, ET>;
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg::SMEM);
            int64_t rows = (int64_t)dims.n[0] * dims.n[1];
            int64_t ntiles = (rows + cfg::ROWS - 1) / cfg::ROWS;
            PRC_LAUNCH_B("fft_z_c2r", st, bytes,
                         kern<<<fast_grid(ntiles, cfg::THREADS), cfg::THREADS, cfg::SMEM, st>>>(si, nin, dims, pitch, e));
            PRC_CHECK_LAUNCH();
            return PRC_OK;
        }
    };
};

// ---- TMA-fed passes ----

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The driver's tensor-map encoder, looked up once through the runtime (no libcuda link).
static EncodeTiledFn tensor_map_encoder() {
    static EncodeTiledFn fn = []() -> EncodeTiledFn {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return (EncodeTiledFn)f;
    }();
    return fn;
}

// PRC_FFT_TMA=0 in the environment keeps the register-prefetch kernels (tests compare both).
static bool tma_enabled() {
    static int cached = -1;
    if (cached < 0) {
        const char* v = getenv("PRC_FFT_TMA");
        cached = (v != nullptr && v[0] == '0') ? 0 : 1;
    }
    return cached == 1 && tensor_map_encoder() != nullptr;
}

// Tensor map over the half spectrum at `base` (rows of p.pitch complex values) in 8-byte elements:
// dims (nh U, n1, n0), box (bcols U, b1, b2).  False when the layout breaks a copy rule (base not
// 16-byte aligned, row stride not a multiple of 16 bytes), so the caller uses the register kernels.
static bool spectrum_map(CUtensorMap* m, const void* base, const Plan3& p, size_t csize, int bcols, int b1, int b2) {
    EncodeTiledFn enc = tensor_map_encoder();
    const cuuint64_t U = csize / 8, row = (cuuint64_t)p.pitch * csize;
    if (!enc || ((uintptr_t)base & 15) != 0 || row % 16 != 0 || (bcols * U * 8) % 16 != 0) return false;
    cuuint64_t dim[3] = {(cuuint64_t)p.nh * U, (cuuint64_t)p.dims.n[1], (cuuint64_t)p.dims.n[0]};
    cuuint64_t stride[2] = {row, row * (cuuint64_t)p.dims.n[1]};
    cuuint32_t box[3] = {(cuuint32_t)(bcols * U), (cuuint32_t)b1, (cuuint32_t)b2};
    cuuint32_t es[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, const_cast<void*>(base), dim, stride, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Persistent grid: as many CTAs as fit on the device at once (occupancy of this kernel), at most
// one per tile.
template <typename K> static int resident_grid(K kern, int threads, size_t smem, int64_t ntiles) {
    // occupancy of (kernel, device), looked up once
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> known;
    int dev = 0;
    cudaGetDevice(&dev);
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = known.find({(const void*)kern, dev});
        if (it != known.end()) per_sm = it->second;
    }
    if (per_sm == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1)
            per_sm = 1;
        std::lock_guard<std::mutex> lock(mu);
        known[{(const void*)kern, dev}] = per_sm;
    }
    const int64_t cap = (int64_t)device_sm_count() * per_sm;
    return (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, cap));
}

constexpr int TMA_UNAVAILABLE = -1;

// Tuning knobs of the TMA-fed passes:
//   PRC_TMA_STAGE_KB   shared memory of tile stages per strided-pass CTA (2 to 4 stages)
//   PRC_TMA_STRIDED_B  columns per strided tile in FP32 (FP64 half as many; 128-byte row segments);
//                      0 = as the register kernel
//   PRC_TMA_C2R_S      row stages of the inverse z pass
#ifndef PRC_TMA_STAGE_KB
#define PRC_TMA_STAGE_KB 96
#endif
#ifndef PRC_TMA_STRIDED_B
#define PRC_TMA_STRIDED_B 16
#endif
#ifndef PRC_TMA_C2R_S
#define PRC_TMA_C2R_S 3
#endif

template <int S0> struct StageCount {
    static constexpr int value = S0 < 2 ? 2 : (S0 > 4 ? 4 : S0);
};

template <typename T, int N> struct StridedTmaB {
    static constexpr int B0 = PRC_TMA_STRIDED_B == 0 ? StridedCfg<T, N>::B
                                                     : (sizeof(T) == 4 ? PRC_TMA_STRIDED_B : PRC_TMA_STRIDED_B / 2);
    static constexpr int value = (N / 8) * B0 <= 1024 ? B0 : 1024 / (N / 8);
};

template <typename T, int N> struct StridedTmaCfg {
    static constexpr int B = StridedTmaB<T, N>::value;
    static constexpr int THREADS = (N / 8) * B;
    static constexpr int S = StageCount<(int)(PRC_TMA_STAGE_KB * 1024 / fast::TileShape<T, N, B>::BYTES)>::value;
    static constexpr size_t SMEM = fast::TmaSmem<T, N, B, S, fast::StridedPP<T, N, B, S>::value ? 1 : 0>::BYTES;
};

template <typename T, int DIR> struct FastStridedTma {
    template <int N> struct K {
        static int run(const Plan3& p, Specs<cplx_t<T>> sp, int nb, Strided s, int axis, const char* name,
                       double bytes, cudaStream_t st) {
            typedef StridedTmaCfg<T, N> cfg;
            typedef fast::TileShape<T, N, cfg::B> TS;
            tma::Maps maps;
            for (int i = 0; i < nb; i++)
                if (!spectrum_map(&maps.m[i], sp.p[i], p, sizeof(cplx_t<T>), cfg::B, axis == 1 ? TS::BOXL : 1,
                                  axis == 1 ? 1 : TS::BOXL))
                    return TMA_UNAVAILABLE;
            auto kern = fast::strided_tma<T, N, cfg::B, cfg::S, DIR>;
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg::SMEM);
            const int64_t ntiles = (int64_t)s.outer * ((s.ncols + cfg::B - 1) / cfg::B) * nb;
            PRC_LAUNCH_B(name, st, bytes,
                         kern<<<resident_grid(kern, cfg::THREADS, cfg::SMEM, ntiles), cfg::THREADS, cfg::SMEM, st>>>(
                             maps, sp, nb, s, axis));
            PRC_CHECK_LAUNCH();
            return PRC_OK;
        }
    };
};

// PRC_TMA_KSPACE_LEAN=1: FP32 k-space kernel with the spectrum kept in shared memory, two CTAs per SM.
#ifndef PRC_TMA_KSPACE_LEAN
#define PRC_TMA_KSPACE_LEAN 0
#endif
template <typename T, int N> struct KSpaceTmaCfg {
    static constexpr bool LEAN = PRC_TMA_KSPACE_LEAN && sizeof(T) == 4;
    static constexpr int B = KSpaceCfg<T, N>::B;
    static constexpr int THREADS = KSpaceCfg<T, N>::THREADS;
    static constexpr int S = 2;
    static constexpr bool PP = fast::KSpacePP<T, N, B, S, LEAN>::value;
    static constexpr size_t SMEM = fast::TmaSmem<T, N, B, S, PP ? 2 : 1, PP ? fast::PadFirst<T, B>::value : 0>::BYTES;
};

template <typename T> struct FastXTma {
    template <int N> struct K {
        template <int KT>
        static int go(const tma::Maps& maps, int nin, Specs<cplx_t<T>> so, const Plan3& p, KOp op, double bytes,
                      cudaStream_t st) {
            typedef KSpaceTmaCfg<T, N> cfg;
            auto kern = fast::x_kspace_tma<T, N, cfg::B, cfg::S, KT, cfg::LEAN>;
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg::SMEM);
            const int64_t ntiles = (int64_t)p.dims.n[1] * ((p.nh + cfg::B - 1) / cfg::B) * nin;
            PRC_LAUNCH_B("fft_x_kspace", st, bytes,
                         kern<<<resident_grid(kern, cfg::THREADS, cfg::SMEM, ntiles), cfg::THREADS, cfg::SMEM, st>>>(
                             maps, nin, so, p.dims, p.pitch, op));
            PRC_CHECK_LAUNCH();
            return PRC_OK;
        }
        static int run(const Plan3& p, Specs<cplx_t<T>> si, int nin, Specs<cplx_t<T>> so, KOp op, double bytes,
                       cudaStream_t st) {
            typedef KSpaceTmaCfg<T, N> cfg;
            typedef fast::TileShape<T, N, cfg::B> TS;
            tma::Maps maps;
            for (int i = 0; i < nin; i++)
                if (!spectrum_map(&maps.m[i], si.p[i], p, sizeof(cplx_t<T>), cfg::B, 1, TS::BOXL))
                    return TMA_UNAVAILABLE;
            switch (op.type) {
                case KOP_GAUSS: return go<KOP_GAUSS>(maps, nin, so, p, op, bytes, st);
                case KOP_PP: return go<KOP_PP>(maps, nin, so, p, op, bytes, st);
                case KOP_ITER_GLOBAL: return go<KOP_ITER_GLOBAL>(maps, nin, so, p, op, bytes, st);
                case KOP_ITER_LOCAL: return go<KOP_ITER_LOCAL>(maps, nin, so, p, op, bytes, st);
                case KOP_PSI: return go<KOP_PSI>(maps, nin, so, p, op, bytes, st);
                case KOP_HESS3: return go<KOP_HESS3>(maps, nin, so, p, op, bytes, st);
                default: return go<KOP_IDENTITY>(maps, nin, so, p, op, bytes, st);
            }
        }
    };
};

// Columns per tile (FP32; FP64 half as many; 0 = as the strided passes) and CTAs per SM the inverse y pass
// of the local-line-of-sight iteration is compiled for.  Two CTAs of 8 columns per SM (64 registers a
// thread) measured 4.30 ms per nmesh-512 reconstruction against 4.57 for one CTA of 16 columns, and
// the ping-pong exchanges below 3.82.
#ifndef PRC_HESS_B
#define PRC_HESS_B 8
#endif
#ifndef PRC_HESS_MINB
#define PRC_HESS_MINB 2
#endif
// PRC_HESS_PP: exchanges through a scratch tile and the consumed stage in turn (half the barriers), with
// PRC_HESS_PP_S stages
#ifndef PRC_HESS_PP
#define PRC_HESS_PP 1
#endif
#ifndef PRC_HESS_PP_S
#define PRC_HESS_PP_S 2
#endif
template <typename T, int N> struct HessTmaCfg {
    static constexpr int B0 = PRC_HESS_B == 0 ? StridedTmaB<T, N>::value
                                              : (sizeof(T) == 4 ? PRC_HESS_B : PRC_HESS_B / 2);
    static constexpr int B = (N / 8) * B0 <= 1024 ? B0 : 1024 / (N / 8);
    static constexpr int THREADS = (N / 8) * B;
    // PRC_HESS_MINB blocks, and at least 16 warps per SM for short lines (192 threads at 192 points)
    static constexpr int MINB0 = THREADS * PRC_HESS_MINB >= 512 ? PRC_HESS_MINB : (511 + THREADS) / THREADS;
    static constexpr int MINB = THREADS * MINB0 <= 1024 ? MINB0 : 1;
    static constexpr int PADX = 0;     // see y_hessian_tma
    static constexpr bool PP =
        PRC_HESS_PP != 0 && fast::TmaSmem<T, N, B, PRC_HESS_PP_S, 1, PADX>::BYTES + 2 * N * sizeof(T) <= 227 * 1024;
    static constexpr int S = PP ? PRC_HESS_PP_S
                                : StageCount<(int)(PRC_TMA_STAGE_KB * 1024 / fast::TileShape<T, N, B>::BYTES)>::value;
    static constexpr size_t SMEM = fast::TmaSmem<T, N, B, S, PP ? 1 : 0, PP ? PADX : 0>::BYTES;
};

template <typename T> struct FastHessTma {
    template <int N> struct K {
        typedef HessTmaCfg<T, N> cfg;
        // probe: only check that the tensor maps can be made (nothing is launched)
        static int run(const Plan3& p, cplx_t<T>* const* d, cplx_t<T>* const* o, fast::HessGeom h, cudaStream_t st,
                       bool probe) {
            typedef fast::TileShape<T, N, cfg::B> TS;
            tma::Maps maps;
            for (int i = 0; i < 3; i++)
                if (!spectrum_map(&maps.m[i], d[i], p, sizeof(cplx_t<T>), cfg::B, TS::BOXL, 1)) return TMA_UNAVAILABLE;
            if (probe) return PRC_OK;
            Specs<cplx_t<T>> so;
            for (int i = 0; i < 3; i++) so.p[i] = o[i];
            Strided s;
            s.n = p.dims.n[1];
            s.ls = p.pitch;
            s.outer = p.dims.n[0];
            s.os = (int64_t)p.dims.n[1] * p.pitch;
            s.ncols = p.nh;
            auto kern = fast::y_hessian_tma<T, N, cfg::B, cfg::S, cfg::MINB, cfg::PP>;
            const size_t smem = cfg::SMEM + 2 * N * sizeof(T);     // + the x1 and k_y tables
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            const int64_t ntiles = (int64_t)s.outer * ((s.ncols + cfg::B - 1) / cfg::B);
            const double bytes = 6.0 * spectrum_values(p) * sizeof(cplx_t<T>);
            PRC_LAUNCH_B("fft_y_inv_hessian", st, bytes,
                         kern<<<resident_grid(kern, cfg::THREADS, smem, ntiles), cfg::THREADS, smem, st>>>(
                             maps, so, s, h));
            PRC_CHECK_LAUNCH();
            return PRC_OK;
        }
    };
};

template <typename T> struct FastZC2RTma {
    template <int M> struct K {
        typedef RowCfg<T, M> cfg;
        static constexpr int S = PRC_TMA_C2R_S;
        typedef fast::TmaRows<T, M, cfg::ROWS, S> Rows;
        static int run(const Plan3& p, Specs<cplx_t<T>> si, int nin, Epi<T> e, double bytes, cudaStream_t st) {
            if (p.pitch != Rows::PS) return TMA_UNAVAILABLE;
            for (int i = 0; i < nin; i++)
                if (((uintptr_t)si.p[i] & 15) != 0) return TMA_UNAVAILABLE;
            switch (e.type) {
                case EPI_DENSITY: return go<EPI_DENSITY>(p, si, nin, e, bytes, st);
                case EPI_DENSITY_NORANDOMS: return go<EPI_DENSITY_NORANDOMS>(p, si, nin, e, bytes, st);
                case EPI_ITER_GLOBAL: return go<EPI_ITER_GLOBAL>(p, si, nin, e, bytes, st);
                case EPI_ITER_LOCAL: return go<EPI_ITER_LOCAL>(p, si, nin, e, bytes, st);
                case EPI_STORE4: return go<EPI_STORE4>(p, si, nin, e, bytes, st);
                case EPI_ITER_POLY: return go<EPI_ITER_POLY>(p, si, nin, e, bytes, st);
                case EPI_ITER_POLY_R2C: return go<EPI_ITER_POLY_R2C>(p, si, nin, e, bytes, st);
                default: return go<EPI_STORE>(p, si, nin, e, bytes, st);
            }
        }
        template <int ET>
        static int go(const Plan3& p, Specs<cplx_t<T>> si, int nin, Epi<T> e, double bytes, cudaStream_t st) {
            auto kern = fast::z_c2r_tma<T, M, cfg::ROWS, ET, S>;
            const size_t smem = fast::C2RTmaSmem<T, M, cfg::ROWS, S>::BYTES;
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            const int64_t rows = (int64_t)p.dims.n[0] * p.dims.n[1];
            const int64_t ntiles = (rows + cfg::ROWS - 1) / cfg::ROWS;
            PRC_LAUNCH_B("fft_z_c2r", st, bytes,
                         kern<<<resident_grid(kern, cfg::THREADS, smem, ntiles), cfg::THREADS, smem, st>>>(si, nin,
                                                                                                       p.dims, e));
            PRC_CHECK_LAUNCH();
            return PRC_OK;
        }
    };
};

template <typename T> struct FFTLaunch {
    typedef cplx_t<T> C;
    static constexpr size_t CS = sizeof(C);
    static constexpr size_t BUDGET = 100 * 1024;

    template <typename TIN>
    static int z_r2c(const Plan3& p, const void* const* in, C* const* out, int nb, cudaStream_t st) {
        if (p.dims.n[2] % 2 == 0 && fast_len(p.dims.n[2] / 2) && !getenv_generic()) {
            RealsIn ri;
            Specs<C> so;
            for (int i = 0; i < nb; i++) {
                ri.p[i] = in[i];
                so.p[i] = out[i];
            }
            int64_t rows = (int64_t)p.dims.n[0] * p.dims.n[1];
            double bytes = (double)nb * rows * (p.dims.n[2] * sizeof(TIN) + p.nh * CS);
            return dispatch_pow2<FastZR2C<T, TIN>::template K>(p.dims.n[2] / 2, ri, so, nb, rows, p.pitch, bytes, st);
        }
        const int n2 = p.dims.n[2], L = n2 % 2 ? n2 : n2 / 2 + 1;
        auto need = [&](int b) { return (size_t)(2 * L * row_pitch(b) + n2) * CS; };
        int B = 16;
        while (B > 1 && need(B) > BUDGET) B >>= 1;
        const size_t smem = need(B);
        RealsIn ri;
        Specs<C> so;
        for (int i = 0; i < nb; i++) {
            ri.p[i] = in[i];
            so.p[i] = out[i];
        }
        cudaFuncSetAttribute(fft_z_r2c<T, TIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int64_t rows = (int64_t)p.dims.n[0] * p.dims.n[1];
        int64_t ntiles = ((rows + B - 1) / B) * nb;
        PRC_LAUNCH_B("fft_z_r2c", st, (double)nb * rows * (p.dims.n[2] * sizeof(TIN) + p.nh * CS), fft_z_r2c<T, TIN><<<fft_grid(ntiles, 2), FFT_THREADS, smem, st>>>(ri, so, nb, p.dims, p.pitch, p.rz, B));
        PRC_CHECK_LAUNCH();
        return PRC_OK;
    }

    template <int DIR> static int strided(const Plan3& p, int axis, C* const* data, int nb, cudaStream_t st) {
        const int nline = axis == 1 ? p.dims.n[1] : p.dims.n[0];
        if (fast_len(nline) && !getenv_generic()) {
            Strided s;
            const int nh = p.nh;
            if (axis == 1) {
                s.n = p.dims.n[1];
                s.ls = p.pitch;
                s.outer = p.dims.n[0];
                s.os = (int64_t)p.dims.n[1] * p.pitch;
            } else {
                s.n = p.dims.n[0];
                s.ls = (int64_t)p.dims.n[1] * p.pitch;
                s.outer = p.dims.n[1];
                s.os = p.pitch;
            }
            s.ncols = nh;
            Specs<C> sp;
            for (int i = 0; i < nb; i++) sp.p[i] = data[i];
            const char* name = DIR < 0 ? (axis == 1 ? "fft_y_fwd" : "fft_x_fwd") : (axis == 1 ? "fft_y_inv" : "fft_x_inv");
            double bytes = 2.0 * nb * spectrum_values(p) * CS;
            if (tma_enabled()) {
                const int r = dispatch_pow2<FastStridedTma<T, DIR>::template K>(nline, p, sp, nb, s, axis, name, bytes, st);
                if (r != TMA_UNAVAILABLE) return r;
            }
            return dispatch_pow2<FastStrided<T, DIR>::template K>(nline, sp, nb, s, name, bytes, st);
        }
        Strided s;
        const int nh = p.nh;
        if (axis == 1) {
            s.n = p.dims.n[1];
            s.ls = p.pitch;
            s.outer = p.dims.n[0];
            s.os = (int64_t)p.dims.n[1] * p.pitch;
        } else {
            s.n = p.dims.n[0];
            s.ls = (int64_t)p.dims.n[1] * p.pitch;
            s.outer = p.dims.n[1];
            s.os = p.pitch;
        }
        s.ncols = nh;
        int B = choose_B(s.n, 2, CS, BUDGET - s.n * CS, 16);
        size_t smem = (size_t)(2 * s.n * B + s.n) * CS;
        Specs<C> sp;
        for (int i = 0; i < nb; i++) sp.p[i] = data[i];
        cudaFuncSetAttribute(fft_strided<T, DIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int64_t ntiles = (int64_t)s.outer * ((nh + B - 1) / B) * nb;
        PRC_LAUNCH_B((DIR < 0 ? (axis == 1 ? "fft_y_fwd" : "fft_x_fwd") : (axis == 1 ? "fft_y_inv" : "fft_x_inv")), st, 2.0 * nb * spectrum_values(p) * CS, fft_strided<T, DIR><<<fft_grid(ntiles, 2), FFT_THREADS, smem, st>>>(sp, nb, s, axis == 1 ? p.ry : p.rx, B));
        PRC_CHECK_LAUNCH();
        return PRC_OK;
    }

    static int x_fused(const Plan3& p, C* const* in, int nin, C* const* out, const KOp& op, cudaStream_t st) {
        const int n0 = p.dims.n[0];
        if (fast_len(n0) && !getenv_generic()) {
            Specs<C> si, so;
            for (int i = 0; i < nin; i++) si.p[i] = in[i];
            for (int i = 0; i < nin * op.nper; i++) so.p[i] = out[i];
            double bytes = (double)nin * (1 + op.nper) * spectrum_values(p) * CS;
            if (tma_enabled()) {
                const int r = dispatch_pow2<FastXTma<T>::template K>(n0, p, si, nin, so, op, bytes, st);
                if (r != TMA_UNAVAILABLE) return r;
            }
            return dispatch_pow2<FastX<T>::template K>(n0, si, nin, so, p.dims, p.pitch, op, bytes, st);
        }
        int B = choose_B(n0, 3, CS, BUDGET - n0 * CS, 16);
        size_t smem = (size_t)(3 * n0 * B + n0) * CS;
        Specs<C> si, so;
        for (int i = 0; i < nin; i++) si.p[i] = in[i];
        for (int i = 0; i < nin * op.nper; i++) so.p[i] = out[i];
        cudaFuncSetAttribute(fft_x_fused<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int64_t ntiles = (int64_t)p.dims.n[1] * ((p.nh + B - 1) / B) * nin;
        PRC_LAUNCH_B("fft_x_kspace", st, (double)nin * (1 + op.nper) * spectrum_values(p) * CS, fft_x_fused<T><<<fft_grid(ntiles, 2), FFT_THREADS, smem, st>>>(si, nin, so, p.dims, p.pitch, p.rx, B, op));
        PRC_CHECK_LAUNCH();
        return PRC_OK;
    }

    // The TMA x pass only (TMA_UNAVAILABLE, with nothing launched, where it cannot run).
    static int x_fused_tma(const Plan3& p, C* const* in, int nin, C* const* out, const KOp& op, cudaStream_t st) {
        const int n0 = p.dims.n[0];
        if (!fast_len(n0) || getenv_generic() || !tma_enabled()) return TMA_UNAVAILABLE;
        Specs<C> si, so;
        for (int i = 0; i < nin; i++) si.p[i] = in[i];
        for (int i = 0; i < nin * op.nper; i++) so.p[i] = out[i];
        const double bytes = (double)nin * (1 + op.nper) * spectrum_values(p) * CS;
        return dispatch_pow2<FastXTma<T>::template K>(n0, p, si, nin, so, op, bytes, st);
    }

    static int z_c2r(const Plan3& p, C* const* in, int nin, const Epi<T>& e, cudaStream_t st) {
        const int M = p.dims.n[2] / 2, nh = M + 1;
        if (p.dims.n[2] % 2 == 0 && fast_len(M) && !getenv_generic()) {
            Specs<C> si;
            for (int i = 0; i < nin; i++) si.p[i] = in[i];
            int64_t rows = (int64_t)p.dims.n[0] * p.dims.n[1];
            double bytes = (double)nin * rows * nh * CS +
                           (double)rows * p.dims.n[2] * sizeof(T) *
                               (e.type == EPI_STORE ? nin : (e.type == EPI_STORE4 ? 4 : (e.delta ? 2 : 1)));
            if (e.type == EPI_ITER_POLY_R2C)   // the spectrum rows written instead of the real rows
                bytes += (double)rows * (nh * CS - (double)p.dims.n[2] * sizeof(T));
            if (tma_enabled()) {
                const int r = dispatch_pow2<FastZC2RTma<T>::template K>(M, p, si, nin, e, bytes, st);
                if (r != TMA_UNAVAILABLE) return r;
            }
            return dispatch_pow2<FastZC2R<T>::template K>(M, si, nin, p.dims, p.pitch, e, bytes, st);
        }
        if (e.type == EPI_ITER_POLY_R2C) return PRC_ERR_ARG;   // register z kernels only
        const int n2 = p.dims.n[2], L = n2 % 2 ? n2 : nh;
        auto need = [&](int b) {
            return (size_t)(2 * L * row_pitch(b) + n2) * CS + (size_t)nin * b * n2 * sizeof(T);
        };
        int B = 16;
        while (B > 1 && need(B) > BUDGET) B >>= 1;
        const size_t smem = need(B);
        Specs<C> si;
        for (int i = 0; i < nin; i++) si.p[i] = in[i];
        cudaFuncSetAttribute(fft_z_c2r<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int64_t rows = (int64_t)p.dims.n[0] * p.dims.n[1];
        int64_t ntiles = (rows + B - 1) / B;
        PRC_LAUNCH_B("fft_z_c2r", st, (double)nin * rows * nh * CS + (double)rows * p.dims.n[2] * sizeof(T) * (e.type == EPI_STORE ? nin : (e.delta ? 2 : 1)), fft_z_c2r<T><<<fft_grid(ntiles, 2), FFT_THREADS, smem, st>>>(si, nin, p.dims, p.pitch, p.rz, B, e));
        PRC_CHECK_LAUNCH();
        return PRC_OK;
    }
};

static void fill_kop_geometry(KOp* op, const Plan3& p, const double boxsize[3], int mesh_bytes) {
    for (int a = 0; a < 3; a++) {
        op->n[a] = p.dims.n[a];
        // numpy: d = boxsize / nmesh (boxsize stored in the mesh dtype), val = 1.0 / (n * d)
        double bs = mesh_bytes == 4 ? (double)(float)boxsize[a] : boxsize[a];
        double d = bs / (double)p.dims.n[a];
        op->fscale[a] = 1.0 / ((double)p.dims.n[a] * d);
        op->radius[a] = 0.;
        op->los[a] = 0.;
    }
    op->beta = 0.;
    op->nper = 1;
    op->norm = 1.0 / ((double)p.dims.n[0] * p.dims.n[1] * p.dims.n[2]);
    op->side = nullptr;
}

template <typename T> static Epi<T> epi_default() {
    Epi<T> e;
    memset(&e, 0, sizeof(e));
    e.type = EPI_STORE;
    e.scale = 1.;
    return e;
}

// Forward z, y then x (x only when `do_x`).
template <typename T, typename TIN>
static int forward_zy(const Plan3& p, const void* const* in, cplx_t<T>* const* spec, int nb, cudaStream_t st) {
    PRC_TRY((FFTLaunch<T>::template z_r2c<TIN>(p, in, spec, nb, st)));
    PRC_TRY(FFTLaunch<T>::template strided<-1>(p, 1, spec, nb, st));
    return PRC_OK;
}

template <typename T> static size_t spec_bytes(const Plan3& p) {
    return (spectrum_elems(p) * sizeof(cplx_t<T>) + 255) & ~(size_t)255;
}

// ---- composites ----

template <typename T>
static int smooth_impl(const void* in, int in_bytes, T* out, const int32_t nmesh[3], const double boxsize[3],
                       const double radius[3], void* ws, size_t wsb, cudaStream_t st) {
    Plan3 p;
    PRC_TRY(make_plan(nmesh, &p));
    pad_pitch<T>(&p);
    if (!ws || wsb < spec_bytes<T>(p)) return PRC_ERR_WORKSPACE;
    cplx_t<T>* S = (cplx_t<T>*)ws;
    const void* ins[1] = {in};
    if (in_bytes == 8) PRC_TRY((forward_zy<T, double>(p, ins, &S, 1, st)));
    else PRC_TRY((forward_zy<T, float>(p, ins, &S, 1, st)));
    KOp op;
    fill_kop_geometry(&op, p, boxsize, sizeof(T));
    op.type = KOP_GAUSS;
    for (int a = 0; a < 3; a++) op.radius[a] = sizeof(T) == 4 ? (double)(float)radius[a] : radius[a];
    PRC_TRY(FFTLaunch<T>::x_fused(p, &S, 1, &S, op, st));
    PRC_TRY(FFTLaunch<T>::template strided<+1>(p, 1, &S, 1, st));
    Epi<T> e = epi_default<T>();
    e.out[0] = out;
    return FFTLaunch<T>::z_c2r(p, &S, 1, e, st);
}

template <typename T>
static int density_impl(const double* md, const double* mr, const double* sums, const int32_t nmesh[3],
                        const double boxsize[3], const double radius[3], double bias, double ran_min,
                        double size_randoms, T* delta, void* ws, size_t wsb, cudaStream_t st) {
    Plan3 p;
    PRC_TRY(make_plan(nmesh, &p));
    pad_pitch<T>(&p);
    const int nb = mr ? 2 : 1;
    if (!ws || wsb < nb * spec_bytes<T>(p)) return PRC_ERR_WORKSPACE;
    cplx_t<T>* S[2] = {(cplx_t<T>*)ws, (cplx_t<T>*)((char*)ws + spec_bytes<T>(p))};
    const void* ins[2] = {md, mr};
    PRC_TRY((forward_zy<T, double>(p, ins, S, nb, st)));
    KOp op;
    fill_kop_geometry(&op, p, boxsize, sizeof(T));
    op.type = KOP_GAUSS;
    for (int a = 0; a < 3; a++) op.radius[a] = sizeof(T) == 4 ? (double)(float)radius[a] : radius[a];
    PRC_TRY(FFTLaunch<T>::x_fused(p, S, nb, S, op, st));
    PRC_TRY(FFTLaunch<T>::template strided<+1>(p, 1, S, nb, st));
    Epi<T> e = epi_default<T>();
    e.type = mr ? EPI_DENSITY : EPI_DENSITY_NORANDOMS;
    e.out[0] = delta;
    e.sums = sums;
    e.bias = bias;
    e.ran_min = ran_min;
    e.size_randoms = size_randoms;
    e.ncells = (double)p.dims.n[0] * p.dims.n[1] * p.dims.n[2];
    return FFTLaunch<T>::z_c2r(p, S, nb, e, st);
}

// Epilogue writing the three displacement meshes: separate (stride 1) or interleaved as
// (x, y, z, 0) per cell (stride 4, psi_y = psi_x + 1, psi_z = psi_x + 2).
template <typename T> static int psi_epilogue(T* px, T* py, T* pz, int stride, Epi<T>* e) {
    *e = epi_default<T>();
    if (stride == 1) {
        e->type = EPI_STORE;
        e->out[0] = px;
        e->out[1] = py;
        e->out[2] = pz;
        return PRC_OK;
    }
    if (stride == 4 && py == px + 1 && pz == px + 2 && ((uintptr_t)px % (4 * sizeof(T))) == 0) {
        e->type = EPI_STORE4;
        e->out[0] = px;
        return PRC_OK;
    }
    return PRC_ERR_ARG;
}

template <typename T>
static int pp_impl(const T* delta, const int32_t nmesh[3], const double boxsize[3], double beta, const double los[3],
                   T* px, T* py, T* pz, int psi_stride, void* ws, size_t wsb, cudaStream_t st) {
    Epi<T> e;
    PRC_TRY(psi_epilogue(px, py, pz, psi_stride, &e));
    Plan3 p;
    PRC_TRY(make_plan(nmesh, &p));
    pad_pitch<T>(&p);
    if (!ws || wsb < 4 * spec_bytes<T>(p)) return PRC_ERR_WORKSPACE;
    cplx_t<T>* S[4];
    for (int i = 0; i < 4; i++) S[i] = (cplx_t<T>*)((char*)ws + i * spec_bytes<T>(p));
    const void* ins[1] = {delta};
    PRC_TRY((forward_zy<T, T>(p, ins, S, 1, st)));
    KOp op;
    fill_kop_geometry(&op, p, boxsize, sizeof(T));
    op.type = KOP_PP;
    op.nper = 3;
    op.beta = beta;
    for (int a = 0; a < 3; a++) op.los[a] = sizeof(T) == 4 ? (double)(float)los[a] : los[a];
    PRC_TRY(FFTLaunch<T>::x_fused(p, S, 1, S + 1, op, st));
    PRC_TRY(FFTLaunch<T>::template strided<+1>(p, 1, S + 1, 3, st));
    return FFTLaunch<T>::z_c2r(p, S + 1, 3, e, st);
}

// Several plane-parallel reconstructions of the same mesh, box and parameters: the meshes go through the
// passes in groups of PP_GROUP, each pass one launch over the (mesh, tile) pairs of its group (the three
// outputs of every mesh fill the pointer tables of the inverse passes); the inverse z pass, whose
// epilogue writes one displacement mesh, runs per mesh.  Each tile is computed as in pp_impl, so the
// results are those of separate calls.
constexpr int PP_GROUP = MAX_BATCH / 3;

template <typename T>
static int pp_batch_impl(const T* const* deltas, T* const* px, T* const* py, T* const* pz, int count,
                         const int32_t nmesh[3], const double boxsize[3], double beta, const double los[3],
                         int psi_stride, void* ws, size_t wsb, cudaStream_t st) {
    Plan3 p;
    PRC_TRY(make_plan(nmesh, &p));
    pad_pitch<T>(&p);
    const size_t sb = spec_bytes<T>(p);
    const int G = std::min(count, PP_GROUP);
    if (!ws || wsb < (size_t)4 * G * sb) return PRC_ERR_WORKSPACE;
    for (int i = 0; i < count; i++) {
        Epi<T> e;
        if (!deltas[i]) return PRC_ERR_ARG;
        PRC_TRY(psi_epilogue(px[i], py[i], pz[i], psi_stride, &e));
    }
    KOp op;
    fill_kop_geometry(&op, p, boxsize, sizeof(T));
    op.type = KOP_PP;
    op.nper = 3;
    op.beta = beta;
    for (int a = 0; a < 3; a++) op.los[a] = sizeof(T) == 4 ? (double)(float)los[a] : los[a];
    cplx_t<T>* F[PP_GROUP];
    cplx_t<T>* O[3 * PP_GROUP];
    for (int i = 0; i < G; i++) F[i] = (cplx_t<T>*)((char*)ws + i * sb);
    for (int i = 0; i < 3 * G; i++) O[i] = (cplx_t<T>*)((char*)ws + (G + i) * sb);
    for (int b = 0; b < count; b += G) {
        const int g = std::min(G, count - b);
        const void* ins[PP_GROUP];
        for (int i = 0; i < g; i++) ins[i] = deltas[b + i];
        PRC_TRY((forward_zy<T, T>(p, ins, F, g, st)));
        PRC_TRY(FFTLaunch<T>::x_fused(p, F, g, O, op, st));
        PRC_TRY(FFTLaunch<T>::template strided<+1>(p, 1, O, 3 * g, st));
        for (int i = 0; i < g; i++) {
            Epi<T> e;
            PRC_TRY(psi_epilogue(px[b + i], py[b + i], pz[b + i], psi_stride, &e));
            PRC_TRY(FFTLaunch<T>::z_c2r(p, O + 3 * i, 3, e, st));
        }
    }
    return PRC_OK;
}

template <typename T>
static int iter_impl(const T* delta, const int32_t nmesh[3], const double boxsize[3], const double boxcenter[3],
                     double beta, const double* los, int niter, T* px, T* py, T* pz, int psi_stride, void* ws,
                     size_t wsb, cudaStream_t st) {
    Epi<T> es;
    PRC_TRY(psi_epilogue(px, py, pz, psi_stride, &es));
    Plan3 p;
    PRC_TRY(make_plan(nmesh, &p));
    pad_pitch<T>(&p);
    const int nout = los ? 1 : 6;
    // spectra: the forward transform + max(nout, 3) outputs (3 for the final displacements)
    const int nspec = 1 + std::max(nout, 3);
    const size_t sb = spec_bytes<T>(p);
    const size_t mesh_b = ((size_t)p.dims.size() * sizeof(T) + 255) & ~(size_t)255;
    const size_t side_b = los ? 0 : (((size_t)(p.nh + p.dims.n[1]) * sizeof(cplx_t<T>) + 255) & ~(size_t)255);
    if (!ws || wsb < (size_t)nspec * sb + mesh_b + side_b) return PRC_ERR_WORKSPACE;
    cplx_t<T>* S[7];
    for (int i = 0; i < nspec; i++) S[i] = (cplx_t<T>*)((char*)ws + i * sb);
    T* dreal = (T*)((char*)ws + nspec * sb);
    cplx_t<T>* side = los ? nullptr : (cplx_t<T>*)((char*)ws + nspec * sb + mesh_b);
    KOp op;
    fill_kop_geometry(&op, p, boxsize, sizeof(T));
    if (los)
        for (int a = 0; a < 3; a++) op.los[a] = sizeof(T) == 4 ? (double)(float)los[a] : los[a];
    Epi<T> e = epi_default<T>();
    e.delta = delta;
    e.out[0] = dreal;
    for (int a = 0; a < 3; a++) {
        // node coordinates of RealMesh.coords (mesh.py:522-527): offset (mesh dtype) + d * i, d in f64
        double bs = sizeof(T) == 4 ? (double)(float)boxsize[a] : boxsize[a];
        double bc = sizeof(T) == 4 ? (double)(float)boxcenter[a] : boxcenter[a];
        e.offset[a] = sizeof(T) == 4 ? (double)(float)((float)bc - (float)bs / 2.f) : bc - bs / 2.;
        e.cell[a] = bs / (double)p.dims.n[a];
    }
    // The Hessian iteration's inverse z pass can hand its rows straight to the next forward z transform
    // (EPI_ITER_POLY_R2C), when both z passes are the register kernels; then S[0] already holds the
    // z-transformed rows and only the y transform is left (knob fft_fuse_z, 0 = store and reload).
    const bool fuse_z = p.dims.n[2] % 2 == 0 && fast_len(p.dims.n[2] / 2) && !getenv_generic() &&
                        tune_get("fft_fuse_z", 0, 1) != 0;
    bool z_done = false;   // S[0] holds the z transform of the next forward input
    auto forward = [&](const void* in) -> int {
        if (z_done) {
            z_done = false;
            return FFTLaunch<T>::template strided<-1>(p, 1, S, 1, st);
        }
        const void* ins[1] = {in};
        return forward_zy<T, T>(p, ins, S, 1, st);
    };
    for (int it = 0; it < niter; it++) {
        PRC_TRY(forward(it == 0 ? (const void*)delta : (const void*)dreal));
        double base = beta;
        if (it == 0) base /= (1. + beta);
        if (los) {
            e.type = EPI_ITER_GLOBAL;
            e.factor[0] = base;
        } else {
            e.type = EPI_ITER_LOCAL;
            const int pi[6] = {0, 0, 0, 1, 1, 2}, pj[6] = {0, 1, 2, 1, 2, 2};
            for (int c = 0; c < 6; c++) e.factor[c] = (1. + (pi[c] != pj[c])) * beta / (it == 0 ? (1. + beta) : 1.);
        }
        if (!los && p.dims.n[2] % 2 == 0 && fast_len(p.dims.n[1]) && !getenv_generic() && tma_enabled()) {
            // x pass to the three spectra E, s_x E, k_x^2 E (S1..S3), inverse y forming the six
            // Hessian terms and combining them into the quadratic in x2 (A, B, C in S4..S6), then
            // the z pass over C, B, A
            fast::HessGeom h;
            h.x0_off = e.offset[0];
            h.x0_cell = e.cell[0];
            h.x1_off = e.offset[1];
            h.x1_cell = e.cell[1];
            for (int c = 0; c < 6; c++) h.f[c] = e.factor[c];
            h.fscale_y = op.fscale[1];
            h.fscale_z = op.fscale[2];
            h.ny = p.dims.n[1];
            h.nz = p.dims.n[2];
            const bool even_x = p.dims.n[0] % 2 == 0;
            h.q01 = even_x && p.dims.n[1] % 2 == 0 ? side : nullptr;
            h.l02 = even_x && p.dims.n[2] % 2 == 0 ? side + p.nh : nullptr;
            cplx_t<T>* outs[3] = {S[4], S[5], S[6]};
            int r = dispatch_pow2<FastHessTma<T>::template K>(p.dims.n[1], p, S + 1, outs, h, st, true);
            if (r == PRC_OK) {
                op.type = KOP_HESS3;
                op.nper = 3;
                op.side = side;
                r = FFTLaunch<T>::x_fused_tma(p, S, 1, S + 1, op, st);
                op.side = nullptr;
            }
            if (r != TMA_UNAVAILABLE) {
                PRC_TRY(r);
                PRC_TRY(dispatch_pow2<FastHessTma<T>::template K>(p.dims.n[1], p, S + 1, outs, h, st, false));
                Epi<T> ep = e;
                ep.type = fuse_z ? EPI_ITER_POLY_R2C : EPI_ITER_POLY;
                ep.spec = S[0];
                ep.spec_pitch = p.pitch;
                cplx_t<T>* cba[3] = {S[6], S[5], S[4]};
                PRC_TRY(FFTLaunch<T>::z_c2r(p, cba, 3, ep, st));
                z_done = fuse_z;
                continue;
            }
        }
        op.type = los ? KOP_ITER_GLOBAL : KOP_ITER_LOCAL;
        op.nper = nout;
        PRC_TRY(FFTLaunch<T>::x_fused(p, S, 1, S + 1, op, st));
        PRC_TRY(FFTLaunch<T>::template strided<+1>(p, 1, S + 1, nout, st));
        PRC_TRY(FFTLaunch<T>::z_c2r(p, S + 1, nout, e, st));
    }
    PRC_TRY(forward(niter > 0 ? (const void*)dreal : (const void*)delta));
    op.type = KOP_PSI;
    op.nper = 3;
    PRC_TRY(FFTLaunch<T>::x_fused(p, S, 1, S + 1, op, st));
    PRC_TRY(FFTLaunch<T>::template strided<+1>(p, 1, S + 1, 3, st));
    return FFTLaunch<T>::z_c2r(p, S + 1, 3, es, st);
}

// Zeldovich displacement of a density contrast, psi_a = IFFT(i k_a delta_k / k^2), delta_k(0) = 0
// (iterative_fft.py:71-82, iterative_fft_particle.py:93-108).
template <typename T>
static int psi_impl(const T* delta, const int32_t nmesh[3], const double boxsize[3], T* px, T* py, T* pz,
                    int psi_stride, void* ws, size_t wsb, cudaStream_t st) {
    Epi<T> es;
    PRC_TRY(psi_epilogue(px, py, pz, psi_stride, &es));
    Plan3 p;
    PRC_TRY(make_plan(nmesh, &p));
    pad_pitch<T>(&p);
    const size_t sb = spec_bytes<T>(p);
    if (!ws || wsb < 4 * sb) return PRC_ERR_WORKSPACE;
    cplx_t<T>* S[4];
    for (int i = 0; i < 4; i++) S[i] = (cplx_t<T>*)((char*)ws + i * sb);
    KOp op;
    fill_kop_geometry(&op, p, boxsize, sizeof(T));
    const void* ins[1] = {delta};
    PRC_TRY((forward_zy<T, T>(p, ins, S, 1, st)));
    op.type = KOP_PSI;
    op.nper = 3;
    PRC_TRY(FFTLaunch<T>::x_fused(p, S, 1, S + 1, op, st));
    PRC_TRY(FFTLaunch<T>::template strided<+1>(p, 1, S + 1, 3, st));
    return FFTLaunch<T>::z_c2r(p, S + 1, 3, es, st);
}

template <typename T>
static int rfft_impl(const void* in, int in_bytes, void* out, const int32_t nmesh[3], cudaStream_t st) {
    Plan3 p;
    PRC_TRY(make_plan(nmesh, &p));
    cplx_t<T>* S = (cplx_t<T>*)out;
    const void* ins[1] = {in};
    if (in_bytes == 8) PRC_TRY((forward_zy<T, double>(p, ins, &S, 1, st)));
    else PRC_TRY((forward_zy<T, float>(p, ins, &S, 1, st)));
    return FFTLaunch<T>::template strided<-1>(p, 0, &S, 1, st);
}

template <typename T>
static int irfft_impl(void* in, T* out, const int32_t nmesh[3], cudaStream_t st) {
    Plan3 p;
    PRC_TRY(make_plan(nmesh, &p));
    cplx_t<T>* S = (cplx_t<T>*)in;
    PRC_TRY(FFTLaunch<T>::template strided<+1>(p, 0, &S, 1, st));
    PRC_TRY(FFTLaunch<T>::template strided<+1>(p, 1, &S, 1, st));
    Epi<T> e = epi_default<T>();
    e.out[0] = out;
    e.scale = 1.0 / ((double)p.dims.n[0] * p.dims.n[1] * p.dims.n[2]);
    return FFTLaunch<T>::z_c2r(p, &S, 1, e, st);
}

}  // namespace prc

using namespace prc;

static bool geom_ok(const int32_t* nmesh, const double* boxsize) {
    if (!nmesh || !boxsize) return false;
    for (int a = 0; a < 3; a++)
        if (!(boxsize[a] > 0)) return false;
    return true;
}

extern "C" {

unsigned int prc_device_fault_flags(int reset) {
    unsigned int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_fault, sizeof(v)) != cudaSuccess) return 0xffffffffu;
    if (reset && v != 0) {
        const unsigned int zero = 0;
        cudaMemcpyToSymbol(g_fault, &zero, sizeof(zero));
    }
    return v;
}

int prc_debug_wait_timeout(int64_t limit_ns, int* out, void* stream) {
    if (!out || limit_ns <= 0 || limit_ns > 1000000000ll) return PRC_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    PRC_LAUNCH("debug_wait_timeout", st, debug_wait_timeout<<<1, 32, 0, st>>>((uint64_t)limit_ns, 256u, out));
    PRC_CHECK_LAUNCH();
    return PRC_OK;
}

int prc_fft_supported(const int32_t nmesh[3]) {
    if (!nmesh) return 0;
    Plan3 p;
    return make_plan(nmesh, &p) == PRC_OK ? 1 : 0;
}

size_t prc_fft_workspace_bytes(const int32_t nmesh[3], int mesh_bytes, int nspectra) {
    Plan3 p;
    if (!nmesh || make_plan(nmesh, &p) != PRC_OK) return 0;
    if (mesh_bytes == 4) {
        pad_pitch<float>(&p);
        return (size_t)nspectra * spec_bytes<float>(p);
    }
    pad_pitch<double>(&p);
    return (size_t)nspectra * spec_bytes<double>(p);
}

prc_status_t prc_rfft3d_f32(const void* in, int in_bytes, void* out, const int32_t nmesh[3], void* stream) {
    if (!in || !out || !nmesh || (in_bytes != 4 && in_bytes != 8)) return PRC_ERR_ARG;
    return rfft_impl<float>(in, in_bytes, out, nmesh, (cudaStream_t)stream);
}
prc_status_t prc_rfft3d_f64(const void* in, int in_bytes, void* out, const int32_t nmesh[3], void* stream) {
    if (!in || !out || !nmesh || (in_bytes != 4 && in_bytes != 8)) return PRC_ERR_ARG;
    return rfft_impl<double>(in, in_bytes, out, nmesh, (cudaStream_t)stream);
}
prc_status_t prc_irfft3d_f32(void* in, float* out, const int32_t nmesh[3], void* stream) {
    if (!in || !out || !nmesh) return PRC_ERR_ARG;
    return irfft_impl<float>(in, out, nmesh, (cudaStream_t)stream);
}
prc_status_t prc_irfft3d_f64(void* in, double* out, const int32_t nmesh[3], void* stream) {
    if (!in || !out || !nmesh) return PRC_ERR_ARG;
    return irfft_impl<double>(in, out, nmesh, (cudaStream_t)stream);
}

prc_status_t prc_smooth_gaussian_f32(const void* in, int in_bytes, float* out, const int32_t nmesh[3],
                                     const double boxsize[3], const double radius[3], void* workspace,
                                     size_t workspace_bytes, void* stream) {
    if (!in || !out || !geom_ok(nmesh, boxsize) || !radius || (in_bytes != 4 && in_bytes != 8)) return PRC_ERR_ARG;
    return smooth_impl<float>(in, in_bytes, out, nmesh, boxsize, radius, workspace, workspace_bytes, (cudaStream_t)stream);
}
prc_status_t prc_smooth_gaussian_f64(const void* in, int in_bytes, double* out, const int32_t nmesh[3],
                                     const double boxsize[3], const double radius[3], void* workspace,
                                     size_t workspace_bytes, void* stream) {
    if (!in || !out || !geom_ok(nmesh, boxsize) || !radius || (in_bytes != 4 && in_bytes != 8)) return PRC_ERR_ARG;
    return smooth_impl<double>(in, in_bytes, out, nmesh, boxsize, radius, workspace, workspace_bytes, (cudaStream_t)stream);
}

size_t prc_density_contrast_workspace_bytes(const int32_t nmesh[3], int mesh_bytes, int with_randoms) {
    return prc_fft_workspace_bytes(nmesh, mesh_bytes, with_randoms ? 2 : 1);
}

prc_status_t prc_density_contrast_f32(const double* mesh_data, const double* mesh_randoms, const double* sums,
                                      const int32_t nmesh[3], const double boxsize[3], const double radius[3],
                                      double bias, double ran_min, double size_randoms, float* delta, void* workspace,
                                      size_t workspace_bytes, void* stream) {
    if (!mesh_data || !sums || !delta || !geom_ok(nmesh, boxsize) || !radius) return PRC_ERR_ARG;
    return density_impl<float>(mesh_data, mesh_randoms, sums, nmesh, boxsize, radius, bias, ran_min, size_randoms,
                               delta, workspace, workspace_bytes, (cudaStream_t)stream);
}
prc_status_t prc_density_contrast_f64(const double* mesh_data, const double* mesh_randoms, const double* sums,
                                      const int32_t nmesh[3], const double boxsize[3], const double radius[3],
                                      double bias, double ran_min, double size_randoms, double* delta, void* workspace,
                                      size_t workspace_bytes, void* stream) {
    if (!mesh_data || !sums || !delta || !geom_ok(nmesh, boxsize) || !radius) return PRC_ERR_ARG;
    return density_impl<double>(mesh_data, mesh_randoms, sums, nmesh, boxsize, radius, bias, ran_min, size_randoms,
                                delta, workspace, workspace_bytes, (cudaStream_t)stream);
}

size_t prc_plane_parallel_workspace_bytes(const int32_t nmesh[3], int mesh_bytes) {
    return prc_fft_workspace_bytes(nmesh, mesh_bytes, 4);
}

prc_status_t prc_plane_parallel_fft_f32(const float* delta, const int32_t nmesh[3], const double boxsize[3], double beta,
                                        const double los[3], float* psi_x, float* psi_y, float* psi_z, int psi_stride,
                                        void* workspace, size_t workspace_bytes, void* stream) {
    if (!delta || !geom_ok(nmesh, boxsize) || !los || !psi_x || !psi_y || !psi_z) return PRC_ERR_ARG;
    return pp_impl<float>(delta, nmesh, boxsize, beta, los, psi_x, psi_y, psi_z, psi_stride, workspace, workspace_bytes,
                          (cudaStream_t)stream);
}
prc_status_t prc_plane_parallel_fft_f64(const double* delta, const int32_t nmesh[3], const double boxsize[3],
                                        double beta, const double los[3], double* psi_x, double* psi_y, double* psi_z,
                                        int psi_stride, void* workspace, size_t workspace_bytes, void* stream) {
    if (!delta || !geom_ok(nmesh, boxsize) || !los || !psi_x || !psi_y || !psi_z) return PRC_ERR_ARG;
    return pp_impl<double>(delta, nmesh, boxsize, beta, los, psi_x, psi_y, psi_z, psi_stride, workspace, workspace_bytes,
                           (cudaStream_t)stream);
}

size_t prc_plane_parallel_batch_workspace_bytes(const int32_t nmesh[3], int mesh_bytes, int count) {
    if (count < 1) return 0;
    return prc_fft_workspace_bytes(nmesh, mesh_bytes, 4 * std::min(count, PP_GROUP));
}

prc_status_t prc_plane_parallel_fft_batch_f32(const float* const* delta, float* const* psi_x, float* const* psi_y,
                                              float* const* psi_z, int count, const int32_t nmesh[3],
                                              const double boxsize[3], double beta, const double los[3],
                                              int psi_stride, void* workspace, size_t workspace_bytes, void* stream) {
    if (!delta || !psi_x || !psi_y || !psi_z || count < 1 || !geom_ok(nmesh, boxsize) || !los) return PRC_ERR_ARG;
    return pp_batch_impl<float>(delta, psi_x, psi_y, psi_z, count, nmesh, boxsize, beta, los, psi_stride, workspace,
                                workspace_bytes, (cudaStream_t)stream);
}
prc_status_t prc_plane_parallel_fft_batch_f64(const double* const* delta, double* const* psi_x, double* const* psi_y,
                                              double* const* psi_z, int count, const int32_t nmesh[3],
                                              const double boxsize[3], double beta, const double los[3],
                                              int psi_stride, void* workspace, size_t workspace_bytes, void* stream) {
    if (!delta || !psi_x || !psi_y || !psi_z || count < 1 || !geom_ok(nmesh, boxsize) || !los) return PRC_ERR_ARG;
    return pp_batch_impl<double>(delta, psi_x, psi_y, psi_z, count, nmesh, boxsize, beta, los, psi_stride, workspace,
                                 workspace_bytes, (cudaStream_t)stream);
}

size_t prc_iterative_fft_workspace_bytes(const int32_t nmesh[3], int mesh_bytes, int local_los) {
    Plan3 p;
    if (!nmesh || make_plan(nmesh, &p) != PRC_OK) return 0;
    size_t mesh_b = ((size_t)p.dims.size() * mesh_bytes + 255) & ~(size_t)255;
    // local line of sight: the two Nyquist lines of the three-spectrum Hessian pass
    size_t side_b = local_los ? (((size_t)(p.nh + p.dims.n[1]) * 2 * mesh_bytes + 255) & ~(size_t)255) : 0;
    return prc_fft_workspace_bytes(nmesh, mesh_bytes, local_los ? 7 : 4) + mesh_b + side_b;
}

prc_status_t prc_iterative_fft_f32(const float* delta, const int32_t nmesh[3], const double boxsize[3],
                                   const double boxcenter[3], double beta, const double* los, int niterations,
                                   float* psi_x, float* psi_y, float* psi_z, int psi_stride, void* workspace,
                                   size_t workspace_bytes, void* stream) {
    if (!delta || !geom_ok(nmesh, boxsize) || !boxcenter || niterations < 0 || !psi_x || !psi_y || !psi_z)
        return PRC_ERR_ARG;
    return iter_impl<float>(delta, nmesh, boxsize, boxcenter, beta, los, niterations, psi_x, psi_y, psi_z, psi_stride,
                            workspace, workspace_bytes, (cudaStream_t)stream);
}
prc_status_t prc_iterative_fft_f64(const double* delta, const int32_t nmesh[3], const double boxsize[3],
                                   const double boxcenter[3], double beta, const double* los, int niterations,
                                   double* psi_x, double* psi_y, double* psi_z, int psi_stride, void* workspace,
                                   size_t workspace_bytes, void* stream) {
    if (!delta || !geom_ok(nmesh, boxsize) || !boxcenter || niterations < 0 || !psi_x || !psi_y || !psi_z)
        return PRC_ERR_ARG;
    return iter_impl<double>(delta, nmesh, boxsize, boxcenter, beta, los, niterations, psi_x, psi_y, psi_z, psi_stride,
                             workspace, workspace_bytes, (cudaStream_t)stream);
}


size_t prc_zeldovich_psi_workspace_bytes(const int32_t nmesh[3], int mesh_bytes) {
    return prc_fft_workspace_bytes(nmesh, mesh_bytes, 4);
}

prc_status_t prc_zeldovich_psi_f32(const float* delta, const int32_t nmesh[3], const double boxsize[3], float* psi_x,
                                   float* psi_y, float* psi_z, int psi_stride, void* workspace, size_t workspace_bytes,
                                   void* stream) {
    if (!delta || !geom_ok(nmesh, boxsize) || !psi_x || !psi_y || !psi_z) return PRC_ERR_ARG;
    return psi_impl<float>(delta, nmesh, boxsize, psi_x, psi_y, psi_z, psi_stride, workspace, workspace_bytes,
                           (cudaStream_t)stream);
}
prc_status_t prc_zeldovich_psi_f64(const double* delta, const int32_t nmesh[3], const double boxsize[3],
                                   double* psi_x, double* psi_y, double* psi_z, int psi_stride, void* workspace,
                                   size_t workspace_bytes, void* stream) {
    if (!delta || !geom_ok(nmesh, boxsize) || !psi_x || !psi_y || !psi_z) return PRC_ERR_ARG;
    return psi_impl<double>(delta, nmesh, boxsize, psi_x, psi_y, psi_z, psi_stride, workspace, workspace_bytes,
                            (cudaStream_t)stream);
}

}  // extern "C"

// Full-multigrid solve of the RSD-modified Poisson equation on a periodic mesh.
//
// Operator, for cell c with p = i + offset / h (local line of sight) or p = los / h (global),
// g = beta / (h^2 |p|^2), G_a = 1/h_a^2 + g p_a^2 (reference src/multigrid.c:63-104):
//   (A v)_c = 2 (G_x + G_y + G_z) v_c - S(v)_c
//   S(v)_c  = sum_a G_a (v_{c+a} + v_{c-a})
//           + g/2 sum_{a<b} p_a p_b (v_{c+a+b} + v_{c-a-b} - v_{c-a+b} - v_{c+a-b})
//           + [local] g sum_a p_a (v_{c+a} - v_{c-a})
// Damped Jacobi: v <- (1 - w) v + w (f + S(v)) / (2 sum G), one fused kernel per sweep
// (the reference writes jac then blends in a second pass).
//
// Schedule = the reference's fixed FMG (src/multigrid.c:270-328): restrict f to the coarsest
// level (while every n > 4 and even), then per level prolong the coarse solution and run
// `vcycle_niterations` V-cycles of `jacobi_niterations` pre- and post-sweeps.
//
// Mixed precision (f32 entry with mixed_precision = 1): the V-cycle is affine and consistent,
// so V(v, f) = v + V(0, f - A v) exactly; each V-cycle is run as an FP64 residual of the FP64
// iterate, an FP32 V-cycle from zero on that defect, and an FP64 correction.
#include "common.cuh"

#include <algorithm>
#include <vector>

namespace prc {

template <typename T> struct Stencil {
    int n[3];
    T h2[3], ih2[3], off[3], losh[3];
    T beta;
    int local;
};

template <typename T>
static Stencil<T> make_stencil(const int n[3], const double boxsize[3], const double boxcenter[3], double beta,
                               const double* los) {
    Stencil<T> s;
    s.local = los == nullptr;
    s.beta = (T)beta;
    for (int d = 0; d < 3; d++) {
        s.n[d] = n[d];
        T bs = (T)boxsize[d], bc = (T)boxcenter[d];
        T h = bs / (T)n[d];                                  // FLOAT / size_t in the reference
        s.h2[d] = h * h;
        s.ih2[d] = (T)(1. / (double)s.h2[d]);
        s.off[d] = (T)(((double)bc - (double)bs / 2.) / (double)h);
        s.losh[d] = s.local ? (T)0 : (T)los[d] / h;
    }
    return s;
}

template <typename T, typename S>
__device__ __forceinline__ void coeffs(const Stencil<S>& s, int x, int y, int z, T p[3], T& g, T G[3]) {
    if (s.local) {
        p[0] = (T)x + (T)s.off[0];
        p[1] = (T)y + (T)s.off[1];
        p[2] = (T)z + (T)s.off[2];
    } else {
        p[0] = (T)s.losh[0];
        p[1] = (T)s.losh[1];
        p[2] = (T)s.losh[2];
    }
    g = (T)s.beta / ((T)s.h2[0] * p[0] * p[0] + (T)s.h2[1] * p[1] * p[1] + (T)s.h2[2] * p[2] * p[2]);
#pragma unroll
    for (int d = 0; d < 3; d++) G[d] = (T)s.ih2[d] + g * p[d] * p[d];
}

// The neighbour terms of S(v) at one cell, accumulated in type A from a mesh of type V.
template <typename A, typename V>
__device__ __forceinline__ A neighbour_sum(const V* __restrict__ v, const int n[3], int x, int y, int z, const A p[3],
                                           A g, const A G[3], int local) {
    const int xp = wrap_up(x, n[0]), xm = wrap_dn(x, n[0]);
    const int yp = wrap_up(y, n[1]), ym = wrap_dn(y, n[1]);
    const int zp = wrap_up(z, n[2]), zm = wrap_dn(z, n[2]);
    const int64_t sx = (int64_t)n[1] * n[2], sy = n[2];
    const int64_t X0 = x * sx, Xp = xp * sx, Xm = xm * sx;
    const int64_t Y0 = y * sy, Yp = yp * sy, Ym = ym * sy;
#define L(a, b, c) ((A)__ldg(v + (a) + (b) + (c)))
    const A vxp = L(Xp, Y0, z), vxm = L(Xm, Y0, z);
    const A vyp = L(X0, Yp, z), vym = L(X0, Ym, z);
    const A vzp = L(X0, Y0, zp), vzm = L(X0, Y0, zm);
    A s = G[0] * (vxp + vxm) + G[1] * (vyp + vym) + G[2] * (vzp + vzm);
    s += g / (A)2 * (p[0] * p[1] * (L(Xp, Yp, z) + L(Xm, Ym, z) - L(Xm, Yp, z) - L(Xp, Ym, z))
                   + p[0] * p[2] * (L(Xp, Y0, zp) + L(Xm, Y0, zm) - L(Xm, Y0, zp) - L(Xp, Y0, zm))
                   + p[1] * p[2] * (L(X0, Yp, zp) + L(X0, Ym, zm) - L(X0, Ym, zp) - L(X0, Yp, zm)));
    if (local) s += g * (p[0] * (vxp - vxm) + p[1] * (vyp - vym) + p[2] * (vzp - vzm));
#undef L
    return s;
}

__device__ __forceinline__ void cell_of(int64_t i, const int n[3], int& x, int& y, int& z) {
    z = (int)(i % n[2]);
    int64_t r = i / n[2];
    y = (int)(r % n[1]);
    x = (int)(r / n[1]);
}

// One damped-Jacobi sweep: vout = (1 - w) v + w (f + S(v)) / (2 sum G).  zero_v: v is
// identically zero (first sweep of a V-cycle started from zero), so S(v) = 0 and v is not read.
template <typename T, typename FT>
__global__ void __launch_bounds__(256) jacobi_sweep(const T* __restrict__ v, const FT* __restrict__ f,
                                                    T* __restrict__ vout, Stencil<T> s, T w, int zero_v) {
    const int64_t N = (int64_t)s.n[0] * s.n[1] * s.n[2];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        int x, y, z;
        cell_of(i, s.n, x, y, z);
        T p[3], g, G[3];
        coeffs<T>(s, x, y, z, p, g, G);
        T jac = (T)f[i];
        T vc = (T)0;
        if (!zero_v) {
            jac += neighbour_sum<T>(v, s.n, x, y, z, p, g, G, s.local);
            vc = v[i];
        }
        jac /= (T)2 * (G[0] + G[1] + G[2]);
        vout[i] = ((T)1 - w) * vc + w * jac;
    }
}

// r = f - A v, evaluated in type A (double for the mixed-precision defect), stored as R.
template <typename A, typename V, typename FT, typename R, typename S>
__global__ void __launch_bounds__(256) residual_kernel(const V* __restrict__ v, const FT* __restrict__ f,
                                                       R* __restrict__ r, Stencil<S> s) {
    const int64_t N = (int64_t)s.n[0] * s.n[1] * s.n[2];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        int x, y, z;
        cell_of(i, s.n, x, y, z);
        A p[3], g, G[3];
        coeffs<A>(s, x, y, z, p, g, G);
        const A nb = neighbour_sum<A>(v, s.n, x, y, z, p, g, G, s.local);
        const A av = (A)2 * (G[0] + G[1] + G[2]) * (A)v[i] - nb;
        r[i] = (R)((A)f[i] - av);
    }
}

// 27-point full weighting, coarse cell (x, y, z) centred on fine (2x, 2y, 2z).
template <typename A, typename TI, typename TO>
__global__ void __launch_bounds__(256) reduce_kernel(const TI* __restrict__ fine, TO* __restrict__ coarse, Dims nf) {
    const int nc[3] = {nf.n[0] / 2, nf.n[1] / 2, nf.n[2] / 2};
    const int64_t N = (int64_t)nc[0] * nc[1] * nc[2];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        int x, y, z;
        cell_of(i, nc, x, y, z);
        const int X[3] = {wrap_dn(2 * x, nf.n[0]), 2 * x, wrap_up(2 * x, nf.n[0])};
        const int Y[3] = {wrap_dn(2 * y, nf.n[1]), 2 * y, wrap_up(2 * y, nf.n[1])};
        const int Z[3] = {wrap_dn(2 * z, nf.n[2]), 2 * z, wrap_up(2 * z, nf.n[2])};
        A acc = 0;
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const TI* row = fine + ((int64_t)X[a] * nf.n[1] + Y[b]) * nf.n[2];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const int side = (a != 1) + (b != 1) + (c != 1);
                    acc += (A)(8 >> side) * (A)__ldg(row + Z[c]);
                }
            }
        coarse[i] = (TO)(acc / (A)64);
    }
}

// Trilinear prolongation of a coarse mesh (nc) onto the fine mesh (2 nc): fine node 2c + e is
// the mean of the coarse nodes c + e' over e' <= e.  ADD: fine += value (V-cycle correction),
// else fine = value.
template <typename A, typename TI, typename TO, bool ADD>
__global__ void __launch_bounds__(256) prolong_kernel(const TI* __restrict__ coarse, TO* __restrict__ fine, Dims nc) {
    const int64_t N = (int64_t)nc.n[0] * nc.n[1] * nc.n[2];
    const int nf1 = 2 * nc.n[1], nf2 = 2 * nc.n[2];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        int x, y, z;
        cell_of(i, nc.n, x, y, z);
        const int xs[2] = {x, wrap_up(x, nc.n[0])}, ys[2] = {y, wrap_up(y, nc.n[1])}, zs[2] = {z, wrap_up(z, nc.n[2])};
        A c[2][2][2];
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++)
#pragma unroll
                for (int d = 0; d < 2; d++)
                    c[a][b][d] = (A)__ldg(coarse + ((int64_t)xs[a] * nc.n[1] + ys[b]) * nc.n[2] + zs[d]);
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const int ex = (e >> 2) & 1, ey = (e >> 1) & 1, ez = e & 1;
            A s = 0;
#pragma unroll
            for (int a = 0; a <= ex; a++)
#pragma unroll
                for (int b = 0; b <= ey; b++)
#pragma unroll
                    for (int d = 0; d <= ez; d++) s += c[a][b][d];
            s /= (A)((1 + ex) * (1 + ey) * (1 + ez));
            TO* dst = fine + ((int64_t)(2 * x + ex) * nf1 + (2 * y + ey)) * nf2 + (2 * z + ez);
            if (ADD) *dst = (TO)((A)*dst + s);
            else *dst = (TO)s;
        }
    }
}

template <typename TI, typename TO>
__global__ void convert_kernel(const TI* __restrict__ in, TO* __restrict__ out, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (TO)in[i];
}

template <typename TA, typename TB>
__global__ void add_kernel(TA* __restrict__ acc, const TB* __restrict__ x, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc[i] = acc[i] + (TA)x[i];
}

static int grid_for(int64_t n) {
    int64_t blocks = (n + 255) / 256;
    return (int)std::max<int64_t>(1, std::min<int64_t>(blocks, (int64_t)device_sm_count() * 16));
}

// ---------------------------------------------------------------------------------------------
// Level hierarchy and the FMG / V-cycle drivers
// ---------------------------------------------------------------------------------------------
struct Level {
    int n[3];
    int64_t size() const { return (int64_t)n[0] * n[1] * n[2]; }
};

static bool coarsenable(const int n[3]) {
    for (int d = 0; d < 3; d++)
        if (!(n[d] > 4 && n[d] % 2 == 0)) return false;
    return true;
}

static std::vector<Level> hierarchy(const int32_t nmesh[3]) {
    std::vector<Level> L;
    Level l;
    for (int d = 0; d < 3; d++) l.n[d] = nmesh[d];
    L.push_back(l);
    while (coarsenable(L.back().n)) {
        Level c;
        for (int d = 0; d < 3; d++) c.n[d] = L.back().n[d] / 2;
        L.push_back(c);
    }
    return L;
}

static size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

// Per-level buffers of one precision.
template <typename T> struct LevelBufs {
    T *v, *f, *r, *tmp;
};

struct Params {
    double boxsize[3], boxcenter[3], los[3];
    int has_los;
    double beta, damping;
    int jn, vn;
};

template <typename T> struct MGRunner {
    std::vector<Level> L;
    std::vector<LevelBufs<T>> B;
    Params P;
    cudaStream_t st;

    Stencil<T> stencil(int l) const {
        return make_stencil<T>(L[l].n, P.boxsize, P.boxcenter, P.beta, P.has_los ? P.los : nullptr);
    }

    // niter sweeps in place on v (ping-pong through tmp); zero_first: v known to be zero.
    int jacobi(int l, T* v, const T* f, T* tmp, int niter, bool zero_first) {
        Stencil<T> s = stencil(l);
        const int64_t N = L[l].size();
        T* src = v;
        T* dst = tmp;
        if (niter == 0 && zero_first && cudaMemsetAsync(v, 0, N * sizeof(T), st) != cudaSuccess) return PRC_ERR_CUDA;
        for (int it = 0; it < niter; it++) {
            PRC_LAUNCH_B("mg_jacobi", st, (double)N * sizeof(T) * ((zero_first && it == 0) ? 2 : 3), jacobi_sweep<T, T><<<grid_for(N), 256, 0, st>>>(src, f, dst, s, (T)P.damping, zero_first && it == 0));
            std::swap(src, dst);
        }
        if (src != v) cudaMemcpyAsync(v, src, N * sizeof(T), cudaMemcpyDeviceToDevice, st);
        PRC_CHECK_LAUNCH();
        return PRC_OK;
    }

    // Recursive V-cycle on level l: v (B[l].v) with right-hand side f.
    int vcycle(int l, T* v, const T* f, bool v_zero) {
        PRC_TRY(jacobi(l, v, f, B[l].tmp, P.jn, v_zero));
        if (l + 1 < (int)L.size()) {
            Stencil<T> s = stencil(l);
            const int64_t N = L[l].size();
            PRC_LAUNCH_B("mg_residual", st, 3.0 * N * sizeof(T), residual_kernel<T, T, T, T, T><<<grid_for(N), 256, 0, st>>>(v, f, B[l].r, s));
            Dims nf = {{L[l].n[0], L[l].n[1], L[l].n[2]}};
            PRC_LAUNCH_B("mg_reduce", st, (double)(N + L[l + 1].size()) * sizeof(T), reduce_kernel<T, T, T><<<grid_for(L[l + 1].size()), 256, 0, st>>>(B[l].r, B[l + 1].f, nf));
            PRC_CHECK_LAUNCH();
            PRC_TRY(vcycle(l + 1, B[l + 1].v, B[l + 1].f, true));
            Dims nc = {{L[l + 1].n[0], L[l + 1].n[1], L[l + 1].n[2]}};
            PRC_LAUNCH_B("mg_prolong_add", st, (double)(2 * N + L[l + 1].size()) * sizeof(T), prolong_kernel<T, T, T, true><<<grid_for(L[l + 1].size()), 256, 0, st>>>(B[l + 1].v, v, nc));
            PRC_CHECK_LAUNCH();
        }
        return jacobi(l, v, f, B[l].tmp, P.jn, false);
    }
};

// Plain FMG in precision T (the reference schedule); f0 is the level-0 right-hand side.
template <typename T> static int fmg_plain(MGRunner<T>& R, const T* f0, T* v0) {
    const int nl = (int)R.L.size();
    cudaStream_t st = R.st;
    // right-hand sides at every level
    R.B[0].f = const_cast<T*>(f0);
    for (int l = 0; l + 1 < nl; l++) {
        Dims nf = {{R.L[l].n[0], R.L[l].n[1], R.L[l].n[2]}};
        PRC_LAUNCH_B("mg_reduce", st, (double)(R.L[l].size() + R.L[l + 1].size()) * sizeof(T), reduce_kernel<T, T, T><<<grid_for(R.L[l + 1].size()), 256, 0, st>>>(R.B[l].f, R.B[l + 1].f, nf));
    }
    PRC_CHECK_LAUNCH();
    // the FMG solution of level l lives in fmg_v[l]; level 0 writes straight into v0
    for (int l = nl - 1; l >= 0; l--) {
        T* v = l == 0 ? v0 : R.B[l].v;
        if (l == nl - 1) {
            if (cudaMemsetAsync(v, 0, R.L[l].size() * sizeof(T), st) != cudaSuccess) return PRC_ERR_CUDA;
        } else {
            Dims nc = {{R.L[l + 1].n[0], R.L[l + 1].n[1], R.L[l + 1].n[2]}};
            PRC_LAUNCH_B("mg_prolong", st, (double)(R.L[l].size() + R.L[l + 1].size()) * sizeof(T), prolong_kernel<T, T, T, false><<<grid_for(R.L[l + 1].size()), 256, 0, st>>>(R.B[l + 1].v, v, nc));
            PRC_CHECK_LAUNCH();
        }
        // V-cycles at level l use the coarser levels' v as scratch: keep this level's FMG
        // solution in `v` and run the recursion with v_zero = false.
        // the next finer level prolongs from R.B[l].v, which is `v` itself for l >= 1
        for (int it = 0; it < R.P.vn; it++) PRC_TRY(R.vcycle(l, v, R.B[l].f, l == nl - 1 && it == 0));
    }
    return PRC_OK;
}

}  // namespace prc

using namespace prc;

namespace {

// Workspace layout for plain FMG in precision T: per level v, f (levels >= 1), r, tmp.
template <typename T> size_t plain_layout(const int32_t nmesh[3], char* base, std::vector<LevelBufs<T>>* out,
                                          std::vector<Level>* lv) {
    std::vector<Level> L = hierarchy(nmesh);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base ? base + off : nullptr;
        off += al(bytes);
        return p;
    };
    std::vector<LevelBufs<T>> B(L.size());
    for (size_t l = 0; l < L.size(); l++) {
        size_t b = (size_t)L[l].size() * sizeof(T);
        B[l].v = l == 0 ? nullptr : (T*)take(b);
        B[l].f = l == 0 ? nullptr : (T*)take(b);
        B[l].r = (T*)take(b);
        B[l].tmp = (T*)take(b);
    }
    if (out) *out = B;
    if (lv) *lv = L;
    return off;
}

// Mixed layout: FP64 f and v per level, plus the FP32 plain buffers for the inner V-cycles.
struct MixedBufs {
    std::vector<double*> f64, v64;
    std::vector<LevelBufs<float>> b32;
    std::vector<Level> L;
};

size_t mixed_layout(const int32_t nmesh[3], char* base, MixedBufs* mb) {
    std::vector<Level> L = hierarchy(nmesh);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base ? base + off : nullptr;
        off += al(bytes);
        return p;
    };
    MixedBufs m;
    m.L = L;
    m.f64.resize(L.size());
    m.v64.resize(L.size());
    m.b32.resize(L.size());
    for (size_t l = 0; l < L.size(); l++) {
        size_t n = (size_t)L[l].size();
        m.f64[l] = (double*)take(n * 8);
        m.v64[l] = (double*)take(n * 8);
        m.b32[l].v = (float*)take(n * 4);
        m.b32[l].f = (float*)take(n * 4);
        m.b32[l].r = (float*)take(n * 4);
        m.b32[l].tmp = (float*)take(n * 4);
    }
    if (mb) *mb = m;
    return off;
}

Params make_params(const double boxsize[3], const double boxcenter[3], double beta, double damping, int jn, int vn,
                   const double* los) {
    Params P;
    for (int d = 0; d < 3; d++) {
        P.boxsize[d] = boxsize[d];
        P.boxcenter[d] = boxcenter[d];
        P.los[d] = los ? los[d] : 0.;
    }
    P.has_los = los != nullptr;
    P.beta = beta;
    P.damping = damping;
    P.jn = jn;
    P.vn = vn;
    return P;
}

bool mg_args_ok(const void* delta, const void* phi, const int32_t nmesh[3], const double* boxsize,
                const double* boxcenter, int jn, int vn) {
    if (!delta || !phi || !nmesh || !boxsize || !boxcenter || jn < 0 || vn < 0) return false;
    for (int d = 0; d < 3; d++)
        if (nmesh[d] < 1 || !(boxsize[d] > 0)) return false;
    return true;
}

template <typename T>
int run_plain(const T* delta, T* phi, const int32_t nmesh[3], const Params& P, void* ws, size_t wsb, cudaStream_t st) {
    if (!ws || wsb < plain_layout<T>(nmesh, nullptr, nullptr, nullptr)) return PRC_ERR_WORKSPACE;
    MGRunner<T> R;
    plain_layout<T>(nmesh, (char*)ws, &R.B, &R.L);
    R.P = P;
    R.st = st;
    return fmg_plain<T>(R, delta, phi);
}

// Mixed precision FMG: every V-cycle is v64 += V32(0, f64 - A v64).
int run_mixed(const float* delta, float* phi, const int32_t nmesh[3], const Params& P, void* ws, size_t wsb,
              cudaStream_t st) {
    if (!ws || wsb < mixed_layout(nmesh, nullptr, nullptr)) return PRC_ERR_WORKSPACE;
    MixedBufs m;
    mixed_layout(nmesh, (char*)ws, &m);
    const int nl = (int)m.L.size();
    MGRunner<float> R;
    R.L = m.L;
    R.B = m.b32;
    R.P = P;
    R.st = st;
    const int64_t N0 = m.L[0].size();
    PRC_LAUNCH_B("mg_convert", st, 12.0 * N0, convert_kernel<float, double><<<grid_for(N0), 256, 0, st>>>(delta, m.f64[0], N0));
    for (int l = 0; l + 1 < nl; l++) {
        Dims nf = {{m.L[l].n[0], m.L[l].n[1], m.L[l].n[2]}};
        PRC_LAUNCH_B("mg_reduce", st, 8.0 * (m.L[l].size() + m.L[l + 1].size()), reduce_kernel<double, double, double><<<grid_for(m.L[l + 1].size()), 256, 0, st>>>(m.f64[l], m.f64[l + 1], nf));
    }
    PRC_CHECK_LAUNCH();
    for (int l = nl - 1; l >= 0; l--) {
        const int64_t N = m.L[l].size();
        if (l == nl - 1) {
            if (cudaMemsetAsync(m.v64[l], 0, N * 8, st) != cudaSuccess) return PRC_ERR_CUDA;
        } else {
            Dims nc = {{m.L[l + 1].n[0], m.L[l + 1].n[1], m.L[l + 1].n[2]}};
            PRC_LAUNCH_B("mg_prolong", st, 8.0 * (m.L[l].size() + m.L[l + 1].size()), prolong_kernel<double, double, double, false><<<grid_for(m.L[l + 1].size()), 256, 0, st>>>(m.v64[l + 1],
                                                                                                    m.v64[l], nc));
        }
        Stencil<double> s64 = make_stencil<double>(m.L[l].n, P.boxsize, P.boxcenter, P.beta,
                                                   P.has_los ? P.los : nullptr);
        for (int it = 0; it < P.vn; it++) {
            // defect in FP64 (stored FP32 as the inner V-cycle's right-hand side)
            PRC_LAUNCH_B("mg_residual_fp64", st, 20.0 * N, residual_kernel<double, double, double, float, double><<<grid_for(N), 256, 0, st>>>(m.v64[l], m.f64[l],
                                                                                            m.b32[l].f, s64));
            PRC_CHECK_LAUNCH();
            PRC_TRY(R.vcycle(l, m.b32[l].v, m.b32[l].f, true));
            PRC_LAUNCH_B("mg_correct_fp64", st, 20.0 * N, add_kernel<double, float><<<grid_for(N), 256, 0, st>>>(m.v64[l], m.b32[l].v, N));
            PRC_CHECK_LAUNCH();
        }
    }
    PRC_LAUNCH_B("mg_convert", st, 12.0 * N0, convert_kernel<double, float><<<grid_for(N0), 256, 0, st>>>(m.v64[0], phi, N0));
    PRC_CHECK_LAUNCH();
    return PRC_OK;
}

}  // namespace

extern "C" {

size_t prc_multigrid_workspace_bytes(const int32_t nmesh[3], int mesh_bytes, int mixed_precision) {
    if (!nmesh) return 0;
    for (int d = 0; d < 3; d++)
        if (nmesh[d] < 1) return 0;
    if (mesh_bytes == 4 && mixed_precision) return mixed_layout(nmesh, nullptr, nullptr);
    if (mesh_bytes == 4) return plain_layout<float>(nmesh, nullptr, nullptr, nullptr);
    return plain_layout<double>(nmesh, nullptr, nullptr, nullptr);
}

prc_status_t prc_multigrid_f32(const float* delta, float* phi, const int32_t nmesh[3], const double boxsize[3],
                               const double boxcenter[3], double beta, double damping, int jacobi_niterations,
                               int vcycle_niterations, const double* los, int mixed_precision, void* workspace,
                               size_t workspace_bytes, void* stream) {
    if (!mg_args_ok(delta, phi, nmesh, boxsize, boxcenter, jacobi_niterations, vcycle_niterations)) return PRC_ERR_ARG;
    Params P = make_params(boxsize, boxcenter, beta, damping, jacobi_niterations, vcycle_niterations, los);
    if (mixed_precision) return run_mixed(delta, phi, nmesh, P, workspace, workspace_bytes, (cudaStream_t)stream);
    return run_plain<float>(delta, phi, nmesh, P, workspace, workspace_bytes, (cudaStream_t)stream);
}

prc_status_t prc_multigrid_f64(const double* delta, double* phi, const int32_t nmesh[3], const double boxsize[3],
                               const double boxcenter[3], double beta, double damping, int jacobi_niterations,
                               int vcycle_niterations, const double* los, void* workspace, size_t workspace_bytes,
                               void* stream) {
    if (!mg_args_ok(delta, phi, nmesh, boxsize, boxcenter, jacobi_niterations, vcycle_niterations)) return PRC_ERR_ARG;
    Params P = make_params(boxsize, boxcenter, beta, damping, jacobi_niterations, vcycle_niterations, los);
    return run_plain<double>(delta, phi, nmesh, P, workspace, workspace_bytes, (cudaStream_t)stream);
}

#define MG_COMPONENTS(SUF, T)                                                                                        \
    prc_status_t prc_mg_jacobi_##SUF(T* v, const T* f, T* scratch, const int32_t nmesh[3], const double boxsize[3], \
                                     const double boxcenter[3], double beta, double damping, int niterations,       \
                                     const double* los, void* stream) {                                             \
        if (!v || !f || !scratch || !nmesh || !boxsize || !boxcenter || niterations < 0) return PRC_ERR_ARG;        \
        MGRunner<T> R;                                                                                               \
        R.L = hierarchy(nmesh);                                                                                      \
        R.P = make_params(boxsize, boxcenter, beta, damping, niterations, 0, los);                                  \
        R.st = (cudaStream_t)stream;                                                                                 \
        return R.jacobi(0, v, f, scratch, niterations, false);                                                      \
    }                                                                                                                \
    prc_status_t prc_mg_residual_##SUF(const T* v, const T* f, T* r, const int32_t nmesh[3],                        \
                                       const double boxsize[3], const double boxcenter[3], double beta,             \
                                       const double* los, void* stream) {                                           \
        if (!v || !f || !r || !nmesh || !boxsize || !boxcenter) return PRC_ERR_ARG;                                 \
        int n[3] = {nmesh[0], nmesh[1], nmesh[2]};                                                                   \
        Stencil<T> s = make_stencil<T>(n, boxsize, boxcenter, beta, los);                                            \
        int64_t N = (int64_t)n[0] * n[1] * n[2];                                                                     \
        PRC_LAUNCH("mg_residual", (cudaStream_t)stream,                                                              \
                   residual_kernel<T, T, T, T, T><<<grid_for(N), 256, 0, (cudaStream_t)stream>>>(v, f, r, s));     \
        PRC_CHECK_LAUNCH();                                                                                          \
        return PRC_OK;                                                                                               \
    }                                                                                                                \
    prc_status_t prc_mg_reduce_##SUF(const T* fine, T* coarse, const int32_t nf[3], void* stream) {                 \
        if (!fine || !coarse || !nf) return PRC_ERR_ARG;                                                             \
        Dims d = {{nf[0], nf[1], nf[2]}};                                                                            \
        int64_t N = (int64_t)(nf[0] / 2) * (nf[1] / 2) * (nf[2] / 2);                                                \
        PRC_LAUNCH("mg_reduce", (cudaStream_t)stream,                                                                \
                   reduce_kernel<T, T, T><<<grid_for(N), 256, 0, (cudaStream_t)stream>>>(fine, coarse, d));       \
        PRC_CHECK_LAUNCH();                                                                                          \
        return PRC_OK;                                                                                               \
    }                                                                                                                \
    prc_status_t prc_mg_prolong_##SUF(const T* coarse, T* fine, const int32_t nc[3], void* stream) {                \
        if (!fine || !coarse || !nc) return PRC_ERR_ARG;                                                             \
        Dims d = {{nc[0], nc[1], nc[2]}};                                                                            \
        int64_t N = (int64_t)nc[0] * nc[1] * nc[2];                                                                  \
        PRC_LAUNCH("mg_prolong", (cudaStream_t)stream,                                                               \
                   prolong_kernel<T, T, T, false><<<grid_for(N), 256, 0, (cudaStream_t)stream>>>(coarse, fine, d)); \
        PRC_CHECK_LAUNCH();                                                                                          \
        return PRC_OK;                                                                                               \
    }

MG_COMPONENTS(f32, float)
MG_COMPONENTS(f64, double)

}  // extern "C"

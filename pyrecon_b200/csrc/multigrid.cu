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
#include <list>
#include <map>
#include <mutex>
#include <stdlib.h>
#include <string>
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

// Operator forms of the quad kernels (template argument MODE).  MG_LOCAL: p = position / h, 19 points
// with the first-derivative term.  MG_GLOBAL: p = los / h, 19 points.  MG_AXIS0..2: a line of sight
// along one axis, where every edge coefficient p_a p_b and all but one p_a^2 are exactly zero, so the
// operator reads 7 points; the terms it leaves out are exact zeros in the 19-point form, so the two agree
// up to the compiler's contraction of the kept terms into multiply-adds (run-time knob mg_axis_stencil = 0
// keeps the 19-point form for comparison).
enum { MG_GLOBAL = 0, MG_LOCAL = 1, MG_AXIS0 = 2, MG_AXIS1 = 3, MG_AXIS2 = 4 };

template <typename T> static int mg_mode(const Stencil<T>& s) {
    if (s.local) return MG_LOCAL;
    int zeros = 0, axis = 0;
    for (int d = 0; d < 3; d++) {
        if (s.losh[d] == (T)0) zeros++;
        else axis = d;
    }
    return zeros == 2 && tune_get("mg_axis_stencil", 0, 1) != 0 ? MG_AXIS0 + axis : MG_GLOBAL;
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

// S(v) from the six axis neighbours and the three edge combinations e_ab = v(+a+b) + v(-a-b) -
// v(-a+b) - v(+a-b); every kernel evaluates it through this one expression.
template <typename A>
__device__ __forceinline__ A stencil_terms(A vxp, A vxm, A vyp, A vym, A vzp, A vzm, A exy, A exz, A eyz, const A p[3],
                                           A g, const A G[3], int local) {
    A s = G[0] * (vxp + vxm) + G[1] * (vyp + vym) + G[2] * (vzp + vzm);
    s += g / (A)2 * (p[0] * p[1] * exy + p[0] * p[2] * exz + p[1] * p[2] * eyz);
    if (local) s += g * (p[0] * (vxp - vxm) + p[1] * (vyp - vym) + p[2] * (vzp - vzm));
    return s;
}

// The neighbour terms of S(v) at one cell, accumulated in type A from a mesh of type V (read-only global
// memory, or shared memory when SMEM).
template <typename A, typename V, bool SMEM = false>
__device__ __forceinline__ A neighbour_sum(const V* __restrict__ v, const int n[3], int x, int y, int z, const A p[3],
                                           A g, const A G[3], int local) {
    const int xp = wrap_up(x, n[0]), xm = wrap_dn(x, n[0]);
    const int yp = wrap_up(y, n[1]), ym = wrap_dn(y, n[1]);
    const int zp = wrap_up(z, n[2]), zm = wrap_dn(z, n[2]);
    const int64_t sx = (int64_t)n[1] * n[2], sy = n[2];
    const int64_t X0 = x * sx, Xp = xp * sx, Xm = xm * sx;
    const int64_t Y0 = y * sy, Yp = yp * sy, Ym = ym * sy;
#define L(a, b, c) ((A)(SMEM ? v[(a) + (b) + (c)] : __ldg(v + (a) + (b) + (c))))
    const A vxp = L(Xp, Y0, z), vxm = L(Xm, Y0, z);
    const A vyp = L(X0, Yp, z), vym = L(X0, Ym, z);
    const A vzp = L(X0, Y0, zp), vzm = L(X0, Y0, zm);
    const A exy = L(Xp, Yp, z) + L(Xm, Ym, z) - L(Xm, Yp, z) - L(Xp, Ym, z);
    const A exz = L(Xp, Y0, zp) + L(Xm, Y0, zm) - L(Xm, Y0, zp) - L(Xp, Y0, zm);
    const A eyz = L(X0, Yp, zp) + L(X0, Ym, zm) - L(X0, Ym, zp) - L(X0, Yp, zm);
#undef L
    return stencil_terms<A>(vxp, vxm, vyp, vym, vzp, vzm, exy, exz, eyz, p, g, G, local);
}

// Kernels run one thread per cell of a 3D launch: (z, y) over the block's (x, y) threads, x over
// blockIdx.z.  A batch of `count` problems of the same shape, stored one after the other, is one
// launch with count n0 planes along blockIdx.z: problem blockIdx.z / n0, plane blockIdx.z % n0.
__device__ __forceinline__ bool cell3(const int n[3], int& x, int& y, int& z) {
    z = blockIdx.x * blockDim.x + threadIdx.x;
    y = blockIdx.y * blockDim.y + threadIdx.y;
    x = gridDim.z == (unsigned)n[0] ? (int)blockIdx.z : (int)(blockIdx.z % n[0]);   // no division unbatched
    return z < n[2] && y < n[1];
}

// Offset of this block's problem in a batch of meshes of shape n.
__device__ __forceinline__ int64_t batch_offset(const int n[3]) {
    if (gridDim.z == (unsigned)n[0]) return 0;
    return (int64_t)(blockIdx.z / n[0]) * ((int64_t)n[0] * n[1] * n[2]);
}

// One damped-Jacobi sweep: vout = (1 - w) v + w (f + S(v)) / (2 sum G).  zero_v: v is
// identically zero (first sweep of a V-cycle started from zero), so S(v) = 0 and v is not read.
template <typename T, typename FT>
__global__ void __launch_bounds__(256) jacobi_sweep(const T* __restrict__ v, const FT* __restrict__ f,
                                                    T* __restrict__ vout, Stencil<T> s, T w, int zero_v) {
    pdl_trigger();
    pdl_wait();
    int x, y, z;
    if (!cell3(s.n, x, y, z)) return;
    const int64_t bo = batch_offset(s.n);
    v += bo, f += bo, vout += bo;
    const int64_t i = ((int64_t)x * s.n[1] + y) * s.n[2] + z;
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

// ---- four cells along z per thread (n2 % 4 == 0, 16-byte aligned meshes) ----
// The thread loads the nine (x +- 1, y +- 1) columns it needs once as vectors (the five that need
// z - 1 and z + 4 as well), so a cell costs ~5 loads instead of 19 and the index arithmetic is
// shared.  Same expression per cell as the one-cell kernels.
template <typename T> __device__ __forceinline__ void load4(const T* __restrict__ p, T (&o)[4]) {
    if constexpr (sizeof(T) == 4) {
        const float4 q = __ldg((const float4*)p);
        o[0] = q.x, o[1] = q.y, o[2] = q.z, o[3] = q.w;
    } else {
        const double2 a = __ldg((const double2*)p), b = __ldg((const double2*)p + 1);
        o[0] = a.x, o[1] = a.y, o[2] = b.x, o[3] = b.y;
    }
}
// values at z0 - 1 .. z0 + 4 of one column (periodic in z)
template <typename T> __device__ __forceinline__ void load6(const T* __restrict__ col, int z0, int n2, T (&o)[6]) {
    T m[4];
    load4(col + z0, m);
    o[0] = __ldg(col + (z0 == 0 ? n2 - 1 : z0 - 1));
    o[1] = m[0], o[2] = m[1], o[3] = m[2], o[4] = m[3];
    o[5] = __ldg(col + (z0 + 4 == n2 ? 0 : z0 + 4));
}

struct Quad {
    int x, y, z0;
    int64_t c;        // offset of (x, y, 0)
};
__device__ __forceinline__ bool quad_of(const int n[3], Quad& q) {
    q.z0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    q.y = blockIdx.y * blockDim.y + threadIdx.y;
    q.x = gridDim.z == (unsigned)n[0] ? (int)blockIdx.z : (int)(blockIdx.z % n[0]);
    q.c = ((int64_t)q.x * n[1] + q.y) * n[2];
    return q.z0 < n[2] && q.y < n[1];
}

// The operator at the four cells of a quad, rearranged so that a cell needs one division.  With
// q = sum_a h_a^2 p_a^2 (so g = beta / q) and P = sum_a p_a^2:
//   U = sum_a (v+a + v-a) / h_a^2
//   W = sum_a p_a^2 (v+a + v-a) + 1/2 sum_{a<b} p_a p_b e_ab [+ sum_a p_a (v+a - v-a), local]
//   S(v) = U + g W,   2 sum_a G_a = 2 (sum_a 1/h_a^2 + g P).
// x and y are fixed for the thread, so the p_0, p_1 terms are computed once for its four cells.
// The nine columns a quad's operator reads: the centre and the four axis neighbours at z0 - 1 .. z0 + 4,
// the four (x +- 1, y +- 1) edge columns at z0 .. z0 + 3.
template <typename V> struct QuadCols {
    V c[6], XP[6], XM[6], YP[6], YM[6], PP[4], MM[4], MP[4], PM[4];
};

// Axis modes read the centre column at z0 - 1 .. z0 + 4 and the four axis neighbours at z0 .. z0 + 3
// (entries 1..4 of their arrays), nothing else.
template <int MODE, typename V, typename S>
__device__ __forceinline__ void quad_load(const V* __restrict__ v, const Stencil<S>& s, const Quad& q, QuadCols<V>& Q) {
    const int n0 = s.n[0], n1 = s.n[1], n2 = s.n[2];
    const int64_t sx = (int64_t)n1 * n2;
    const int64_t xp = (int64_t)wrap_up(q.x, n0) * sx, xm = (int64_t)wrap_dn(q.x, n0) * sx, x0 = (int64_t)q.x * sx;
    const int64_t yp = (int64_t)wrap_up(q.y, n1) * n2, ym = (int64_t)wrap_dn(q.y, n1) * n2, y0 = (int64_t)q.y * n2;
    load6(v + x0 + y0, q.z0, n2, Q.c);
    if constexpr (MODE >= MG_AXIS0) {
        V t[4];
        load4(v + xp + y0 + q.z0, t);
#pragma unroll
        for (int k = 0; k < 4; k++) Q.XP[k + 1] = t[k];
        load4(v + xm + y0 + q.z0, t);
#pragma unroll
        for (int k = 0; k < 4; k++) Q.XM[k + 1] = t[k];
        load4(v + x0 + yp + q.z0, t);
#pragma unroll
        for (int k = 0; k < 4; k++) Q.YP[k + 1] = t[k];
        load4(v + x0 + ym + q.z0, t);
#pragma unroll
        for (int k = 0; k < 4; k++) Q.YM[k + 1] = t[k];
        return;
    }
    load6(v + xp + y0, q.z0, n2, Q.XP);
    load6(v + xm + y0, q.z0, n2, Q.XM);
    load6(v + x0 + yp, q.z0, n2, Q.YP);
    load6(v + x0 + ym, q.z0, n2, Q.YM);
    load4(v + xp + yp + q.z0, Q.PP);
    load4(v + xm + ym + q.z0, Q.MM);
    load4(v + xm + yp + q.z0, Q.MP);
    load4(v + xp + ym + q.z0, Q.PM);
}

// The operator at the four cells of a quad (x, y, z0 .. z0 + 3), rearranged so that a cell needs one
// division.  With q = sum_a h_a^2 p_a^2 (so g = beta / q) and P = sum_a p_a^2:
//   U = sum_a (v+a + v-a) / h_a^2
//   W = sum_a p_a^2 (v+a + v-a) + 1/2 sum_{a<b} p_a p_b e_ab [+ sum_a p_a (v+a - v-a), local]
//   S(v) = U + g W,   2 sum_a G_a = 2 (sum_a 1/h_a^2 + g P).
// x and y are fixed for the thread, so the p_0, p_1 terms are computed once for its four cells.  Every
// quad kernel (one sweep from global memory, two sweeps from shared memory) evaluates this function.
template <typename A, typename V, typename S, int MODE>
__device__ __forceinline__ void quad_compute(const QuadCols<V>& Q, const Stencil<S>& s, int x, int y, int z0,
                                             A (&U)[4], A (&W)[4], A (&qq)[4], A (&P)[4]) {
    constexpr bool LOCAL = MODE == MG_LOCAL;
    const V(&c)[6] = Q.c;
    const V(&XP)[6] = Q.XP;
    const V(&XM)[6] = Q.XM;
    const V(&YP)[6] = Q.YP;
    const V(&YM)[6] = Q.YM;
    const V(&PP)[4] = Q.PP;
    const V(&MM)[4] = Q.MM;
    const V(&MP)[4] = Q.MP;
    const V(&PM)[4] = Q.PM;
    const A ih0 = (A)s.ih2[0], ih1 = (A)s.ih2[1], ih2 = (A)s.ih2[2];
    A p0, p1, p2b;
    if (LOCAL) {
        p0 = (A)x + (A)s.off[0];
        p1 = (A)y + (A)s.off[1];
        p2b = (A)z0 + (A)s.off[2];
    } else {
        p0 = (A)s.losh[0];
        p1 = (A)s.losh[1];
        p2b = (A)s.losh[2];
    }
    const A s0 = p0 * p0, s1 = p1 * p1;
    const A q01 = (A)s.h2[0] * s0 + (A)s.h2[1] * s1, P01 = s0 + s1;
    const A e01 = (A)0.5 * p0 * p1, hp0 = (A)0.5 * p0, hp1 = (A)0.5 * p1;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const A p2 = LOCAL ? p2b + (A)k : p2b;
        const A s2 = p2 * p2;
        const A xpv = (A)XP[k + 1], xmv = (A)XM[k + 1], ypv = (A)YP[k + 1], ymv = (A)YM[k + 1];
        const A zpv = (A)c[k + 2], zmv = (A)c[k];
        if constexpr (MODE >= MG_AXIS0) {
            U[k] = ih0 * (xpv + xmv) + ih1 * (ypv + ymv) + ih2 * (zpv + zmv);
            if constexpr (MODE == MG_AXIS0) W[k] = s0 * (xpv + xmv);
            else if constexpr (MODE == MG_AXIS1) W[k] = s1 * (ypv + ymv);
            else W[k] = s2 * (zpv + zmv);
            qq[k] = q01 + (A)s.h2[2] * s2;
            P[k] = P01 + s2;
            continue;
        }
        const A exy = ((A)PP[k] + (A)MM[k]) - ((A)MP[k] + (A)PM[k]);
        const A exz = ((A)XP[k + 2] + (A)XM[k]) - ((A)XM[k + 2] + (A)XP[k]);
        const A eyz = ((A)YP[k + 2] + (A)YM[k]) - ((A)YM[k + 2] + (A)YP[k]);
        U[k] = ih0 * (xpv + xmv) + ih1 * (ypv + ymv) + ih2 * (zpv + zmv);
        A w;
        if (LOCAL)
            w = (s0 + p0) * xpv + (s0 - p0) * xmv + (s1 + p1) * ypv + (s1 - p1) * ymv + (s2 + p2) * zpv +
                (s2 - p2) * zmv;
        else
            w = s0 * (xpv + xmv) + s1 * (ypv + ymv) + s2 * (zpv + zmv);
        W[k] = w + e01 * exy + hp0 * p2 * exz + hp1 * p2 * eyz;
        qq[k] = q01 + (A)s.h2[2] * s2;
        P[k] = P01 + s2;
    }
}


template <typename A, typename V, typename S, int MODE>
__device__ __forceinline__ void quad_terms(const V* __restrict__ v, const Stencil<S>& s, const Quad& q, A (&U)[4],
                                           A (&W)[4], A (&qq)[4], A (&P)[4]) {
    QuadCols<V> Q;
    quad_load<MODE>(v, s, q, Q);
    quad_compute<A, V, S, MODE>(Q, s, q.x, q.y, q.z0, U, W, qq, P);
}

template <typename T> __device__ __forceinline__ T quotient(T a, T b) {
    if constexpr (sizeof(T) == 4) return __fdividef(a, b);   // FP32 sweeps: fast reciprocal (2 ulp)
    else return a / b;
}

// quad_compute's terms where v is identically zero (the first sweep of a V-cycle started from zero).
template <typename T, bool LOCAL>
__device__ __forceinline__ void quad_zero_terms(const Stencil<T>& s, int x, int y, int z0, T (&U)[4], T (&W)[4],
                                                T (&qq)[4], T (&P)[4], T (&vc)[4]) {
    const T p0 = LOCAL ? (T)x + s.off[0] : s.losh[0], p1 = LOCAL ? (T)y + s.off[1] : s.losh[1];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const T p2 = LOCAL ? (T)(z0 + k) + s.off[2] : s.losh[2];
        const T s2 = p2 * p2;
        qq[k] = s.h2[0] * p0 * p0 + s.h2[1] * p1 * p1 + s.h2[2] * s2;
        P[k] = p0 * p0 + p1 * p1 + s2;
        U[k] = W[k] = vc[k] = (T)0;
    }
}

// The damped-Jacobi update of a quad: jac = (q (f + U) + beta W) / (2 (q sum 1/h^2 + beta P)),
// o = v + w (jac - v).
template <typename T>
__device__ __forceinline__ void quad_blend(const Stencil<T>& s, T w, const T (&fv)[4], const T (&vc)[4],
                                           const T (&U)[4], const T (&W)[4], const T (&qq)[4], const T (&P)[4],
                                           T (&o)[4]) {
    const T sih = s.ih2[0] + s.ih2[1] + s.ih2[2];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const T jac = quotient<T>(qq[k] * (fv[k] + U[k]) + s.beta * W[k], (T)2 * (qq[k] * sih + s.beta * P[k]));
        o[k] = vc[k] + w * (jac - vc[k]);
    }
}

// Damped-Jacobi sweep of four cells per thread:
//   jac = (f + S) / (2 sum G) = (q (f + U) + beta W) / (2 (q sum 1/h^2 + beta P)),
//   vout = v + w (jac - v).
template <typename T, int MODE>
__global__ void __launch_bounds__(256) jacobi_sweep4(const T* __restrict__ v, const T* __restrict__ f,
                                                     T* __restrict__ vout, Stencil<T> s, T w, int zero_v) {
    pdl_trigger();
    pdl_wait();
    Quad q;
    if (!quad_of(s.n, q)) return;
    const int64_t bo = batch_offset(s.n);
    v += bo, f += bo, vout += bo;
    T fv[4], vc[4], U[4], W[4], qq[4], P[4];
    load4(f + q.c + q.z0, fv);
    if (zero_v) {
        quad_zero_terms<T, MODE == MG_LOCAL>(s, q.x, q.y, q.z0, U, W, qq, P, vc);
    } else {
        quad_terms<T, T, T, MODE>(v, s, q, U, W, qq, P);
        load4(v + q.c + q.z0, vc);
    }
    T o[4];
    quad_blend(s, w, fv, vc, U, W, qq, P, o);
    if constexpr (sizeof(T) == 4) {
        *(float4*)(vout + q.c + q.z0) = make_float4(o[0], o[1], o[2], o[3]);
    } else {
        ((double2*)(vout + q.c + q.z0))[0] = make_double2(o[0], o[1]);
        ((double2*)(vout + q.c + q.z0))[1] = make_double2(o[2], o[3]);
    }
}

// ---- two sweeps per pass (temporal blocking) ----
// A block owns a tile of TY rows (y) x 4 TQ cells (z) and marches along x through a slab of planes.  At
// plane step x it stages plane x + 1 of v (the tile grown by two rows and eight cells on each side;
// planes x - 1 and x are already there), runs the first sweep at plane x over the tile grown by one
// row and one quad on each side into a ring of three planes in shared memory, then the second sweep at
// plane x - 1 over the tile from the ring's planes x - 2 .. x.  v and f are read from DRAM once and the
// result written once per two sweeps (the halo of the first sweep is recomputed by the neighbouring
// tiles).  Every quad goes through quad_compute / quad_blend, the arithmetic of jacobi_sweep4, so two
// sweeps here equal two jacobi_sweep4 launches bit for bit.  Periodic in every axis: staged rows and
// 4-cell chunks wrap (n2 % 4 == 0 keeps every chunk contiguous and aligned).
template <typename T, int TY, int TQ> struct TbShape {
    static constexpr int ZP = 4 * TQ + 16;         // row pitch: cells z0 - 8 .. z0 + 4 TQ + 8
    static constexpr int R0 = TY + 4;              // rows of a staged v plane: y0 - 2 .. y0 + TY + 1
    static constexpr int R1 = TY + 2;              // rows of a first-sweep plane: y0 - 1 .. y0 + TY
    static constexpr int Q1 = TQ + 2;              // quads of a first-sweep row: z0 - 4 .. z0 + 4 TQ + 3
    static constexpr int THREADS = TQ * TY;
};

__device__ __forceinline__ int wrap_mod(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

template <typename T>
__device__ __forceinline__ void smem_quad6(const T* row, int i, T (&o)[6]) {   // cells i - 1 .. i + 4, i % 4 == 0
    T m[4];
    if constexpr (sizeof(T) == 4) {
        const float4 a = *(const float4*)(row + i);
        m[0] = a.x, m[1] = a.y, m[2] = a.z, m[3] = a.w;
    } else {
        const double2 a = *(const double2*)(row + i), b = *(const double2*)(row + i + 2);
        m[0] = a.x, m[1] = a.y, m[2] = b.x, m[3] = b.y;
    }
    o[0] = row[i - 1], o[1] = m[0], o[2] = m[1], o[3] = m[2], o[4] = m[3], o[5] = row[i + 4];
}
template <typename T> __device__ __forceinline__ void smem_quad4(const T* row, int i, T (&o)[4]) {
    if constexpr (sizeof(T) == 4) {
        const float4 a = *(const float4*)(row + i);
        o[0] = a.x, o[1] = a.y, o[2] = a.z, o[3] = a.w;
    } else {
        const double2 a = *(const double2*)(row + i), b = *(const double2*)(row + i + 2);
        o[0] = a.x, o[1] = a.y, o[2] = b.x, o[3] = b.y;
    }
}
template <typename T> __device__ __forceinline__ void smem_store4(T* row, int i, const T (&o)[4]) {
    if constexpr (sizeof(T) == 4) {
        *(float4*)(row + i) = make_float4(o[0], o[1], o[2], o[3]);
    } else {
        *(double2*)(row + i) = make_double2(o[0], o[1]);
        *(double2*)(row + i + 2) = make_double2(o[2], o[3]);
    }
}

// The columns of the quad at (row r, cell index i) of plane `mid`, its neighbours in planes `lo` (x - 1)
// and `hi` (x + 1), all with row pitch ZP.
template <typename T, int ZP>
__device__ __forceinline__ void smem_cols(const T* lo, const T* mid, const T* hi, int r, int i, QuadCols<T>& Q) {
    smem_quad6(mid + r * ZP, i, Q.c);
    smem_quad6(hi + r * ZP, i, Q.XP);
    smem_quad6(lo + r * ZP, i, Q.XM);
    smem_quad6(mid + (r + 1) * ZP, i, Q.YP);
    smem_quad6(mid + (r - 1) * ZP, i, Q.YM);
    smem_quad4(hi + (r + 1) * ZP, i, Q.PP);
    smem_quad4(lo + (r - 1) * ZP, i, Q.MM);
    smem_quad4(lo + (r + 1) * ZP, i, Q.MP);
    smem_quad4(hi + (r - 1) * ZP, i, Q.PM);
}

template <typename T, bool LOCAL, int TY, int TQ>
__global__ void __launch_bounds__(TQ * TY, (sizeof(T) == 4 ? 6 : 4)) jacobi_sweep2_tb(const T* __restrict__ v, const T* __restrict__ f,
                                                             T* __restrict__ vout, Stencil<T> s, T w, int zero_v,
                                                             int slab, int nslab) {
    pdl_trigger();
    pdl_wait();
    typedef TbShape<T, TY, TQ> SH;
    constexpr int ZP = SH::ZP;
    constexpr int PL0 = SH::R0 * ZP, PL1 = SH::R1 * ZP;
    __shared__ __align__(16) T v0s[3 * PL0];       // planes x - 1, x, x + 1 of v (ring)
    __shared__ __align__(16) T v1s[3 * PL1];       // first-sweep planes x - 2, x - 1, x (ring)
    const int n0 = s.n[0], n1 = s.n[1], n2 = s.n[2];
    const int64_t N = (int64_t)n0 * n1 * n2;
    const int prob = blockIdx.z / nslab;
    const int x0 = (blockIdx.z % nslab) * slab, x1 = min(x0 + slab, n0);
    v += prob * N, f += prob * N, vout += prob * N;
    const int y0 = blockIdx.y * TY, z0 = blockIdx.x * (4 * TQ);
    const int tid = threadIdx.x;
    const int64_t sx = (int64_t)n1 * n2;

    // stage plane x (periodic) of v into ring slot x mod 3
    auto stage = [&](int x) {
        T* dst = v0s + wrap_mod(x, 3) * PL0;
        const int64_t xo = (int64_t)wrap_mod(x, n0) * sx;
        constexpr int CH = ZP / 4;                 // 4-cell chunks per staged row
        for (int q = tid; q < SH::R0 * CH; q += SH::THREADS) {
            const int r = q / CH, ch = q % CH;
            const int gy = wrap_mod(y0 - 2 + r, n1), gz = wrap_mod(z0 - 8 + 4 * ch, n2);
            T m[4];
            load4(v + xo + (int64_t)gy * n2 + gz, m);
            smem_store4(dst + r * ZP, 4 * ch, m);
        }
    };
    if (!zero_v) {
        stage(x0 - 2);
        stage(x0 - 1);
    }
    for (int x = x0 - 1; x <= x1; x++) {
        if (!zero_v) stage(x + 1);
        __syncthreads();
        // first sweep at plane x over rows y0 - 1 .. y0 + TY, quads z0 - 4 .. z0 + 4 TQ
        {
            const int gx = wrap_mod(x, n0);
            const T* lo = v0s + wrap_mod(x - 1, 3) * PL0;
            const T* mid = v0s + wrap_mod(x, 3) * PL0;
            const T* hi = v0s + wrap_mod(x + 1, 3) * PL0;
            T* out = v1s + wrap_mod(x, 3) * PL1;
            for (int q = tid; q < SH::R1 * SH::Q1; q += SH::THREADS) {
                const int r = q / SH::Q1, k = q % SH::Q1;
                const int gy = wrap_mod(y0 - 1 + r, n1), gz = wrap_mod(z0 - 4 + 4 * k, n2);
                T fv[4], vc[4], U[4], W[4], qq[4], P[4], o[4];
                load4(f + (int64_t)gx * sx + (int64_t)gy * n2 + gz, fv);
                if (zero_v) {
                    quad_zero_terms<T, LOCAL>(s, gx, gy, gz, U, W, qq, P, vc);
                } else {
                    QuadCols<T> Q;
                    smem_cols<T, ZP>(lo, mid, hi, r + 1, 4 * k + 4, Q);
                    quad_compute<T, T, T, LOCAL>(Q, s, gx, gy, gz, U, W, qq, P);
                    smem_quad4(mid + (r + 1) * ZP, 4 * k + 4, vc);
                }
                quad_blend(s, w, fv, vc, U, W, qq, P, o);
                smem_store4(out + r * ZP, 4 * k + 4, o);
            }
        }
        __syncthreads();
        // second sweep at plane x - 1 over the tile
        const int xo = x - 1;
        if (xo >= x0) {
            const T* lo = v1s + wrap_mod(xo - 1, 3) * PL1;
            const T* mid = v1s + wrap_mod(xo, 3) * PL1;
            const T* hi = v1s + wrap_mod(xo + 1, 3) * PL1;
            const int r = tid / TQ, k = tid % TQ;
            const int gy = y0 + r, gz = z0 + 4 * k;
            if (gy < n1 && gz < n2) {
                const int64_t at = (int64_t)xo * sx + (int64_t)gy * n2 + gz;
                T fv[4], vc[4], U[4], W[4], qq[4], P[4], o[4];
                load4(f + at, fv);
                QuadCols<T> Q;
                smem_cols<T, ZP>(lo, mid, hi, r + 1, 4 * k + 8, Q);
                quad_compute<T, T, T, LOCAL>(Q, s, xo, gy, gz, U, W, qq, P);
                smem_quad4(mid + (r + 1) * ZP, 4 * k + 8, vc);
                quad_blend(s, w, fv, vc, U, W, qq, P, o);
                if constexpr (sizeof(T) == 4) {
                    *(float4*)(vout + at) = make_float4(o[0], o[1], o[2], o[3]);
                } else {
                    ((double2*)(vout + at))[0] = make_double2(o[0], o[1]);
                    ((double2*)(vout + at))[1] = make_double2(o[2], o[3]);
                }
            }
        }
    }
}

// r = f - A v = (f + U - 2 v sum 1/h^2) + g (W - 2 P v), g = beta / q, evaluated in type A.
template <typename A, typename V, typename FT, typename R, typename S, int MODE>
__global__ void __launch_bounds__(256) residual_kernel4(const V* __restrict__ v, const FT* __restrict__ f,
                                                        R* __restrict__ r, Stencil<S> s) {
    pdl_trigger();
    pdl_wait();
    Quad q;
    if (!quad_of(s.n, q)) return;
    const int64_t bo = batch_offset(s.n);
    v += bo, f += bo, r += bo;
    A U[4], W[4], qq[4], P[4];
    quad_terms<A, V, S, MODE>(v, s, q, U, W, qq, P);
    V vc[4];
    FT fv[4];
    load4(v + q.c + q.z0, vc);
    load4(f + q.c + q.z0, fv);
    const A sih2 = (A)2 * ((A)s.ih2[0] + (A)s.ih2[1] + (A)s.ih2[2]);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const A g = quotient<A>((A)s.beta, qq[k]);
        const A x = (A)vc[k];
        r[q.c + q.z0 + k] = (R)(((A)fv[k] + U[k] - sih2 * x) + g * (W[k] - (A)2 * P[k] * x));
    }
}

// r = f - A v, evaluated in type A (double for the mixed-precision defect), stored as R.
template <typename A, typename V, typename FT, typename R, typename S>
__global__ void __launch_bounds__(256) residual_kernel(const V* __restrict__ v, const FT* __restrict__ f,
                                                       R* __restrict__ r, Stencil<S> s) {
    pdl_trigger();
    pdl_wait();
    int x, y, z;
    if (!cell3(s.n, x, y, z)) return;
    const int64_t bo = batch_offset(s.n);
    v += bo, f += bo, r += bo;
    const int64_t i = ((int64_t)x * s.n[1] + y) * s.n[2] + z;
    A p[3], g, G[3];
    coeffs<A>(s, x, y, z, p, g, G);
    const A nb = neighbour_sum<A>(v, s.n, x, y, z, p, g, G, s.local);
    const A av = (A)2 * (G[0] + G[1] + G[2]) * (A)v[i] - nb;
    r[i] = (R)((A)f[i] - av);
}

// The quad kernels' instance for an operator form (mg_mode).
template <typename T> static decltype(&jacobi_sweep4<T, MG_GLOBAL>) sweep4_kernel(int mode) {
    switch (mode) {
    case MG_LOCAL: return jacobi_sweep4<T, MG_LOCAL>;
    case MG_AXIS0: return jacobi_sweep4<T, MG_AXIS0>;
    case MG_AXIS1: return jacobi_sweep4<T, MG_AXIS1>;
    case MG_AXIS2: return jacobi_sweep4<T, MG_AXIS2>;
    default: return jacobi_sweep4<T, MG_GLOBAL>;
    }
}
template <typename A, typename V, typename FT, typename R, typename S>
static decltype(&residual_kernel4<A, V, FT, R, S, MG_GLOBAL>) residual4_kernel(int mode) {
    switch (mode) {
    case MG_LOCAL: return residual_kernel4<A, V, FT, R, S, MG_LOCAL>;
    case MG_AXIS0: return residual_kernel4<A, V, FT, R, S, MG_AXIS0>;
    case MG_AXIS1: return residual_kernel4<A, V, FT, R, S, MG_AXIS1>;
    case MG_AXIS2: return residual_kernel4<A, V, FT, R, S, MG_AXIS2>;
    default: return residual_kernel4<A, V, FT, R, S, MG_GLOBAL>;
    }
}

// 27-point full weighting, coarse cell (x, y, z) centred on fine (2x, 2y, 2z).
template <typename A, typename TI, typename TO>
__global__ void __launch_bounds__(256) reduce_kernel(const TI* __restrict__ fine, TO* __restrict__ coarse, Dims nf) {
    pdl_trigger();
    pdl_wait();
    const int nc[3] = {nf.n[0] / 2, nf.n[1] / 2, nf.n[2] / 2};
    {
        int x, y, z;
        if (!cell3(nc, x, y, z)) return;
        const int64_t bc = batch_offset(nc);
        fine += 8 * bc, coarse += bc;
        const int64_t i = ((int64_t)x * nc[1] + y) * nc[2] + z;
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
    pdl_trigger();
    pdl_wait();
    const int nf1 = 2 * nc.n[1], nf2 = 2 * nc.n[2];
    {
        int x, y, z;
        if (!cell3(nc.n, x, y, z)) return;
        const int64_t bc = batch_offset(nc.n);
        coarse += bc, fine += 8 * bc;
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
    pdl_trigger();
    pdl_wait();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (TO)in[i];
}

template <typename TA, typename TB>
__global__ void add_kernel(TA* __restrict__ acc, const TB* __restrict__ x, int64_t n) {
    pdl_trigger();
    pdl_wait();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc[i] = acc[i] + (TA)x[i];
}

static int grid_for(int64_t n) {
    int64_t blocks = (n + 255) / 256;
    return (int)std::max<int64_t>(1, std::min<int64_t>(blocks, (int64_t)device_sm_count() * 16));
}

// 3D launch over an (n0, n1, n2) mesh for the cell3 kernels: up to 32 z x 8 y threads per block.
struct Grid3 {
    dim3 grid, block;
};
// `count` problems of that shape: count n0 blocks along z (see cell3).
static Grid3 grid3(const int n[3], int count = 1) {
    int bx = 1, by = 1;
    while (bx < n[2] && bx < 32) bx <<= 1;
    while (by < n[1] && bx * by < 256) by <<= 1;
    Grid3 g;
    g.block = dim3(bx, by, 1);
    g.grid = dim3((n[2] + bx - 1) / bx, (n[1] + by - 1) / by, n[0] * count);
    return g;
}
static Grid3 grid3_coarse(const int nf[3], int count = 1) {
    const int nc[3] = {nf[0] / 2, nf[1] / 2, nf[2] / 2};
    return grid3(nc, count);
}
// Launch of the four-cells-per-thread kernels, usable when n2 % 4 == 0 and the meshes are
// 16-byte aligned.
static Grid3 grid3_quad(const int n[3], int count = 1) {
    const int nq[3] = {n[0], n[1], n[2] / 4};
    return grid3(nq, count);
}
static bool quad_ok(const int n[3], const void* a, const void* b, const void* c) {
    return n[2] % 4 == 0 && (((uintptr_t)a | (uintptr_t)b | (uintptr_t)c) & 15) == 0;
}

// Tile of the temporal-blocked sweeps: TB_TY rows x 4 TB_TQ cells.
constexpr int TB_TY = 8, TB_TQ = 16;

// Slab length of the temporal-blocked sweeps for a level with no tuning-table entry (0: one sweep per
// pass).
static int mg_tb_default(const int n[3], size_t tsize) {
    (void)n;
    (void)tsize;
    return 0;
}

// ---- the V-cycle of the smallest levels in one block per problem ----
// Below a few thousand cells a level costs more in launches than in work: a V-cycle visit of the levels
// under 16^3 is ~40 kernels of a few microseconds each.  vcycle_small runs the V-cycle of levels
// l0 .. l0 + nl - 1 (MGRunner::vcycle's pre-sweeps, residual, restriction, prolongation and post-sweeps,
// with the one-cell expressions of jacobi_sweep, residual_kernel, reduce_kernel and prolong_kernel) in one
// block, each level's v, f and scratch in shared memory, a block barrier between steps.  The problems of
// a batch are one block each.
constexpr int MG_SMALL_LEVELS = 8;
constexpr int MG_SMALL_THREADS = 512;
// Default top level of vcycle_small: 8^3.  Measured per 256^3 local-line-of-sight solve, 10.40 ms with every
// step its own graph node, 10.05 ms from 8^3 down, 11.98 ms from 16^3 down (one block then does ~93k cell
// updates per visit on one SM, slower than the ~40 launches it replaces).
constexpr int MG_SMALL_DEFAULT_CELLS = 512;
constexpr size_t MG_SMALL_MAX_SMEM = 200 * 1024;

template <typename T> struct SmallVCycle {
    int nl;
    Stencil<T> s[MG_SMALL_LEVELS];
    int off[MG_SMALL_LEVELS];    // level l's arrays v, f, scratch (cells(l) values each) start at off[l]
    T w;
    int jn;
    int zero_v;                  // the top level's v starts at zero (not read)
};

__device__ __forceinline__ int cells_of(const int n[3]) { return n[0] * n[1] * n[2]; }

__device__ __forceinline__ void cell_xyz(int i, const int n[3], int& x, int& y, int& z) {
    z = i % n[2];
    y = (i / n[2]) % n[1];
    x = i / (n[1] * n[2]);
}

template <typename T>
__device__ void small_sweeps(const Stencil<T>& s, T*& v, const T* f, T*& tmp, T w, int niter, bool zero) {
    const int N = cells_of(s.n);
    if (niter == 0 && zero)
        for (int i = threadIdx.x; i < N; i += blockDim.x) v[i] = (T)0;
    for (int it = 0; it < niter; it++) {
        const bool z0 = zero && it == 0;
        for (int i = threadIdx.x; i < N; i += blockDim.x) {
            int x, y, z;
            cell_xyz(i, s.n, x, y, z);
            T p[3], g, G[3];
            coeffs<T>(s, x, y, z, p, g, G);
            T jac = f[i];
            T vc = (T)0;
            if (!z0) {
                jac += neighbour_sum<T, T, true>(v, s.n, x, y, z, p, g, G, s.local);
                vc = v[i];
            }
            jac /= (T)2 * (G[0] + G[1] + G[2]);
            tmp[i] = ((T)1 - w) * vc + w * jac;
        }
        T* t = v;
        v = tmp;
        tmp = t;
        __syncthreads();
    }
    __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(MG_SMALL_THREADS) vcycle_small(const T* __restrict__ fg, T* __restrict__ vg,
                                                                 SmallVCycle<T> P) {
    pdl_trigger();
    pdl_wait();
    extern __shared__ __align__(16) unsigned char mg_smem[];
    T* sm = (T*)mg_smem;
    const int N0 = cells_of(P.s[0].n);
    fg += (int64_t)blockIdx.x * N0;
    vg += (int64_t)blockIdx.x * N0;
    T *v[MG_SMALL_LEVELS], *f[MG_SMALL_LEVELS], *t[MG_SMALL_LEVELS];
    for (int l = 0; l < P.nl; l++) {
        const int N = cells_of(P.s[l].n);
        v[l] = sm + P.off[l];
        f[l] = v[l] + N;
        t[l] = f[l] + N;
    }
    for (int i = threadIdx.x; i < N0; i += blockDim.x) {
        f[0][i] = fg[i];
        if (!P.zero_v) v[0][i] = vg[i];
    }
    __syncthreads();
    // down: pre-sweeps, then the residual restricted to the next level's right-hand side
    for (int l = 0; l < P.nl; l++) {
        const Stencil<T>& s = P.s[l];
        small_sweeps(s, v[l], f[l], t[l], P.w, P.jn, l > 0 || P.zero_v);
        if (l + 1 == P.nl) break;
        const int N = cells_of(s.n);
        for (int i = threadIdx.x; i < N; i += blockDim.x) {
            int x, y, z;
            cell_xyz(i, s.n, x, y, z);
            T p[3], g, G[3];
            coeffs<T>(s, x, y, z, p, g, G);
            const T nb = neighbour_sum<T, T, true>(v[l], s.n, x, y, z, p, g, G, s.local);
            const T av = (T)2 * (G[0] + G[1] + G[2]) * v[l][i] - nb;
            t[l][i] = f[l][i] - av;
        }
        __syncthreads();
        const int* nf = s.n;
        const int* nc = P.s[l + 1].n;
        const int Nc = cells_of(nc);
        for (int i = threadIdx.x; i < Nc; i += blockDim.x) {
            int x, y, z;
            cell_xyz(i, nc, x, y, z);
            const int X[3] = {wrap_dn(2 * x, nf[0]), 2 * x, wrap_up(2 * x, nf[0])};
            const int Y[3] = {wrap_dn(2 * y, nf[1]), 2 * y, wrap_up(2 * y, nf[1])};
            const int Z[3] = {wrap_dn(2 * z, nf[2]), 2 * z, wrap_up(2 * z, nf[2])};
            T acc = 0;
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++) {
                    const T* row = t[l] + (X[a] * nf[1] + Y[b]) * nf[2];
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const int side = (a != 1) + (b != 1) + (c != 1);
                        acc += (T)(8 >> side) * row[Z[c]];
                    }
                }
            f[l + 1][i] = acc / (T)64;
        }
        __syncthreads();
    }
    // up: the coarse correction prolonged and added, then post-sweeps
    for (int l = P.nl - 1; l >= 0; l--) {
        if (l + 1 < P.nl) {
            const int* nc = P.s[l + 1].n;
            const int Nc = cells_of(nc);
            const int nf1 = 2 * nc[1], nf2 = 2 * nc[2];
            for (int i = threadIdx.x; i < Nc; i += blockDim.x) {
                int x, y, z;
                cell_xyz(i, nc, x, y, z);
                const int xs[2] = {x, wrap_up(x, nc[0])}, ys[2] = {y, wrap_up(y, nc[1])}, zs[2] = {z, wrap_up(z, nc[2])};
                T c[2][2][2];
#pragma unroll
                for (int a = 0; a < 2; a++)
#pragma unroll
                    for (int b = 0; b < 2; b++)
#pragma unroll
                        for (int d = 0; d < 2; d++) c[a][b][d] = v[l + 1][(xs[a] * nc[1] + ys[b]) * nc[2] + zs[d]];
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const int ex = (e >> 2) & 1, ey = (e >> 1) & 1, ez = e & 1;
                    T sum = 0;
#pragma unroll
                    for (int a = 0; a <= ex; a++)
#pragma unroll
                        for (int b = 0; b <= ey; b++)
#pragma unroll
                            for (int d = 0; d <= ez; d++) sum += c[a][b][d];
                    sum /= (T)((1 + ex) * (1 + ey) * (1 + ez));
                    T* dst = v[l] + ((2 * x + ex) * nf1 + (2 * y + ey)) * nf2 + (2 * z + ez);
                    *dst = *dst + sum;
                }
            }
            __syncthreads();
        }
        small_sweeps(P.s[l], v[l], f[l], t[l], P.w, P.jn, false);
    }
    for (int i = threadIdx.x; i < N0; i += blockDim.x) vg[i] = v[0][i];
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
    std::vector<LevelBufs<T>> B;     // per level: count problems one after the other in each buffer
    Params P;
    cudaStream_t st;
    int count = 1;

    Stencil<T> stencil(int l) const {
        return make_stencil<T>(L[l].n, P.boxsize, P.boxcenter, P.beta, P.has_los ? P.los : nullptr);
    }

    // niter sweeps ping-ponging between v and tmp; on return v points at the result and tmp at the
    // other buffer (the pointers are swapped instead of copying back).  zero_first: v known zero.
    // Pairs of sweeps run as one temporal-blocked pass when the tuning table's "mg_jacobi" (FP32) or
    // "mg_jacobi_f64" entry for the level (keyed by n0) is a slab length > 0 (mg_tb_default otherwise).
    int jacobi(int l, T*& v, const T* f, T*& tmp, int niter, bool zero_first) {
        Stencil<T> s = stencil(l);
        const int64_t N = L[l].size() * count;
        const Grid3 g = grid3(L[l].n, count);
        if (niter == 0 && zero_first && cudaMemsetAsync(v, 0, N * sizeof(T), st) != cudaSuccess) return PRC_ERR_CUDA;
        const bool quad = quad_ok(L[l].n, v, f, tmp);
        const Grid3 gq = grid3_quad(L[l].n, count);
        int it = 0;
        const int slab =
            quad ? tune_get(sizeof(T) == 4 ? "mg_jacobi" : "mg_jacobi_f64", L[l].n[0], mg_tb_default(L[l].n, sizeof(T)))
                 : 0;
        if (slab > 0) {
            const int nslab = (L[l].n[0] + slab - 1) / slab;
            const dim3 grid((L[l].n[2] + 4 * TB_TQ - 1) / (4 * TB_TQ), (L[l].n[1] + TB_TY - 1) / TB_TY, nslab * count);
            if ((int64_t)nslab * count <= 65535) {
                for (; it + 1 < niter; it += 2) {
                    const bool z0 = zero_first && it == 0;
                    PRC_LAUNCH_B("mg_jacobi2", st, (double)N * sizeof(T) * (z0 ? 2 : 3),
                                 launch_pdl((s.local ? jacobi_sweep2_tb<T, true, TB_TY, TB_TQ>
                                          : jacobi_sweep2_tb<T, false, TB_TY, TB_TQ>), grid, TB_TY * TB_TQ, 0, st, v, f, tmp, s, (T)P.damping, z0, slab, nslab));
                    std::swap(v, tmp);
                }
            }
        }
        for (; it < niter; it++) {
            const bool z0 = zero_first && it == 0;
            if (quad)
                PRC_LAUNCH_B("mg_jacobi", st, (double)N * sizeof(T) * (z0 ? 2 : 3),
                             launch_pdl(sweep4_kernel<T>(mg_mode(s)), gq.grid, gq.block, 0, st, v, f, tmp, s, (T)P.damping, z0));
            else
                PRC_LAUNCH_B("mg_jacobi", st, (double)N * sizeof(T) * (z0 ? 2 : 3),
                             launch_pdl(jacobi_sweep<T, T>, g.grid, g.block, 0, st, v, f, tmp, s, (T)P.damping, z0));
            std::swap(v, tmp);
        }
        PRC_CHECK_LAUNCH();
        return PRC_OK;
    }

    // The V-cycle from level l down as one vcycle_small launch, when level l has at most "mg_small_cells"
    // cells (run-time knob, key 0; 0 runs every step as its own kernel) and its levels fit in shared memory.
    int small_vcycle(int l, T* v, const T* f, bool v_zero, bool* done) {
        *done = false;
        const int limit = tune_get("mg_small_cells", 0, MG_SMALL_DEFAULT_CELLS);
        const int nl = (int)L.size() - l;
        if (limit <= 0 || L[l].size() > limit || nl > MG_SMALL_LEVELS) return PRC_OK;
        SmallVCycle<T> sv;
        size_t off = 0;
        sv.nl = nl;
        for (int j = 0; j < nl; j++) {
            sv.s[j] = stencil(l + j);
            sv.off[j] = (int)off;
            off = (off + 3 * (size_t)L[l + j].size() + 3) & ~(size_t)3;
        }
        const size_t smem = off * sizeof(T);
        if (smem > MG_SMALL_MAX_SMEM) return PRC_OK;
        sv.w = (T)P.damping;
        sv.jn = P.jn;
        sv.zero_v = v_zero ? 1 : 0;
        if (smem > 48 * 1024 &&
            cudaFuncSetAttribute(vcycle_small<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return PRC_ERR_CUDA;
        PRC_LAUNCH_B("mg_vcycle_small", st, (double)L[l].size() * count * sizeof(T) * (v_zero ? 2 : 3),
                     launch_pdl(vcycle_small<T>, dim3(count), dim3(MG_SMALL_THREADS), smem, st, f, v, sv));
        PRC_CHECK_LAUNCH();
        *done = true;
        return PRC_OK;
    }

    // Recursive V-cycle on level l: v (B[l].v, or the caller's level-0 pointer) with right-hand side f.
    int vcycle(int l, T*& v, const T* f, bool v_zero) {
        bool small = false;
        PRC_TRY(small_vcycle(l, v, f, v_zero, &small));
        if (small) return PRC_OK;
        PRC_TRY(jacobi(l, v, f, B[l].tmp, P.jn, v_zero));
        if (l + 1 < (int)L.size()) {
            Stencil<T> s = stencil(l);
            const int64_t N = L[l].size() * count;
            const Grid3 g = grid3(L[l].n, count), gc = grid3_coarse(L[l].n, count);
            if (quad_ok(L[l].n, v, f, B[l].r)) {
                const Grid3 gq = grid3_quad(L[l].n, count);
                PRC_LAUNCH_B("mg_residual", st, 3.0 * N * sizeof(T),
                             launch_pdl(residual4_kernel<T, T, T, T, T>(mg_mode(s)), gq.grid, gq.block, 0, st, v, f, B[l].r, s));
            } else {
                PRC_LAUNCH_B("mg_residual", st, 3.0 * N * sizeof(T),
                             launch_pdl(residual_kernel<T, T, T, T, T>, g.grid, g.block, 0, st, v, f, B[l].r, s));
            }
            Dims nf = {{L[l].n[0], L[l].n[1], L[l].n[2]}};
            PRC_LAUNCH_B("mg_reduce", st, (double)(N + L[l + 1].size() * count) * sizeof(T),
                         launch_pdl(reduce_kernel<T, T, T>, gc.grid, gc.block, 0, st, B[l].r, B[l + 1].f, nf));
            PRC_CHECK_LAUNCH();
            PRC_TRY(vcycle(l + 1, B[l + 1].v, B[l + 1].f, true));
            Dims nc = {{L[l + 1].n[0], L[l + 1].n[1], L[l + 1].n[2]}};
            PRC_LAUNCH_B("mg_prolong_add", st, (double)(2 * N + L[l + 1].size() * count) * sizeof(T),
                         launch_pdl(prolong_kernel<T, T, T, true>, gc.grid, gc.block, 0, st, B[l + 1].v, v, nc));
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
    const int cnt = R.count;
    for (int l = 0; l + 1 < nl; l++) {
        Dims nf = {{R.L[l].n[0], R.L[l].n[1], R.L[l].n[2]}};
        const Grid3 gc = grid3_coarse(R.L[l].n, cnt);
        PRC_LAUNCH_B("mg_reduce", st, (double)(R.L[l].size() + R.L[l + 1].size()) * cnt * sizeof(T),
                     launch_pdl(reduce_kernel<T, T, T>, gc.grid, gc.block, 0, st, R.B[l].f, R.B[l + 1].f, nf));
    }
    PRC_CHECK_LAUNCH();
    // the FMG solution of level l >= 1 lives in B[l].v; level 0 starts in v0 and may end in
    // B[0].tmp (pointer swaps), in which case it is copied to v0 once at the end
    T* v0cur = v0;
    for (int l = nl - 1; l >= 0; l--) {
        T*& v = l == 0 ? v0cur : R.B[l].v;
        if (l == nl - 1) {
            if (cudaMemsetAsync(v, 0, R.L[l].size() * cnt * sizeof(T), st) != cudaSuccess) return PRC_ERR_CUDA;
        } else {
            Dims nc = {{R.L[l + 1].n[0], R.L[l + 1].n[1], R.L[l + 1].n[2]}};
            const Grid3 gc = grid3(R.L[l + 1].n, cnt);
            PRC_LAUNCH_B("mg_prolong", st, (double)(R.L[l].size() + R.L[l + 1].size()) * cnt * sizeof(T),
                         launch_pdl(prolong_kernel<T, T, T, false>, gc.grid, gc.block, 0, st, R.B[l + 1].v, v, nc));
            PRC_CHECK_LAUNCH();
        }
        for (int it = 0; it < R.P.vn; it++) PRC_TRY(R.vcycle(l, v, R.B[l].f, l == nl - 1 && it == 0));
    }
    if (v0cur != v0 &&
        cudaMemcpyAsync(v0, v0cur, R.L[0].size() * cnt * sizeof(T), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return PRC_ERR_CUDA;
    return PRC_OK;
}

}  // namespace prc

using namespace prc;

namespace {

// Workspace layout for plain FMG in precision T: per level v, f, r, tmp (level 0's f and v receive the
// caller's right-hand side and return the solution, so the solve itself touches the workspace only).
template <typename T> size_t plain_layout(const int32_t nmesh[3], char* base, std::vector<LevelBufs<T>>* out,
                                          std::vector<Level>* lv, int count = 1) {
    std::vector<Level> L = hierarchy(nmesh);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base ? base + off : nullptr;
        off += al(bytes);
        return p;
    };
    std::vector<LevelBufs<T>> B(L.size());
    for (size_t l = 0; l < L.size(); l++) {
        size_t b = (size_t)L[l].size() * count * sizeof(T);
        B[l].v = (T*)take(b);
        B[l].f = (T*)take(b);
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

size_t mixed_layout(const int32_t nmesh[3], char* base, MixedBufs* mb, int count = 1) {
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
        size_t n = (size_t)L[l].size() * count;
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

// Plain solve of the right-hand side held in the workspace's level-0 f into its level-0 v.
template <typename T> int solve_plain(const int32_t nmesh[3], const Params& P, void* ws, cudaStream_t st,
                                      int count = 1) {
    MGRunner<T> R;
    plain_layout<T>(nmesh, (char*)ws, &R.B, &R.L, count);
    R.P = P;
    R.st = st;
    R.count = count;
    T* f0 = R.B[0].f;
    T* v0 = R.B[0].v;
    return fmg_plain<T>(R, f0, v0);
}

// Mixed precision FMG: every V-cycle is v64 += V32(0, f64 - A v64); the FP64 right-hand side is in the
// workspace's level-0 f64 and the solution is left in its level-0 v64.
int solve_mixed(const int32_t nmesh[3], const Params& P, void* ws, cudaStream_t st, int count = 1) {
    MixedBufs m;
    mixed_layout(nmesh, (char*)ws, &m, count);
    const int nl = (int)m.L.size();
    MGRunner<float> R;
    R.L = m.L;
    R.B = m.b32;
    R.P = P;
    R.st = st;
    R.count = count;
    for (int l = 0; l + 1 < nl; l++) {
        Dims nf = {{m.L[l].n[0], m.L[l].n[1], m.L[l].n[2]}};
        const Grid3 gc = grid3_coarse(m.L[l].n, count);
        PRC_LAUNCH_B("mg_reduce", st, 8.0 * (m.L[l].size() + m.L[l + 1].size()) * count,
                     launch_pdl(reduce_kernel<double, double, double>, gc.grid, gc.block, 0, st, m.f64[l], m.f64[l + 1], nf));
    }
    PRC_CHECK_LAUNCH();
    for (int l = nl - 1; l >= 0; l--) {
        const int64_t N = m.L[l].size() * count;
        const Grid3 g = grid3(m.L[l].n, count);
        if (l == nl - 1) {
            if (cudaMemsetAsync(m.v64[l], 0, N * 8, st) != cudaSuccess) return PRC_ERR_CUDA;
        } else {
            Dims nc = {{m.L[l + 1].n[0], m.L[l + 1].n[1], m.L[l + 1].n[2]}};
            const Grid3 gc = grid3(m.L[l + 1].n, count);
            PRC_LAUNCH_B("mg_prolong", st, 8.0 * (m.L[l].size() + m.L[l + 1].size()) * count,
                         launch_pdl(prolong_kernel<double, double, double, false>, gc.grid, gc.block, 0, st, m.v64[l + 1],
                                                                                                  m.v64[l], nc));
        }
        Stencil<double> s64 = make_stencil<double>(m.L[l].n, P.boxsize, P.boxcenter, P.beta,
                                                   P.has_los ? P.los : nullptr);
        for (int it = 0; it < P.vn; it++) {
            // defect in FP64 (stored FP32 as the inner V-cycle's right-hand side)
            if (quad_ok(m.L[l].n, m.v64[l], m.f64[l], R.B[l].f)) {
                const Grid3 gq = grid3_quad(m.L[l].n, count);
                PRC_LAUNCH_B("mg_residual_fp64", st, 20.0 * N,
                             launch_pdl(residual4_kernel<double, double, double, float, double>(mg_mode(s64)), gq.grid, gq.block, 0, st, m.v64[l], m.f64[l], R.B[l].f, s64));
            } else {
                PRC_LAUNCH_B("mg_residual_fp64", st, 20.0 * N,
                             launch_pdl(residual_kernel<double, double, double, float, double>, g.grid, g.block, 0, st, m.v64[l], m.f64[l], R.B[l].f, s64));
            }
            PRC_CHECK_LAUNCH();
            PRC_TRY(R.vcycle(l, R.B[l].v, R.B[l].f, true));
            PRC_LAUNCH_B("mg_correct_fp64", st, 20.0 * N,
                         launch_pdl(add_kernel<double, float>, grid_for(N), 256, 0, st, m.v64[l], R.B[l].v, N));
            PRC_CHECK_LAUNCH();
        }
    }
    return PRC_OK;
}

// ---- the whole solve as a CUDA graph ----
//
// A solve is a fixed sequence of some thousands of small launches (most on the coarse levels),
// set by the mesh, the parameters and the workspace address (the caller's right-hand side and
// solution are copied in and out around it, so they are not part of it).  It is captured once into a CUDA graph
// and replayed while those stay the same (a small cache keyed on all of them), on the caller's stream
// (on a library stream joined to it by events when the caller gives the legacy default stream, which
// cannot be captured).  PRC_MG_GRAPH=0 launches directly.
struct GraphEntry {
    std::string key;
    int device;
    cudaGraphExec_t exec;
    unsigned long long launches;
    double bytes;
};
struct SideStream {
    cudaStream_t s = nullptr;
    cudaEvent_t in = nullptr, out = nullptr;
};
std::mutex g_graph_mutex;
std::list<GraphEntry> g_graphs;
std::map<int, SideStream> g_side;
constexpr size_t GRAPH_CACHE = 64;

bool graphs_enabled() {
    static int cached = -1;
    if (cached < 0) {
        const char* v = getenv("PRC_MG_GRAPH");
        cached = (v != nullptr && v[0] == '0') ? 0 : 1;
    }
    return cached == 1;
}

template <typename V> void key_add(std::string& k, const V& v) { k.append((const char*)&v, sizeof(V)); }

std::string solve_key(int tsize, int mixed, const int32_t nmesh[3], const Params& P, const void* ws, size_t wsb,
                      int count) {
    std::string k;
    key_add(k, tsize);
    key_add(k, mixed);
    key_add(k, count);
    for (int d = 0; d < 3; d++) {
        key_add(k, nmesh[d]);
        key_add(k, P.boxsize[d]);
        key_add(k, P.boxcenter[d]);
        key_add(k, P.los[d]);
    }
    key_add(k, P.has_los);
    key_add(k, P.beta);
    key_add(k, P.damping);
    key_add(k, P.jn);
    key_add(k, P.vn);
    key_add(k, ws);
    key_add(k, wsb);
    key_add(k, tune_generation());   // kernel choices of the tuning table
    return k;
}

template <typename F> int run_graph(const std::string& key, cudaStream_t st, F body) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (!graphs_enabled() || cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
        return body(st);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PRC_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_graph_mutex);
    const bool legacy = st == nullptr || st == cudaStreamLegacy;
    SideStream& side = g_side[dev];
    if (legacy && side.s == nullptr) {
        if (cudaStreamCreateWithFlags(&side.s, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&side.in, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&side.out, cudaEventDisableTiming) != cudaSuccess) {
            side = SideStream();
            return body(st);
        }
    }
    const cudaStream_t run_st = legacy ? side.s : st;
    if (legacy &&
        (cudaEventRecord(side.in, st) != cudaSuccess || cudaStreamWaitEvent(side.s, side.in, 0) != cudaSuccess))
        return PRC_ERR_CUDA;
    auto it = g_graphs.begin();
    for (; it != g_graphs.end(); ++it)
        if (it->device == dev && it->key == key) break;
    if (it != g_graphs.end()) {
        g_graphs.splice(g_graphs.begin(), g_graphs, it);
    } else {
        capture_tally(nullptr, nullptr);
        if (cudaStreamBeginCapture(run_st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return PRC_ERR_CUDA;
        const int r = body(run_st);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(run_st, &g);
        GraphEntry ent;
        capture_tally(&ent.launches, &ent.bytes);
        if (r != PRC_OK || e != cudaSuccess || g == nullptr) {
            if (g != nullptr) cudaGraphDestroy(g);
            cudaGetLastError();
            return r != PRC_OK ? r : PRC_ERR_CUDA;
        }
        const cudaError_t ei = cudaGraphInstantiate(&ent.exec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) return PRC_ERR_CUDA;
        ent.key = key;
        ent.device = dev;
        g_graphs.push_front(ent);
        while (g_graphs.size() > GRAPH_CACHE) {
            const GraphEntry& old = g_graphs.back();
            int cur = dev;
            if (old.device != cur) cudaSetDevice(old.device);
            cudaDeviceSynchronize();
            cudaGraphExecDestroy(old.exec);
            if (old.device != cur) cudaSetDevice(cur);
            g_graphs.pop_back();
        }
    }
    const GraphEntry& ent = g_graphs.front();
    {
        KernelScope scope("mg_solve_graph", run_st, ent.bytes, false);
        if (cudaGraphLaunch(ent.exec, run_st) != cudaSuccess) return PRC_ERR_CUDA;
    }
    add_launches(ent.launches);
    if (legacy &&
        (cudaEventRecord(side.out, side.s) != cudaSuccess || cudaStreamWaitEvent(st, side.out, 0) != cudaSuccess))
        return PRC_ERR_CUDA;
    return PRC_OK;
}

// Solve through the workspace: each problem's right-hand side is copied into its slot of level 0's f
// (FP64 f for the mixed precision solve), the (graph-captured) solve runs on the workspace alone,
// and each slot of level 0's v is copied out.
template <typename T>
int run_plain_io(const T* const* delta, T* const* phi, int count, const int32_t nmesh[3], const Params& P, void* ws,
                 const std::string& key, cudaStream_t st) {
    std::vector<LevelBufs<T>> B;
    plain_layout<T>(nmesh, (char*)ws, &B, nullptr, count);
    const int64_t N = (int64_t)nmesh[0] * nmesh[1] * nmesh[2];
    for (int b = 0; b < count; b++)
        if (cudaMemcpyAsync(B[0].f + b * N, delta[b], N * sizeof(T), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return PRC_ERR_CUDA;
    PRC_TRY(run_graph(key, st, [&](cudaStream_t s) { return solve_plain<T>(nmesh, P, ws, s, count); }));
    for (int b = 0; b < count; b++)
        if (cudaMemcpyAsync(phi[b], B[0].v + b * N, N * sizeof(T), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return PRC_ERR_CUDA;
    return PRC_OK;
}

int run_mixed_io(const float* const* delta, float* const* phi, double* const* phi64, int count, const int32_t nmesh[3],
                 const Params& P, void* ws, const std::string& key, cudaStream_t st) {
    MixedBufs m;
    mixed_layout(nmesh, (char*)ws, &m, count);
    const int64_t N = (int64_t)nmesh[0] * nmesh[1] * nmesh[2];
    for (int b = 0; b < count; b++)
        PRC_LAUNCH_B("mg_convert", st, 12.0 * N,
                     convert_kernel<float, double><<<grid_for(N), 256, 0, st>>>(delta[b], m.f64[0] + b * N, N));
    PRC_CHECK_LAUNCH();
    PRC_TRY(run_graph(key, st, [&](cudaStream_t s) { return solve_mixed(nmesh, P, ws, s, count); }));
    for (int b = 0; b < count; b++) {
        PRC_LAUNCH_B("mg_convert", st, 12.0 * N,
                     convert_kernel<double, float><<<grid_for(N), 256, 0, st>>>(m.v64[0] + b * N, phi[b], N));
        if (phi64 && phi64[b] &&
            cudaMemcpyAsync(phi64[b], m.v64[0] + b * N, N * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return PRC_ERR_CUDA;
    }
    PRC_CHECK_LAUNCH();
    return PRC_OK;
}

// The batch shares one launch per step along z: count n0 planes (see cell3).
bool batch_ok(const int32_t nmesh[3], int count) { return count >= 1 && (int64_t)nmesh[0] * count <= 65535; }

}  // namespace

extern "C" {

size_t prc_multigrid_batch_workspace_bytes(const int32_t nmesh[3], int mesh_bytes, int mixed_precision, int count) {
    if (!nmesh || count < 1) return 0;
    for (int d = 0; d < 3; d++)
        if (nmesh[d] < 1) return 0;
    if (mesh_bytes == 4 && mixed_precision) return mixed_layout(nmesh, nullptr, nullptr, count);
    if (mesh_bytes == 4) return plain_layout<float>(nmesh, nullptr, nullptr, nullptr, count);
    return plain_layout<double>(nmesh, nullptr, nullptr, nullptr, count);
}

size_t prc_multigrid_workspace_bytes(const int32_t nmesh[3], int mesh_bytes, int mixed_precision) {
    return prc_multigrid_batch_workspace_bytes(nmesh, mesh_bytes, mixed_precision, 1);
}

prc_status_t prc_multigrid_batch_f32(const float* const* delta, float* const* phi, int count, const int32_t nmesh[3],
                                     const double boxsize[3], const double boxcenter[3], double beta, double damping,
                                     int jacobi_niterations, int vcycle_niterations, const double* los,
                                     int mixed_precision, void* workspace, size_t workspace_bytes, void* stream) {
    if (!delta || !phi || !batch_ok(nmesh, count)) return PRC_ERR_ARG;
    for (int b = 0; b < count; b++)
        if (!mg_args_ok(delta[b], phi[b], nmesh, boxsize, boxcenter, jacobi_niterations, vcycle_niterations))
            return PRC_ERR_ARG;
    Params P = make_params(boxsize, boxcenter, beta, damping, jacobi_niterations, vcycle_niterations, los);
    if (!workspace || workspace_bytes < prc_multigrid_batch_workspace_bytes(nmesh, 4, mixed_precision, count))
        return PRC_ERR_WORKSPACE;
    cudaStream_t st = (cudaStream_t)stream;
    const std::string key = solve_key(4, mixed_precision ? 1 : 0, nmesh, P, workspace, workspace_bytes, count);
    if (mixed_precision) return run_mixed_io(delta, phi, nullptr, count, nmesh, P, workspace, key, st);
    return run_plain_io<float>(delta, phi, count, nmesh, P, workspace, key, st);
}

prc_status_t prc_multigrid_batch_mixed_f32(const float* const* delta, float* const* phi, double* const* phi64,
                                           int count, const int32_t nmesh[3], const double boxsize[3],
                                           const double boxcenter[3], double beta, double damping,
                                           int jacobi_niterations, int vcycle_niterations, const double* los,
                                           void* workspace, size_t workspace_bytes, void* stream) {
    if (!delta || !phi || !batch_ok(nmesh, count)) return PRC_ERR_ARG;
    for (int b = 0; b < count; b++)
        if (!mg_args_ok(delta[b], phi[b], nmesh, boxsize, boxcenter, jacobi_niterations, vcycle_niterations))
            return PRC_ERR_ARG;
    Params P = make_params(boxsize, boxcenter, beta, damping, jacobi_niterations, vcycle_niterations, los);
    if (!workspace || workspace_bytes < prc_multigrid_batch_workspace_bytes(nmesh, 4, 1, count))
        return PRC_ERR_WORKSPACE;
    const std::string key = solve_key(4, 1, nmesh, P, workspace, workspace_bytes, count);
    return run_mixed_io(delta, phi, phi64, count, nmesh, P, workspace, key, (cudaStream_t)stream);
}

prc_status_t prc_multigrid_mixed_f32(const float* delta, float* phi, double* phi64, const int32_t nmesh[3],
                                     const double boxsize[3], const double boxcenter[3], double beta, double damping,
                                     int jacobi_niterations, int vcycle_niterations, const double* los,
                                     void* workspace, size_t workspace_bytes, void* stream) {
    return prc_multigrid_batch_mixed_f32(&delta, &phi, &phi64, 1, nmesh, boxsize, boxcenter, beta, damping,
                                         jacobi_niterations, vcycle_niterations, los, workspace, workspace_bytes,
                                         stream);
}

prc_status_t prc_multigrid_batch_f64(const double* const* delta, double* const* phi, int count,
                                     const int32_t nmesh[3], const double boxsize[3], const double boxcenter[3],
                                     double beta, double damping, int jacobi_niterations, int vcycle_niterations,
                                     const double* los, void* workspace, size_t workspace_bytes, void* stream) {
    if (!delta || !phi || !batch_ok(nmesh, count)) return PRC_ERR_ARG;
    for (int b = 0; b < count; b++)
        if (!mg_args_ok(delta[b], phi[b], nmesh, boxsize, boxcenter, jacobi_niterations, vcycle_niterations))
            return PRC_ERR_ARG;
    Params P = make_params(boxsize, boxcenter, beta, damping, jacobi_niterations, vcycle_niterations, los);
    if (!workspace || workspace_bytes < prc_multigrid_batch_workspace_bytes(nmesh, 8, 0, count)) return PRC_ERR_WORKSPACE;
    const std::string key = solve_key(8, 0, nmesh, P, workspace, workspace_bytes, count);
    return run_plain_io<double>(delta, phi, count, nmesh, P, workspace, key, (cudaStream_t)stream);
}

prc_status_t prc_multigrid_f32(const float* delta, float* phi, const int32_t nmesh[3], const double boxsize[3],
                               const double boxcenter[3], double beta, double damping, int jacobi_niterations,
                               int vcycle_niterations, const double* los, int mixed_precision, void* workspace,
                               size_t workspace_bytes, void* stream) {
    return prc_multigrid_batch_f32(&delta, &phi, 1, nmesh, boxsize, boxcenter, beta, damping, jacobi_niterations,
                                   vcycle_niterations, los, mixed_precision, workspace, workspace_bytes, stream);
}

prc_status_t prc_multigrid_f64(const double* delta, double* phi, const int32_t nmesh[3], const double boxsize[3],
                               const double boxcenter[3], double beta, double damping, int jacobi_niterations,
                               int vcycle_niterations, const double* los, void* workspace, size_t workspace_bytes,
                               void* stream) {
    return prc_multigrid_batch_f64(&delta, &phi, 1, nmesh, boxsize, boxcenter, beta, damping, jacobi_niterations,
                                   vcycle_niterations, los, workspace, workspace_bytes, stream);
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
        T *cur = v, *other = scratch;                                                                                \
        PRC_TRY(R.jacobi(0, cur, f, other, niterations, false));                                                     \
        if (cur != v && cudaMemcpyAsync(v, cur, (size_t)R.L[0].size() * sizeof(T), cudaMemcpyDeviceToDevice,       \
                                        (cudaStream_t)stream) != cudaSuccess)                                        \
            return PRC_ERR_CUDA;                                                                                     \
        return PRC_OK;                                                                                               \
    }                                                                                                                \
    prc_status_t prc_mg_residual_##SUF(const T* v, const T* f, T* r, const int32_t nmesh[3],                        \
                                       const double boxsize[3], const double boxcenter[3], double beta,             \
                                       const double* los, void* stream) {                                           \
        if (!v || !f || !r || !nmesh || !boxsize || !boxcenter) return PRC_ERR_ARG;                                 \
        int n[3] = {nmesh[0], nmesh[1], nmesh[2]};                                                                   \
        Stencil<T> s = make_stencil<T>(n, boxsize, boxcenter, beta, los);                                            \
        const double bytes = 3.0 * sizeof(T) * n[0] * n[1] * n[2];                                                   \
        if (quad_ok(n, v, f, r))                                                                                     \
            PRC_LAUNCH_B("mg_residual", (cudaStream_t)stream, bytes,                                                 \
                         residual4_kernel<T, T, T, T, T>(mg_mode(s))                                              \
                             <<<grid3_quad(n).grid, grid3_quad(n).block, 0, (cudaStream_t)stream>>>(v, f, r, s));     \
        else                                                                                                         \
            PRC_LAUNCH_B("mg_residual", (cudaStream_t)stream, bytes,                                                 \
                         residual_kernel<T, T, T, T, T><<<grid3(n).grid, grid3(n).block, 0, (cudaStream_t)stream>>>(  \
                             v, f, r, s));                                                                           \
        PRC_CHECK_LAUNCH();                                                                                          \
        return PRC_OK;                                                                                               \
    }                                                                                                                \
    prc_status_t prc_mg_reduce_##SUF(const T* fine, T* coarse, const int32_t nf[3], void* stream) {                 \
        if (!fine || !coarse || !nf) return PRC_ERR_ARG;                                                             \
        Dims d = {{nf[0], nf[1], nf[2]}};                                                                            \
        PRC_LAUNCH("mg_reduce", (cudaStream_t)stream,                                                                \
                   reduce_kernel<T, T, T><<<grid3_coarse(nf).grid, grid3_coarse(nf).block, 0, (cudaStream_t)stream>>>(fine, coarse, d)); \
        PRC_CHECK_LAUNCH();                                                                                          \
        return PRC_OK;                                                                                               \
    }                                                                                                                \
    prc_status_t prc_mg_prolong_##SUF(const T* coarse, T* fine, const int32_t nc[3], void* stream) {                \
        if (!fine || !coarse || !nc) return PRC_ERR_ARG;                                                             \
        Dims d = {{nc[0], nc[1], nc[2]}};                                                                            \
        PRC_LAUNCH("mg_prolong", (cudaStream_t)stream,                                                               \
                   prolong_kernel<T, T, T, false><<<grid3(nc).grid, grid3(nc).block, 0, (cudaStream_t)stream>>>(coarse, fine, d)); \
        PRC_CHECK_LAUNCH();                                                                                          \
        return PRC_OK;                                                                                               \
    }

MG_COMPONENTS(f32, float)
MG_COMPONENTS(f64, double)

}  // extern "C"

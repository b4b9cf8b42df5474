/*
 * TEST INFRASTRUCTURE ONLY -- not part of the product.
 *
 * CPU oracle: a plain-C restatement of pyrecon's full-multigrid solver of
 * the RSD-modified Poisson equation (reference src/multigrid.c), used by the
 * test-suite and by bench.py's CPU-baseline leg as the checker for the CUDA
 * multigrid.  The product (pyrecon_b200) never links or calls this file.
 *
 * Compiled as real_t = float (-DORACLE_F32) and real_t = double, like the
 * reference's multigrid_float.so / multigrid_double.so.
 *
 * The discrete operator, for cell c with p = (i + offset/h) (local line of
 * sight) or p = los/h (global line of sight), g = beta / (h^2 |p|^2) and
 * G_a = 1/h_a^2 + g p_a^2, is
 *   (A v)_c = 2 (G_x + G_y + G_z) v_c - S(v)_c
 *   S(v)_c  = sum_a G_a (v_{c+a} + v_{c-a})
 *           + g/2 sum_{a<b} p_a p_b (v_{c+a+b} + v_{c-a-b} - v_{c-a+b} - v_{c+a-b})
 *           + [local only] g sum_a p_a (v_{c+a} - v_{c-a})
 * (src/multigrid.c:63-103 for Jacobi, :107-164 for the residual).
 */
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef ORACLE_F32
typedef float real_t;
#else
typedef double real_t;
#endif

typedef struct {
    int64_t n[3];
    real_t h2[3];      /* cell size squared per axis */
    real_t ih2[3];     /* 1 / cell size squared */
    real_t off[3];     /* (boxcenter - boxsize/2) / cell, local line of sight */
    real_t losh[3];    /* los / cell, global line of sight */
    int local;         /* 1 when the line of sight varies per cell */
    real_t beta;
} level_t;

static level_t make_level(const int64_t *n, const real_t *boxsize, const real_t *boxcenter,
                          real_t beta, const real_t *los)
{
    level_t L;
    L.local = (los == NULL);
    L.beta = beta;
    for (int d = 0; d < 3; d++) {
        L.n[d] = n[d];
        real_t h = boxsize[d] / (real_t)n[d];
        L.h2[d] = h * h;
        L.ih2[d] = (real_t)(1. / L.h2[d]);
        L.off[d] = (real_t)((boxcenter[d] - boxsize[d] / 2.) / h);
        L.losh[d] = L.local ? 0 : los[d] / h;
    }
    return L;
}

static inline size_t idx3(const level_t *L, size_t x, size_t y, size_t z)
{
    return (x * (size_t)L->n[1] + y) * (size_t)L->n[2] + z;
}

static inline size_t up(size_t i, int64_t n) { return (i + 1) % (size_t)n; }
static inline size_t dn(size_t i, int64_t n) { return (i + (size_t)n - 1) % (size_t)n; }

/* Coefficients of the operator at cell (x, y, z): p, g, G (see header). */
static inline void coeffs(const level_t *L, size_t x, size_t y, size_t z,
                          real_t p[3], real_t *g, real_t G[3])
{
    if (L->local) {
        p[0] = (real_t)x + L->off[0];
        p[1] = (real_t)y + L->off[1];
        p[2] = (real_t)z + L->off[2];
    } else {
        p[0] = L->losh[0]; p[1] = L->losh[1]; p[2] = L->losh[2];
    }
    *g = L->beta / (L->h2[0] * p[0] * p[0] + L->h2[1] * p[1] * p[1] + L->h2[2] * p[2] * p[2]);
    for (int d = 0; d < 3; d++) G[d] = L->ih2[d] + *g * p[d] * p[d];
}

/* The four groups of neighbour terms of S(v) at one cell, returned separately
 * so Jacobi and the residual can add them in the reference's order. */
typedef struct { real_t face, mixed, deriv; } terms_t;

static terms_t stencil(const level_t *L, const real_t *v, size_t x, size_t y, size_t z,
                       const real_t p[3], real_t g, const real_t G[3])
{
    size_t xp = up(x, L->n[0]), xm = dn(x, L->n[0]);
    size_t yp = up(y, L->n[1]), ym = dn(y, L->n[1]);
    size_t zp = up(z, L->n[2]), zm = dn(z, L->n[2]);
#define V(a, b, c) v[idx3(L, a, b, c)]
    terms_t t;
    t.face = G[0] * (V(xp, y, z) + V(xm, y, z))
           + G[1] * (V(x, yp, z) + V(x, ym, z))
           + G[2] * (V(x, y, zp) + V(x, y, zm));
    t.mixed = g / 2 * (p[0] * p[1] * (V(xp, yp, z) + V(xm, ym, z) - V(xm, yp, z) - V(xp, ym, z))
                     + p[0] * p[2] * (V(xp, y, zp) + V(xm, y, zm) - V(xm, y, zp) - V(xp, y, zm))
                     + p[1] * p[2] * (V(x, yp, zp) + V(x, ym, zm) - V(x, ym, zp) - V(x, yp, zm)));
    t.deriv = 0;
    if (L->local)
        t.deriv = g * (p[0] * (V(xp, y, z) - V(xm, y, z))
                     + p[1] * (V(x, yp, z) - V(x, ym, z))
                     + p[2] * (V(x, y, zp) - V(x, y, zm)));
#undef V
    return t;
}

/* niter damped-Jacobi sweeps: v <- (1-w) v + w (f + S(v)) / (2 sum G).
 * Follows src/multigrid.c:44-104. */
static void jacobi(const level_t *L, real_t *v, const real_t *f, real_t w, int niter)
{
    size_t size = (size_t)(L->n[0] * L->n[1] * L->n[2]);
    real_t *jac = (real_t *)malloc(size * sizeof(real_t));
    for (int it = 0; it < niter; it++) {
        for (size_t x = 0; x < (size_t)L->n[0]; x++)
            for (size_t y = 0; y < (size_t)L->n[1]; y++)
                for (size_t z = 0; z < (size_t)L->n[2]; z++) {
                    real_t p[3], g, G[3];
                    coeffs(L, x, y, z, p, &g, G);
                    terms_t t = stencil(L, v, x, y, z, p, g, G);
                    size_t i = idx3(L, x, y, z);
                    real_t j = f[i] + t.face + t.mixed;
                    if (L->local) j += t.deriv;
                    jac[i] = j / (2 * (G[0] + G[1] + G[2]));
                }
        for (size_t i = 0; i < size; i++) v[i] = (1 - w) * v[i] + w * jac[i];
    }
    free(jac);
}

/* r = f - A v.  Follows src/multigrid.c:107-164. */
static void residual(const level_t *L, const real_t *v, const real_t *f, real_t *r)
{
    for (size_t x = 0; x < (size_t)L->n[0]; x++)
        for (size_t y = 0; y < (size_t)L->n[1]; y++)
            for (size_t z = 0; z < (size_t)L->n[2]; z++) {
                real_t p[3], g, G[3];
                coeffs(L, x, y, z, p, &g, G);
                terms_t t = stencil(L, v, x, y, z, p, g, G);
                size_t i = idx3(L, x, y, z);
                real_t a = 2 * (G[0] + G[1] + G[2]) * v[i] - (t.face + t.mixed);
                if (L->local) a -= t.deriv;
                r[i] = f[i] - a;
            }
}

/* Coarse (n/2) to fine (n) trilinear prolongation, overwriting fine.
 * Follows src/multigrid.c:167-209: fine node 2c + e (e in {0,1}^3) is the
 * mean of the coarse nodes c + e' over the e' <= e (componentwise). */
static void prolong(const level_t *Lc, const real_t *coarse, real_t *fine)
{
    int64_t nf[3] = {2 * Lc->n[0], 2 * Lc->n[1], 2 * Lc->n[2]};
    for (size_t x = 0; x < (size_t)Lc->n[0]; x++)
        for (size_t y = 0; y < (size_t)Lc->n[1]; y++)
            for (size_t z = 0; z < (size_t)Lc->n[2]; z++) {
                size_t cx[2] = {x, up(x, Lc->n[0])}, cy[2] = {y, up(y, Lc->n[1])}, cz[2] = {z, up(z, Lc->n[2])};
                for (int e = 0; e < 8; e++) {
                    int ex = (e >> 2) & 1, ey = (e >> 1) & 1, ez = e & 1;
                    real_t s = 0;
                    int cnt = 0;
                    for (int a = 0; a <= ex; a++)
                        for (int b = 0; b <= ey; b++)
                            for (int c = 0; c <= ez; c++) {
                                s += coarse[idx3(Lc, cx[a], cy[b], cz[c])];
                                cnt++;
                            }
                    size_t fi = ((2 * x + ex) * (size_t)nf[1] + (2 * y + ey)) * (size_t)nf[2] + (2 * z + ez);
                    fine[fi] = s / cnt;
                }
            }
}

/* Fine (n) to coarse (n/2) full-weighting restriction (27-point, weights
 * 8/4/2/1 for centre/face/edge/corner, divided by 64).
 * Follows src/multigrid.c:212-266. */
static void reduce(const level_t *Lf, const real_t *fine, real_t *coarse)
{
    int64_t nc[3] = {Lf->n[0] / 2, Lf->n[1] / 2, Lf->n[2] / 2};
    for (size_t x = 0; x < (size_t)nc[0]; x++)
        for (size_t y = 0; y < (size_t)nc[1]; y++)
            for (size_t z = 0; z < (size_t)nc[2]; z++) {
                size_t X[3] = {dn(2 * x, Lf->n[0]), 2 * x, up(2 * x, Lf->n[0])};
                size_t Y[3] = {dn(2 * y, Lf->n[1]), 2 * y, up(2 * y, Lf->n[1])};
                size_t Z[3] = {dn(2 * z, Lf->n[2]), 2 * z, up(2 * z, Lf->n[2])};
                real_t s = 0;
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++)
                        for (int c = 0; c < 3; c++) {
                            int nside = (a != 1) + (b != 1) + (c != 1);
                            real_t wgt = (real_t)(8 >> nside);
                            s += wgt * fine[idx3(Lf, X[a], Y[b], Z[c])];
                        }
                coarse[(x * (size_t)nc[1] + y) * (size_t)nc[2] + z] = s / (real_t)64.0;
            }
}

static int coarsenable(const int64_t *n)
{
    for (int d = 0; d < 3; d++)
        if (!(n[d] > 4 && n[d] % 2 == 0)) return 0;
    return 1;
}

typedef struct {
    const real_t *boxsize, *boxcenter, *los;
    real_t beta, w;
    int jn;
} params_t;

/* One recursive V-cycle.  Follows src/multigrid.c:270-300. */
static void vcycle(const params_t *P, const int64_t *n, real_t *v, const real_t *f)
{
    level_t L = make_level(n, P->boxsize, P->boxcenter, P->beta, P->los);
    jacobi(&L, v, f, P->w, P->jn);
    if (coarsenable(n)) {
        int64_t nc[3] = {n[0] / 2, n[1] / 2, n[2] / 2};
        size_t size = (size_t)(n[0] * n[1] * n[2]), sizec = size / 8;
        real_t *r = (real_t *)malloc(size * sizeof(real_t));
        residual(&L, v, f, r);
        real_t *fc = (real_t *)malloc(sizec * sizeof(real_t));
        reduce(&L, r, fc);
        free(r);
        real_t *vc = (real_t *)calloc(sizec, sizeof(real_t));
        vcycle(P, nc, vc, fc);
        free(fc);
        level_t Lc = make_level(nc, P->boxsize, P->boxcenter, P->beta, P->los);
        real_t *corr = (real_t *)malloc(size * sizeof(real_t));
        prolong(&Lc, vc, corr);
        free(vc);
        for (size_t i = 0; i < size; i++) v[i] += corr[i];
        free(corr);
    }
    jacobi(&L, v, f, P->w, P->jn);
}

/* Full multigrid; v (length n0*n1*n2) must be zero on entry.
 * Follows src/multigrid.c:303-328: restrict f to the coarsest level (while
 * every n > 4 and even), then on the way up prolong the coarse solution as
 * the initial guess and run vn V-cycles at each level. */
static void fmg_level(const params_t *P, const int64_t *n, const real_t *f, real_t *v, int vn)
{
    if (coarsenable(n)) {
        int64_t nc[3] = {n[0] / 2, n[1] / 2, n[2] / 2};
        size_t sizec = (size_t)(nc[0] * nc[1] * nc[2]);
        level_t L = make_level(n, P->boxsize, P->boxcenter, P->beta, P->los);
        real_t *fc = (real_t *)malloc(sizec * sizeof(real_t));
        reduce(&L, f, fc);
        real_t *vc = (real_t *)calloc(sizec, sizeof(real_t));
        fmg_level(P, nc, fc, vc, vn);
        free(fc);
        level_t Lc = make_level(nc, P->boxsize, P->boxcenter, P->beta, P->los);
        prolong(&Lc, vc, v);
        free(vc);
    }
    for (int it = 0; it < vn; it++) vcycle(P, n, v, f);
}

int oracle_fmg(const real_t *f, real_t *v, const int64_t *n, const real_t *boxsize,
               const real_t *boxcenter, real_t beta, real_t damping, int jacobi_niter,
               int vcycle_niter, const real_t *los)
{
    params_t P = {boxsize, boxcenter, los, beta, damping, jacobi_niter};
    fmg_level(&P, n, f, v, vcycle_niter);
    return 0;
}

/* Single components, exported so tests can pin the CUDA kernels one by one. */
int oracle_mg_jacobi(real_t *v, const real_t *f, const int64_t *n, const real_t *boxsize,
                     const real_t *boxcenter, real_t beta, real_t damping, int niter,
                     const real_t *los)
{
    level_t L = make_level(n, boxsize, boxcenter, beta, los);
    jacobi(&L, v, f, damping, niter);
    return 0;
}

int oracle_mg_residual(const real_t *v, const real_t *f, real_t *r, const int64_t *n,
                       const real_t *boxsize, const real_t *boxcenter, real_t beta,
                       const real_t *los)
{
    level_t L = make_level(n, boxsize, boxcenter, beta, los);
    residual(&L, v, f, r);
    return 0;
}

int oracle_mg_reduce(const real_t *fine, real_t *coarse, const int64_t *n)
{
    level_t L;
    memset(&L, 0, sizeof(L));
    for (int d = 0; d < 3; d++) L.n[d] = n[d];
    reduce(&L, fine, coarse);
    return 0;
}

int oracle_mg_prolong(const real_t *coarse, real_t *fine, const int64_t *ncoarse)
{
    level_t L;
    memset(&L, 0, sizeof(L));
    for (int d = 0; d < 3; d++) L.n[d] = ncoarse[d];
    prolong(&L, coarse, fine);
    return 0;
}

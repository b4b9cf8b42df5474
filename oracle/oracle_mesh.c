/*
 * TEST INFRASTRUCTURE ONLY -- not part of the product.
 *
 * CPU oracle: a plain-C restatement of pyrecon's mesh kernels, used by the
 * test-suite, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg
 * as the checker for the CUDA path.  The product (pyrecon_b200) never links
 * or calls this file.
 *
 * Compiled twice by oracle/Makefile: with -DORACLE_F32 (real_t = float) and
 * without (real_t = double), mirroring the reference's mesh_float.so /
 * mesh_double.so pair (reference src/Makefile:11-15, src/utils.h:8-18).
 *
 * Every routine takes positions already mapped to index space, i.e.
 * ((p - boxcenter) / boxsize + 0.5) * nmesh cast to real_t, exactly as the
 * reference's Python layer hands them to C (pyrecon/mesh.py:554-555).
 */
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <math.h>

#ifdef ORACLE_F32
typedef float real_t;
#else
typedef double real_t;
#endif

/* Flat C-order offset of (ix, iy, iz) in a mesh of shape n[0] x n[1] x n[2]. */
static inline size_t flat(const int64_t *n, size_t ix, size_t iy, size_t iz)
{
    return (ix * (size_t)n[1] + iy) * (size_t)n[2] + iz;
}

/* Base cell of one coordinate: truncation toward zero, then modulo the mesh
 * size (reference src/mesh.c:35-37 and :278-283 use the same int cast). */
static inline size_t base_cell(real_t p, int64_t n)
{
    return (size_t)((int)p) % (size_t)n;
}

/*
 * CIC scatter, sequential over particles in input order.
 * Follows src/mesh.c:26-63 (assign_cic): the fractional offset is taken
 * AFTER the modulo (dx = p - (i mod n)), so a coordinate exactly equal to n
 * lands in cell 0 with dx = n; the 8 corner weights are the products
 * w_x * w_y * w_z * weight, accumulated with += in real_t.
 */
int oracle_assign_cic(real_t *mesh, const int64_t *n, const real_t *pos,
                      const real_t *weights, int64_t npos)
{
    for (int64_t ip = 0; ip < npos; ip++) {
        const real_t *p = pos + 3 * ip;
        size_t lo[3], hi[3];
        real_t fr[3][2];
        for (int d = 0; d < 3; d++) {
            lo[d] = base_cell(p[d], n[d]);
            hi[d] = (lo[d] + 1) % (size_t)n[d];
            real_t t = p[d] - (real_t)lo[d];
            fr[d][0] = 1 - t;
            fr[d][1] = t;
        }
        /* Corner order (x, y, z) in {0,1}^3, z fastest, as mesh.c:55-62. */
        for (int c = 0; c < 8; c++) {
            int cx = (c >> 2) & 1, cy = (c >> 1) & 1, cz = c & 1;
            size_t ix = cx ? hi[0] : lo[0];
            size_t iy = cy ? hi[1] : lo[1];
            size_t iz = cz ? hi[2] : lo[2];
            mesh[flat(n, ix, iy, iz)] += fr[0][cx] * fr[1][cy] * fr[2][cz] * weights[ip];
        }
    }
    return 0;
}

/*
 * CIC gather of a scalar mesh at each position.
 * Follows src/mesh.c:269-310 (read_cic): the fractional offset is taken
 * BEFORE the modulo (dx = p - (int)p); the sum is accumulated over the 8
 * corners in (x, y, z) order with z fastest.
 */
int oracle_read_cic(const real_t *mesh, const int64_t *n, const real_t *pos,
                    real_t *out, int64_t npos)
{
    for (int64_t ip = 0; ip < npos; ip++) {
        const real_t *p = pos + 3 * ip;
        size_t lo[3], hi[3];
        real_t fr[3][2];
        for (int d = 0; d < 3; d++) {
            real_t t = p[d] - (real_t)((int)p[d]);
            lo[d] = base_cell(p[d], n[d]);
            hi[d] = (lo[d] + 1) % (size_t)n[d];
            fr[d][0] = 1 - t;
            fr[d][1] = t;
        }
        real_t acc = 0;
        for (int c = 0; c < 8; c++) {
            int cx = (c >> 2) & 1, cy = (c >> 1) & 1, cz = c & 1;
            size_t ix = cx ? hi[0] : lo[0];
            size_t iy = cy ? hi[1] : lo[1];
            size_t iz = cz ? hi[2] : lo[2];
            acc += mesh[flat(n, ix, iy, iz)] * fr[0][cx] * fr[1][cy] * fr[2][cz];
        }
        out[ip] = acc;
    }
    return 0;
}

/*
 * Central-difference gradient of a scalar mesh, CIC-interpolated at each
 * position, divided by 2 * boxsize / n per axis.
 * Follows src/mesh.c:187-266 (read_finite_difference_cic): fractional
 * offsets before the modulo; for each of the 8 corners c the gradient
 * along axis a is mesh[c + e_a] - mesh[c - e_a] (periodic), weighted by the
 * corner's CIC weight; corners visited in the reference's order
 * 000, 100, 010, 001, 110, 101, 011, 111 (x, y, z).
 */
int oracle_read_finite_difference_cic(const real_t *mesh, const int64_t *n,
                                      const real_t *boxsize, const real_t *pos,
                                      real_t *out, int64_t npos)
{
    static const int corner_order[8][3] = {
        {0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
        {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
    real_t twocell[3];
    for (int d = 0; d < 3; d++) twocell[d] = (real_t)(2.0 * boxsize[d] / (double)n[d]);
    for (int64_t ip = 0; ip < npos; ip++) {
        const real_t *p = pos + 3 * ip;
        size_t lo[3];
        real_t fr[3][2];
        for (int d = 0; d < 3; d++) {
            real_t t = p[d] - (real_t)((int)p[d]);
            lo[d] = base_cell(p[d], n[d]);
            fr[d][0] = 1 - t;
            fr[d][1] = t;
        }
        real_t grad[3] = {0, 0, 0};
        for (int k = 0; k < 8; k++) {
            size_t c[3];
            for (int d = 0; d < 3; d++) c[d] = (lo[d] + (size_t)corner_order[k][d]) % (size_t)n[d];
            real_t wt = fr[0][corner_order[k][0]] * fr[1][corner_order[k][1]] * fr[2][corner_order[k][2]];
            for (int a = 0; a < 3; a++) {
                size_t up[3] = {c[0], c[1], c[2]}, dn[3] = {c[0], c[1], c[2]};
                up[a] = (c[a] + 1) % (size_t)n[a];
                dn[a] = (c[a] + (size_t)n[a] - 1) % (size_t)n[a];
                grad[a] += (mesh[flat(n, up[0], up[1], up[2])] - mesh[flat(n, dn[0], dn[1], dn[2])]) * wt;
            }
        }
        for (int a = 0; a < 3; a++) out[3 * ip + a] = grad[a] / twocell[a];
    }
    return 0;
}

/*
 * mesh[ix, iy, iz] *= (ax[ix] + ay[iy] + az[iz]) ** exp on a real-valued
 * array of shape n (for a complex mesh the caller passes the interleaved
 * view with n[2] doubled and az repeated).
 * Follows src/mesh.c:327-365 (prod_sum); coords holds az, ay, ax in that
 * order, as the reference's Python layer concatenates them (mesh.py:724).
 */
int oracle_prod_sum(real_t *mesh, const int64_t *n, const real_t *coords, int exp)
{
    const real_t *az = coords, *ay = coords + n[2], *ax = coords + n[2] + n[1];
    for (int64_t ix = 0; ix < n[0]; ix++)
        for (int64_t iy = 0; iy < n[1]; iy++) {
            real_t sxy = ay[iy] + ax[ix];
            real_t *row = mesh + flat(n, (size_t)ix, (size_t)iy, 0);
            for (int64_t iz = 0; iz < n[2]; iz++) {
                real_t s = sxy + az[iz];
                if (exp == -1) row[iz] /= s;
                else if (exp == 1) row[iz] *= s;
#ifdef ORACLE_F32
                else row[iz] *= powf(s, (float)exp);
#else
                else row[iz] *= pow(s, (double)exp);
#endif
            }
        }
    return 0;
}

/*
 * Gaussian smoothing by brute-force periodic convolution, in place.
 * Follows src/mesh.c:117-143 (smooth_gaussian) and :66-115 (convolve):
 * half-width rad = (size_t)(nsigmas * radius * n + 1.0) cells per axis
 * (radius in box units; the product in real_t, the + 1.0 in double),
 * fact = 1 / (n radius)^2 rounded to real_t, tap exp(-r2 / 2) evaluated in
 * double where r2 = sum fact dx^2 < nsigmas^2 (else 0); every output is the
 * sum of tap * input over dx, dy, dz ascending, in real_t, divided by the sum
 * of all taps.  Neighbours wrap as ((i + d + n) mod 2^64) % n.  The taps are
 * stored in the order the convolution reads them.
 */
int oracle_smooth_gaussian(real_t *mesh, const int64_t *n, const real_t *radius, real_t nsigmas)
{
    int64_t rad[3], nk[3];
    real_t fact[3];
    for (int a = 0; a < 3; a++) {
        rad[a] = (int64_t)(size_t)((double)(nsigmas * radius[a] * (real_t)n[a]) + 1.0);
        nk[a] = 2 * rad[a] + 1;
        real_t nr = (real_t)n[a] * radius[a];
        fact[a] = (real_t)(1.0 / (double)nr / (double)nr);
    }
    size_t ntaps = (size_t)(nk[0] * nk[1] * nk[2]);
    real_t *taps = (real_t *)malloc(ntaps * sizeof(real_t));
    size_t size = (size_t)(n[0] * n[1] * n[2]);
    real_t *copy = (real_t *)malloc(size * sizeof(real_t));
    if (!taps || !copy) {
        free(taps);
        free(copy);
        return -1;
    }
    real_t total = 0;
    size_t it = 0;
    for (int64_t dx = -rad[0]; dx <= rad[0]; dx++)
        for (int64_t dy = -rad[1]; dy <= rad[1]; dy++)
            for (int64_t dz = -rad[2]; dz <= rad[2]; dz++) {
                real_t r2 = fact[0] * (real_t)dx * (real_t)dx + fact[1] * (real_t)dy * (real_t)dy
                            + fact[2] * (real_t)dz * (real_t)dz;
                real_t k = 0;
                if (r2 < nsigmas * nsigmas) k = (real_t)exp((double)(-r2 / (real_t)2));
                taps[it++] = k;
                total += k;
            }
    for (size_t i = 0; i < size; i++) copy[i] = mesh[i];
    for (int64_t ix = 0; ix < n[0]; ix++)
        for (int64_t iy = 0; iy < n[1]; iy++)
            for (int64_t iz = 0; iz < n[2]; iz++) {
                real_t acc = 0;
                size_t t = 0;
                for (int64_t dx = -rad[0]; dx <= rad[0]; dx++) {
                    size_t jx = (size_t)(ix + dx + n[0]) % (size_t)n[0];
                    for (int64_t dy = -rad[1]; dy <= rad[1]; dy++) {
                        size_t jy = (size_t)(iy + dy + n[1]) % (size_t)n[1];
                        for (int64_t dz = -rad[2]; dz <= rad[2]; dz++) {
                            size_t jz = (size_t)(iz + dz + n[2]) % (size_t)n[2];
                            real_t prod = taps[t++] * copy[flat(n, jx, jy, jz)];
                            acc += prod;
                        }
                    }
                }
                mesh[flat(n, (size_t)ix, (size_t)iy, (size_t)iz)] = acc / total;
            }
    free(taps);
    free(copy);
    return 0;
}

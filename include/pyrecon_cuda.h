/*
 * pyrecon_cuda.h -- C ABI of libpyrecon_cuda.so, the sm_100a (B200) implementation of
 * pyrecon's reconstruction hot path.
 *
 * Every entry point:
 *   - takes DEVICE pointers for meshes, particles and workspaces, and HOST pointers for the
 *     small 3-vectors (nmesh, boxsize, boxcenter, los, radius);
 *   - takes the CUDA stream as `void *stream` (a cudaStream_t; NULL = legacy default stream)
 *     and only enqueues work on it (no host synchronisation, no device allocation: scratch
 *     comes from the caller through `workspace`, sized by the matching *_workspace_bytes);
 *   - returns a prc_status_t; argument checks happen before anything is enqueued.
 * Conditions found while running (positions outside the box, NaN/inf) are OR-ed into the
 * caller's device word `flags` (PRC_FLAG_*); kernels downstream of a raised flag in the same
 * call skip their writes, so the output mesh is left untouched, as the reference leaves it
 * when it raises MeshError (pyrecon/mesh.py:549-553); a paint that does not accumulate
 * (accumulate = 0, the mesh's previous contents unused) writes zeros instead.
 *
 * Meshes are C-ordered (n0, n1, n2); half spectra are (n0, n1, n2/2+1) interleaved complex;
 * positions are (N, 3) row-major float32 or float64 (`pos_bytes` = 4 or 8).  `_f32` / `_f64`
 * suffixes select the mesh precision, as the reference's mesh_float.so / mesh_double.so and
 * multigrid_float.so / multigrid_double.so do (reference src/Makefile:11-21).
 */
#ifndef PYRECON_CUDA_H
#define PYRECON_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int prc_status_t;

#if defined(__GNUC__)
#define PRC_API __attribute__((visibility("default")))
#else
#define PRC_API
#endif

#define PRC_OK 0
#define PRC_ERR_ARG 1          /* invalid argument (null pointer, bad size, bad enum) */
#define PRC_ERR_WORKSPACE 2    /* workspace smaller than *_workspace_bytes */
#define PRC_ERR_CUDA 3         /* a kernel launch or CUDA runtime call failed */
#define PRC_ERR_UNSUPPORTED 4  /* mesh size this build does not handle (FFT radix / limits) */
#define PRC_ERR_TIMEOUT 5      /* a bounded device-side wait gave up */

#define PRC_FLAG_OUT_OF_BOX 1  /* a position outside [boxcenter - boxsize/2, boxcenter + boxsize/2] */
#define PRC_FLAG_NONFINITE 2   /* a NaN/inf position or weight */
#define PRC_FLAG_DEVICE_WAIT 4 /* a bounded wait between the CTAs of a kernel gave up (the paint's sort) */

#define PRC_FIELD_DISP 0       /* Zeldovich displacement only */
#define PRC_FIELD_RSD 1        /* RSD displacement f (s.l) l only */
#define PRC_FIELD_DISP_RSD 2   /* both */

/* Library version string. */
PRC_API const char *prc_version(void);

/* Human-readable name of a status code. */
PRC_API const char *prc_status_string(prc_status_t status);

/* Number of kernels this library has launched since it was loaded (all devices, all streams). */
PRC_API unsigned long long prc_launch_count(void);

/* Per-kernel device timing: enable(1) clears previous records and brackets every later launch
 * with CUDA events on its stream; enable(0) stops recording.  collect() waits for the recorded
 * events, writes {"kernel name": [launches, total ms, compulsory bytes], ...} (JSON,
 * NUL-terminated, truncated to cap) into buf, clears the records and returns the size the full
 * text needs.  Compulsory bytes = what each launch must read and write at least (its algorithmic
 * DRAM traffic), so bytes / ms is the achieved bandwidth against the HBM roofline. */
PRC_API void prc_profile_enable(int on);
PRC_API int prc_profile_collect(char *buf, size_t cap);

/* 1 if every axis of nmesh is handled by the FFT kernels, else 0: any length 2 <= n <= 2048 (the
 * reference's numpy / FFTW engines take any size, pyrecon/mesh.py:974-1118; a 2048^3 FP32 mesh is
 * 34 GB, so a reconstruction's meshes reach the device memory before this limit).  Powers of two up to
 * 1024 run the register-resident kernels, every other length (radices 2-8, any larger prime factor by
 * direct summation, an odd last axis as a full-length transform) the shared-memory kernels. */
PRC_API int prc_fft_supported(const int32_t nmesh[3]);

/* ------------------------------------------------------------------------------------------
 * Painting.  Replaces assign_cic (reference src/mesh.c:26-63) together with the index
 * transform, wrap and box / NaN checks of RealMesh.assign_cic (pyrecon/mesh.py:529-568).
 * Deterministic: particles are radix-sorted by base cell (stable), then each mesh column
 * sums its contributions in a fixed order in FP64.  `mesh` is an FP64 accumulator that
 * `accumulate` = 1 adds into (repeated assign_* calls), 0 overwrites.  `column_sums`
 * (n0*n1 doubles, may be NULL) receives the sum of every final mesh column (z axis).
 * `mesh_bytes` (4 or 8) is the reference mesh dtype that fixes the index-space precision;
 * `weights` may be NULL (unit weights), else `weight_bytes` = 4 or 8.
 * ------------------------------------------------------------------------------------------ */
PRC_API size_t prc_assign_cic_workspace_bytes(const int32_t nmesh[3], int64_t npos, int mesh_bytes);
PRC_API prc_status_t prc_assign_cic(double *mesh, double *column_sums, const int32_t nmesh[3],
                            const double boxsize[3], const double boxcenter[3], int mesh_bytes,
                            const void *positions, int pos_bytes, const void *weights,
                            int weight_bytes, int64_t npos, int wrap, int accumulate,
                            int32_t *flags, void *workspace, size_t workspace_bytes, void *stream);
/* prc_assign_cic that also writes `order` (npos uint32): the particles' indices sorted by base cell
 * (stable), the order in which the paint summed them; a read-out of the same positions given it
 * gathers in cell order (prc_read_shifts_*). */
PRC_API prc_status_t prc_assign_cic_order(double *mesh, double *column_sums, const int32_t nmesh[3],
                                  const double boxsize[3], const double boxcenter[3], int mesh_bytes,
                                  const void *positions, int pos_bytes, const void *weights,
                                  int weight_bytes, int64_t npos, int wrap, int accumulate,
                                  int32_t *flags, void *workspace, size_t workspace_bytes, void *stream,
                                  uint32_t *order);

/* prc_assign_cic_order that also writes the positions themselves in that order (sorted_positions:
 * npos x 3 of the positions' dtype, particle order[i] at row i), so that a read-out of the same positions
 * in cell order (prc_read_shifts_* with order and sorted_positions) streams them instead of gathering
 * through the permutation.  Extends assign_cic (src/mesh.c:26-63) the same way prc_assign_cic_order does. */
PRC_API prc_status_t prc_assign_cic_sorted(double *mesh, double *column_sums, const int32_t nmesh[3],
                                   const double boxsize[3], const double boxcenter[3], int mesh_bytes,
                                   const void *positions, int pos_bytes, const void *weights,
                                   int weight_bytes, int64_t npos, int wrap, int accumulate,
                                   int32_t *flags, void *workspace, size_t workspace_bytes, void *stream,
                                   uint32_t *order, void *sorted_positions);

/* Allocation-free variant of prc_assign_cic, with no counterpart in the reference.  For callers
 * that cannot allocate device memory (no allocator of their own, or code running where a
 * cudaMalloc is not allowed): it takes no workspace and calls no cudaMalloc / cudaFree; its
 * scratch is a 17 MiB array in the library's own device memory (held on every GPU that loads
 * the library until the process exits).  Same arguments, results and flags as prc_assign_cic
 * (equal to it to FP64 rounding), but particles are painted in chunks of 2^18, each accumulated
 * into the mesh.  Meshes with more than 2^20 (x, y) columns, or n2 > 4096, are rejected with
 * PRC_ERR_UNSUPPORTED.  The first call on a device (per driver context: each context holds its own
 * copy of the array) looks up the array's address (make it before any stream capture).  Every call
 * shares the array: calls that overlap on the GPU (other streams, other host threads) race and must
 * be serialised by the caller. */
PRC_API prc_status_t prc_assign_cic_noalloc(double *mesh, double *column_sums, const int32_t nmesh[3],
                                            const double boxsize[3], const double boxcenter[3], int mesh_bytes,
                                            const void *positions, int pos_bytes, const void *weights,
                                            int weight_bytes, int64_t npos, int wrap, int accumulate,
                                            int32_t *flags, void *stream);

/* Base-cell keys and the stable order that sorts them (the permutation the paint uses):
 * keys_sorted[i] = key[order[i]], key = (ix * n1 + iy) * n2 + iz.  Exposed so the sort can be
 * checked bit for bit against a stable argsort. Uses the paint workspace. */
PRC_API prc_status_t prc_cic_cell_order(uint32_t *keys_sorted, uint32_t *order, const int32_t nmesh[3],
                                const double boxsize[3], const double boxcenter[3], int mesh_bytes,
                                const void *positions, int pos_bytes, int64_t npos, int wrap,
                                int32_t *flags, void *workspace, size_t workspace_bytes, void *stream);

/* Deterministic FP64 sum of n doubles into *out (device).  Replaces np.sum of a mesh. */
PRC_API size_t prc_sum_workspace_bytes(int64_t n);
PRC_API prc_status_t prc_sum_f64(const double *x, int64_t n, double *out, void *workspace,
                         size_t workspace_bytes, void *stream);

/* ------------------------------------------------------------------------------------------
 * Gathers.  Output `out` has the positions' dtype (the reference casts back,
 * pyrecon/mesh.py:610,653).
 * ------------------------------------------------------------------------------------------ */
/* Replaces read_cic (reference src/mesh.c:269-310) + RealMesh.read_cic (mesh.py:570-610). */
PRC_API prc_status_t prc_read_cic_f32(const float *mesh, const int32_t nmesh[3], const double boxsize[3],
                              const double boxcenter[3], const void *positions, int pos_bytes,
                              int64_t npos, int wrap, void *out, int32_t *flags, void *stream);
PRC_API prc_status_t prc_read_cic_f64(const double *mesh, const int32_t nmesh[3], const double boxsize[3],
                              const double boxcenter[3], const void *positions, int pos_bytes,
                              int64_t npos, int wrap, void *out, int32_t *flags, void *stream);

/* Replaces read_finite_difference_cic (reference src/mesh.c:187-266) +
 * RealMesh.read_finite_difference_cic (mesh.py:612-653); out is (npos, 3). */
PRC_API prc_status_t prc_read_finite_difference_cic_f32(const float *mesh, const int32_t nmesh[3],
                                                const double boxsize[3], const double boxcenter[3],
                                                const void *positions, int pos_bytes, int64_t npos,
                                                int wrap, void *out, int32_t *flags, void *stream);
PRC_API prc_status_t prc_read_finite_difference_cic_f64(const double *mesh, const int32_t nmesh[3],
                                                const double boxsize[3], const double boxcenter[3],
                                                const void *positions, int pos_bytes, int64_t npos,
                                                int wrap, void *out, int32_t *flags, void *stream);

/* Fused shift read-out of the FFT algorithms: three CIC gathers of psi_x, psi_y, psi_z, the RSD
 * term f (s.l) l with l = los (global, unit 3-vector) or p/|p| of the wrapped positions (los =
 * NULL), field selection and, if `shifted`, positions - shifts wrapped when `wrap`.
 * Replaces BaseReconstruction.read_shifts / read_shifted_positions (pyrecon/recon.py:255-325).
 * psi_stride: 1 for three separate meshes, 4 for one interleaved (x, y, z, 0) mesh with
 * psi_y = psi_x + 1, psi_z = psi_x + 2 (one vector load per CIC corner).
 * out is (npos, 3) in `out_bytes` precision.  `order` (may be NULL) is a permutation of 0..npos-1
 * in which to visit the particles, e.g. the cell order prc_assign_cic_order returned when these
 * positions were painted: neighbouring threads then gather neighbouring cells.  Results do not
 * depend on it.  sorted_positions (optional, with order): the same positions in that order, as
 * prc_assign_cic_sorted wrote them; they are read from there (a stream) instead of positions[order[k]]. */
PRC_API prc_status_t prc_read_shifts_psi_f32(const float *psi_x, const float *psi_y, const float *psi_z, int psi_stride,
                                     const int32_t nmesh[3], const double boxsize[3],
                                     const double boxcenter[3], const void *positions, int pos_bytes,
                                     int64_t npos, const uint32_t *order, double f, const double *los, int field,
                                     int shifted, int wrap, void *out, int out_bytes, int32_t *flags, void *stream, const void *sorted_positions);
PRC_API prc_status_t prc_read_shifts_psi_f64(const double *psi_x, const double *psi_y, const double *psi_z,
                                     int psi_stride, const int32_t nmesh[3], const double boxsize[3],
                                     const double boxcenter[3], const void *positions, int pos_bytes,
                                     int64_t npos, const uint32_t *order, double f, const double *los, int field,
                                     int shifted, int wrap, void *out, int out_bytes, int32_t *flags, void *stream, const void *sorted_positions);

/* Same for the multigrid potential: finite-difference CIC gradient of phi, RSD direction from
 * the UNWRAPPED positions (pyrecon/multigrid.py:137-158). */
PRC_API prc_status_t prc_read_shifts_phi_f32(const float *phi, const int32_t nmesh[3], const double boxsize[3],
                                     const double boxcenter[3], const void *positions, int pos_bytes,
                                     int64_t npos, const uint32_t *order, double f, const double *los, int field,
                                     int shifted, int wrap, void *out, int out_bytes, int32_t *flags, void *stream, const void *sorted_positions);
PRC_API prc_status_t prc_read_shifts_phi_f64(const double *phi, const int32_t nmesh[3], const double boxsize[3],
                                     const double boxcenter[3], const void *positions, int pos_bytes,
                                     int64_t npos, const uint32_t *order, double f, const double *los, int field,
                                     int shifted, int wrap, void *out, int out_bytes, int32_t *flags, void *stream, const void *sorted_positions);

/* Sum of a float mesh accumulated in float64 (deterministic, as prc_sum_f64); replaces np.sum of the
 * smoothed meshes in IterativeFFTParticleReconstruction.set_density_contrast
 * (pyrecon/iterative_fft_particle.py:52). */
PRC_API prc_status_t prc_sum_f32(const float *x, int64_t n, double *out, void *workspace, size_t workspace_bytes,
                                 void *stream);

/* Density contrast of meshes that are already smoothed (IterativeFFTParticleReconstruction.set_density_contrast,
 * pyrecon/iterative_fft_particle.py:35-63): delta = (d - alpha r) / (b alpha r) where r > ran_min * sum(r) /
 * size_randoms (else 0), alpha = sum(d) / sum(r); without randoms (mesh_randoms NULL) delta = (d / mean(d) - 1) / b.
 * Inputs of `in_bytes` precision (8: the paint accumulators, 4: FP32 meshes); sums = device {sum d, sum r}. */
PRC_API prc_status_t prc_delta_from_meshes_f32(const void *mesh_data, const void *mesh_randoms, int in_bytes,
                                               const double *sums, const int32_t nmesh[3], double bias, double ran_min,
                                               double size_randoms, float *delta, void *stream);
PRC_API prc_status_t prc_delta_from_meshes_f64(const void *mesh_data, const void *mesh_randoms, int in_bytes,
                                               const double *sums, const int32_t nmesh[3], double bias, double ran_min,
                                               double size_randoms, double *delta, void *stream);

/* Zeldovich displacement of a density contrast, psi_a = IFFT(i k_a delta_k / k^2) with delta_k(0) = 0
 * (pyrecon/iterative_fft.py:71-82, pyrecon/iterative_fft_particle.py:93-108); psi_stride as for
 * prc_read_shifts_psi_*. */
PRC_API size_t prc_zeldovich_psi_workspace_bytes(const int32_t nmesh[3], int mesh_bytes);
PRC_API prc_status_t prc_zeldovich_psi_f32(const float *delta, const int32_t nmesh[3], const double boxsize[3],
                                           float *psi_x, float *psi_y, float *psi_z, int psi_stride, void *workspace,
                                           size_t workspace_bytes, void *stream);
PRC_API prc_status_t prc_zeldovich_psi_f64(const double *delta, const int32_t nmesh[3], const double boxsize[3],
                                           double *psi_x, double *psi_y, double *psi_z, int psi_stride,
                                           void *workspace, size_t workspace_bytes, void *stream);

/* One iteration's particle update of IterativeFFTParticleReconstruction (pyrecon/iterative_fft_particle.py:106-139):
 * s = CIC read of the interleaved (x, y, z, 0) displacement psi4 at the wrapped pos_rec; on the first iteration
 * s -= beta / (1 + beta) (s.l) l; then pos_rec = x - f (s.l) l, with x = pos_data (wrapped when wrap_data) and
 * l = los (global, unit 3-vector) or x / |x| (los = NULL).  Float64 arithmetic, stored in the positions dtype. */
PRC_API prc_status_t prc_ifftp_update_f32(const float *psi4, const int32_t nmesh[3], const double boxsize[3],
                                          const double boxcenter[3], const void *pos_data, void *pos_rec, int pos_bytes,
                                          int64_t npos, double f, double beta, int first, const double *los,
                                          int wrap_data, int32_t *flags, void *stream);
PRC_API prc_status_t prc_ifftp_update_f64(const double *psi4, const int32_t nmesh[3], const double boxsize[3],
                                          const double boxcenter[3], const void *pos_data, void *pos_rec, int pos_bytes,
                                          int64_t npos, double f, double beta, int first, const double *los,
                                          int wrap_data, int32_t *flags, void *stream);

/* Shift read-out of IterativeFFTParticleReconstruction (pyrecon/iterative_fft_particle.py:148-244).  With
 * pos_rec (the data, `positions` = the data positions): shifts at the reconstructed positions and
 * RSD = data - reconstructed.  Without: at positions p (wrapped when wrap), disp = psi(p),
 * rsd = f (disp.l) l, disp+rsd = psi(p - rsd, wrapped) + rsd.  `shifted`: positions - shifts, wrapped
 * when wrap.  out (npos, 3) in `out_bytes` precision.  `order` (may be NULL): the particles' indices in the
 * cell order of their paint (prc_assign_cic_order), the order the gathers visit them in (same results). */
PRC_API prc_status_t prc_ifftp_read_f32(const float *psi4, const int32_t nmesh[3], const double boxsize[3],
                                        const double boxcenter[3], const void *positions, const void *pos_rec,
                                        int pos_bytes, int64_t npos, double f, const double *los, int field,
                                        int shifted, int wrap, void *out, int out_bytes, int32_t *flags,
                                        const uint32_t *order, void *stream);
PRC_API prc_status_t prc_ifftp_read_f64(const double *psi4, const int32_t nmesh[3], const double boxsize[3],
                                        const double boxcenter[3], const void *positions, const void *pos_rec,
                                        int pos_bytes, int64_t npos, double f, const double *los, int field,
                                        int shifted, int wrap, void *out, int out_bytes, int32_t *flags,
                                        const uint32_t *order, void *stream);

/* Device fault word of the FFT kernels on the current device (no counterpart in the reference,
 * whose FFTs run on the host): PRC_FAULT_WAIT_TIMEOUT when a kernel gave up a bounded wait for its
 * own tile copies (its outputs are then incomplete), PRC_FAULT_SMEM_ALIGN when shared memory was
 * misaligned for the copy unit.  Synchronises with the device; reset != 0 clears the word. */
#define PRC_FAULT_WAIT_TIMEOUT 1u
#define PRC_FAULT_SMEM_ALIGN 2u
PRC_API unsigned int prc_device_fault_flags(int reset);

/* Run-time tuning table (no counterpart in the reference; its nearest relative is the FFTW wisdom of
 * pyrecon/mesh.py:1050-1081): integer knob `name` for key `key` (a mesh axis length), read by the
 * launchers at launch time; value < 0 removes an entry, prc_tune_clear removes all.  Knobs:
 *   "mg_jacobi" (FP32 sweeps), "mg_jacobi_f64" (FP64 sweeps), key = level n0: 0 = one damped-Jacobi
 *   sweep per pass, s > 0 = two sweeps per pass (temporal blocking), each block marching through slabs
 *   of s planes along x.
 * pyrecon_b200.tuning times the choices on the device and stores them as JSON wisdom. */
PRC_API int prc_tune_set(const char *name, int key, int value);
PRC_API int prc_tune_get(const char *name, int key, int dflt);
PRC_API void prc_tune_clear(void);

/* Test hook of the failure path (no counterpart in the reference): one CTA arms its transaction
 * barrier for bytes that no copy delivers (none is issued, so nothing is ever in flight), waits at
 * most limit_ns (0 < limit_ns <= 1 s) through the same bounded wait the FFT kernels use, sets
 * PRC_FAULT_WAIT_TIMEOUT in the fault word and returns; out (device int) = 1 when the wait gave up. */
PRC_API int prc_debug_wait_timeout(int64_t limit_ns, int* out, void* stream);

/* ------------------------------------------------------------------------------------------
 * FFTs and the k-space steps (the numpy / pyfftw sites of pyrecon/mesh.py:974-1118 and the
 * algorithm modules).  Forward transforms are unnormalised; inverse ones divide by n0*n1*n2,
 * as numpy's fftn / ifftn.  Spectra are the r2c half; multipliers are applied in their
 * Hermitian-symmetrised form so results equal the reference's c2c transform followed by .real.
 * ------------------------------------------------------------------------------------------ */
/* Workspace of `nspectra` half spectra as the composite entry points below lay them out inside
 * their workspace (rows padded to a multiple of 32 bytes). */
PRC_API size_t prc_fft_workspace_bytes(const int32_t nmesh[3], int mesh_bytes, int nspectra);

/* Forward r2c: in is a real mesh of `in_bytes` (4 or 8) precision, out the half spectrum. */
PRC_API prc_status_t prc_rfft3d_f32(const void *in, int in_bytes, void *out, const int32_t nmesh[3], void *stream);
PRC_API prc_status_t prc_rfft3d_f64(const void *in, int in_bytes, void *out, const int32_t nmesh[3], void *stream);
/* Inverse c2r of a half spectrum (overwritten) into a real mesh. */
PRC_API prc_status_t prc_irfft3d_f32(void *in, float *out, const int32_t nmesh[3], void *stream);
PRC_API prc_status_t prc_irfft3d_f64(void *in, double *out, const int32_t nmesh[3], void *stream);

/* Gaussian smoothing exp(-1/2 sum (r_a k_a)^2) of a real mesh (in: `in_bytes` precision,
 * may equal out).  Replaces RealMesh.smooth_gaussian(method='fft') (mesh.py:655-680). */
PRC_API prc_status_t prc_smooth_gaussian_f32(const void *in, int in_bytes, float *out, const int32_t nmesh[3],
                                     const double boxsize[3], const double radius[3], void *workspace,
                                     size_t workspace_bytes, void *stream);
PRC_API prc_status_t prc_smooth_gaussian_f64(const void *in, int in_bytes, double *out, const int32_t nmesh[3],
                                     const double boxsize[3], const double radius[3], void *workspace,
                                     size_t workspace_bytes, void *stream);

/* Gaussian smoothing in real space: periodic convolution with exp(-r^2 / 2) truncated at r < nsigmas,
 * normalised by the sum of its taps.  Replaces RealMesh.smooth_gaussian(method='real')
 * (pyrecon/mesh.py:684-695) and the reference C smooth_gaussian / convolve (src/mesh.c:66-143), whose
 * arguments it keeps: `radius` in units of the box side per axis (the reference's radius / boxsize,
 * rounded to the mesh precision), `nsigmas` (rounded likewise).  Outputs equal the reference's bit for
 * bit.  Out of place (in != out).  The taps are built on the host and copied into the workspace
 * (from pageable memory: not for stream capture).  PRC_ERR_UNSUPPORTED when a half-width
 * nsigmas * radius * nmesh exceeds 2047 cells.  The reference's kernel array is only fully written
 * when its x and z widths agree; elsewhere this uses the layout its convolution reads. */
PRC_API size_t prc_smooth_gaussian_real_workspace_bytes(const int32_t nmesh[3], const double radius[3], double nsigmas,
                                                        int mesh_bytes);
PRC_API prc_status_t prc_smooth_gaussian_real_f32(const float *in, float *out, const int32_t nmesh[3],
                                                  const double radius[3], double nsigmas, void *workspace,
                                                  size_t workspace_bytes, void *stream);
PRC_API prc_status_t prc_smooth_gaussian_real_f64(const double *in, double *out, const int32_t nmesh[3],
                                                  const double radius[3], double nsigmas, void *workspace,
                                                  size_t workspace_bytes, void *stream);

/* Martin's density contrast of OriginalMultiGridReconstruction.set_density_contrast
 * (pyrecon/multigrid.py:49-97), before its smoothing, from the FP64 data and randoms paint meshes
 * (randoms may be NULL): data set to 0 where 0 < randoms < ran_min, alpha = sum(data) / sum of
 * randoms >= ran_min, delta = (data / (alpha randoms) - 1) / bias where randoms >= ran_min, else 0,
 * then the mean of the non-zero delta removed from them.  Without randoms delta = (data / mean - 1) /
 * bias.  The caller smooths delta afterwards (prc_smooth_gaussian_* or prc_smooth_gaussian_real_*). */
PRC_API size_t prc_density_contrast_original_workspace_bytes(void);
PRC_API prc_status_t prc_density_contrast_original_f32(const double *mesh_data, const double *mesh_randoms,
                                                       const int32_t nmesh[3], double bias, double ran_min,
                                                       float *delta, void *workspace, size_t workspace_bytes,
                                                       void *stream);
PRC_API prc_status_t prc_density_contrast_original_f64(const double *mesh_data, const double *mesh_randoms,
                                                       const int32_t nmesh[3], double bias, double ran_min,
                                                       double *delta, void *workspace, size_t workspace_bytes,
                                                       void *stream);

/* set_density_contrast of BaseReconstruction (pyrecon/recon.py:198-249): smooths the FP64 data
 * (and randoms, may be NULL) meshes, then delta = (d - alpha r) / (bias alpha r) where
 * r > ran_min * sum_r / size_randoms, else 0 (no randoms: d / mean(d) - 1, / bias).
 * `sums` is a device pointer to {sum of data mesh, sum of randoms mesh} (FP64, e.g. from
 * prc_sum_f64 on the paint's column sums); smoothing conserves the sum, so alpha = sums[0] /
 * sums[1]. */
PRC_API size_t prc_density_contrast_workspace_bytes(const int32_t nmesh[3], int mesh_bytes, int with_randoms);
PRC_API prc_status_t prc_density_contrast_f32(const double *mesh_data, const double *mesh_randoms,
                                      const double *sums, const int32_t nmesh[3], const double boxsize[3],
                                      const double radius[3], double bias, double ran_min,
                                      double size_randoms, float *delta, void *workspace,
                                      size_t workspace_bytes, void *stream);
PRC_API prc_status_t prc_density_contrast_f64(const double *mesh_data, const double *mesh_randoms,
                                      const double *sums, const int32_t nmesh[3], const double boxsize[3],
                                      const double radius[3], double bias, double ran_min,
                                      double size_randoms, double *delta, void *workspace,
                                      size_t workspace_bytes, void *stream);

/* PlaneParallelFFTReconstruction.run (pyrecon/plane_parallel_fft.py:41-55):
 * psi_a = IFFT(i k_a delta_k / (k^2 (1 + beta mu^2))), los a unit 3-vector.
 * psi_stride (here and in prc_iterative_fft_*): 1 writes three separate meshes, 4 writes one
 * interleaved (x, y, z, 0) mesh at psi_x (psi_y = psi_x + 1, psi_z = psi_x + 2, 16/32-byte aligned). */
PRC_API size_t prc_plane_parallel_workspace_bytes(const int32_t nmesh[3], int mesh_bytes);
PRC_API prc_status_t prc_plane_parallel_fft_f32(const float *delta, const int32_t nmesh[3], const double boxsize[3],
                                        double beta, const double los[3], float *psi_x, float *psi_y,
                                        float *psi_z, int psi_stride, void *workspace, size_t workspace_bytes,
                                        void *stream);
PRC_API prc_status_t prc_plane_parallel_fft_f64(const double *delta, const int32_t nmesh[3], const double boxsize[3],
                                        double beta, const double los[3], double *psi_x, double *psi_y,
                                        double *psi_z, int psi_stride, void *workspace, size_t workspace_bytes,
                                        void *stream);

/* `count` PlaneParallelFFTReconstruction.run (pyrecon/plane_parallel_fft.py:41-55) of catalogues in the
 * same box with the same beta and line of sight: the meshes share the launches of each FFT pass, two at
 * a time (one launch over the tiles of both).  delta, psi_x, psi_y, psi_z are host arrays of `count`
 * device pointers (psi_stride as above); the workspace does not grow past two meshes' worth; results
 * equal `count` separate calls. */
PRC_API size_t prc_plane_parallel_batch_workspace_bytes(const int32_t nmesh[3], int mesh_bytes, int count);
PRC_API prc_status_t prc_plane_parallel_fft_batch_f32(const float *const *delta, float *const *psi_x,
                                              float *const *psi_y, float *const *psi_z, int count,
                                              const int32_t nmesh[3], const double boxsize[3], double beta,
                                              const double los[3], int psi_stride, void *workspace,
                                              size_t workspace_bytes, void *stream);
PRC_API prc_status_t prc_plane_parallel_fft_batch_f64(const double *const *delta, double *const *psi_x,
                                              double *const *psi_y, double *const *psi_z, int count,
                                              const int32_t nmesh[3], const double boxsize[3], double beta,
                                              const double los[3], int psi_stride, void *workspace,
                                              size_t workspace_bytes, void *stream);

/* IterativeFFTReconstruction.run (pyrecon/iterative_fft.py:12-82), niterations of the
 * Burden et al. 2015 field-level iteration then psi_a = IFFT(i k_a delta_k / k^2).
 * los = NULL selects the local line of sight. */
PRC_API size_t prc_iterative_fft_workspace_bytes(const int32_t nmesh[3], int mesh_bytes, int local_los);
PRC_API prc_status_t prc_iterative_fft_f32(const float *delta, const int32_t nmesh[3], const double boxsize[3],
                                   const double boxcenter[3], double beta, const double *los,
                                   int niterations, float *psi_x, float *psi_y, float *psi_z, int psi_stride,
                                   void *workspace, size_t workspace_bytes, void *stream);
PRC_API prc_status_t prc_iterative_fft_f64(const double *delta, const int32_t nmesh[3], const double boxsize[3],
                                   const double boxcenter[3], double beta, const double *los,
                                   int niterations, double *psi_x, double *psi_y, double *psi_z, int psi_stride,
                                   void *workspace, size_t workspace_bytes, void *stream);

/* Mirror of prod_sum (reference src/mesh.c:327-365): mesh *= (ax[i] + ay[j] + az[k])^exp on a
 * real array of `shape`, coords = concatenation az, ay, ax (exp = -1, 1 or any integer). */
PRC_API prc_status_t prc_prod_sum_f32(float *mesh, const int32_t shape[3], const float *coords, int exp, void *stream);
PRC_API prc_status_t prc_prod_sum_f64(double *mesh, const int32_t shape[3], const double *coords, int exp, void *stream);

/* ------------------------------------------------------------------------------------------
 * Multigrid.  Replaces fmg (reference src/multigrid.c:303-328) and its components.
 * los = NULL selects the local line of sight (19-point stencil with the first-derivative term).
 * _f32 with mixed_precision = 1: every V-cycle is computed as v += V(0, f - A v) with the
 * residual and v in FP64 and the V-cycle itself in FP32 (identical in exact arithmetic to the
 * reference's fixed FMG schedule); mixed_precision = 0 runs the whole schedule in FP32.
 * ------------------------------------------------------------------------------------------ */
PRC_API size_t prc_multigrid_workspace_bytes(const int32_t nmesh[3], int mesh_bytes, int mixed_precision);
PRC_API prc_status_t prc_multigrid_f32(const float *delta, float *phi, const int32_t nmesh[3], const double boxsize[3],
                               const double boxcenter[3], double beta, double damping, int jacobi_niterations,
                               int vcycle_niterations, const double *los, int mixed_precision, void *workspace,
                               size_t workspace_bytes, void *stream);
PRC_API prc_status_t prc_multigrid_f64(const double *delta, double *phi, const int32_t nmesh[3], const double boxsize[3],
                               const double boxcenter[3], double beta, double damping, int jacobi_niterations,
                               int vcycle_niterations, const double *los, void *workspace,
                               size_t workspace_bytes, void *stream);

/* `count` solves of the same mesh and parameters at once (several OriginalMultiGridReconstruction.run,
 * pyrecon/multigrid.py:99-135, of catalogues in the same box): every kernel of the schedule runs over
 * all of them in one launch (count * nmesh[0] <= 65535).  delta and phi are host arrays of `count`
 * device pointers; results equal `count` separate calls. */
PRC_API size_t prc_multigrid_batch_workspace_bytes(const int32_t nmesh[3], int mesh_bytes, int mixed_precision,
                                                   int count);
PRC_API prc_status_t prc_multigrid_batch_f32(const float *const *delta, float *const *phi, int count,
                                             const int32_t nmesh[3], const double boxsize[3],
                                             const double boxcenter[3], double beta, double damping,
                                             int jacobi_niterations, int vcycle_niterations, const double *los,
                                             int mixed_precision, void *workspace, size_t workspace_bytes,
                                             void *stream);
PRC_API prc_status_t prc_multigrid_batch_f64(const double *const *delta, double *const *phi, int count,
                                             const int32_t nmesh[3], const double boxsize[3],
                                             const double boxcenter[3], double beta, double damping,
                                             int jacobi_niterations, int vcycle_niterations, const double *los,
                                             void *workspace, size_t workspace_bytes, void *stream);

/* The mixed-precision FP32 solve (prc_multigrid_f32 / prc_multigrid_batch_f32 with mixed_precision = 1)
 * that also returns its FP64 iterate: phi (FP32, the mesh dtype) and phi64 (FP64; NULL entries, or a
 * NULL array, skip it).  The reference stores phi in the mesh dtype (pyrecon/multigrid.py:115-133), so
 * its FP32 finite-difference read-out inherits the FP32 rounding of phi (|phi| ~ 1e5 at 2000 Mpc/h and
 * nmesh 256: ~1e-3 Mpc/h on the shifts); reading shifts from phi64 (prc_read_shifts_phi_f64 with the
 * same positions) keeps the refinement's accuracy.  Same workspace as the mixed FP32 solve. */
PRC_API prc_status_t prc_multigrid_mixed_f32(const float *delta, float *phi, double *phi64, const int32_t nmesh[3],
                                             const double boxsize[3], const double boxcenter[3], double beta,
                                             double damping, int jacobi_niterations, int vcycle_niterations,
                                             const double *los, void *workspace, size_t workspace_bytes,
                                             void *stream);
PRC_API prc_status_t prc_multigrid_batch_mixed_f32(const float *const *delta, float *const *phi,
                                                   double *const *phi64, int count, const int32_t nmesh[3],
                                                   const double boxsize[3], const double boxcenter[3], double beta,
                                                   double damping, int jacobi_niterations, int vcycle_niterations,
                                                   const double *los, void *workspace, size_t workspace_bytes,
                                                   void *stream);

/* Components, one level (jacobi: src/multigrid.c:44-104, residual :107-164, prolong :167-209,
 * reduce :212-266).  jacobi runs `niterations` sweeps in place on v using `scratch` (one mesh). */
PRC_API prc_status_t prc_mg_jacobi_f32(float *v, const float *f, float *scratch, const int32_t nmesh[3],
                               const double boxsize[3], const double boxcenter[3], double beta, double damping,
                               int niterations, const double *los, void *stream);
PRC_API prc_status_t prc_mg_jacobi_f64(double *v, const double *f, double *scratch, const int32_t nmesh[3],
                               const double boxsize[3], const double boxcenter[3], double beta, double damping,
                               int niterations, const double *los, void *stream);
PRC_API prc_status_t prc_mg_residual_f32(const float *v, const float *f, float *r, const int32_t nmesh[3],
                                 const double boxsize[3], const double boxcenter[3], double beta,
                                 const double *los, void *stream);
PRC_API prc_status_t prc_mg_residual_f64(const double *v, const double *f, double *r, const int32_t nmesh[3],
                                 const double boxsize[3], const double boxcenter[3], double beta,
                                 const double *los, void *stream);
PRC_API prc_status_t prc_mg_reduce_f32(const float *fine, float *coarse, const int32_t nmesh_fine[3], void *stream);
PRC_API prc_status_t prc_mg_reduce_f64(const double *fine, double *coarse, const int32_t nmesh_fine[3], void *stream);
PRC_API prc_status_t prc_mg_prolong_f32(const float *coarse, float *fine, const int32_t nmesh_coarse[3], void *stream);
PRC_API prc_status_t prc_mg_prolong_f64(const double *coarse, double *fine, const int32_t nmesh_coarse[3], void *stream);

#ifdef __cplusplus
}
#endif

#endif /* PYRECON_CUDA_H */

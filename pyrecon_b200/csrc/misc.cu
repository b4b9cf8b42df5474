// Library metadata and the element-wise mesh kernels of the reference's C ABI.
#include "common.cuh"

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <vector>
#include <math.h>
#include <stdio.h>
#include <string.h>

namespace prc {

// ---------------------------------------------------------------------------------------------
// Launch counter and optional per-kernel event timing
// ---------------------------------------------------------------------------------------------
namespace {
std::atomic<unsigned long long> g_launches{0};
std::atomic<int> g_profiling{0};
struct TimedLaunch {
    const char* name;
    cudaEvent_t start, stop;
    double bytes;
};
std::mutex g_mutex;
std::vector<TimedLaunch> g_timed;
// Recycled timing events per device (creating an event per launch would add host time to every
// profiled launch).
std::map<int, std::vector<cudaEvent_t>> g_event_pool;

cudaEvent_t take_event() {
    int dev = 0;
    cudaGetDevice(&dev);
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        auto& pool = g_event_pool[dev];
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}

// Caller holds g_mutex.
void recycle_event(cudaEvent_t e) {
    int dev = 0;
    cudaGetDevice(&dev);
    g_event_pool[dev].push_back(e);
}
}  // namespace

void add_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

namespace {
thread_local unsigned long long t_capture_launches = 0;
thread_local double t_capture_bytes = 0.;
}  // namespace

void capture_tally(unsigned long long* launches, double* bytes) {
    if (launches) *launches = t_capture_launches;
    if (bytes) *bytes = t_capture_bytes;
    t_capture_launches = 0;
    t_capture_bytes = 0.;
}

KernelScope::KernelScope(const char* n, cudaStream_t s, double b, bool count)
    : name(n), st(s), start(nullptr), bytes(b) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
        // inside a capture: tallied for the graph, neither counted nor timed here
        t_capture_launches += 1;
        t_capture_bytes += b;
        return;
    }
    if (count) g_launches.fetch_add(1, std::memory_order_relaxed);
    if (g_profiling.load(std::memory_order_relaxed)) {
        start = take_event();
        if (start != nullptr) cudaEventRecord(start, st);
    }
}

KernelScope::~KernelScope() {
    if (start == nullptr) return;
    cudaEvent_t stop = take_event();
    if (stop == nullptr) {
        std::lock_guard<std::mutex> lock(g_mutex);
        recycle_event(start);
        return;
    }
    cudaEventRecord(stop, st);
    std::lock_guard<std::mutex> lock(g_mutex);
    g_timed.push_back({name, start, stop, bytes});
}

// mesh[ix, iy, iz] *= (ax[ix] + ay[iy] + az[iz])^exp, coords = az | ay | ax (src/mesh.c:327-365).
template <typename T>
__global__ void prod_sum_kernel(T* __restrict__ mesh, Dims d, const T* __restrict__ coords, int exp) {
    const int64_t N = d.size();
    const T* az = coords;
    const T* ay = coords + d.n[2];
    const T* ax = coords + d.n[2] + d.n[1];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int iz = (int)(i % d.n[2]);
        const int64_t r = i / d.n[2];
        const int iy = (int)(r % d.n[1]), ix = (int)(r / d.n[1]);
        const T s = (ay[iy] + ax[ix]) + az[iz];
        if (exp == -1) mesh[i] = mesh[i] / s;
        else if (exp == 1) mesh[i] = mesh[i] * s;
        else mesh[i] = mesh[i] * (T)pow((double)s, (double)exp);
    }
}

template <typename T> static int prod_sum(T* mesh, const int32_t shape[3], const T* coords, int exp, cudaStream_t st) {
    if (!mesh || !shape || !coords) return PRC_ERR_ARG;
    Dims d = {{shape[0], shape[1], shape[2]}};
    if (d.size() <= 0) return PRC_ERR_ARG;
    int64_t blocks = std::min<int64_t>((d.size() + 255) / 256, (int64_t)device_sm_count() * 16);
    PRC_LAUNCH("prod_sum", st, prod_sum_kernel<T><<<(int)blocks, 256, 0, st>>>(mesh, d, coords, exp));
    PRC_CHECK_LAUNCH();
    return PRC_OK;
}

static bool mesh_dims_ok(const int32_t nmesh[3]) {
    return nmesh && nmesh[0] > 0 && nmesh[1] > 0 && nmesh[2] > 0;
}

// ---------------------------------------------------------------------------------------------
// Real-space Gaussian smoothing: periodic brute-force convolution with a Gaussian truncated at
// nsigmas (RealMesh.smooth_gaussian(method='real'), pyrecon/mesh.py:684-695, src/mesh.c:66-143).
//
// The taps are built on the host as the reference builds its kernel: extents, factors and r^2 in
// the mesh precision, exp evaluated in double and rounded to the mesh precision, the normalisation
// summed tap by tap in the mesh precision.  Every output sums its taps in the reference's order
// (dx, then dy, then dz ascending) with round-to-nearest multiplies and adds and is divided by the
// normalisation, so outputs equal the reference's bit for bit.  Taps at or beyond nsigmas are 0 in
// the reference and left out here: adding 0 * v (finite v) to a sum that starts at +0 never changes
// it.  Neighbour indices wrap with the reference's unsigned arithmetic, ((i + d + n) mod 2^64) % n.
//
// Layout: the taps form rows of consecutive dz at fixed (dx, dy): int4 {dx, dy, first dz, count},
// in order, followed by the weights of all rows back to back.
// ---------------------------------------------------------------------------------------------
constexpr int SMOOTH_BZ = 32;      // output cells per block along z (one warp)
constexpr int SMOOTH_BY = 8;       // along y (warps per block)
constexpr int SMOOTH_QX = 4;       // along x (per thread)
constexpr int SMOOTH_MAX_RAD = 2048;

template <typename T> struct RealSmoothPlan {
    int rad[3];
    std::vector<int4> rows;
    std::vector<T> w;
    T sumw;
};

template <typename T>
static int real_smooth_plan(const int32_t nmesh[3], const double radius_in[3], double nsigmas_in, RealSmoothPlan<T>* p) {
    if (!mesh_dims_ok(nmesh) || !radius_in) return PRC_ERR_ARG;
    const T nsigmas = (T)nsigmas_in;
    T fact[3];
    for (int a = 0; a < 3; a++) {
        const T r = (T)radius_in[a];
        if (!(r > 0) || !(nsigmas > 0)) return PRC_ERR_ARG;
        // (size_t)(nsigmas * r * n + 1.0): product in the mesh precision, the + 1.0 in double
        const double ext = (double)(nsigmas * r * (T)nmesh[a]) + 1.0;
        if (!(ext < (double)SMOOTH_MAX_RAD + 1.)) return PRC_ERR_UNSUPPORTED;
        p->rad[a] = (int)(size_t)ext;
        const T nr = (T)nmesh[a] * r;
        fact[a] = (T)(1.0 / (double)nr / (double)nr);
    }
    const T cut = nsigmas * nsigmas;
    p->rows.clear();
    p->w.clear();
    T sumw = 0;
    for (int dx = -p->rad[0]; dx <= p->rad[0]; dx++) {
        for (int dy = -p->rad[1]; dy <= p->rad[1]; dy++) {
            int first = 0, count = 0;
            for (int dz = -p->rad[2]; dz <= p->rad[2] + 1; dz++) {
                bool in = false;
                T k = 0;
                if (dz <= p->rad[2]) {
                    const T r2 = fact[0] * dx * dx + fact[1] * dy * dy + fact[2] * dz * dz;
                    if (r2 < cut) {
                        const T e = -r2 / (T)2;
                        k = (T)::exp((double)e);
                        in = true;
                    }
                }
                if (in) {
                    if (count == 0) first = dz;
                    count++;
                    p->w.push_back(k);
                    sumw += k;
                } else if (count > 0) {
                    p->rows.push_back(make_int4(dx, dy, first, count));
                    count = 0;
                }
            }
        }
    }
    p->sumw = sumw;
    return PRC_OK;
}

template <typename T> static size_t real_smooth_bytes(const RealSmoothPlan<T>& p) {
    return ((p.rows.size() * sizeof(int4) + 255) / 256) * 256 + p.w.size() * sizeof(T);
}

// Reference neighbour index along one axis for i + d = s.
__device__ __forceinline__ int wrap_ref(int64_t s, int n) {
    return (int)((uint64_t)(s + (int64_t)n) % (uint64_t)n);
}

template <typename T>
__global__ void __launch_bounds__(SMOOTH_BZ * SMOOTH_BY) smooth_real_kernel(const T* __restrict__ in, T* __restrict__ out,
                                                                            Dims d, const int4* __restrict__ rows,
                                                                            int nrows, const T* __restrict__ w, int r0,
                                                                            int r1, int r2, T sumw) {
    extern __shared__ int tab[];
    const int z0 = blockIdx.x * SMOOTH_BZ, y0 = blockIdx.y * SMOOTH_BY, x0 = blockIdx.z * SMOOTH_QX;
    const int nx = SMOOTH_QX + 2 * r0, ny = SMOOTH_BY + 2 * r1, nz = SMOOTH_BZ + 2 * r2;
    int* tx = tab;
    int* ty = tx + nx;
    int* tz = ty + ny;
    for (int i = threadIdx.x; i < nx + ny + nz; i += blockDim.x) {
        if (i < nx) tx[i] = wrap_ref((int64_t)x0 - r0 + i, d.n[0]);
        else if (i < nx + ny) ty[i - nx] = wrap_ref((int64_t)y0 - r1 + (i - nx), d.n[1]);
        else tz[i - nx - ny] = wrap_ref((int64_t)z0 - r2 + (i - nx - ny), d.n[2]);
    }
    __syncthreads();
    const int zl = threadIdx.x % SMOOTH_BZ, yl = threadIdx.x / SMOOTH_BZ;
    const int z = z0 + zl, y = y0 + yl;
    if (z >= d.n[2] || y >= d.n[1]) return;
    const int64_t n12 = (int64_t)d.n[1] * d.n[2];
    T acc[SMOOTH_QX];
#pragma unroll
    for (int q = 0; q < SMOOTH_QX; q++) acc[q] = 0;
    int woff = 0;
    for (int r = 0; r < nrows; r++) {
        const int4 row = __ldg(rows + r);
        const int64_t yb = (int64_t)ty[yl + r1 + row.y] * d.n[2];
        const T* src[SMOOTH_QX];
#pragma unroll
        for (int q = 0; q < SMOOTH_QX; q++) src[q] = in + (int64_t)tx[q + r0 + row.x] * n12 + yb;
        const int* zi = tz + zl + r2 + row.z;
        const T* wr = w + woff;
        for (int j = 0; j < row.w; j++) {
            const T wt = __ldg(wr + j);
            const int iz = zi[j];
#pragma unroll
            for (int q = 0; q < SMOOTH_QX; q++) acc[q] = rn_add(acc[q], rn_mul(wt, __ldg(src[q] + iz)));
        }
        woff += row.w;
    }
#pragma unroll
    for (int q = 0; q < SMOOTH_QX; q++)
        if (x0 + q < d.n[0]) out[(int64_t)(x0 + q) * n12 + (int64_t)y * d.n[2] + z] = rn_div(acc[q], sumw);
}

template <typename T>
static int smooth_real(const T* in, T* out, const int32_t nmesh[3], const double radius[3], double nsigmas, void* ws,
                       size_t wsb, cudaStream_t st) {
    if (!in || !out || in == out) return PRC_ERR_ARG;
    RealSmoothPlan<T> p;
    PRC_TRY(real_smooth_plan<T>(nmesh, radius, nsigmas, &p));
    if (!ws || wsb < real_smooth_bytes(p)) return PRC_ERR_WORKSPACE;
    if (((uintptr_t)ws % 16) != 0) return PRC_ERR_ARG;
    const size_t row_bytes = ((p.rows.size() * sizeof(int4) + 255) / 256) * 256;
    int4* rows = (int4*)ws;
    T* w = (T*)((char*)ws + row_bytes);
    // from pageable host memory: the copy is staged before the call returns
    if (!p.rows.empty() &&
        cudaMemcpyAsync(rows, p.rows.data(), p.rows.size() * sizeof(int4), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return PRC_ERR_CUDA;
    if (!p.w.empty() && cudaMemcpyAsync(w, p.w.data(), p.w.size() * sizeof(T), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return PRC_ERR_CUDA;
    Dims d = {{nmesh[0], nmesh[1], nmesh[2]}};
    const dim3 grid((unsigned)ceil_div(d.n[2], SMOOTH_BZ), (unsigned)ceil_div(d.n[1], SMOOTH_BY),
                    (unsigned)ceil_div(d.n[0], SMOOTH_QX));
    if (grid.y > 65535 || grid.z > 65535) return PRC_ERR_UNSUPPORTED;
    const size_t smem = sizeof(int) * (SMOOTH_QX + SMOOTH_BY + SMOOTH_BZ + 2 * (p.rad[0] + p.rad[1] + p.rad[2]));
    if (smem > 48 * 1024) return PRC_ERR_UNSUPPORTED;
    PRC_LAUNCH_B("smooth_real", st, 2. * sizeof(T) * (double)d.size(),
                 smooth_real_kernel<T><<<grid, SMOOTH_BZ * SMOOTH_BY, smem, st>>>(
                     in, out, d, rows, (int)p.rows.size(), w, p.rad[0], p.rad[1], p.rad[2], p.sumw));
    PRC_CHECK_LAUNCH();
    return PRC_OK;
}

// ---------------------------------------------------------------------------------------------
// Martin's density contrast (OriginalMultiGridReconstruction.set_density_contrast,
// pyrecon/multigrid.py:49-97), before its smoothing, from the FP64 paint meshes d (data) and r
// (randoms):
//   d' = 0 where 0 < r < ran_min, else d;  mask = r >= ran_min;  alpha = sum d' / sum_{mask} r;
//   delta = mask ? (d / (alpha r) - 1) / bias : 0;  then delta -= mean of the non-zero delta
//   where delta != 0.
// Without randoms: delta = (d / mean(d) - 1) / bias.  Arithmetic in double, delta stored in the
// mesh precision (the mean of the non-zero cells is taken over the stored values).  The sums are
// deterministic: fixed grid, per-block tree, every block combining the partials in the same order.
// ---------------------------------------------------------------------------------------------
constexpr int MARTIN_BLOCKS = 512;
constexpr int MARTIN_THREADS = 256;

// Sum of the MARTIN_BLOCKS partials of one quantity, the same on every block.
__device__ __forceinline__ double martin_total(const double* __restrict__ partial, double* s) {
    double acc = 0.;
    for (int i = threadIdx.x; i < MARTIN_BLOCKS; i += MARTIN_THREADS) acc += partial[i];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = MARTIN_THREADS / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    const double t = s[0];
    __syncthreads();
    return t;
}

__device__ __forceinline__ void martin_block_sum(double a, double b, double* sa, double* sb, double* out_a,
                                                 double* out_b) {
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for (int o = MARTIN_THREADS / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sa[threadIdx.x] += sa[threadIdx.x + o];
            sb[threadIdx.x] += sb[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out_a[blockIdx.x] = sa[0];
        out_b[blockIdx.x] = sb[0];
    }
}

// partial[0:B] = sum d', partial[B:2B] = sum of r over the mask (0 without randoms).
__global__ void __launch_bounds__(MARTIN_THREADS) martin_sums(const double* __restrict__ d, const double* __restrict__ r,
                                                              int64_t n, double ran_min, double* __restrict__ partial) {
    __shared__ double sa[MARTIN_THREADS], sb[MARTIN_THREADS];
    double a = 0., b = 0.;
    for (int64_t i = (int64_t)blockIdx.x * MARTIN_THREADS + threadIdx.x; i < n; i += (int64_t)MARTIN_BLOCKS * MARTIN_THREADS) {
        const double dv = d[i];
        if (r) {
            const double rv = r[i];
            a += (rv > 0. && rv < ran_min) ? 0. : dv;
            if (rv >= ran_min) b += rv;
        } else {
            a += dv;
        }
    }
    martin_block_sum(a, b, sa, sb, partial, partial + MARTIN_BLOCKS);
}

// delta, and partial[2B:3B] = sum of the non-zero stored delta, partial[3B:4B] = their count.
template <typename T>
__global__ void __launch_bounds__(MARTIN_THREADS) martin_delta(const double* __restrict__ d, const double* __restrict__ r,
                                                               int64_t n, double bias, double ran_min,
                                                               double* __restrict__ partial, T* __restrict__ delta) {
    __shared__ double sa[MARTIN_THREADS], sb[MARTIN_THREADS];
    const double sd = martin_total(partial, sa);
    const double sr = r ? martin_total(partial + MARTIN_BLOCKS, sa) : 0.;
    const double alpha = r ? sd / sr : 0.;
    const double mean = sd / (double)n;
    double a = 0., c = 0.;
    for (int64_t i = (int64_t)blockIdx.x * MARTIN_THREADS + threadIdx.x; i < n; i += (int64_t)MARTIN_BLOCKS * MARTIN_THREADS) {
        const double dv = d[i];
        double o;
        if (r) {
            const double rv = r[i];
            o = rv >= ran_min ? (dv / (alpha * rv) - 1.) / bias : 0.;
        } else {
            o = (dv / mean - 1.) / bias;
        }
        const T v = (T)o;
        delta[i] = v;
        if (v != (T)0) {
            a += (double)v;
            c += 1.;
        }
    }
    martin_block_sum(a, c, sa, sb, partial + 2 * MARTIN_BLOCKS, partial + 3 * MARTIN_BLOCKS);
}

template <typename T>
__global__ void __launch_bounds__(MARTIN_THREADS) martin_center(const double* __restrict__ partial, int64_t n,
                                                                T* __restrict__ delta) {
    __shared__ double s[MARTIN_THREADS];
    const double sum = martin_total(partial + 2 * MARTIN_BLOCKS, s);
    const double count = martin_total(partial + 3 * MARTIN_BLOCKS, s);
    if (count == 0.) return;
    const double mean = sum / count;
    for (int64_t i = (int64_t)blockIdx.x * MARTIN_THREADS + threadIdx.x; i < n; i += (int64_t)MARTIN_BLOCKS * MARTIN_THREADS) {
        const T v = delta[i];
        if (v != (T)0) delta[i] = (T)((double)v - mean);
    }
}

template <typename T>
static int density_original(const double* d, const double* r, const int32_t nmesh[3], double bias, double ran_min,
                            T* delta, void* ws, size_t wsb, cudaStream_t st) {
    if (!d || !delta || !mesh_dims_ok(nmesh)) return PRC_ERR_ARG;
    if (!ws || wsb < 4 * MARTIN_BLOCKS * sizeof(double)) return PRC_ERR_WORKSPACE;
    const int64_t n = (int64_t)nmesh[0] * nmesh[1] * nmesh[2];
    double* partial = (double*)ws;
    const double in_bytes = 8. * (double)n * (r ? 2 : 1);
    PRC_LAUNCH_B("martin_sums", st, in_bytes,
                 martin_sums<<<MARTIN_BLOCKS, MARTIN_THREADS, 0, st>>>(d, r, n, ran_min, partial));
    PRC_LAUNCH_B("martin_delta", st, in_bytes + sizeof(T) * (double)n,
                 martin_delta<T><<<MARTIN_BLOCKS, MARTIN_THREADS, 0, st>>>(d, r, n, bias, ran_min, partial, delta));
    if (r)
        PRC_LAUNCH_B("martin_center", st, 2. * sizeof(T) * (double)n,
                     martin_center<T><<<MARTIN_BLOCKS, MARTIN_THREADS, 0, st>>>(partial, n, delta));
    PRC_CHECK_LAUNCH();
    return PRC_OK;
}

}  // namespace prc

extern "C" {

const char* prc_version(void) { return "pyrecon_b200 0.1.0 (sm_100a)"; }

const char* prc_status_string(prc_status_t status) {
    switch (status) {
        case PRC_OK: return "ok";
        case PRC_ERR_ARG: return "invalid argument";
        case PRC_ERR_WORKSPACE: return "workspace too small";
        case PRC_ERR_CUDA: return "CUDA launch or runtime error";
        case PRC_ERR_UNSUPPORTED: return "unsupported mesh size";
        case PRC_ERR_TIMEOUT: return "device wait timed out";
        default: return "unknown status";
    }
}

unsigned long long prc_launch_count(void) { return prc::g_launches.load(); }

void prc_profile_enable(int on) {
    std::lock_guard<std::mutex> lock(prc::g_mutex);
    for (auto& t : prc::g_timed) {
        cudaEventSynchronize(t.stop);
        prc::recycle_event(t.start);
        prc::recycle_event(t.stop);
    }
    prc::g_timed.clear();
    prc::g_profiling.store(on ? 1 : 0);
}

int prc_profile_collect(char* buf, size_t cap) {
    struct Agg { long long n = 0; double ms = 0., bytes = 0.; };
    std::map<std::string, Agg> agg;
    {
        std::lock_guard<std::mutex> lock(prc::g_mutex);
        for (auto& t : prc::g_timed) {
            float ms = 0.f;
            if (cudaEventSynchronize(t.stop) == cudaSuccess && cudaEventElapsedTime(&ms, t.start, t.stop) == cudaSuccess) {
                auto& a = agg[t.name];
                a.n += 1;
                a.ms += ms;
                a.bytes += t.bytes;
            }
            prc::recycle_event(t.start);
            prc::recycle_event(t.stop);
        }
        prc::g_timed.clear();
    }
    std::string out = "{";
    bool first = true;
    for (auto& kv : agg) {
        char item[256];
        snprintf(item, sizeof(item), "%s\"%s\": [%lld, %.6f, %.1f]", first ? "" : ", ", kv.first.c_str(), kv.second.n,
                 kv.second.ms, kv.second.bytes);
        out += item;
        first = false;
    }
    out += "}";
    if (buf && cap > 0) {
        size_t n = std::min(cap - 1, out.size());
        memcpy(buf, out.data(), n);
        buf[n] = 0;
    }
    return (int)out.size() + 1;
}

prc_status_t prc_prod_sum_f32(float* mesh, const int32_t shape[3], const float* coords, int exp, void* stream) {
    return prc::prod_sum<float>(mesh, shape, coords, exp, (cudaStream_t)stream);
}

prc_status_t prc_prod_sum_f64(double* mesh, const int32_t shape[3], const double* coords, int exp, void* stream) {
    return prc::prod_sum<double>(mesh, shape, coords, exp, (cudaStream_t)stream);
}

size_t prc_smooth_gaussian_real_workspace_bytes(const int32_t nmesh[3], const double radius[3], double nsigmas,
                                                int mesh_bytes) {
    if (mesh_bytes == 4) {
        prc::RealSmoothPlan<float> p;
        return prc::real_smooth_plan<float>(nmesh, radius, nsigmas, &p) == PRC_OK ? prc::real_smooth_bytes(p) : 0;
    }
    prc::RealSmoothPlan<double> p;
    return prc::real_smooth_plan<double>(nmesh, radius, nsigmas, &p) == PRC_OK ? prc::real_smooth_bytes(p) : 0;
}

prc_status_t prc_smooth_gaussian_real_f32(const float* in, float* out, const int32_t nmesh[3], const double radius[3],
                                          double nsigmas, void* workspace, size_t workspace_bytes, void* stream) {
    return prc::smooth_real<float>(in, out, nmesh, radius, nsigmas, workspace, workspace_bytes, (cudaStream_t)stream);
}

prc_status_t prc_smooth_gaussian_real_f64(const double* in, double* out, const int32_t nmesh[3], const double radius[3],
                                          double nsigmas, void* workspace, size_t workspace_bytes, void* stream) {
    return prc::smooth_real<double>(in, out, nmesh, radius, nsigmas, workspace, workspace_bytes, (cudaStream_t)stream);
}

size_t prc_density_contrast_original_workspace_bytes(void) { return 4 * prc::MARTIN_BLOCKS * sizeof(double); }

prc_status_t prc_density_contrast_original_f32(const double* mesh_data, const double* mesh_randoms,
                                               const int32_t nmesh[3], double bias, double ran_min, float* delta,
                                               void* workspace, size_t workspace_bytes, void* stream) {
    return prc::density_original<float>(mesh_data, mesh_randoms, nmesh, bias, ran_min, delta, workspace,
                                         workspace_bytes, (cudaStream_t)stream);
}

prc_status_t prc_density_contrast_original_f64(const double* mesh_data, const double* mesh_randoms,
                                               const int32_t nmesh[3], double bias, double ran_min, double* delta,
                                               void* workspace, size_t workspace_bytes, void* stream) {
    return prc::density_original<double>(mesh_data, mesh_randoms, nmesh, bias, ran_min, delta, workspace,
                                          workspace_bytes, (cudaStream_t)stream);
}

}  // extern "C"

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

}  // extern "C"

// Shared definitions for the pyrecon_b200 CUDA library (sm_100a).
//
// Conventions used by every kernel and entry point:
//   * meshes are C-ordered (n0, n1, n2) arrays, index (ix * n1 + iy) * n2 + iz;
//   * half spectra are (n0, n1, n2/2 + 1) interleaved complex arrays;
//   * positions are (N, 3) row-major arrays of float or double;
//   * every entry point returns a prc_status_t and launches on the caller's
//     stream; nothing here allocates device memory.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/pyrecon_cuda.h"

#define PRC_CHECK_LAUNCH()                                   \
    do {                                                     \
        cudaError_t _e = cudaGetLastError();                 \
        if (_e != cudaSuccess) return PRC_ERR_CUDA;          \
    } while (0)

#define PRC_TRY(expr)                                        \
    do {                                                     \
        int _s = (expr);                                     \
        if (_s != PRC_OK) return _s;                         \
    } while (0)

namespace prc {

// ---------------------------------------------------------------------------------------------
// Complex arithmetic on float2 / double2
// ---------------------------------------------------------------------------------------------
template <typename T> struct cplx_of;
template <> struct cplx_of<float> { typedef float2 type; };
template <> struct cplx_of<double> { typedef double2 type; };

template <typename T> using cplx_t = typename cplx_of<T>::type;

template <typename C> __host__ __device__ __forceinline__ C cmake(decltype(C().x) re, decltype(C().x) im) {
    C c;
    c.x = re;
    c.y = im;
    return c;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return cmake<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return cmake<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    return cmake<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C> __device__ __forceinline__ C cconj(C a) { return cmake<C>(a.x, -a.y); }
template <typename C, typename T> __device__ __forceinline__ C cscale(C a, T s) { return cmake<C>(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse): dir = -1 forward, +1 inverse
template <typename C> __device__ __forceinline__ C cmul_i(C a, int dir) {
    return dir < 0 ? cmake<C>(a.y, -a.x) : cmake<C>(-a.y, a.x);
}

// Four-component vectors for interleaved (x, y, z, 0) meshes
template <typename T> struct vec4_of;
template <> struct vec4_of<float> { typedef float4 type; };
template <> struct vec4_of<double> { typedef double4 type; };
template <typename T> __host__ __device__ __forceinline__ typename vec4_of<T>::type make_vec4(T x, T y, T z) {
    typename vec4_of<T>::type v;
    v.x = x;
    v.y = y;
    v.z = z;
    v.w = 0;
    return v;
}

// ---------------------------------------------------------------------------------------------
// Mesh geometry passed by value to kernels
// ---------------------------------------------------------------------------------------------
struct Dims {
    int n[3];
    __host__ __device__ __forceinline__ int64_t size() const { return (int64_t)n[0] * n[1] * n[2]; }
};

__host__ __device__ __forceinline__ int wrap_up(int i, int n) { return i + 1 == n ? 0 : i + 1; }
__host__ __device__ __forceinline__ int wrap_dn(int i, int n) { return i == 0 ? n - 1 : i - 1; }

// IEEE round-to-nearest arithmetic that the compiler may not contract into FMAs,
// used where the reference's numpy / C arithmetic must be reproduced bit for bit.
__device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float rn_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float rn_div(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double rn_div(double a, double b) { return __ddiv_rn(a, b); }

// numpy's result type of (positions dtype, mesh dtype) arithmetic: double unless both are float.
template <typename P, typename F> struct promote { typedef double type; };
template <> struct promote<float, float> { typedef float type; };

// Python's float modulo (result has the sign of the divisor), as numpy's `%` on floats.
template <typename T> __device__ __forceinline__ T py_fmod(T a, T b) {
    T r = fmod(a, b);
    if (r != 0 && ((r < 0) != (b < 0))) r += b;
    return r;
}

// Geometry of one mesh for particle kernels.  boxsize / boxcenter hold the values the
// reference stores in the mesh dtype (pyrecon/mesh.py:447-455), widened to double.
struct BoxGeom {
    int n[3];
    double boxsize[3];
    double boxcenter[3];
};

// Index-space coordinate of one position component, exactly as numpy evaluates
// ((p - boxcenter) / boxsize + 0.5) * nmesh followed by .astype(FLOAT)
// (pyrecon/mesh.py:554-555): arithmetic in the promoted type of (P, F), the
// nmesh multiply in double whenever F is float (int32 array promotion), then
// rounded to F.  The final multiply by an integer is exact in double for the
// float case, so evaluating it in the promoted type gives the same rounding.
template <typename P, typename F>
__device__ __forceinline__ F index_coord(P p, const BoxGeom& g, int d) {
    typedef typename promote<P, F>::type T;
    T t = rn_sub((T)p, (T)(F)g.boxcenter[d]);
    t = rn_div(t, (T)(F)g.boxsize[d]);
    t = rn_add(t, (T)0.5);
    double s = rn_mul((double)t, (double)g.n[d]);
    return (F)s;
}

// numpy's wrap of a position into the box: ((p - offset) % boxsize) + offset, computed in
// the promoted type T of (P, F) with offset = boxcenter - boxsize / 2 in F (mesh.py:477-479).
// The result stays in T, as the wrapped numpy array does.
template <typename P, typename F>
__device__ __forceinline__ typename promote<P, F>::type wrap_position(P p, const BoxGeom& g, int d) {
    typedef typename promote<P, F>::type T;
    F bs = (F)g.boxsize[d], bc = (F)g.boxcenter[d];
    F off = rn_sub(bc, rn_div(bs, (F)2));
    T r = py_fmod<T>(rn_sub((T)p, (T)off), (T)bs);
    return rn_add(r, (T)off);
}

// Grid-stride helpers
__host__ __forceinline__ int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

int device_sm_count();
// Run-time tuning table (tune.cu): knob `name` for key `key` (a mesh axis length), or `dflt` when unset;
// the generation counter changes with every update.
int tune_get(const char* name, int key, int dflt);
unsigned tune_generation();

// Programmatic dependent launch.  A kernel launched by launch_pdl may be scheduled while its predecessor
// on the stream (or in a captured graph) is still finishing: its blocks call pdl_wait() before reading
// anything the predecessor wrote (the wait returns once the predecessor grid has completed and its
// memory is visible; at once when there is no programmatic predecessor), and pdl_trigger() to let
// their own successor be scheduled as soon as every block of this grid has started.  No spin of ours:
// the ordering is the hardware's.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// PRC_PDL=0 in the environment launches these kernels without the attribute (plain stream order).
bool pdl_enabled();

template <typename... K, typename... A>
inline cudaError_t launch_pdl(void (*kernel)(K...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              A&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<K>(args)...);
}

// Adds n to the launch counter (kernels replayed inside a CUDA graph launch).
void add_launches(unsigned long long n);
// Launches and compulsory bytes recorded by this thread's captures since the last call (reset).
void capture_tally(unsigned long long* launches, double* bytes);

// Every kernel launch goes through PRC_LAUNCH: it counts launches (prc_launch_count) and, when
// prc_profile_enable(1) is on, brackets the launch with CUDA events on its stream so the
// per-kernel device time can be read back with prc_profile_collect.
// `bytes` is the launch's compulsory DRAM traffic (what it must read and write at least), so
// the profile reports achieved bandwidth against the HBM roofline.
// Launches made while the calling thread captures a stream are not counted or timed; they are
// tallied per thread (capture_tally) so a replayed graph can report them.
struct KernelScope {
    KernelScope(const char* name, cudaStream_t st, double bytes = 0., bool count = true);
    ~KernelScope();
    const char* name;
    cudaStream_t st;
    cudaEvent_t start;
    double bytes;
};

}  // namespace prc

#define PRC_LAUNCH(NAME, STREAM, ...)                 \
    do {                                              \
        ::prc::KernelScope _prc_scope(NAME, STREAM);  \
        __VA_ARGS__;                                  \
    } while (0)

#define PRC_LAUNCH_B(NAME, STREAM, BYTES, ...)                 \
    do {                                                       \
        ::prc::KernelScope _prc_scope(NAME, STREAM, BYTES);    \
        __VA_ARGS__;                                           \
    } while (0)

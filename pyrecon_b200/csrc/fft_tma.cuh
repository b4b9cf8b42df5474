// TMA-fed versions of the strided FFT passes (y and x axes) and of the x pass with the k-space
// step (included by fft.cu after fft_fast.cuh).
//
// A tile (B adjacent z-columns x N points along the line) is brought into shared memory by the
// tensor-memory-access unit: one elected thread arms the stage's transaction barrier and issues the
// tiled copies (N / 256 boxes of B columns x 256 points), while the CTA computes earlier tiles.
// S stages rotate; a stage is re-armed with the tile S steps ahead as soon as its FFT has read it.
// Threads hold 8 points each in registers exactly as the register kernels in fft_fast.cuh; the
// exchanges of the passes reuse the tile's own stage buffer (the k-space kernel keeps one extra
// buffer for the inverse transforms of its outputs), and results are stored straight from
// registers.  The box layout in shared memory, point k of column c at k * B + c, is the layout
// of ColAddr.
#pragma once

#include "tma.cuh"

namespace fast {

template <typename T, int N, int B> struct TileShape {
    typedef cplx_t<T> C;
    static constexpr int U = (int)(sizeof(C) / 8);    // 8-byte map elements per complex value
    static constexpr int BOXL = N < 256 ? N : 256;    // points per copy (a box extent is at most 256)
    static constexpr int NCHUNK = N / BOXL;
    static constexpr int ELEMS = N * B;
    static constexpr uint32_t BYTES = (uint32_t)(ELEMS * sizeof(C));
};

// Copies of one tile into `stage`, completing on `bar`.  Spectrum maps are (nh U, n1, n0) in 8-byte
// elements; axis 1 (y lines) uses boxes (B U, BOXL, 1) at (c0 U, q BOXL, o), axis 0 (x lines) boxes
// (B U, 1, BOXL) at (c0 U, o, q BOXL).  c0 is a multiple of B, so c0 U * 8 bytes is a multiple of 16.
template <typename T, int N, int B>
__device__ __forceinline__ void issue_tile(cplx_t<T>* stage, const CUtensorMap* map, uint64_t* bar, int axis, int o,
                                           int c0) {
    typedef TileShape<T, N, B> TS;
    prc::tma::arrive_expect_tx(bar, TS::BYTES);
#pragma unroll
    for (int q = 0; q < TS::NCHUNK; q++) {
        if (axis == 1) prc::tma::load_3d(stage + q * TS::BOXL * B, map, bar, c0 * TS::U, q * TS::BOXL, o);
        else prc::tma::load_3d(stage + q * TS::BOXL * B, map, bar, c0 * TS::U, o, q * TS::BOXL);
    }
}

// Tile t of a pass over nbatch spectra: batch index, outer position, first column.
struct TileAt {
    int bi, o, c0;
};
__device__ __forceinline__ TileAt tile_at(int64_t tile, int64_t tiles_per, int ctiles, int B) {
    TileAt a;
    a.bi = (int)(tile / tiles_per);
    const int64_t r = tile % tiles_per;
    a.o = (int)(r / ctiles);
    a.c0 = (int)(r % ctiles) * B;
    return a;
}

// Called by thread 0 after a wait ran out at local step j: wait (bounded) for the copies still in
// flight, those of steps j .. j + S - 1, so none lands after the CTA has exited.
template <int S>
__device__ __forceinline__ void drain(uint64_t* bars, int64_t j, int64_t ntiles) {
    atomicOr(&prc::g_fault, prc::tma::FAULT_WAIT_TIMEOUT);
    for (int d = 0; d < S; d++) {
        const int64_t jj = j + d;
        if ((int64_t)blockIdx.x + jj * gridDim.x >= ntiles) break;
        prc::tma::wait(&bars[jj % S], (uint32_t)((jj / S) & 1));
    }
}

// Shared memory of S stages (+ `extra` tile buffers) and the pass twiddles, then the barriers.
template <typename T, int N, int B, int S, int EXTRA> struct TmaSmem {
    typedef TileShape<T, N, B> TS;
    static constexpr size_t TILES = (size_t)(S + EXTRA) * TS::ELEMS * sizeof(cplx_t<T>);
    static constexpr size_t TW = (size_t)N * sizeof(cplx_t<T>);
    static constexpr size_t BYTES = TILES + TW + S * sizeof(uint64_t);
};

template <typename T, int N, int B, int S, int DIR>
__global__ void __launch_bounds__(N / 8 * B) strided_tma(const __grid_constant__ prc::tma::Maps maps,
                                                         Specs<cplx_t<T>> data, int nbatch, Strided s, int axis) {
    typedef cplx_t<T> C;
    typedef TileShape<T, N, B> TS;
    constexpr int TL = N / 8;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    C* stages = (C*)smem_raw;
    C* tw = stages + S * TS::ELEMS;
    uint64_t* bars = (uint64_t*)(tw + N);
    const int tid = threadIdx.x, col = tid % B, t = tid / B;
    const ColAddr addr{B, col};
    if (tid == 0) {
        for (int i = 0; i < S; i++) prc::tma::barrier_init(&bars[i], 1);
        prc::tma::fence_barrier_init();
    }
    fill_pass_twiddles<C, N>(tw);
    const int ctiles = (s.ncols + B - 1) / B;
    const int64_t tiles_per = (int64_t)s.outer * ctiles;
    const int64_t ntiles = tiles_per * nbatch;
    __syncthreads();
    if ((prc::tma::smem_addr(stages) & 127) != 0) {
        if (tid == 0) atomicOr(&prc::g_fault, prc::tma::FAULT_SMEM_ALIGN);
        return;
    }
    if (tid == 0) {
        for (int j = 0; j < S; j++) {
            const int64_t tile = blockIdx.x + (int64_t)j * gridDim.x;
            if (tile >= ntiles) break;
            const TileAt a = tile_at(tile, tiles_per, ctiles, B);
            issue_tile<T, N, B>(stages + j * TS::ELEMS, &maps.m[a.bi], &bars[j], axis, a.o, a.c0);
        }
    }
    int64_t j = 0;
    for (;; j++) {
        const int64_t tile = blockIdx.x + j * gridDim.x;
        if (tile >= ntiles) break;
        const int st = (int)(j % S);
        const bool ok = prc::tma::wait(&bars[st], (uint32_t)((j / S) & 1));
        if (__syncthreads_or(!ok)) {
            if (tid == 0) drain<S>(bars, j, ntiles);
            return;
        }
        C* sb = stages + st * TS::ELEMS;
        const TileAt a = tile_at(tile, tiles_per, ctiles, B);
        C v[8];
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = sb[(t + i * TL) * B + col];
        __syncthreads();
        fft_regs<C, N, DIR>(v, t, sb, addr, tw);   // ends with a barrier when it exchanged through sb
        if (tid == 0) {
            const int64_t next = tile + (int64_t)S * gridDim.x;
            if (next < ntiles) {
                const TileAt b = tile_at(next, tiles_per, ctiles, B);
                prc::tma::fence_proxy_async();
                issue_tile<T, N, B>(sb, &maps.m[b.bi], &bars[st], axis, b.o, b.c0);
            }
        }
        if (a.c0 + col < s.ncols) {
            C* g = data.p[a.bi] + (int64_t)a.o * s.os + a.c0 + col;
#pragma unroll
            for (int i = 0; i < 8; i++) g[(int64_t)(t + i * TL) * s.ls] = v[i];
        }
    }
}

// LEAN: the forward spectrum is kept in the tile's stage (not in registers) and the per-point
// multiplier terms are recomputed for every output, so two CTAs fit on an SM (FP32); the stage is
// re-armed only after the tile's last output.
template <typename T, int N, int B, int S, int KT, bool LEAN>
__global__ void __launch_bounds__(N / 8 * B, (MinBlocks<T, N / 8 * B, LEAN ? 2 : PRC_KSPACE_MINB>::value))
    x_kspace_tma(const __grid_constant__ prc::tma::Maps maps, int nin, Specs<cplx_t<T>> out, Dims dims, int pitch,
                 KOp op) {
    typedef cplx_t<T> C;
    typedef TileShape<T, N, B> TS;
    constexpr int TL = N / 8;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    C* stages = (C*)smem_raw;
    C* xbuf = stages + S * TS::ELEMS;
    C* tw = xbuf + TS::ELEMS;
    uint64_t* bars = (uint64_t*)(tw + N);
    const int tid = threadIdx.x, col = tid % B, t = tid / B;
    const ColAddr addr{B, col};
    if (tid == 0) {
        for (int i = 0; i < S; i++) prc::tma::barrier_init(&bars[i], 1);
        prc::tma::fence_barrier_init();
    }
    fill_pass_twiddles<C, N>(tw);
    const int n1 = dims.n[1], nh = dims.n[2] / 2 + 1;
    const int64_t ls = (int64_t)n1 * pitch;
    const int ctiles = (nh + B - 1) / B;
    const int64_t tiles_per = (int64_t)n1 * ctiles;
    const int64_t ntiles = tiles_per * nin;
    __syncthreads();
    if ((prc::tma::smem_addr(stages) & 127) != 0) {
        if (tid == 0) atomicOr(&prc::g_fault, prc::tma::FAULT_SMEM_ALIGN);
        return;
    }
    if (tid == 0) {
        for (int j = 0; j < S; j++) {
            const int64_t tile = blockIdx.x + (int64_t)j * gridDim.x;
            if (tile >= ntiles) break;
            const TileAt a = tile_at(tile, tiles_per, ctiles, B);
            issue_tile<T, N, B>(stages + j * TS::ELEMS, &maps.m[a.bi], &bars[j], 0, a.o, a.c0);
        }
    }
    int64_t j = 0;
    for (;; j++) {
        const int64_t tile = blockIdx.x + j * gridDim.x;
        if (tile >= ntiles) break;
        const int st = (int)(j % S);
        const bool ok = prc::tma::wait(&bars[st], (uint32_t)((j / S) & 1));
        if (__syncthreads_or(!ok)) {
            if (tid == 0) drain<S>(bars, j, ntiles);
            return;
        }
        C* sb = stages + st * TS::ELEMS;
        const TileAt a = tile_at(tile, tiles_per, ctiles, B);
        const int iy = a.o, iz = a.c0 + col;
        auto refill = [&]() {
            if (tid == 0) {
                const int64_t next = tile + (int64_t)S * gridDim.x;
                if (next < ntiles) {
                    const TileAt b = tile_at(next, tiles_per, ctiles, B);
                    prc::tma::fence_proxy_async();
                    issue_tile<T, N, B>(sb, &maps.m[b.bi], &bars[st], 0, b.o, b.c0);
                }
            }
        };
        const int64_t off = (int64_t)iy * pitch + iz;
        if constexpr (LEAN) {
            {
                C v[8];
#pragma unroll
                for (int i = 0; i < 8; i++) v[i] = sb[(t + i * TL) * B + col];
                __syncthreads();
                fft_regs<C, N, -1>(v, t, sb, addr, tw);
                if constexpr (Plan<N>::NPASS == 1) __syncthreads();
#pragma unroll
                for (int i = 0; i < 8; i++) sb[(t + i * TL) * B + col] = v[i];
            }
            for (int o = 0; o < op.nper; o++) {
                C u[8];
                {
                    C v[8];
#pragma unroll
                    for (int i = 0; i < 8; i++) v[i] = sb[(t + i * TL) * B + col];
                    KLine<T, N, KT> kl;
                    kl.setup(op, dims, t, iy, iz);
                    kl.apply(op, dims, t, o, v, u);
                }
                fft_regs<C, N, +1>(u, t, xbuf, addr, tw);
                if (iz < nh) {
                    C* go = out.p[a.bi * op.nper + o] + off;
#pragma unroll
                    for (int i = 0; i < 8; i++) go[(int64_t)(t + i * TL) * ls] = u[i];
                }
            }
            __syncthreads();
            refill();
        } else {
            C v[8];
#pragma unroll
            for (int i = 0; i < 8; i++) v[i] = sb[(t + i * TL) * B + col];
            __syncthreads();
            fft_regs<C, N, -1>(v, t, sb, addr, tw);
            refill();
            KLine<T, N, KT> kl;
            kl.setup(op, dims, t, iy, iz);
            for (int o = 0; o < op.nper; o++) {
                C u[8];
                kl.apply(op, dims, t, o, v, u);
                fft_regs<C, N, +1>(u, t, xbuf, addr, tw);
                if (iz < nh) {
                    C* go = out.p[a.bi * op.nper + o] + off;
#pragma unroll
                    for (int i = 0; i < 8; i++) go[(int64_t)(t + i * TL) * ls] = u[i];
                }
            }
        }
    }
}

// Input rows of the inverse z pass staged by bulk copies.  Unit u = (tile u / nin, input u % nin):
// the tile's ROWS rows of that input, contiguous in memory (rows of PS complex values, PS the padded
// pitch), copied into stage u % S; a stage is re-armed with unit u + S once its rows have been read
// into registers.  Units are consumed in the order z_c2r_body asks for them: inputs 0 .. nin - 1 of
// each tile, tiles blockIdx.x, blockIdx.x + gridDim.x, ...
template <typename T, int M, int ROWS, int S> struct TmaRows {
    typedef cplx_t<T> C;
    static constexpr int Q = (int)(32 / sizeof(C));
    static constexpr int PS = (M + 1 + Q - 1) / Q * Q;
    static constexpr int STAGE = ROWS * PS;
    C* stages;
    uint64_t* bars;
    const Specs<C>& in;
    int nin;
    int64_t rows, ntiles;
    int64_t next = 0;        // next unit this thread consumes
    int64_t issued = 0;      // thread 0: units issued
    int64_t first_fail = -1; // thread 0: unit whose wait ran out first
    bool failed = false;

    __device__ __forceinline__ TmaRows(C* st, uint64_t* b, const Specs<C>& i, int n, int64_t r)
        : stages(st), bars(b), in(i), nin(n), rows(r), ntiles((r + ROWS - 1) / ROWS) {}

    __device__ __forceinline__ void issue(int64_t u) {
        const int64_t tile = blockIdx.x + (u / nin) * gridDim.x;
        if (tile >= ntiles) return;
        const int64_t row0 = tile * ROWS;
        const int64_t nr = rows - row0 < ROWS ? rows - row0 : ROWS;
        const uint32_t bytes = (uint32_t)(nr * PS * sizeof(C));
        const int st = (int)(u % S);
        prc::tma::arrive_expect_tx(&bars[st], bytes);
        prc::tma::load_1d(stages + st * STAGE, select6(in, (int)(u % nin)) + row0 * PS, bytes, &bars[st]);
        issued = u + 1;
    }

    __device__ __forceinline__ void start() {
        if (threadIdx.x == 0)
            for (int u = 0; u < S; u++) issue(u);
    }

    // Same result as row_c2r, the row read from the stage instead of global memory.
    __device__ __forceinline__ void row(int, int64_t, bool, int t, C* buf, const RowAddr& addr, const C* tw,
                                        const C* wk, C (&v)[8]) {
        constexpr int TL = M / 8;
        const int st = (int)(next % S);
        if (!prc::tma::wait(&bars[st], (uint32_t)((next / S) & 1))) {
            if (!failed && threadIdx.x == 0) first_fail = next;
            failed = true;
        }
        const C* x = stages + st * STAGE + (threadIdx.x / TL) * PS;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int k = t + i * TL;
            const C xk = x[k];
            const C xc = cconj(x[M - k]);
            const C ev = cadd(xk, xc);
            const C od = cmul(cconj(wk[k]), csub(xk, xc));
            v[i] = cadd(ev, cmul_i(od, +1));
        }
        __syncthreads();
        if (threadIdx.x == 0 && !failed) {
            prc::tma::fence_proxy_async();
            issue(next + S);
        }
        next++;
        fft_regs<C, M, +1>(v, t, buf, addr, tw);
    }

    // End of a tile: if any thread's wait ran out, thread 0 waits (bounded) for the copies it issued
    // and has not seen land, and every thread leaves the kernel.
    __device__ __forceinline__ bool stop() {
        if (!__syncthreads_or(failed)) return false;
        if (threadIdx.x == 0) {
            atomicOr(&prc::g_fault, prc::tma::FAULT_WAIT_TIMEOUT);
            int64_t u = first_fail >= 0 && first_fail < next ? first_fail : next;
            for (; u < issued; u++) prc::tma::wait(&bars[u % S], (uint32_t)((u / S) & 1));
        }
        return true;
    }
};

template <typename T, int M, int ROWS, int S> struct C2RTmaSmem {
    typedef cplx_t<T> C;
    static constexpr size_t STAGES = (size_t)S * TmaRows<T, M, ROWS, S>::STAGE * sizeof(C);
    static constexpr size_t BUF = (size_t)ROWS * row_stride(M) * sizeof(C);
    static constexpr size_t BYTES = STAGES + BUF + (size_t)(2 * M + 1) * sizeof(C) + 8 + S * sizeof(uint64_t);
};

template <typename T, int M, int ROWS, int ET, int S>
__global__ void __launch_bounds__(M / 8 * ROWS, (MinBlocks<T, M / 8 * ROWS, PRC_C2R_MINB>::value))
    z_c2r_tma(Specs<cplx_t<T>> in, int nin, Dims dims, Epi<T> e) {
    typedef cplx_t<T> C;
    typedef TmaRows<T, M, ROWS, S> Rows;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    C* stages = (C*)smem_raw;
    C* buf = stages + S * Rows::STAGE;
    C* tw = buf + ROWS * row_stride(M);
    C* wk = tw + M;
    uint64_t* bars = (uint64_t*)(((uintptr_t)(wk + M + 1) + 7) & ~(uintptr_t)7);
    if (threadIdx.x == 0) {
        for (int i = 0; i < S; i++) prc::tma::barrier_init(&bars[i], 1);
        prc::tma::fence_barrier_init();
    }
    fill_pass_twiddles<C, M>(tw);
    fill_roots(wk, M + 1, 2 * M);
    __syncthreads();
    if ((prc::tma::smem_addr(stages) & 15) != 0) {
        if (threadIdx.x == 0) atomicOr(&prc::g_fault, prc::tma::FAULT_SMEM_ALIGN);
        return;
    }
    Rows src(stages, bars, in, nin, (int64_t)dims.n[0] * dims.n[1]);
    src.start();
    z_c2r_body<T, M, ROWS, ET>(src, nin, dims, e, tw, wk, buf);
}

// Inverse y pass of the six Hessian spectra D_ij = k_i k_j delta(k) / k^2 of the local-line-of-sight
// iteration, combined on the fly.  After the inverse x (done) and y transforms, x0 (fixed per tile)
// and x1 (per point) are known, so the weighted sum over (i, j) of f_ij x_i x_j d_ij, which the
// real-space update needs, is a quadratic in x2 with coefficients
//   A = f00 x0^2 D00 + f01 x0 x1 D01 + f11 x1^2 D11,   B = f02 x0 D02 + f12 x1 D12,   C = f22 D22
// that are formed here, before the inverse z transform (which they commute with, being constant along
// z).  The three are written in place of D00, D01, D02, so the z pass reads 3 spectra instead of 6
// and runs 3 row transforms instead of 6.  Inputs stream through S stages in the order
// D00, D01, D11 | D02, D12 | D22, one accumulator per output.
struct HessGeom {
    double x0_off, x0_cell;   // x0 = x0_off + x0_cell * ix (mesh-dtype offset, float64 cell as the epilogue)
    double x1_off, x1_cell;   // x1 = x1_off + x1_cell * iy
    double f[6];              // f_ij in the order (0,0) (0,1) (0,2) (1,1) (1,2) (2,2)
};

template <typename T, int N, int B, int S>
__global__ void __launch_bounds__(N / 8 * B) y_hessian_tma(const __grid_constant__ prc::tma::Maps maps,
                                                           Specs<cplx_t<T>> out, Strided s, HessGeom h) {
    typedef cplx_t<T> C;
    typedef TileShape<T, N, B> TS;
    constexpr int TL = N / 8;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    C* stages = (C*)smem_raw;
    C* tw = stages + S * TS::ELEMS;
    uint64_t* bars = (uint64_t*)(tw + N);
    const int tid = threadIdx.x, col = tid % B, t = tid / B;
    const ColAddr addr{B, col};
    if (tid == 0) {
        for (int i = 0; i < S; i++) prc::tma::barrier_init(&bars[i], 1);
        prc::tma::fence_barrier_init();
    }
    fill_pass_twiddles<C, N>(tw);
    const int ctiles = (s.ncols + B - 1) / B;
    const int64_t ntiles = (int64_t)s.outer * ctiles;
    __syncthreads();
    if ((prc::tma::smem_addr(stages) & 127) != 0) {
        if (tid == 0) atomicOr(&prc::g_fault, prc::tma::FAULT_SMEM_ALIGN);
        return;
    }
    // unit u: tile blockIdx.x + (u / 6) gridDim.x, spectrum ORDER[u % 6]
    auto spectrum_of = [](int k) { return k < 2 ? k : (k == 2 ? 3 : (k == 3 ? 2 : k)); };
    auto issue = [&](int64_t u) {
        const int64_t tile = blockIdx.x + (u / 6) * gridDim.x;
        if (tile >= ntiles) return;
        const TileAt a = tile_at(tile, ntiles, ctiles, B);
        issue_tile<T, N, B>(stages + (u % S) * TS::ELEMS, &maps.m[spectrum_of((int)(u % 6))], &bars[u % S], 1, a.o,
                            a.c0);
    };
    if (tid == 0)
        for (int u = 0; u < S; u++) issue(u);
    int64_t u = 0;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const TileAt a = tile_at(tile, ntiles, ctiles, B);
        const T x0 = (T)(h.x0_off + h.x0_cell * a.o);
        T x1[8];
#pragma unroll
        for (int i = 0; i < 8; i++) x1[i] = (T)(h.x1_off + h.x1_cell * (t + i * TL));
        const bool store = a.c0 + col < s.ncols;
        const int64_t off = (int64_t)a.o * s.os + a.c0 + col;
#pragma unroll 1
        for (int g = 0; g < 3; g++) {
            C acc[8];
#pragma unroll
            for (int i = 0; i < 8; i++) acc[i] = cmake<C>(0, 0);
            const int nterm = g == 0 ? 3 : (g == 1 ? 2 : 1);
#pragma unroll 1
            for (int q = 0; q < nterm; q++, u++) {
                const int st = (int)(u % S);
                const bool ok = prc::tma::wait(&bars[st], (uint32_t)((u / S) & 1));
                if (__syncthreads_or(!ok)) {
                    if (tid == 0) {
                        atomicOr(&prc::g_fault, prc::tma::FAULT_WAIT_TIMEOUT);
                        for (int d = 0; d < S; d++) {
                            const int64_t uu = u + d;
                            if ((int64_t)blockIdx.x + (uu / 6) * gridDim.x >= ntiles) break;
                            prc::tma::wait(&bars[uu % S], (uint32_t)((uu / S) & 1));
                        }
                    }
                    return;
                }
                C* sb = stages + st * TS::ELEMS;
                C v[8];
#pragma unroll
                for (int i = 0; i < 8; i++) v[i] = sb[(t + i * TL) * B + col];
                __syncthreads();
                fft_regs<C, N, +1>(v, t, sb, addr, tw);
                if (tid == 0) {
                    prc::tma::fence_proxy_async();
                    issue(u + S);
                }
                const int k = g == 0 ? (q == 0 ? 0 : (q == 1 ? 1 : 3)) : (g == 1 ? (q == 0 ? 2 : 4) : 5);
                const T f = (T)(k == 0 ? h.f[0] : k == 1 ? h.f[1] : k == 2 ? h.f[2] : k == 3 ? h.f[3] : k == 4 ? h.f[4] : h.f[5]);
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    // weight of D_k at this point: f x0^2 | f x0 x1 | f x1^2 | f x0 | f x1 | f
                    const T w = k == 0 ? f * (x0 * x0) : k == 1 ? f * (x0 * x1[i]) : k == 3 ? f * (x1[i] * x1[i])
                              : k == 2 ? f * x0 : k == 4 ? f * x1[i] : f;
                    acc[i] = cmake<C>(acc[i].x + w * v[i].x, acc[i].y + w * v[i].y);
                }
            }
            if (store) {
                C* o = (g == 0 ? out.p[0] : (g == 1 ? out.p[1] : out.p[2])) + off;
#pragma unroll
                for (int i = 0; i < 8; i++) o[(int64_t)(t + i * TL) * s.ls] = acc[i];
            }
        }
    }
}

}  // namespace fast

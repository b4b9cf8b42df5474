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
    // points per copy: a box extent is at most 256 and divides N (384 = 2 x 192)
    static constexpr int BOXL = N <= 256 ? N : (N % 256 == 0 ? 256 : N / 2);
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
// PADX: the first of the EXTRA tiles is a padded first-exchange buffer (PadAddr, N / 8 more rows).
template <typename T, int N, int B, int S, int EXTRA, int PADX = 0> struct TmaSmem {
    typedef TileShape<T, N, B> TS;
    static constexpr size_t TILES = ((size_t)(S + EXTRA) * TS::ELEMS + (size_t)PADX * (N / 8) * B) * sizeof(cplx_t<T>);
    static constexpr size_t TW = (size_t)N * sizeof(cplx_t<T>);
    static constexpr size_t BYTES = TILES + TW + S * sizeof(uint64_t);
};

// The first exchange of a tile of B columns is padded where a row is half the banks wide (B * complex =
// 64 bytes, FP32 with B = 8): see PadAddr.
template <typename T, int B> struct PadFirst {
    static constexpr int value = B * sizeof(cplx_t<T>) == 64 ? 1 : 0;
};

// PRC_STRIDED_PP: the strided passes exchange through a scratch tile, then the consumed stage
// (fft_regs_pp), where shared memory has room for the scratch tile.
#ifndef PRC_STRIDED_PP
#define PRC_STRIDED_PP 1
#endif
template <typename T, int N, int B, int S> struct StridedPP {
    static constexpr bool value = PRC_STRIDED_PP && TmaSmem<T, N, B, S, 1>::BYTES <= 227 * 1024;
};

template <typename T, int N, int B, int S, int DIR>
__global__ void __launch_bounds__(N / 8 * B) strided_tma(const __grid_constant__ prc::tma::Maps maps,
                                                         Specs<cplx_t<T>> data, int nbatch, Strided s, int axis) {
    typedef cplx_t<T> C;
    typedef TileShape<T, N, B> TS;
    constexpr int TL = N / 8;
    constexpr bool PP = StridedPP<T, N, B, S>::value;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    C* stages = (C*)smem_raw;
    C* xscr = stages + S * TS::ELEMS;           // PP: the exchange scratch tile
    C* tw = xscr + (PP ? TS::ELEMS : 0);
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
        if constexpr (PP) {
            // the second exchange goes through the stage: a barrier after the last reads, before its re-arm
            fft_regs_pp<C, N, DIR>(v, t, xscr, sb, addr, tw);
            __syncthreads();
        } else {
            __syncthreads();
            fft_regs<C, N, DIR>(v, t, sb, addr, tw);   // ends with a barrier when it exchanged through sb
        }
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

// PRC_KSPACE_PP: the transforms of the k-space pass exchange through two scratch tiles in turn
// (fft_regs_pp, one barrier per exchange), where the CTA's shared memory has room for both.
#ifndef PRC_KSPACE_PP
#define PRC_KSPACE_PP 1
#endif
template <typename T, int N, int B, int S, bool LEAN> struct KSpacePP {
    static constexpr bool value =
        PRC_KSPACE_PP && !LEAN && TmaSmem<T, N, B, S, 2, PadFirst<T, B>::value>::BYTES <= 227 * 1024;
};

// LEAN: the forward spectrum is kept in the tile's stage (not in registers) and the per-point
// multiplier terms are recomputed for every output, so two CTAs fit on an SM (FP32); the stage is
// re-armed only after the tile's last output.
// Blocks per SM asked of the register allocator: at least 16 warps per SM in FP32 (a tile of B columns of
// a short line has few threads: 256 at 256 points, 128 at 128, 384 at 384), so at most 128 registers a
// thread (85 for 384 threads); tiles of less than a warp (lines of 8 or 16 points) are left free.
// CEIL = false (lines of 3 2^k points, whose radix-3 step needs more registers): 512 / THREADS rounded
// down; rounded up, the 384-point pass (80 registers, ~100 bytes spilled) measured 2.91 against 2.66 ms
// per nmesh-384 reconstruction.
template <typename T, int THREADS, bool CEIL = true> struct KSpaceMinBlocks {
    static constexpr int value =
        MinBlocks<T, THREADS,
                  (PRC_KSPACE_MINB > 1 ? PRC_KSPACE_MINB
                                       : (THREADS >= 512 || THREADS < 32 ? 1
                                                                         : (CEIL ? (511 + THREADS) / THREADS : 512 / THREADS)))>::value;
};

template <typename T, int N, int B, int S, int KT, bool LEAN>
__global__ void __launch_bounds__(N / 8 * B, (LEAN ? MinBlocks<T, N / 8 * B, 2>::value
                                                  : KSpaceMinBlocks<T, N / 8 * B, N % 3 != 0>::value))
    x_kspace_tma(const __grid_constant__ prc::tma::Maps maps, int nin, Specs<cplx_t<T>> out, Dims dims, int pitch,
                 KOp op) {
    typedef cplx_t<T> C;
    typedef TileShape<T, N, B> TS;
    constexpr int TL = N / 8;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    C* stages = (C*)smem_raw;
    constexpr bool PP = KSpacePP<T, N, B, S, LEAN>::value;
    // with an odd number of exchanges per transform, consecutive transforms would start on the buffer
    // the previous one read last: a barrier separates them (as it does a transform without exchanges
    // from the stage re-arm)
    constexpr bool PP_SYNC = Shape<N>::NX % 2 == 1 || Shape<N>::NX == 0;
    constexpr int PADX = PP ? PadFirst<T, B>::value : 0;   // PP: xbuf, the first exchange's, padded
    C* xbuf = stages + S * TS::ELEMS;
    C* ybuf = xbuf + TS::ELEMS + PADX * (N / 8) * B;   // PP: the second scratch tile
    C* tw = ybuf + (PP ? TS::ELEMS : 0);
    uint64_t* bars = (uint64_t*)(tw + N);
    const int tid = threadIdx.x, col = tid % B, t = tid / B;
    const ColAddr addr{B, col};
    const PadAddr paddr{B, col};
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
                if constexpr (Shape<N>::NX == 0) __syncthreads();
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
                    if constexpr (KT == KOP_HESS3)
                        if (o == 0) kl.nyquist_lines(op, dims, t, iy, iz, v);
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
            if constexpr (PP) {
                // the stage is free once every thread is past the first exchange's barrier
                if constexpr (PADX) fft_regs_pp<C, N, -1>(v, t, xbuf, paddr, ybuf, addr, tw);
                else fft_regs_pp<C, N, -1>(v, t, xbuf, ybuf, addr, tw);
                if constexpr (PP_SYNC) __syncthreads();
            } else {
                __syncthreads();
                fft_regs<C, N, -1>(v, t, sb, addr, tw);
            }
            refill();
            KLine<T, N, KT> kl;
            kl.setup(op, dims, t, iy, iz);
            if constexpr (KT == KOP_HESS3) kl.nyquist_lines(op, dims, t, iy, iz, v);
            for (int o = 0; o < op.nper; o++) {
                C u[8];
                kl.apply(op, dims, t, o, v, u);
                if constexpr (PP) {
                    if constexpr (PADX) fft_regs_pp<C, N, +1>(u, t, xbuf, paddr, ybuf, addr, tw);
                    else fft_regs_pp<C, N, +1>(u, t, xbuf, ybuf, addr, tw);
                    if constexpr (PP_SYNC) __syncthreads();
                } else {
                    fft_regs<C, N, +1>(u, t, xbuf, addr, tw);
                }
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
// PRC_C2R_PP: the row transforms exchange through two row buffers in turn (fft_regs_pp); the barrier
// before a stage is re-armed also orders each row's first exchange after the previous row's reads.
// Rows in whole warps (RowWarp): no block barrier per unit.  Each warp releases a stage once it has read
// its rows (one arrival on the stage's `empty` barrier, which counts the warps), and thread 0 re-arms the
// stage of the previous unit once every warp has released it (a bounded wait that normally finds it
// done): S - 1 units stay in flight ahead of the one being read, and the warps of a block drift apart
// instead of meeting at every row transform.
#ifndef PRC_C2R_PP
#define PRC_C2R_PP 1
#endif
template <typename T, int M, int ROWS, int S> struct TmaRows {
    typedef cplx_t<T> C;
    static constexpr int Q = (int)(32 / sizeof(C));
    static constexpr int PS = (M + 1 + Q - 1) / Q * Q;
    static constexpr int STAGE = ROWS * PS;
    static constexpr bool PP = PRC_C2R_PP;   // the row transforms alternate between buf1 and buf2
    static constexpr bool WR = RowWarp<M, ROWS>::value;   // stages released per warp
    C* stages;
    C* buf1 = nullptr;       // PRC_C2R_PP: the row buffer the caller passes, and the second one
    C* buf2 = nullptr;       // (same layout, so a row's offset in buf1 is its offset in buf2)
    uint64_t* bars;
    uint64_t* empty = nullptr;   // WR: per stage, the warps that have read its unit
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

    // Same result as row_c2r, the row read from the stage instead of global memory.  The barrier before
    // the stage is re-armed stays the block's (every row of the tile reads the stage); WS: the row's
    // transform exchanges synchronise per warp.
    template <bool WS>
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
        if constexpr (WR) {
            __syncwarp();
            if ((threadIdx.x & 31) == 0) prc::tma::arrive(&empty[st]);
            if (threadIdx.x == 0 && !failed && next >= 1) {
                const int64_t u = next - 1;
                if (prc::tma::wait(&empty[u % S], (uint32_t)((u / S) & 1))) {
                    prc::tma::fence_proxy_async();
                    issue(u + S);
                } else {
                    if (first_fail < 0) first_fail = next;
                    failed = true;
                }
            }
        } else {
            __syncthreads();
            if (threadIdx.x == 0 && !failed) {
                prc::tma::fence_proxy_async();
                issue(next + S);
            }
        }
        next++;
        if constexpr (PRC_C2R_PP) fft_regs_pp<C, M, +1, WS>(v, t, buf, buf2 + (buf - buf1), addr, tw);
        else fft_regs<C, M, +1, WS>(v, t, buf, addr, tw);
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
    static constexpr size_t BYTES =
        STAGES + (PRC_C2R_PP ? 2 : 1) * BUF + (size_t)(2 * M + 1) * sizeof(C) + 8 + 2 * S * sizeof(uint64_t);
};

template <typename T, int M, int ROWS, int ET, int S>
__global__ void __launch_bounds__(M / 8 * ROWS, (MinBlocks<T, M / 8 * ROWS, PRC_C2R_MINB>::value))
    z_c2r_tma(Specs<cplx_t<T>> in, int nin, Dims dims, Epi<T> e) {
    typedef cplx_t<T> C;
    typedef TmaRows<T, M, ROWS, S> Rows;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    C* stages = (C*)smem_raw;
    C* buf = stages + S * Rows::STAGE;
    C* buf2 = buf + ROWS * row_stride(M);        // PRC_C2R_PP: the second row buffer
    C* tw = buf2 + (PRC_C2R_PP ? ROWS * row_stride(M) : 0);
    C* wk = tw + M;
    uint64_t* bars = (uint64_t*)(((uintptr_t)(wk + M + 1) + 7) & ~(uintptr_t)7);
    uint64_t* empty = bars + S;
    if (threadIdx.x == 0) {
        for (int i = 0; i < S; i++) prc::tma::barrier_init(&bars[i], 1);
        if constexpr (Rows::WR)
            for (int i = 0; i < S; i++) prc::tma::barrier_init(&empty[i], blockDim.x / 32);
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
    src.buf1 = buf;
    src.buf2 = buf2;
    src.empty = empty;
    src.start();
    z_c2r_body<T, M, ROWS, ET>(src, nin, dims, e, tw, wk, buf);
}

// Inverse y pass of the local-line-of-sight iteration.  The update needs the six Hessian fields
// d_ij = IFFT(k_i k_j E), E = delta(k) / k^2, weighted by f_ij x_i x_j.  Along an x line k_y and k_z are
// constant, so the x pass only transforms three spectra
//   F0 = IFFT_x(E),  F1 = IFFT_x(s_x E),  F2 = IFFT_x(k_x^2 E)
// (s_a = k_a, or 0 on the Nyquist plane of axis a, which is what the symmetrised multiplier of an odd
// factor reduces to), and the six follow in y-k space as D00 = F2, D01 = s_y F1, D02 = s_z F1,
// D11 = k_y^2 F0, D12 = s_y s_z F0, D22 = k_z^2 F0 (k_z constant along y).  After the inverse y
// transforms, x0 (fixed per tile) and x1 (per point) are known, so the weighted sum is a quadratic in
// x2 with coefficients
//   A = f00 x0^2 D00 + f01 x0 x1 D01 + f11 x1^2 D11,   B = f02 x0 D02 + f12 x1 D12,   C = f22 D22
// formed here, before the inverse z transform (which they commute with, being constant along z); the
// z pass then reads 3 spectra and runs 3 row transforms.  Where two axes are both at their Nyquist
// index the symmetrised k_a k_b is not s_a s_b but k_a k_b: D01 gains q01[iz] (-1)^(x + y) (the
// single mode at the x and y Nyquist indices, transformed), D02 on the z-Nyquist column is
// IFFT_y((-1)^x l02) and D12 on it is k_z IFFT_y(k_y [y Nyquist] F0).  Six units per tile stream through S stages:
// (F2, 1) (F1, s_y) (F0, k_y^2) -> A | (F1, 1) (F0, s_y) -> B | (F0, 1) -> C; a tile's second and third
// reads of F0 / F1 come from L2.
struct HessGeom {
    double x0_off, x0_cell;   // x0 = x0_off + x0_cell * ix (mesh-dtype offset, float64 cell as the epilogue)
    double x1_off, x1_cell;   // x1 = x1_off + x1_cell * iy
    double f[6];              // f_ij in the order (0,0) (0,1) (0,2) (1,1) (1,2) (2,2)
    double fscale_y, fscale_z; // numpy fftfreq spacing of the y and z wavenumbers
    int ny, nz;
    // Nyquist lines written by the x pass (null where an axis is odd): q01[iz] = k_x k_y E at
    // (x, y Nyquist), l02[iy] = k_x k_z E at (x, z Nyquist).  The symmetrised multiplier of k_a k_b is
    // k_a k_b where a and b are both Nyquist or both not, so D01 and D02 need these beyond s_a s_b.
    const void* q01;
    const void* l02;
};

// PP: the transforms exchange through a scratch tile and the consumed stage in turn (fft_regs_pp), with
// one barrier per exchange; a stage is then re-armed at the next unit's barrier, once every thread has
// finished with it, so S - 1 units are in flight ahead of the one being transformed.
template <typename T, int N, int B, int S, int MINB, bool PP>
__global__ void __launch_bounds__(N / 8 * B, (MinBlocks<T, N / 8 * B, MINB>::value)) y_hessian_tma(const __grid_constant__ prc::tma::Maps maps,
                                                           Specs<cplx_t<T>> out, Strided s, HessGeom h) {
    typedef cplx_t<T> C;
    typedef TileShape<T, N, B> TS;
    constexpr int TL = N / 8;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    C* stages = (C*)smem_raw;
    // the padded first-exchange buffer measured no faster here (3.85 against 3.79 ms per reconstruction:
    // two CTAs per SM leave less shared memory to spare), unlike the k-space pass
    constexpr int PADX = 0;
    C* xscr = stages + S * TS::ELEMS;          // PP: the exchange scratch tile
    C* tw = xscr + (PP ? TS::ELEMS + PADX * (N / 8) * B : 0);
    uint64_t* bars = (uint64_t*)(tw + N);
    T* x1tab = (T*)(bars + S);     // x1 and k_y of every y index (2 N values after the barriers)
    T* kytab = x1tab + N;
    const int tid = threadIdx.x, col = tid % B, t = tid / B;
    const ColAddr addr{B, col};
    const PadAddr paddr{B, col};
    if (tid == 0) {
        for (int i = 0; i < S; i++) prc::tma::barrier_init(&bars[i], 1);
        prc::tma::fence_barrier_init();
    }
    fill_pass_twiddles<C, N>(tw);
    for (int i = tid; i < N; i += blockDim.x) {
        x1tab[i] = (T)(h.x1_off + h.x1_cell * i);
        kytab[i] = kval<T>(i, h.ny, (T)h.fscale_y);
    }
    const int ctiles = (s.ncols + B - 1) / B;
    const int64_t ntiles = (int64_t)s.outer * ctiles;
    __syncthreads();
    if ((prc::tma::smem_addr(stages) & 127) != 0) {
        if (tid == 0) atomicOr(&prc::g_fault, prc::tma::FAULT_SMEM_ALIGN);
        return;
    }
    // unit u: tile blockIdx.x + (u / 6) gridDim.x, input spectrum F[2, 1, 0, 1, 0, 0][u % 6]
    auto input_of = [](int q) { return q == 0 ? 2 : (q == 1 || q == 3 ? 1 : 0); };
    auto issue = [&](int64_t u) {
        const int64_t tile = blockIdx.x + (u / 6) * gridDim.x;
        if (tile >= ntiles) return;
        const TileAt a = tile_at(tile, ntiles, ctiles, B);
        issue_tile<T, N, B>(stages + (u % S) * TS::ELEMS, &maps.m[input_of((int)(u % 6))], &bars[u % S], 1, a.o,
                            a.c0);
    };
    if (tid == 0)
        for (int u = 0; u < S; u++) issue(u);
    const int ynyq = h.ny % 2 == 0 ? h.ny / 2 : -1;
    const C* q01 = (const C*)h.q01;
    const C* l02 = (const C*)h.l02;
    int64_t u = 0;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const TileAt a = tile_at(tile, ntiles, ctiles, B);
        const T x0 = (T)(h.x0_off + h.x0_cell * a.o);
        const int iz = a.c0 + col;
        const T kz = kval<T>(iz, h.nz, (T)h.fscale_z);
        const bool znyq = nyquist(iz, h.nz);
        const T sz = znyq ? (T)0 : kz;
        const bool store = iz < s.ncols;
        const T xsign = (a.o & 1) ? (T)-1 : (T)1;     // (-1)^x
        const int64_t off = (int64_t)a.o * s.os + iz;
#pragma unroll 1
        for (int g = 0; g < 3; g++) {
            C acc[8];
#pragma unroll
            for (int i = 0; i < 8; i++) acc[i] = cmake<C>(0, 0);
            const int nterm = g == 0 ? 3 : (g == 1 ? 2 : 1);
#pragma unroll 1
            for (int j = 0; j < nterm; j++, u++) {
                const int st = (int)(u % S);
                const bool ok = prc::tma::wait(&bars[st], (uint32_t)((u / S) & 1));
                const bool failed = __syncthreads_or(!ok);
                if (PP && !failed && tid == 0 && u > 0) {
                    // every thread is past unit u - 1: its stage takes unit u - 1 + S
                    prc::tma::fence_proxy_async();
                    issue(u - 1 + S);
                }
                if (failed) {
                    if (tid == 0) {
                        atomicOr(&prc::g_fault, prc::tma::FAULT_WAIT_TIMEOUT);
                        // units u .. u + S - 1 (u + S - 2 under PP) were issued and may be in flight
                        for (int d = 0; d < (PP ? S - 1 : S); d++) {
                            const int64_t uu = u + d;
                            if ((int64_t)blockIdx.x + (uu / 6) * gridDim.x >= ntiles) break;
                            prc::tma::wait(&bars[uu % S], (uint32_t)((uu / S) & 1));
                        }
                    }
                    return;
                }
                const int q = (int)(u % 6);
                C* sb = stages + st * TS::ELEMS;
                // D02 on the z-Nyquist column: the x-Nyquist mode of the line, (-1)^x l02
                const bool sub02 = q == 3 && znyq && l02 != nullptr;
                C v[8];
                // y factor before the transform (q is the same for the whole CTA, so each case is one
                // uniform branch): k_y^2 (D11), s_y (D01, D12), k_y on the Nyquist index only (D12, z Nyquist)
                if (q == 2) {
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        const T ky = kytab[t + i * TL];
                        v[i] = cscale(sb[(t + i * TL) * B + col], ky * ky);
                    }
                } else if (q == 1 || q == 4) {
                    const bool on_nyq = q == 4 && znyq;
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        const int iy = t + i * TL;
                        const T yf = (on_nyq == (iy == ynyq)) ? kytab[iy] : (T)0;
                        v[i] = cscale(sb[iy * B + col], yf);
                    }
                } else if (sub02) {
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        const C x = l02[t + i * TL];
                        v[i] = cmake<C>(xsign * x.x, xsign * x.y);
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 8; i++) v[i] = sb[(t + i * TL) * B + col];
                }
                if constexpr (PP) {
                    // scratch first: the stage is written only by the second exchange, behind the first
                    // exchange's barrier, when every thread has read its points from it
                    if constexpr (PADX) fft_regs_pp<C, N, +1>(v, t, xscr, paddr, sb, addr, tw);
                    else fft_regs_pp<C, N, +1>(v, t, xscr, sb, addr, tw);
                } else {
                    __syncthreads();
                    fft_regs<C, N, +1>(v, t, sb, addr, tw);
                    if (tid == 0) {
                        prc::tma::fence_proxy_async();
                        issue(u + S);
                    }
                }
                if (q == 1 && q01 != nullptr && iz < s.ncols) {
                    // D01 at the x and y Nyquist indices: q01[iz] (-1)^(x + y)
                    const C c = q01[iz];
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        const T sg = ((t + i * TL) & 1) ? -xsign : xsign;
                        v[i] = cmake<C>(v[i].x + sg * c.x, v[i].y + sg * c.y);
                    }
                }
                // weight at this point: f00 x0^2 | f01 x0 x1 | f11 x1^2 | f02 x0 s_z (1 where substituted) |
                // f12 x1 k_z | f22 k_z^2
                if (q == 1 || q == 2 || q == 4) {
                    const T f = (T)(q == 1 ? h.f[1] : q == 2 ? h.f[3] : h.f[4]);
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        const T x1 = x1tab[t + i * TL];
                        const T w = q == 1 ? f * (x0 * x1) : q == 2 ? f * (x1 * x1) : f * x1 * kz;
                        acc[i] = cmake<C>(acc[i].x + w * v[i].x, acc[i].y + w * v[i].y);
                    }
                } else {
                    const T f = (T)(q == 0 ? h.f[0] : q == 3 ? h.f[2] : h.f[5]);
                    const T w = q == 0 ? f * (x0 * x0) : q == 3 ? f * x0 * (sub02 ? (T)1 : sz) : f * (kz * kz);
#pragma unroll
                    for (int i = 0; i < 8; i++) acc[i] = cmake<C>(acc[i].x + w * v[i].x, acc[i].y + w * v[i].y);
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

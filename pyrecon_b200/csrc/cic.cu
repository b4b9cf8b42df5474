// Cloud-in-cell painting (deterministic, sort-by-cell) and the particle gathers.
//
// Paint pipeline for N particles on an n0 x n1 x n2 mesh (prc_assign_cic):
//   1. keys:     per particle, wrap / box check / index transform exactly as numpy does it
//                (pyrecon/mesh.py:546-555), base cell key = (ix*n1 + iy)*n2 + iz (mesh.c:35-37);
//   2. sort:     stable LSD radix sort of (key, particle id), <= 9-bit digits;
//   3. payload:  particles gathered in sorted order as (dx, dy, dz, w) in the mesh dtype, with
//                the post-modulo fractional offsets of src/mesh.c:45-47;
//   4. columns:  start offset of every (ix, iy) column in the sorted array;
//   5. pull:     one warp per OUTPUT column (X, Y) sums, in a fixed order, the contributions of
//                the four base columns (X-cx, Y-cy) in FP64 shared memory: per 32-particle chunk
//                the k-th particles of the runs of equal iz add in round k (distinct cells per
//                round), the z = iz terms before the z = iz + 1 terms, so every cell sums its
//                particles in sorted order.  Same inputs -> same bits, run after run.
#include "common.cuh"

#include <cuda.h>

#include <limits.h>

#include <algorithm>
#include <map>
#include <mutex>

namespace prc {

// ---------------------------------------------------------------------------------------------
// Radix sort of (uint32 key, uint32 value), stable
// ---------------------------------------------------------------------------------------------
namespace rsort {

constexpr int THREADS = 256;
constexpr int WARPS = THREADS / 32;
constexpr int ITEMS = 16;                      // per thread
constexpr int TILE = THREADS * ITEMS;          // 4096 items per tile
constexpr int MAXBITS = 9;
constexpr int MAXRADIX = 1 << MAXBITS;
static_assert(2 * THREADS >= MAXRADIX, "downsweep scans two digits per thread");

__global__ void __launch_bounds__(THREADS) upsweep(const uint32_t* __restrict__ keys, int64_t n, int shift,
                                                   int radix, int ntiles, uint32_t* __restrict__ hist) {
    __shared__ uint32_t cnt[MAXRADIX];
    const uint32_t mask = (uint32_t)radix - 1;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        for (int d = threadIdx.x; d < radix; d += THREADS) cnt[d] = 0;
        __syncthreads();
        int64_t base = (int64_t)tile * TILE;
        for (int k = 0; k < ITEMS; k++) {
            int64_t i = base + (int64_t)k * THREADS + threadIdx.x;
            if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & mask], 1u);
        }
        __syncthreads();
        for (int d = threadIdx.x; d < radix; d += THREADS) hist[(int64_t)d * ntiles + tile] = cnt[d];
        __syncthreads();
    }
}

// Exclusive scan of `count` uint32 in place, by one block per SCAN_TILE chunk + one pass over
// the chunk totals.  Sizes here stay below 2^32 (digit counts of < 2^32 items).
constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* s_warp, uint32_t* total) {
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        s_warp[lane] = w;   // inclusive warp-total prefix
    }
    __syncthreads();
    uint32_t before = warp > 0 ? s_warp[warp - 1] : 0u;
    uint32_t res = before + x - v;
    if (total) *total = s_warp[(blockDim.x >> 5) - 1];
    __syncthreads();
    return res;
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_tiles(uint32_t* __restrict__ data, int64_t count,
                                                           uint32_t* __restrict__ tile_sums) {
    __shared__ uint32_t s_warp[32];
    int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS], sum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        v[k] = base + k < count ? data[base + k] : 0u;
        sum += v[k];
    }
    uint32_t total;
    uint32_t run = block_exclusive_scan(sum, s_warp, &total);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        if (base + k < count) data[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_totals(uint32_t* __restrict__ sums, int count) {
    __shared__ uint32_t s_warp[32];
    uint32_t carry = 0;
    for (int base = 0; base < count; base += SCAN_THREADS) {
        int i = base + threadIdx.x;
        uint32_t v = i < count ? sums[i] : 0u;
        uint32_t total;
        uint32_t ex = block_exclusive_scan(v, s_warp, &total);
        if (i < count) sums[i] = carry + ex;
        carry += total;
    }
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_add(uint32_t* __restrict__ data, int64_t count,
                                                         const uint32_t* __restrict__ tile_sums) {
    int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
    uint32_t add = tile_sums[blockIdx.x];
    for (int k = threadIdx.x; k < SCAN_TILE; k += SCAN_THREADS)
        if (base + k < count) data[base + k] += add;
}

// Stable scatter of one tile: each warp ranks its contiguous 512-item slice chunk by chunk
// (ballots group equal digits; lanes keep input order), warps are then offset by the
// counts of the warps before them.  The tile is first reordered by digit in shared memory, so the
// writes to the output run over consecutive addresses of each digit's range (coalesced) instead of
// scattering single items; the tile's base in each digit's range comes from the scanned histogram.
__global__ void __launch_bounds__(THREADS, 3) downsweep(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                     uint32_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                     int64_t n, int shift, int radix, int ntiles,
                                                     const uint32_t* __restrict__ offsets) {
    extern __shared__ uint32_t smem[];
    uint32_t* s_key = smem;                       // TILE
    uint32_t* s_val = s_key + TILE;               // TILE
    uint32_t* s_rank = s_val + TILE;              // TILE: rank in the warp's digit group, then local index
    uint32_t* s_cnt = s_rank + TILE;              // WARPS * radix
    uint32_t* s_loc = s_cnt + WARPS * radix;      // radix: first local index of each digit
    uint32_t* s_glob = s_loc + radix;             // radix: the tile's first output index of each digit
    __shared__ uint32_t s_warp[32];
    const uint32_t mask = (uint32_t)radix - 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    constexpr int SLICE = TILE / WARPS;

    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int64_t base = (int64_t)tile * TILE;
        int valid = (int)min((int64_t)TILE, n - base);
        for (int k = threadIdx.x; k < TILE; k += THREADS) {
            if (k < valid) {
                s_key[k] = kin[base + k];
                s_val[k] = vin[base + k];
            }
        }
        for (int k = threadIdx.x; k < WARPS * radix; k += THREADS) s_cnt[k] = 0u;
        __syncthreads();
        uint32_t* cnt = s_cnt + warp * radix;
        for (int c = 0; c < SLICE; c += 32) {
            int k = warp * SLICE + c + lane;
            bool ok = k < valid;
            uint32_t d = ok ? (s_key[k] >> shift) & mask : 0u;
            // lanes with the same digit (the set __match_any_sync returns), from one vote per digit bit and
            // one for validity: short-latency votes instead of the match instruction
            const uint32_t okm = __ballot_sync(0xffffffffu, ok);
            uint32_t peers = ok ? okm : ~okm;
#pragma unroll
            for (int b = 0; b < MAXBITS; b++) {
                const bool bit = (d >> b) & 1u;
                const uint32_t v = __ballot_sync(0xffffffffu, bit);
                peers &= bit ? v : ~v;
            }
            uint32_t before = ok ? cnt[d] : 0u;
            __syncwarp();
            if (ok) {
                s_rank[k] = before + __popc(peers & lt);
                if ((peers & lt) == 0u) cnt[d] = before + __popc(peers);
            }
            __syncwarp();
        }
        __syncthreads();
        // per digit: offsets of the warps within the digit's group, and the group size
        uint32_t tot[2] = {0u, 0u};
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int d = 2 * threadIdx.x + j;
            if (d < radix) {
                uint32_t run = 0u;
                for (int w = 0; w < WARPS; w++) {
                    uint32_t c = s_cnt[w * radix + d];
                    s_cnt[w * radix + d] = run;
                    run += c;
                }
                tot[j] = run;
                s_glob[d] = offsets[(int64_t)d * ntiles + tile];
            }
        }
        // local start of every digit: exclusive scan of the group sizes (2 digits per thread)
        const uint32_t ex = block_exclusive_scan(tot[0] + tot[1], s_warp, nullptr);
        if (2 * threadIdx.x < radix) s_loc[2 * threadIdx.x] = ex;
        if (2 * threadIdx.x + 1 < radix) s_loc[2 * threadIdx.x + 1] = ex + tot[0];
        __syncthreads();
        // local index of every item (its own slot of s_rank), then the reorder through registers
        uint32_t rk[ITEMS], rv[ITEMS], ri[ITEMS];
#pragma unroll
        for (int j = 0; j < ITEMS; j++) {
            const int k = j * THREADS + threadIdx.x;
            if (k < valid) {
                const uint32_t key = s_key[k];
                const uint32_t d = (key >> shift) & mask;
                rk[j] = key;
                rv[j] = s_val[k];
                ri[j] = s_loc[d] + s_cnt[(k / SLICE) * radix + d] + s_rank[k];
            }
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < ITEMS; j++) {
            const int k = j * THREADS + threadIdx.x;
            if (k < valid) {
                s_key[ri[j]] = rk[j];
                s_val[ri[j]] = rv[j];
            }
        }
        __syncthreads();
        for (int k = threadIdx.x; k < valid; k += THREADS) {
            const uint32_t key = s_key[k];
            const uint32_t d = (key >> shift) & mask;
            const uint32_t pos = s_glob[d] + ((uint32_t)k - s_loc[d]);
            kout[pos] = key;
            vout[pos] = s_val[k];
        }
        __syncthreads();
    }
}

inline size_t downsweep_smem(int radix) { return (size_t)(3 * TILE + WARPS * radix + 2 * radix) * sizeof(uint32_t); }

// ---- one sweep per digit (decoupled look-back) ----
// The digit histograms of every pass come from one read of the keys; then each pass is one kernel whose
// CTAs take tiles in the order they start (a tile counter), rank a tile as the downsweep does, publish
// the tile's count of every digit, and find the tile's output offset for a digit by looking back over
// the tiles before it: a predecessor that has published its inclusive prefix ends the walk, one that has
// only published its count adds it and the walk goes on.  Status words: 2 flag bits (count / prefix)
// over a 30-bit value, so a sort of up to 2^30 - 1 items; larger ones take the reduce-then-scan passes.
// A predecessor always runs (it took its tile earlier) and publishes its counts before it looks back
// itself, so every wait ends; it is bounded all the same (WAIT_LIMIT_NS): one that runs out raises
// PRC_FLAG_DEVICE_WAIT in the caller's flags, which the kernels downstream honour.
constexpr uint32_t LB_VALUE = (1u << 30) - 1;
constexpr uint32_t LB_COUNT = 1u << 30, LB_PREFIX = 2u << 30;
constexpr int MAXPASS = 4;
constexpr uint64_t WAIT_LIMIT_NS = 200ull * 1000 * 1000;

// The look-back exchanges only the status words themselves (a count is the whole message, in the same
// word as its flag), so relaxed loads and stores at GPU scope suffice: no fence, and several loads can
// be in flight at once.
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
constexpr int LB_WINDOW = 8;    // predecessors read at once by a look-back step (per digit)
__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Digit counts of every pass (dbits-bit digits, npass of them) over all keys, added into hist[p * radix + d].
__global__ void __launch_bounds__(THREADS) digit_histograms(const uint32_t* __restrict__ keys, int64_t n, int dbits,
                                                            int npass, uint32_t* __restrict__ hist) {
    __shared__ uint32_t cnt[MAXPASS * MAXRADIX];
    const int radix = 1 << dbits;
    const uint32_t mask = (uint32_t)radix - 1;
    for (int i = threadIdx.x; i < npass * radix; i += THREADS) cnt[i] = 0u;
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * THREADS) {
        const uint32_t k = keys[i];
        for (int p = 0; p < npass; p++) atomicAdd(&cnt[p * radix + ((k >> (p * dbits)) & mask)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < npass * radix; i += THREADS)
        if (cnt[i]) atomicAdd(&hist[i], cnt[i]);
}

// One pass of the sort: the ranking and the shared-memory reorder of downsweep, the tile's offset in each
// digit's range from the look-back.  hist: this pass's digit counts; lookback (ntiles * radix) and
// *tile_counter zeroed before the launch.
__global__ void __launch_bounds__(THREADS, 3) onesweep(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                    uint32_t* __restrict__ kout, uint32_t* __restrict__ vout, int64_t n,
                                                    int shift, int radix, int ntiles, const uint32_t* __restrict__ hist,
                                                    uint32_t* lookback, uint32_t* tile_counter, int32_t* flags) {
    extern __shared__ uint32_t smem[];
    uint32_t* s_key = smem;                       // TILE
    uint32_t* s_val = s_key + TILE;               // TILE
    uint32_t* s_rank = s_val + TILE;              // TILE: rank in the warp's digit group, then local index
    uint32_t* s_cnt = s_rank + TILE;              // WARPS * radix
    uint32_t* s_loc = s_cnt + WARPS * radix;      // radix: first local index of each digit
    uint32_t* s_glob = s_loc + radix;             // radix: the tile's first output index of each digit
    uint32_t* s_base = s_glob + radix;            // radix: first output index of each digit (all tiles)
    __shared__ uint32_t s_warp[32];
    __shared__ int s_tile;
    const uint32_t mask = (uint32_t)radix - 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    constexpr int SLICE = TILE / WARPS;
    {
        const uint32_t g0 = 2 * threadIdx.x < radix ? hist[2 * threadIdx.x] : 0u;
        const uint32_t g1 = 2 * threadIdx.x + 1 < radix ? hist[2 * threadIdx.x + 1] : 0u;
        const uint32_t ex = block_exclusive_scan(g0 + g1, s_warp, nullptr);
        if (2 * threadIdx.x < radix) s_base[2 * threadIdx.x] = ex;
        if (2 * threadIdx.x + 1 < radix) s_base[2 * threadIdx.x + 1] = ex + g0;
    }
    bool gave_up = false;
    for (;;) {
        if (threadIdx.x == 0) s_tile = (int)atomicAdd(tile_counter, 1u);
        __syncthreads();
        const int tile = s_tile;
        if (tile >= ntiles) break;
        int64_t base = (int64_t)tile * TILE;
        int valid = (int)min((int64_t)TILE, n - base);
        for (int k = threadIdx.x; k < TILE; k += THREADS) {
            if (k < valid) {
                s_key[k] = kin[base + k];
                s_val[k] = vin[base + k];
            }
        }
        for (int k = threadIdx.x; k < WARPS * radix; k += THREADS) s_cnt[k] = 0u;
        for (int d = threadIdx.x; d < radix; d += THREADS) s_glob[d] = 0u;
        __syncthreads();
        // the tile's digit counts (in s_glob until the look-back), published before the ranking so the tiles
        // after this one can look back past it early
        for (int k = threadIdx.x; k < valid; k += THREADS) atomicAdd(&s_glob[(s_key[k] >> shift) & mask], 1u);
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int d = 2 * threadIdx.x + j;
            if (d < radix) st_relaxed(lookback + (int64_t)tile * radix + d, (tile == 0 ? LB_PREFIX : LB_COUNT) | s_glob[d]);
        }
        uint32_t* cnt = s_cnt + warp * radix;
        for (int c = 0; c < SLICE; c += 32) {
            int k = warp * SLICE + c + lane;
            bool ok = k < valid;
            uint32_t d = ok ? (s_key[k] >> shift) & mask : 0u;
            const uint32_t okm = __ballot_sync(0xffffffffu, ok);
            uint32_t peers = ok ? okm : ~okm;
#pragma unroll
            for (int b = 0; b < MAXBITS; b++) {
                const bool bit = (d >> b) & 1u;
                const uint32_t v = __ballot_sync(0xffffffffu, bit);
                peers &= bit ? v : ~v;
            }
            uint32_t before = ok ? cnt[d] : 0u;
            __syncwarp();
            if (ok) {
                s_rank[k] = before + __popc(peers & lt);
                if ((peers & lt) == 0u) cnt[d] = before + __popc(peers);
            }
            __syncwarp();
        }
        __syncthreads();
        uint32_t tot[2] = {0u, 0u};
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int d = 2 * threadIdx.x + j;
            if (d < radix) {
                uint32_t run = 0u;
                for (int w = 0; w < WARPS; w++) {
                    uint32_t c = s_cnt[w * radix + d];
                    s_cnt[w * radix + d] = run;
                    run += c;
                }
                tot[j] = run;
            }
        }
        {
            // each digit's offset in the output: walk back over the predecessors LB_WINDOW at a time (both
            // digits' words read together), adding counts up to the first inclusive prefix; a word not yet
            // published stops the walk there and it is read again (bounded)
            int t[2] = {tile - 1, tile - 1};
            uint32_t excl[2] = {0u, 0u};
            bool done[2] = {tile == 0 || 2 * (int)threadIdx.x >= radix, tile == 0 || 2 * (int)threadIdx.x + 1 >= radix};
            uint64_t t0 = 0;
            while (!(done[0] && done[1])) {
                uint32_t w[2][LB_WINDOW];
#pragma unroll
                for (int j = 0; j < 2; j++)
#pragma unroll
                    for (int i = 0; i < LB_WINDOW; i++)
                        w[j][i] = !done[j] && t[j] - i >= 0
                                      ? ld_relaxed(lookback + (int64_t)(t[j] - i) * radix + 2 * threadIdx.x + j)
                                      : LB_PREFIX;
                bool stalled = false;
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    if (done[j]) continue;
                    int used = 0;
                    bool fin = false;
#pragma unroll
                    for (int i = 0; i < LB_WINDOW; i++) {
                        if (fin || used < i) continue;                 // stopped earlier in the window
                        if ((w[j][i] & ~LB_VALUE) == 0u) continue;     // not published: the walk waits here
                        excl[j] += w[j][i] & LB_VALUE;
                        used = i + 1;
                        fin = (w[j][i] & LB_PREFIX) != 0u;
                    }
                    t[j] -= used;
                    done[j] = fin;
                    if (!fin && used < LB_WINDOW) stalled = true;
                }
                if (stalled) {
                    const uint64_t now = global_ns();
                    if (t0 == 0) t0 = now;
                    else if (now - t0 > WAIT_LIMIT_NS) {
                        gave_up = true;
                        break;
                    }
                    __nanosleep(32);
                }
            }
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const int d = 2 * threadIdx.x + j;
                if (d < radix) {
                    if (tile > 0) st_relaxed(lookback + (int64_t)tile * radix + d, LB_PREFIX | (excl[j] + tot[j]));
                    s_glob[d] = s_base[d] + excl[j];
                }
            }
        }
        const uint32_t ex = block_exclusive_scan(tot[0] + tot[1], s_warp, nullptr);
        if (2 * threadIdx.x < radix) s_loc[2 * threadIdx.x] = ex;
        if (2 * threadIdx.x + 1 < radix) s_loc[2 * threadIdx.x + 1] = ex + tot[0];
        __syncthreads();
        uint32_t rk[ITEMS], rv[ITEMS], ri[ITEMS];
#pragma unroll
        for (int j = 0; j < ITEMS; j++) {
            const int k = j * THREADS + threadIdx.x;
            if (k < valid) {
                const uint32_t key = s_key[k];
                const uint32_t d = (key >> shift) & mask;
                rk[j] = key;
                rv[j] = s_val[k];
                ri[j] = s_loc[d] + s_cnt[(k / SLICE) * radix + d] + s_rank[k];
            }
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < ITEMS; j++) {
            const int k = j * THREADS + threadIdx.x;
            if (k < valid) {
                s_key[ri[j]] = rk[j];
                s_val[ri[j]] = rv[j];
            }
        }
        __syncthreads();
        for (int k = threadIdx.x; k < valid; k += THREADS) {
            const uint32_t key = s_key[k];
            const uint32_t d = (key >> shift) & mask;
            const uint32_t pos = s_glob[d] + ((uint32_t)k - s_loc[d]);
            kout[pos] = key;
            vout[pos] = s_val[k];
        }
        __syncthreads();
    }
    if (gave_up) atomicOr(flags, PRC_FLAG_DEVICE_WAIT);
}

inline size_t onesweep_smem(int radix) { return downsweep_smem(radix) + (size_t)radix * sizeof(uint32_t); }

inline int num_tiles(int64_t n) { return (int)((n + TILE - 1) / TILE); }

inline int64_t scan_count(int64_t n, int radix) { return (int64_t)num_tiles(n) * radix; }

inline int scan_blocks(int64_t count) { return (int)((count + SCAN_TILE - 1) / SCAN_TILE); }

// Bytes of scratch for sorting n items with the largest digit: the reduce-then-scan passes' tile
// histograms and scan tile sums, or the one-sweep passes' digit counts, tile counters and look-back
// words (the larger of the two).
inline size_t scratch_bytes(int64_t n) {
    int64_t c = scan_count(n, MAXRADIX);
    const int64_t rts = c + scan_blocks(c) + 64;
    const int64_t one = (int64_t)MAXPASS * MAXRADIX + 64 + c;
    return (size_t)std::max(rts, one) * sizeof(uint32_t);
}

// Sorts (k0, v0) by the low `bits` bits of the key.  Ping-pongs with (k1, v1); returns through
// *kres / *vres which pair holds the result.  One kernel per digit (onesweep) up to 2^30 - 1 items
// (run-time knob sort_onesweep = 0: the reduce-then-scan passes, the same result), else per digit a
// histogram pass, a scan and a scatter pass.  flags: the caller's status word (PRC_FLAG_DEVICE_WAIT).
int sort_pairs(uint32_t* k0, uint32_t* v0, uint32_t* k1, uint32_t* v1, int64_t n, int bits, uint32_t* scratch,
               uint32_t** kres, uint32_t** vres, int32_t* flags, cudaStream_t st) {
    *kres = k0;
    *vres = v0;
    if (n <= 1 || bits <= 0) return PRC_OK;
    int npass = (bits + MAXBITS - 1) / MAXBITS;
    int dbits = (bits + npass - 1) / npass;
    int radix = 1 << dbits;
    int ntiles = num_tiles(n);
    int64_t count = (int64_t)ntiles * radix;
    int sms = device_sm_count();
    uint32_t *ka = k0, *va = v0, *kb = k1, *vb = v1;
    if (n <= (int64_t)LB_VALUE && npass <= MAXPASS && tune_get("sort_onesweep", 0, 1) != 0) {
        static bool attr_set1 = false;
        if (!attr_set1) {
            cudaFuncSetAttribute(onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)onesweep_smem(MAXRADIX));
            attr_set1 = true;
        }
        uint32_t* hist = scratch;                                   // MAXPASS * MAXRADIX
        uint32_t* counters = scratch + MAXPASS * MAXRADIX;          // MAXPASS (64 words)
        uint32_t* lookback = counters + 64;                         // ntiles * radix
        if (cudaMemsetAsync(scratch, 0, (MAXPASS * MAXRADIX + 64) * sizeof(uint32_t), st) != cudaSuccess)
            return PRC_ERR_CUDA;
        const int hgrid = (int)std::max<int64_t>(1, std::min<int64_t>((n + THREADS - 1) / THREADS, (int64_t)sms * 4));
        PRC_LAUNCH_B("sort_histograms", st, 4.0 * n, digit_histograms<<<hgrid, THREADS, 0, st>>>(ka, n, dbits, npass, hist));
        const int grid = min(ntiles, sms * 3);
        for (int p = 0; p < npass; p++) {
            if (cudaMemsetAsync(lookback, 0, (size_t)count * sizeof(uint32_t), st) != cudaSuccess) return PRC_ERR_CUDA;
            PRC_LAUNCH_B("sort_onesweep", st, 16.0 * n + 4.0 * radix,
                         onesweep<<<grid, THREADS, onesweep_smem(radix), st>>>(ka, va, kb, vb, n, p * dbits, radix, ntiles,
                                                                              hist + p * radix, lookback, counters + p, flags));
            PRC_CHECK_LAUNCH();
            uint32_t* t;
            t = ka; ka = kb; kb = t;
            t = va; va = vb; vb = t;
        }
        *kres = ka;
        *vres = va;
        return PRC_OK;
    }
    uint32_t* hist = scratch;
    uint32_t* tsums = scratch + count;
    int grid = min(ntiles, sms * 8);
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(downsweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)downsweep_smem(MAXRADIX));
        attr_set = true;
    }
    for (int p = 0; p < npass; p++) {
        int shift = p * dbits;
        PRC_LAUNCH_B("sort_upsweep", st, 4.0 * n + 4.0 * count, upsweep<<<grid, THREADS, 0, st>>>(ka, n, shift, radix, ntiles, hist));
        int sb = scan_blocks(count);
        PRC_LAUNCH_B("sort_scan", st, 8.0 * count, scan_tiles<<<sb, SCAN_THREADS, 0, st>>>(hist, count, tsums));
        PRC_LAUNCH("sort_scan", st, scan_totals<<<1, SCAN_THREADS, 0, st>>>(tsums, sb));
        PRC_LAUNCH_B("sort_scan", st, 8.0 * count, scan_add<<<sb, SCAN_THREADS, 0, st>>>(hist, count, tsums));
        PRC_LAUNCH_B("sort_downsweep", st, 16.0 * n + 4.0 * count, downsweep<<<grid, THREADS, downsweep_smem(radix), st>>>(ka, va, kb, vb, n, shift, radix, ntiles, hist));
        PRC_CHECK_LAUNCH();
        uint32_t* t;
        t = ka; ka = kb; kb = t;
        t = va; va = vb; vb = t;
    }
    *kres = ka;
    *vres = va;
    return PRC_OK;
}

}  // namespace rsort

// ---------------------------------------------------------------------------------------------
// Particle helpers
// ---------------------------------------------------------------------------------------------

template <typename T> __device__ __forceinline__ bool finite3(T a, T b, T c) {
    return isfinite(a) && isfinite(b) && isfinite(c);
}

// Box check of pyrecon/mesh.py:549-551 (inclusive on both faces), compared in the promoted type.
template <typename P, typename F> __device__ __forceinline__ bool in_box(P p, const BoxGeom& g, int d) {
    typedef typename promote<P, F>::type T;
    F bs = (F)g.boxsize[d], bc = (F)g.boxcenter[d];
    F half = rn_div(bs, (F)2);
    F low = rn_sub(bc, half), high = rn_add(bc, half);
    return (T)p >= (T)low && (T)p <= (T)high;
}

// Index-space coordinates (mesh dtype F) of particle i, after the optional wrap; flags
// out-of-box / non-finite.  Returns false when the particle is invalid.
template <typename P, typename F>
__device__ __forceinline__ bool particle_index_of(const P (&p)[3], const BoxGeom& g, int wrap, F q[3], int* bad) {
    typedef typename promote<P, F>::type T;
    if (wrap) {
        T w[3];
#pragma unroll
        for (int d = 0; d < 3; d++) w[d] = wrap_position<P, F>(p[d], g, d);
        if (!finite3(w[0], w[1], w[2])) {
            *bad |= PRC_FLAG_NONFINITE;
            return false;
        }
#pragma unroll
        for (int d = 0; d < 3; d++) q[d] = index_coord<T, F>(w[d], g, d);
    } else {
        bool inside = in_box<P, F>(p[0], g, 0) && in_box<P, F>(p[1], g, 1) && in_box<P, F>(p[2], g, 2);
        if (!inside) {
            *bad |= PRC_FLAG_OUT_OF_BOX;   // NaN compares false: reported as out of box, as numpy does
            return false;
        }
        if (!finite3(p[0], p[1], p[2])) {
            *bad |= PRC_FLAG_NONFINITE;
            return false;
        }
#pragma unroll
        for (int d = 0; d < 3; d++) q[d] = index_coord<P, F>(p[d], g, d);
    }
    return true;
}

template <typename P, typename F>
__device__ __forceinline__ bool particle_index(const P* __restrict__ pos, int64_t i, const BoxGeom& g, int wrap,
                                               F q[3], int* bad) {
    const P p[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    return particle_index_of<P, F>(p, g, wrap, q, bad);
}

// Base cell: C (int) truncation, then modulo n (src/mesh.c:35-37); kept in [0, n) for any input.
template <typename F> __device__ __forceinline__ int base_cell(F q, int n) {
    int b = (int)q;
    b %= n;
    return b < 0 ? b + n : b;
}

__device__ __forceinline__ void raise_flags(int32_t* flags, int bad) {
    // one atomic per warp that saw a problem
    unsigned m = __ballot_sync(0xffffffffu, bad != 0);
    int all = bad;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) all |= __shfl_xor_sync(0xffffffffu, all, o);
    if (m && (threadIdx.x & 31) == __ffs(m) - 1) atomicOr(flags, all);
}

// ---------------------------------------------------------------------------------------------
// Paint kernels
// ---------------------------------------------------------------------------------------------

template <typename P, typename F, typename W>
__global__ void __launch_bounds__(256) paint_keys(const P* __restrict__ pos, const W* __restrict__ weights, int64_t n,
                                                  BoxGeom g, int wrap, uint32_t* __restrict__ keys,
                                                  uint32_t* __restrict__ ids, int32_t* __restrict__ flags) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t start = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    // iterate a warp-uniform number of times so raise_flags' warp collectives see every lane
    int64_t nround = (n + stride - 1) / stride;
    for (int64_t r = 0; r < nround; r++) {
        int64_t i = start + r * stride;
        int bad = 0;
        if (i < n) {
            F q[3];
            uint32_t key = 0;
            if (particle_index<P, F>(pos, i, g, wrap, q, &bad)) {
                if (weights != nullptr && !isfinite((double)weights[i])) bad |= PRC_FLAG_NONFINITE;
                int ix = base_cell(q[0], g.n[0]), iy = base_cell(q[1], g.n[1]), iz = base_cell(q[2], g.n[2]);
                key = ((uint32_t)ix * (uint32_t)g.n[1] + (uint32_t)iy) * (uint32_t)g.n[2] + (uint32_t)iz;
            }
            keys[i] = key;
            ids[i] = (uint32_t)i;
        }
        raise_flags(flags, bad);
    }
}

// (dx, dy, dz, w) of every particle in sorted order, in the mesh dtype F; the fractional
// offsets are taken after the modulo as src/mesh.c:45-47 does.
template <typename F> struct alignas(4 * sizeof(F)) Payload { F t[3]; F w; };

// sorted_pos (optional): the positions themselves in the same order (pos of particle order[i] at i), so a
// later read-out in cell order streams them instead of gathering through the permutation.
template <typename P, typename F, typename W>
__global__ void __launch_bounds__(256) paint_payload(const P* __restrict__ pos, const W* __restrict__ weights, int64_t n,
                                                     BoxGeom g, int wrap, const uint32_t* __restrict__ order,
                                                     Payload<F>* __restrict__ out, P* __restrict__ sorted_pos,
                                                     const int32_t* __restrict__ flags) {
    if (*flags) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t id = order[i];
        F q[3];
        int bad = 0;
        Payload<F> pl;
        particle_index<P, F>(pos, id, g, wrap, q, &bad);
#pragma unroll
        for (int d = 0; d < 3; d++) pl.t[d] = rn_sub(q[d], (F)base_cell(q[d], g.n[d]));
        pl.w = weights != nullptr ? (F)weights[id] : (F)1;
        out[i] = pl;
        if (sorted_pos != nullptr) {
#pragma unroll
            for (int d = 0; d < 3; d++) sorted_pos[3 * i + d] = pos[3 * id + d];
        }
    }
}

// col_start[c] = first sorted index whose column (key / n2) is >= c, for c in [0, ncol].
__global__ void column_starts(const uint32_t* __restrict__ keys, int64_t n, int n2, int64_t ncol,
                              uint32_t* __restrict__ col_start, const int32_t* __restrict__ flags) {
    if (*flags) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t col = i < n ? (int64_t)(keys[i] / (uint32_t)n2) : ncol;
        int64_t prev = i > 0 ? (int64_t)(keys[i - 1] / (uint32_t)n2) : -1;
        for (int64_t c = prev + 1; c <= col; c++) col_start[c] = (uint32_t)i;
    }
}

constexpr int PULL_WARPS = 4;

template <typename F>
__global__ void __launch_bounds__(PULL_WARPS * 32) paint_pull(const uint32_t* __restrict__ keys,
                                                              const Payload<F>* __restrict__ payload,
                                                              const uint32_t* __restrict__ col_start, Dims dims,
                                                              int accumulate, double* __restrict__ mesh,
                                                              double* __restrict__ column_sums,
                                                              const int32_t* __restrict__ flags) {
    extern __shared__ double s_col[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n0 = dims.n[0], n1 = dims.n[1], n2 = dims.n[2];
    double* col = s_col + (size_t)warp * n2;
    const int64_t ncol = (int64_t)n0 * n1;
    if (*flags) {
        // bad catalogue: an accumulated mesh is left as it was, a fresh one comes out zero
        if (!accumulate)
            for (int64_t c = (int64_t)blockIdx.x * PULL_WARPS + warp; c < ncol; c += (int64_t)gridDim.x * PULL_WARPS) {
                for (int z = lane; z < n2; z += 32) mesh[c * n2 + z] = 0.;
                if (column_sums != nullptr && lane == 0) column_sums[c] = 0.;
            }
        return;
    }
    for (int64_t c = (int64_t)blockIdx.x * PULL_WARPS + warp; c < ncol; c += (int64_t)gridDim.x * PULL_WARPS) {
        const int X = (int)(c / n1), Y = (int)(c % n1);
        for (int z = lane; z < n2; z += 32) col[z] = 0.;
        __syncwarp();
        // base columns contributing corner (cx, cy) to this column, in a fixed order
#pragma unroll 1
        for (int s = 0; s < 4; s++) {
            const int cx = s >> 1, cy = s & 1;
            const int Xs = cx ? wrap_dn(X, n0) : X, Ys = cy ? wrap_dn(Y, n1) : Y;
            const int64_t src = (int64_t)Xs * n1 + Ys;
            const int64_t beg = col_start[src], end = col_start[src + 1];
            for (int64_t b0 = beg; b0 < end; b0 += 32) {
                const int64_t i = b0 + lane;
                const bool ok = i < end;
                int iz = INT_MAX;
                double a = 0., b = 0.;
                if (ok) {
                    iz = (int)(keys[i] % (uint32_t)n2);
                    const Payload<F> pl = payload[i];
                    const F wx = cx ? pl.t[0] : rn_sub((F)1, pl.t[0]);
                    const F wy = cy ? pl.t[1] : rn_sub((F)1, pl.t[1]);
                    const F wxy = rn_mul(wx, wy);
                    // ((wx * wy) * wz) * weight, the reference's evaluation order (mesh.c:55-62)
                    a = (double)rn_mul(rn_mul(wxy, rn_sub((F)1, pl.t[2])), pl.w);
                    b = (double)rn_mul(rn_mul(wxy, pl.t[2]), pl.w);
                }
                // runs of equal iz (keys are sorted within a column): the r-th particle of every run adds
                // in round r, so the lanes of a round write distinct cells and every cell sums its
                // particles in their sorted order; a's (cell iz) and b's (cell iz + 1) in separate phases
                const int pz = __shfl_up_sync(0xffffffffu, iz, 1);
                const uint32_t heads = __ballot_sync(0xffffffffu, ok && (lane == 0 || pz != iz));
                const uint32_t upto = heads & ((2u << lane) - 1u);       // lane 31: every head
                const int rank = ok ? lane - (31 - __clz(upto)) : 0;
                const int rmax = __reduce_max_sync(0xffffffffu, (unsigned)rank);
                const int iz1 = iz + 1 == n2 ? 0 : iz + 1;
                for (int r = 0; r <= rmax; r++) {
                    if (ok && rank == r) col[iz] += a;
                    __syncwarp();
                }
                for (int r = 0; r <= rmax; r++) {
                    if (ok && rank == r) col[iz1] += b;
                    __syncwarp();
                }
            }
        }
        double* dst = mesh + c * (int64_t)n2;
        double part = 0.;
        for (int z = lane; z < n2; z += 32) {
            double v = col[z];
            if (accumulate) v += dst[z];
            dst[z] = v;
            part += v;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if (column_sums != nullptr && lane == 0) column_sums[c] = part;
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------------------------
// Deterministic sum
// ---------------------------------------------------------------------------------------------
constexpr int SUM_THREADS = 256;
constexpr int SUM_BLOCKS = 512;

template <typename X>
__global__ void __launch_bounds__(SUM_THREADS) sum_partials(const X* __restrict__ x, int64_t n,
                                                            double* __restrict__ partial) {
    __shared__ double s[SUM_THREADS];
    double acc = 0.;
    for (int64_t i = (int64_t)blockIdx.x * SUM_THREADS + threadIdx.x; i < n; i += (int64_t)SUM_BLOCKS * SUM_THREADS)
        acc += x[i];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = SUM_THREADS / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

__global__ void __launch_bounds__(SUM_THREADS) sum_final(const double* __restrict__ partial, double* __restrict__ out) {
    __shared__ double s[SUM_THREADS];
    double acc = 0.;
    for (int i = threadIdx.x; i < SUM_BLOCKS; i += SUM_THREADS) acc += partial[i];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = SUM_THREADS / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

// ---------------------------------------------------------------------------------------------
// Gathers
// ---------------------------------------------------------------------------------------------

// Fractional offset before the modulo (src/mesh.c:278-283) and base cells.
template <typename F> struct Cic {
    int lo[3], hi[3];
    F w[3][2];
};

template <typename F> __device__ __forceinline__ Cic<F> cic_setup(const F q[3], const int n[3]) {
    Cic<F> c;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        F t = rn_sub(q[d], (F)(int)q[d]);
        c.lo[d] = base_cell(q[d], n[d]);
        c.hi[d] = wrap_up(c.lo[d], n[d]);
        c.w[d][0] = rn_sub((F)1, t);
        c.w[d][1] = t;
    }
    return c;
}

__device__ __forceinline__ int64_t at3(const int n[3], int x, int y, int z) {
    return ((int64_t)x * n[1] + y) * n[2] + z;
}

// CIC read of one mesh: corners in (x, y, z) order with z fastest, each term
// ((m * w_x) * w_y) * w_z accumulated in order (src/mesh.c:294-301).
template <typename F> __device__ __forceinline__ F cic_read(const F* __restrict__ m, const Cic<F>& c, const int n[3]) {
    F acc = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int cx = (k >> 2) & 1, cy = (k >> 1) & 1, cz = k & 1;
        const F v = __ldg(m + at3(n, cx ? c.hi[0] : c.lo[0], cy ? c.hi[1] : c.lo[1], cz ? c.hi[2] : c.lo[2]));
        const F term = rn_mul(rn_mul(rn_mul(v, c.w[0][cx]), c.w[1][cy]), c.w[2][cz]);
        acc = k == 0 ? term : rn_add(acc, term);
    }
    return acc;
}

template <typename F> __device__ __forceinline__ typename vec4_of<F>::type load4(const typename vec4_of<F>::type* p);
template <> __device__ __forceinline__ float4 load4<float>(const float4* p) { return __ldg(p); }
template <> __device__ __forceinline__ double4 load4<double>(const double4* p) {
    const double2* q = (const double2*)p;
    const double2 a = __ldg(q), b = __ldg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

// Same as cic_read for the three components of an interleaved (x, y, z, 0) mesh at once: one
// vector load per corner, each component accumulated in the same order as cic_read.
template <typename F>
__device__ __forceinline__ void cic_read3(const typename vec4_of<F>::type* __restrict__ m, const Cic<F>& c,
                                          const int n[3], F out[3]) {
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int cx = (k >> 2) & 1, cy = (k >> 1) & 1, cz = k & 1;
        const typename vec4_of<F>::type v =
            load4<F>(m + at3(n, cx ? c.hi[0] : c.lo[0], cy ? c.hi[1] : c.lo[1], cz ? c.hi[2] : c.lo[2]));
        const F comp[3] = {v.x, v.y, v.z};
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const F term = rn_mul(rn_mul(rn_mul(comp[a], c.w[0][cx]), c.w[1][cy]), c.w[2][cz]);
            out[a] = k == 0 ? term : rn_add(out[a], term);
        }
    }
}

// Finite-difference gradient CIC read (src/mesh.c:187-266): corners in the order
// 000, 100, 010, 001, 110, 101, 011, 111; divided by 2 * boxsize / n in F.
template <typename F>
__device__ __forceinline__ void fd_read(const F* __restrict__ m, const Cic<F>& c, const int n[3], const F twocell[3],
                                        F out[3]) {
    // Along each axis the eight corners and their +-1 neighbours span four nodes, lo - 1, lo, hi, hi + 1
    // (periodic), indexed 0..3: corner c (0 or 1) sits at index c + 1, its neighbours at c and c + 2.  The
    // 32 distinct values are loaded once from precomputed plane, row and cell offsets; the arithmetic and
    // its order are those of the corner loop of src/mesh.c:187-266.
    const int64_t sx = (int64_t)n[1] * n[2];
    const int64_t X[4] = {wrap_dn(c.lo[0], n[0]) * sx, c.lo[0] * sx, c.hi[0] * sx, wrap_up(c.hi[0], n[0]) * sx};
    const int64_t Y[4] = {(int64_t)wrap_dn(c.lo[1], n[1]) * n[2], (int64_t)c.lo[1] * n[2], (int64_t)c.hi[1] * n[2],
                          (int64_t)wrap_up(c.hi[1], n[1]) * n[2]};
    const int Z[4] = {wrap_dn(c.lo[2], n[2]), c.lo[2], c.hi[2], wrap_up(c.hi[2], n[2])};
    F xv[4][2][2], yv[2][4][2], zv[2][2][4];   // [axis index 0..3 along the derivative's axis][corner][corner]
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 2; b++) {
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const bool core = e == 1 || e == 2;
                xv[e][a][b] = __ldg(m + X[e] + Y[a + 1] + Z[b + 1]);
                yv[a][e][b] = core ? F(0) : __ldg(m + X[a + 1] + Y[e] + Z[b + 1]);
                zv[a][b][e] = core ? F(0) : __ldg(m + X[a + 1] + Y[b + 1] + Z[e]);
            }
        }
    // core nodes (indices 1, 2 on every axis) come from the x table
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 2; b++)
#pragma unroll
            for (int e = 1; e < 3; e++) {
                yv[a][e][b] = xv[a + 1][e - 1][b];
                zv[a][b][e] = xv[a + 1][b][e - 1];
            }
    const int order[8] = {0, 4, 2, 1, 6, 5, 3, 7};   // (cx<<2 | cy<<1 | cz)
    F g[3] = {0, 0, 0};
#pragma unroll
    for (int kk = 0; kk < 8; kk++) {
        const int k = order[kk];
        const int cx = (k >> 2) & 1, cy = (k >> 1) & 1, cz = k & 1;
        const F wt = rn_mul(rn_mul(c.w[0][cx], c.w[1][cy]), c.w[2][cz]);
        const F gx = rn_mul(rn_sub(xv[cx + 2][cy][cz], xv[cx][cy][cz]), wt);
        const F gy = rn_mul(rn_sub(yv[cx][cy + 2][cz], yv[cx][cy][cz]), wt);
        const F gz = rn_mul(rn_sub(zv[cx][cy][cz + 2], zv[cx][cy][cz]), wt);
        if (kk == 0) {
            g[0] = gx; g[1] = gy; g[2] = gz;
        } else {
            g[0] = rn_add(g[0], gx); g[1] = rn_add(g[1], gy); g[2] = rn_add(g[2], gz);
        }
    }
#pragma unroll
    for (int a = 0; a < 3; a++) out[a] = rn_div(g[a], twocell[a]);
}

template <typename P, typename F>
__global__ void __launch_bounds__(256) read_cic_kernel(const F* __restrict__ mesh, BoxGeom g, const P* __restrict__ pos,
                                                       int64_t n, int wrap, P* __restrict__ out, int32_t* flags) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t nround = (n + stride - 1) / stride;
    for (int64_t r = 0; r < nround; r++) {
        int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x + r * stride;
        int bad = 0;
        if (i < n) {
            F q[3] = {0, 0, 0};
            P v = (P)NAN;
            if (particle_index<P, F>(pos, i, g, wrap, q, &bad)) v = (P)cic_read(mesh, cic_setup(q, g.n), g.n);
            out[i] = v;
        }
        raise_flags(flags, bad & PRC_FLAG_OUT_OF_BOX);   // non-finite only warns in the reference
    }
}

template <typename F> __host__ __forceinline__ void twocell_of(const BoxGeom& g, F out[3]) {
    for (int d = 0; d < 3; d++) out[d] = (F)(2.0 * (double)(F)g.boxsize[d] / (double)g.n[d]);
}

template <typename P, typename F>
__global__ void __launch_bounds__(256) read_fd_kernel(const F* __restrict__ mesh, BoxGeom g, F tc0, F tc1, F tc2,
                                                      const P* __restrict__ pos, int64_t n, int wrap,
                                                      P* __restrict__ out, int32_t* flags) {
    const F twocell[3] = {tc0, tc1, tc2};
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t nround = (n + stride - 1) / stride;
    for (int64_t r = 0; r < nround; r++) {
        int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x + r * stride;
        int bad = 0;
        if (i < n) {
            F q[3] = {0, 0, 0}, s[3] = {(F)NAN, (F)NAN, (F)NAN};
            if (particle_index<P, F>(pos, i, g, wrap, q, &bad)) fd_read(mesh, cic_setup(q, g.n), g.n, twocell, s);
#pragma unroll
            for (int a = 0; a < 3; a++) out[3 * i + a] = (P)s[a];
        }
        raise_flags(flags, bad & PRC_FLAG_OUT_OF_BOX);
    }
}

// Fused shifts.  Type flow of the reference (pyrecon/recon.py:255-325, multigrid.py:137-158):
// displacement read in F then cast to P (the shifts array has the positions' dtype); RSD in
// R = promoted type of (shifts, los); result cast back to P; positions - shifts in P, then
// wrapped in T = promote(P, F) when `wrap`; the output type O is chosen by the caller.
// PRC_READ_MINB: blocks per SM asked of the register allocator for the CIC shift read-out (its gathers
// are latency-bound: ncu shows long-scoreboard stalls first).  Measured per nmesh-512 reconstruction,
// with the next round's position loaded ahead: 1.73 ms free (100 registers, 2 blocks), 1.72 ms at 3
// blocks (80), 1.84 ms at 4 (64), and 5 blocks (48, a few spilled) slower still, so the default leaves
// the allocator free; the finite-difference read-out (48 loads a particle) always is.
#ifndef PRC_READ_MINB
#define PRC_READ_MINB 1
#endif

template <typename P, typename F, typename O, bool PHI, bool IL>
__global__ void __launch_bounds__(256, (PHI ? 1 : PRC_READ_MINB)) read_shifts_kernel(const F* __restrict__ m0, const F* __restrict__ m1,
                                                          const F* __restrict__ m2, BoxGeom g, F tc0, F tc1, F tc2,
                                                          const P* __restrict__ pos, int64_t n, double f,
                                                          int global_los, double l0, double l1, double l2, int field,
                                                          int shifted, int wrap, O* __restrict__ out, int32_t* flags,
                                                          const uint32_t* __restrict__ order,
                                                          const P* __restrict__ sorted_pos) {
    typedef typename promote<P, F>::type T;
    const F twocell[3] = {tc0, tc1, tc2};
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t nround = (n + stride - 1) / stride;
    // particles visited in `order` (cell-sorted, from the paint): neighbouring threads gather neighbouring
    // cells; each particle's result only depends on its own position, read from the paint's cell-ordered
    // copy when there is one (a stream, not a gather).  The next round's position (and output index) is
    // loaded one round ahead, so a round waits on memory only for its mesh gathers.
    const P* src = sorted_pos != nullptr ? sorted_pos : pos;
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t inext = 0;
    P pnext[3] = {(P)0, (P)0, (P)0};
    auto fetch = [&](int64_t kk) {
        inext = order != nullptr ? (int64_t)order[kk] : kk;
        const int64_t at = sorted_pos != nullptr ? kk : inext;
        pnext[0] = src[3 * at];
        pnext[1] = src[3 * at + 1];
        pnext[2] = src[3 * at + 2];
    };
    if (k < n) fetch(k);
    for (int64_t r = 0; r < nround; r++, k += stride) {
        int bad = 0;
        const int64_t i = inext;
        const P p[3] = {pnext[0], pnext[1], pnext[2]};
        if (k + stride < n) fetch(k + stride);
        if (k < n) {
            F q[3] = {0, 0, 0};
            P s[3];
            const bool ok = particle_index_of<P, F>(p, g, wrap, q, &bad);
            const Cic<F> c = cic_setup(q, g.n);
            if (PHI) {
                F d[3] = {(F)NAN, (F)NAN, (F)NAN};
                if (ok) fd_read(m0, c, g.n, twocell, d);
#pragma unroll
                for (int a = 0; a < 3; a++) s[a] = (P)d[a];
            } else if (IL) {
                F d[3] = {(F)NAN, (F)NAN, (F)NAN};
                if (ok) cic_read3<F>((const typename vec4_of<F>::type*)m0, c, g.n, d);
#pragma unroll
                for (int a = 0; a < 3; a++) s[a] = (P)d[a];
            } else {
                s[0] = ok ? (P)cic_read(m0, c, g.n) : (P)NAN;
                s[1] = ok ? (P)cic_read(m1, c, g.n) : (P)NAN;
                s[2] = ok ? (P)cic_read(m2, c, g.n) : (P)NAN;
            }
            if (field != PRC_FIELD_DISP) {
                // line of sight: global (mesh dtype) or p / |p| of the positions the reference uses
                // (wrapped ones for psi, unwrapped ones for phi); all in double here, then the sum
                // s.l is accumulated in order ((s0 l0 + s1 l1) + s2 l2) as numpy's reduction does.
                double l[3];
                if (global_los) {
                    l[0] = (double)(F)l0; l[1] = (double)(F)l1; l[2] = (double)(F)l2;
                } else {
                    double x[3];
#pragma unroll
                    for (int a = 0; a < 3; a++) x[a] = (!PHI && wrap) ? (double)wrap_position<P, F>(p[a], g, a) : (double)p[a];
                    double dist = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
#pragma unroll
                    for (int a = 0; a < 3; a++) l[a] = x[a] / dist;
                }
                double proj = (double)s[0] * l[0];
                proj = rn_add(proj, rn_mul((double)s[1], l[1]));
                proj = rn_add(proj, rn_mul((double)s[2], l[2]));
                proj *= f;
                P rsd[3];
#pragma unroll
                for (int a = 0; a < 3; a++) rsd[a] = (P)(proj * l[a]);
                if (field == PRC_FIELD_RSD) {
#pragma unroll
                    for (int a = 0; a < 3; a++) s[a] = rsd[a];
                } else {
#pragma unroll
                    for (int a = 0; a < 3; a++) s[a] = (P)rn_add(s[a], rsd[a]);
                }
            }
            if (shifted) {
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    P v = rn_sub(p[a], s[a]);
                    out[3 * i + a] = wrap ? (O)wrap_position<P, F>(v, g, a) : (O)v;
                }
            } else {
#pragma unroll
                for (int a = 0; a < 3; a++) out[3 * i + a] = (O)s[a];
            }
        }
        raise_flags(flags, bad & PRC_FLAG_OUT_OF_BOX);
    }
}

// ---------------------------------------------------------------------------------------------
// IterativeFFTParticleReconstruction (pyrecon/iterative_fft_particle.py): density contrast of
// already smoothed meshes, the per-iteration particle update and the particle read-out.
// Arithmetic of the particle steps in float64, results stored in the positions dtype.
// ---------------------------------------------------------------------------------------------

// delta of set_density_contrast (iterative_fft_particle.py:50-63) from meshes of type X.
template <typename X, typename T>
__global__ void __launch_bounds__(256) delta_meshes_kernel(const X* __restrict__ d, const X* __restrict__ r,
                                                           const double* __restrict__ sums, int64_t n, double bias,
                                                           double ran_min, double size_randoms, T* __restrict__ delta) {
    const double sd = sums[0];
    const double sr = r ? sums[1] : 0.;
    const double alpha = r ? sd * 1. / sr : 0.;
    const double threshold = r ? ran_min * sr / size_randoms : 0.;
    const double mean = sd / (double)n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double dv = (double)d[i];
        double o;
        if (r) {
            const double rv = (double)r[i];
            o = rv > threshold ? (dv - alpha * rv) / (bias * alpha * rv) : 0.;
        } else {
            o = (dv / mean - 1.) / bias;
        }
        delta[i] = (T)o;
    }
}

// Displacement (3 components, in P) at coordinates p, read with RealMesh.read_cic's wrap (wrap = 1)
// or its box check (wrap = 0); NaN where invalid.
template <typename P, typename F>
__device__ __forceinline__ void psi_at(const typename vec4_of<F>::type* __restrict__ psi, const BoxGeom& g,
                                       const P (&p)[3], int wrap, P (&s)[3], int* bad) {
    F q[3] = {0, 0, 0};
    const bool ok = particle_index<P, F>(p, 0, g, wrap, q, bad);
    F d[3] = {(F)NAN, (F)NAN, (F)NAN};
    if (ok) cic_read3<F>(psi, cic_setup(q, g.n), g.n, d);
#pragma unroll
    for (int a = 0; a < 3; a++) s[a] = (P)d[a];
}

// Line of sight: the global one (mesh dtype) or the unit vector of x.
__device__ __forceinline__ void los_of(int global, double l0, double l1, double l2, const double (&x)[3],
                                       double (&l)[3]) {
    if (global) {
        l[0] = l0, l[1] = l1, l[2] = l2;
        return;
    }
    const double dist = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
#pragma unroll
    for (int a = 0; a < 3; a++) l[a] = x[a] / dist;
}

__device__ __forceinline__ double dot3(const double (&a)[3], const double (&b)[3]) {
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}

// One iteration's update (iterative_fft_particle.py:106-139): shifts read at the current
// reconstructed positions (wrapped), the first iteration's RSD correction, then
// x_rec = x_data - f (s.l) l with l from the data positions (wrapped when wrap_data).
template <typename P, typename F>
__global__ void __launch_bounds__(256) ifftp_update_kernel(const typename vec4_of<F>::type* __restrict__ psi, BoxGeom g,
                                                           const P* __restrict__ pos_data, P* __restrict__ pos_rec,
                                                           int64_t n, double f, double beta, int first, int global_los,
                                                           double l0, double l1, double l2, int wrap_data,
                                                           int32_t* flags) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t nround = (n + stride - 1) / stride;
    for (int64_t r = 0; r < nround; r++) {
        const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x + r * stride;
        int bad = 0;
        if (i < n) {
            const P pr[3] = {pos_rec[3 * i], pos_rec[3 * i + 1], pos_rec[3 * i + 2]};
            P s[3];
            psi_at<P, F>(psi, g, pr, 1, s, &bad);
            double x[3];
#pragma unroll
            for (int a = 0; a < 3; a++)
                x[a] = wrap_data ? (double)(P)wrap_position<P, F>(pos_data[3 * i + a], g, a) : (double)pos_data[3 * i + a];
            double l[3];
            los_of(global_los, l0, l1, l2, x, l);
            double sd[3] = {(double)s[0], (double)s[1], (double)s[2]};
            double dot = dot3(sd, l);
            if (first) {
                const double c = beta / (1. + beta) * dot;
#pragma unroll
                for (int a = 0; a < 3; a++) sd[a] = (double)(P)(sd[a] - c * l[a]);
                dot = dot3(sd, l);
            }
            const double fd = f * dot;
#pragma unroll
            for (int a = 0; a < 3; a++) pos_rec[3 * i + a] = (P)(x[a] - fd * l[a]);
        }
        raise_flags(flags, bad & PRC_FLAG_NONFINITE);
    }
}

// Read-out (iterative_fft_particle.py:148-244).  data mode (pos_rec != NULL, pos = the data):
// shifts at the reconstructed positions, RSD = data - reconstructed.  Otherwise, at positions p
// (wrapped when wrap): disp = psi(p); rsd = f (disp.l) l; disp+rsd = psi(p - rsd, wrapped) + rsd.
// shifted: input positions - shifts, wrapped when wrap.
template <typename P, typename F, typename O>
__global__ void __launch_bounds__(256) ifftp_read_kernel(const typename vec4_of<F>::type* __restrict__ psi, BoxGeom g,
                                                         const P* __restrict__ pos, const P* __restrict__ pos_rec,
                                                         int64_t n, double f, int global_los, double l0, double l1,
                                                         double l2, int field, int shifted, int wrap,
                                                         O* __restrict__ out, int32_t* flags,
                                                         const uint32_t* __restrict__ order) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t nround = (n + stride - 1) / stride;
    for (int64_t r = 0; r < nround; r++) {
        const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x + r * stride;
        int bad = 0;
        if (k < n) {
            // particles visited in `order` when given (the cell order of their paint), as read_shifts_kernel
            const int64_t i = order != nullptr ? (int64_t)order[k] : k;
            double base[3], sh[3];
            if (pos_rec != nullptr) {
                const P pr[3] = {pos_rec[3 * i], pos_rec[3 * i + 1], pos_rec[3 * i + 2]};
                P s[3];
                psi_at<P, F>(psi, g, pr, 1, s, &bad);
                P pd[3];
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    pd[a] = wrap ? (P)wrap_position<P, F>(pos[3 * i + a], g, a) : pos[3 * i + a];
                    base[a] = (double)pd[a];
                    const P rsd = (P)(pd[a] - pr[a]);
                    sh[a] = field == PRC_FIELD_DISP ? (double)s[a]
                          : (field == PRC_FIELD_RSD ? (double)rsd : (double)(P)(s[a] + rsd));
                }
            } else {
                P p[3];
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    base[a] = (double)pos[3 * i + a];
                    p[a] = wrap ? (P)wrap_position<P, F>(pos[3 * i + a], g, a) : pos[3 * i + a];
                }
                P s[3];
                psi_at<P, F>(psi, g, p, 0, s, &bad);
                if (field == PRC_FIELD_DISP) {
#pragma unroll
                    for (int a = 0; a < 3; a++) sh[a] = (double)s[a];
                } else {
                    double x[3] = {(double)p[0], (double)p[1], (double)p[2]}, l[3];
                    los_of(global_los, l0, l1, l2, x, l);
                    const double sd[3] = {(double)s[0], (double)s[1], (double)s[2]};
                    const double fd = f * dot3(sd, l);
                    P rsd[3];
#pragma unroll
                    for (int a = 0; a < 3; a++) rsd[a] = (P)(fd * l[a]);
                    if (field == PRC_FIELD_RSD) {
#pragma unroll
                        for (int a = 0; a < 3; a++) sh[a] = (double)rsd[a];
                    } else {
                        P real[3], s2[3];
#pragma unroll
                        for (int a = 0; a < 3; a++) real[a] = (P)(p[a] - rsd[a]);
                        psi_at<P, F>(psi, g, real, 1, s2, &bad);
#pragma unroll
                        for (int a = 0; a < 3; a++) sh[a] = (double)(P)(s2[a] + rsd[a]);
                    }
                }
            }
#pragma unroll
            for (int a = 0; a < 3; a++) {
                if (shifted) {
                    const P v = (P)(base[a] - sh[a]);
                    out[3 * i + a] = wrap ? (O)wrap_position<P, F>(v, g, a) : (O)v;
                } else {
                    out[3 * i + a] = (O)sh[a];
                }
            }
        }
        raise_flags(flags, bad);
    }
}

int device_sm_count() {
    static int cached = -1;
    if (cached < 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cached = sms > 0 ? sms : 148;
    }
    return cached;
}

inline BoxGeom make_geom(const int32_t nmesh[3], const double boxsize[3], const double boxcenter[3]) {
    BoxGeom g;
    for (int d = 0; d < 3; d++) {
        g.n[d] = nmesh[d];
        g.boxsize[d] = boxsize[d];
        g.boxcenter[d] = boxcenter[d];
    }
    return g;
}

inline bool valid_nmesh(const int32_t* nmesh) {
    if (!nmesh) return false;
    for (int d = 0; d < 3; d++)
        if (nmesh[d] < 1 || nmesh[d] > 65536) return false;
    return (int64_t)nmesh[0] * nmesh[1] * nmesh[2] < ((int64_t)1 << 32);
}

inline int key_bits(const int32_t* nmesh) {
    uint64_t N = (uint64_t)nmesh[0] * nmesh[1] * nmesh[2];
    int b = 0;
    while (((uint64_t)1 << b) < N) b++;
    return b;
}

inline int particle_grid(int64_t n) {
    int64_t blocks = (n + 255) / 256;
    int64_t cap = (int64_t)device_sm_count() * 16;
    return (int)std::max<int64_t>(1, std::min(blocks, cap));
}

// Workspace layout of the paint.
struct PaintWs {
    uint32_t *k0, *v0, *k1, *v1, *col_start, *scratch;
    void* payload;
};

inline size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

inline size_t paint_layout(const int32_t nmesh[3], int64_t npos, int mesh_bytes, char* base, PaintWs* ws) {
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base ? base + off : nullptr;
        off += align_up(bytes);
        return p;
    };
    int64_t ncol = (int64_t)nmesh[0] * nmesh[1];
    size_t kb = (size_t)std::max<int64_t>(npos, 1) * sizeof(uint32_t);
    PaintWs w;
    w.k0 = (uint32_t*)take(kb);
    w.v0 = (uint32_t*)take(kb);
    w.k1 = (uint32_t*)take(kb);
    w.v1 = (uint32_t*)take(kb);
    w.col_start = (uint32_t*)take((size_t)(ncol + 1) * sizeof(uint32_t));
    w.scratch = (uint32_t*)take(rsort::scratch_bytes(std::max<int64_t>(npos, 1)));
    w.payload = take((size_t)std::max<int64_t>(npos, 1) * 4 * (mesh_bytes == 4 ? 4 : 8));
    if (ws) *ws = w;
    return off;
}

template <typename P, typename F, typename W>
int paint_sort(const P* pos, const W* w, int64_t n, const BoxGeom& g, int wrap, const PaintWs& ws, int32_t* flags,
               uint32_t** keys, uint32_t** order, cudaStream_t st) {
    PRC_LAUNCH_B("paint_keys", st, (double)n * (3 * sizeof(P) + (w ? sizeof(W) : 0) + 8), paint_keys<P, F, W><<<particle_grid(n), 256, 0, st>>>(pos, w, n, g, wrap, ws.k0, ws.v0, flags));
    PRC_CHECK_LAUNCH();
    int32_t nm[3] = {g.n[0], g.n[1], g.n[2]};
    return rsort::sort_pairs(ws.k0, ws.v0, ws.k1, ws.v1, n, key_bits(nm), ws.scratch, keys, order, flags, st);
}

template <typename P, typename F, typename W>
int paint_run(double* mesh, double* colsums, const BoxGeom& g, const P* pos, const W* w, int64_t n, int wrap,
              int accumulate, int32_t* flags, const PaintWs& ws, cudaStream_t st, uint32_t* order_out = nullptr,
              P* sorted_out = nullptr) {
    uint32_t *keys = nullptr, *order = nullptr;
    if (n > 0) PRC_TRY((paint_sort<P, F, W>(pos, w, n, g, wrap, ws, flags, &keys, &order, st)));
    if (n > 0 && order_out != nullptr &&
        cudaMemcpyAsync(order_out, order, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return PRC_ERR_CUDA;
    Payload<F>* pl = (Payload<F>*)ws.payload;
    if (n > 0) {
        PRC_LAUNCH_B("paint_payload", st,
                     (double)n * (4 + 3 * sizeof(P) * (sorted_out ? 2 : 1) + (w ? sizeof(W) : 0) + sizeof(Payload<F>)),
                     paint_payload<P, F, W><<<particle_grid(n), 256, 0, st>>>(pos, w, n, g, wrap, order, pl, sorted_out,
                                                                             flags));
        PRC_CHECK_LAUNCH();
    } else {
        keys = ws.k0;
    }
    int64_t ncol = (int64_t)g.n[0] * g.n[1];
    PRC_LAUNCH_B("paint_columns", st, 8.0 * n + 4.0 * ncol, column_starts<<<particle_grid(n + 1), 256, 0, st>>>(keys, n, g.n[2], ncol, ws.col_start, flags));
    PRC_CHECK_LAUNCH();
    size_t smem = (size_t)PULL_WARPS * g.n[2] * sizeof(double);
    if (smem > 48 * 1024) cudaFuncSetAttribute(paint_pull<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int64_t blocks = (ncol + PULL_WARPS - 1) / PULL_WARPS;
    int grid = (int)std::min<int64_t>(blocks, (int64_t)device_sm_count() * 16);
    Dims dims = {{g.n[0], g.n[1], g.n[2]}};
    PRC_LAUNCH_B("paint_pull", st, (double)n * (4 + sizeof(Payload<F>)) + 4.0 * ncol + 8.0 * (accumulate ? 2 : 1) * ncol * g.n[2] + 8.0 * ncol, paint_pull<F><<<grid, PULL_WARPS * 32, smem, st>>>(keys, pl, ws.col_start, dims, accumulate, mesh, colsums, flags));
    PRC_CHECK_LAUNCH();
    return PRC_OK;
}

template <typename P, typename F>
int paint_dispatch_w(double* mesh, double* colsums, const BoxGeom& g, const void* pos, const void* w, int wb, int64_t n,
                     int wrap, int acc, int32_t* flags, const PaintWs& ws, cudaStream_t st, uint32_t* order_out,
                     void* sorted_out) {
    P* so = (P*)sorted_out;
    if (w == nullptr)
        return paint_run<P, F, F>(mesh, colsums, g, (const P*)pos, (const F*)nullptr, n, wrap, acc, flags, ws, st, order_out, so);
    if (wb == 4)
        return paint_run<P, F, float>(mesh, colsums, g, (const P*)pos, (const float*)w, n, wrap, acc, flags, ws, st, order_out, so);
    return paint_run<P, F, double>(mesh, colsums, g, (const P*)pos, (const double*)w, n, wrap, acc, flags, ws, st, order_out, so);
}

template <typename P, typename F>
int read_shifts_launch(const F* m0, const F* m1, const F* m2, int stride, bool phi, const BoxGeom& g, const void* pos,
                       int64_t n, const uint32_t* order, double f, const double* los, int field, int shifted, int wrap,
                       void* out, int ob, int32_t* flags, cudaStream_t st, const void* sorted_pos) {
    if (sorted_pos != nullptr && order == nullptr) return PRC_ERR_ARG;
    const bool il = !phi && stride == 4;
    if (il && (m1 != m0 + 1 || m2 != m0 + 2 || ((uintptr_t)m0 % (4 * sizeof(F))) != 0)) return PRC_ERR_ARG;
    if (!phi && !il && stride != 1) return PRC_ERR_ARG;
    F tc[3];
    twocell_of(g, tc);
    double l[3] = {0, 0, 0};
    if (los)
        for (int a = 0; a < 3; a++) l[a] = los[a];
    int grid = particle_grid(n);
    // particles in and out, plus every mesh cell the gathers touch (at most 8 or 32 per particle)
    const double ncell = (double)g.n[0] * g.n[1] * g.n[2];
    const double gather_bytes = (double)n * 3 * (sizeof(P) + ob) +
                                (phi ? std::min(ncell, 32.0 * n) : 3 * std::min(ncell, 8.0 * n)) * sizeof(F);
#define LAUNCH(O, PH, IL)                                                                                          \
    PRC_LAUNCH_B(PH ? "read_shifts_phi" : "read_shifts_psi", st, gather_bytes,                                     \
                 read_shifts_kernel<P, F, O, PH, IL><<<grid, 256, 0, st>>>(m0, m1, m2, g, tc[0], tc[1], tc[2],     \
                                                                         (const P*)pos, n, f, los != nullptr, l[0], \
                                                                         l[1], l[2], field, shifted, wrap,          \
                                                                         (O*)out, flags, order,             \
                                                                         (const P*)sorted_pos))
    if (phi) {
        if (ob == 4) LAUNCH(float, true, false); else LAUNCH(double, true, false);
    } else if (il) {
        if (ob == 4) LAUNCH(float, false, true); else LAUNCH(double, false, true);
    } else {
        if (ob == 4) LAUNCH(float, false, false); else LAUNCH(double, false, false);
    }
#undef LAUNCH
    PRC_CHECK_LAUNCH();
    return PRC_OK;
}

// ---------------------------------------------------------------------------------------------
// Allocation-free paint: scratch in a file-scope device array
// ---------------------------------------------------------------------------------------------
// Particles are painted in chunks of at most NOALLOC_CHUNK (each chunk accumulates into the mesh,
// so the scratch does not grow with the catalogue); meshes up to NOALLOC_MAX_COLUMNS (x, y)
// columns.  The array lives in every GPU that loads this library until the process exits.
constexpr int64_t NOALLOC_CHUNK = (int64_t)1 << 18;
constexpr int64_t NOALLOC_MAX_COLUMNS = (int64_t)1 << 20;
constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)17 << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// The calling thread's current driver context (null when none is current yet: the runtime then uses
// the device's primary context), fetched through the runtime so the library does not link libcuda.
static void* current_context() {
    typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
    static CtxGetCurrentFn fn = []() -> CtxGetCurrentFn {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return (CtxGetCurrentFn)f;
    }();
    CUcontext c = nullptr;
    if (fn != nullptr && fn(&c) != CUDA_SUCCESS) c = nullptr;
    return (void*)c;
}

// Device address of g_noalloc_scratch in the current context of the current device, looked up once per
// (device, context): every context that loads the module holds its own copy of the array, so an address
// is only valid in the context it was looked up in.
static void* noalloc_scratch_address() {
    static std::mutex mu;
    static std::map<std::pair<int, void*>, void*> cache;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    const std::pair<int, void*> key(dev, current_context());
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) return nullptr;
    cache[key] = p;
    return p;
}

template <typename P, typename F, typename W>
int paint_noalloc(double* mesh, double* colsums, const BoxGeom& g, const P* pos, const W* w, int64_t n, int wrap,
                  int accumulate, int32_t* flags, const PaintWs& ws, cudaStream_t st) {
    // validate every particle first (raises flags; the painting kernels of all chunks then skip,
    // leaving the mesh untouched as the single-call paint does)
    for (int64_t off = 0; off < n; off += NOALLOC_CHUNK) {
        const int64_t cnt = std::min(NOALLOC_CHUNK, n - off);
        PRC_LAUNCH_B("paint_keys", st, (double)cnt * (3 * sizeof(P) + (w ? sizeof(W) : 0) + 8),
                     paint_keys<P, F, W><<<particle_grid(cnt), 256, 0, st>>>(pos + 3 * off, w ? w + off : nullptr, cnt,
                                                                            g, wrap, ws.k0, ws.v0, flags));
        PRC_CHECK_LAUNCH();
    }
    if (n == 0) return paint_run<P, F, W>(mesh, colsums, g, pos, w, 0, wrap, accumulate, flags, ws, st);
    for (int64_t off = 0; off < n; off += NOALLOC_CHUNK) {
        const int64_t cnt = std::min(NOALLOC_CHUNK, n - off);
        PRC_TRY((paint_run<P, F, W>(mesh, colsums, g, pos + 3 * off, w ? w + off : nullptr, cnt, wrap,
                                    off == 0 ? accumulate : 1, flags, ws, st)));
    }
    return PRC_OK;
}

template <typename P, typename F>
int paint_noalloc_w(double* mesh, double* colsums, const BoxGeom& g, const void* pos, const void* w, int wb, int64_t n,
                    int wrap, int acc, int32_t* flags, const PaintWs& ws, cudaStream_t st) {
    if (w == nullptr) return paint_noalloc<P, F, F>(mesh, colsums, g, (const P*)pos, (const F*)nullptr, n, wrap, acc, flags, ws, st);
    if (wb == 4) return paint_noalloc<P, F, float>(mesh, colsums, g, (const P*)pos, (const float*)w, n, wrap, acc, flags, ws, st);
    return paint_noalloc<P, F, double>(mesh, colsums, g, (const P*)pos, (const double*)w, n, wrap, acc, flags, ws, st);
}

}  // namespace prc

using namespace prc;

extern "C" {

prc_status_t prc_assign_cic_noalloc(double* mesh, double* column_sums, const int32_t nmesh[3], const double boxsize[3],
                                    const double boxcenter[3], int mesh_bytes, const void* positions, int pos_bytes,
                                    const void* weights, int weight_bytes, int64_t npos, int wrap, int accumulate,
                                    int32_t* flags, void* stream) {
    if (!mesh || !valid_nmesh(nmesh) || !boxsize || !boxcenter || !flags || npos < 0) return PRC_ERR_ARG;
    if (npos >= ((int64_t)1 << 32) || (npos > 0 && !positions)) return PRC_ERR_ARG;
    if ((mesh_bytes != 4 && mesh_bytes != 8) || (pos_bytes != 4 && pos_bytes != 8)) return PRC_ERR_ARG;
    if (weights && weight_bytes != 4 && weight_bytes != 8) return PRC_ERR_ARG;
    if (nmesh[2] > 4096 || (int64_t)nmesh[0] * nmesh[1] > NOALLOC_MAX_COLUMNS) return PRC_ERR_UNSUPPORTED;
    if (paint_layout(nmesh, std::min(npos, NOALLOC_CHUNK), mesh_bytes, nullptr, nullptr) > NOALLOC_SCRATCH_BYTES)
        return PRC_ERR_UNSUPPORTED;
    void* scratch = noalloc_scratch_address();
    if (scratch == nullptr) return PRC_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    PaintWs ws;
    paint_layout(nmesh, std::min(npos, NOALLOC_CHUNK), mesh_bytes, (char*)scratch, &ws);
    BoxGeom g = make_geom(nmesh, boxsize, boxcenter);
    if (cudaMemsetAsync(flags, 0, sizeof(int32_t), st) != cudaSuccess) return PRC_ERR_CUDA;
    if (pos_bytes == 4 && mesh_bytes == 4)
        return paint_noalloc_w<float, float>(mesh, column_sums, g, positions, weights, weight_bytes, npos, wrap, accumulate, flags, ws, st);
    if (pos_bytes == 4 && mesh_bytes == 8)
        return paint_noalloc_w<float, double>(mesh, column_sums, g, positions, weights, weight_bytes, npos, wrap, accumulate, flags, ws, st);
    if (pos_bytes == 8 && mesh_bytes == 4)
        return paint_noalloc_w<double, float>(mesh, column_sums, g, positions, weights, weight_bytes, npos, wrap, accumulate, flags, ws, st);
    return paint_noalloc_w<double, double>(mesh, column_sums, g, positions, weights, weight_bytes, npos, wrap, accumulate, flags, ws, st);
}

size_t prc_assign_cic_workspace_bytes(const int32_t nmesh[3], int64_t npos, int mesh_bytes) {
    if (!valid_nmesh(nmesh) || npos < 0) return 0;
    return paint_layout(nmesh, npos, mesh_bytes, nullptr, nullptr);
}

static prc_status_t assign_cic_impl(double* mesh, double* column_sums, const int32_t nmesh[3], const double boxsize[3],
                                    const double boxcenter[3], int mesh_bytes, const void* positions, int pos_bytes,
                                    const void* weights, int weight_bytes, int64_t npos, int wrap, int accumulate,
                                    int32_t* flags, void* workspace, size_t workspace_bytes, void* stream,
                                    uint32_t* order_out, void* sorted_out = nullptr) {
    if (!mesh || !valid_nmesh(nmesh) || !boxsize || !boxcenter || !flags || npos < 0) return PRC_ERR_ARG;
    if (npos >= ((int64_t)1 << 32) || (npos > 0 && !positions)) return PRC_ERR_ARG;
    if ((mesh_bytes != 4 && mesh_bytes != 8) || (pos_bytes != 4 && pos_bytes != 8)) return PRC_ERR_ARG;
    if (weights && weight_bytes != 4 && weight_bytes != 8) return PRC_ERR_ARG;
    if (nmesh[2] > 4096) return PRC_ERR_UNSUPPORTED;   // one FP64 column per warp in shared memory
    if (workspace_bytes < prc_assign_cic_workspace_bytes(nmesh, npos, mesh_bytes) || !workspace) return PRC_ERR_WORKSPACE;
    cudaStream_t st = (cudaStream_t)stream;
    PaintWs ws;
    paint_layout(nmesh, npos, mesh_bytes, (char*)workspace, &ws);
    BoxGeom g = make_geom(nmesh, boxsize, boxcenter);
    if (cudaMemsetAsync(flags, 0, sizeof(int32_t), st) != cudaSuccess) return PRC_ERR_CUDA;
    if (pos_bytes == 4 && mesh_bytes == 4)
        return paint_dispatch_w<float, float>(mesh, column_sums, g, positions, weights, weight_bytes, npos, wrap, accumulate, flags, ws, st, order_out, sorted_out);
    if (pos_bytes == 4 && mesh_bytes == 8)
        return paint_dispatch_w<float, double>(mesh, column_sums, g, positions, weights, weight_bytes, npos, wrap, accumulate, flags, ws, st, order_out, sorted_out);
    if (pos_bytes == 8 && mesh_bytes == 4)
        return paint_dispatch_w<double, float>(mesh, column_sums, g, positions, weights, weight_bytes, npos, wrap, accumulate, flags, ws, st, order_out, sorted_out);
    return paint_dispatch_w<double, double>(mesh, column_sums, g, positions, weights, weight_bytes, npos, wrap, accumulate, flags, ws, st, order_out, sorted_out);
}

prc_status_t prc_assign_cic(double* mesh, double* column_sums, const int32_t nmesh[3], const double boxsize[3],
                            const double boxcenter[3], int mesh_bytes, const void* positions, int pos_bytes,
                            const void* weights, int weight_bytes, int64_t npos, int wrap, int accumulate,
                            int32_t* flags, void* workspace, size_t workspace_bytes, void* stream) {
    return assign_cic_impl(mesh, column_sums, nmesh, boxsize, boxcenter, mesh_bytes, positions, pos_bytes, weights,
                           weight_bytes, npos, wrap, accumulate, flags, workspace, workspace_bytes, stream, nullptr);
}

prc_status_t prc_assign_cic_order(double* mesh, double* column_sums, const int32_t nmesh[3], const double boxsize[3],
                                  const double boxcenter[3], int mesh_bytes, const void* positions, int pos_bytes,
                                  const void* weights, int weight_bytes, int64_t npos, int wrap, int accumulate,
                                  int32_t* flags, void* workspace, size_t workspace_bytes, void* stream,
                                  uint32_t* order) {
    if (!order && npos > 0) return PRC_ERR_ARG;
    return assign_cic_impl(mesh, column_sums, nmesh, boxsize, boxcenter, mesh_bytes, positions, pos_bytes, weights,
                           weight_bytes, npos, wrap, accumulate, flags, workspace, workspace_bytes, stream, order);
}

prc_status_t prc_assign_cic_sorted(double* mesh, double* column_sums, const int32_t nmesh[3], const double boxsize[3],
                                   const double boxcenter[3], int mesh_bytes, const void* positions, int pos_bytes,
                                   const void* weights, int weight_bytes, int64_t npos, int wrap, int accumulate,
                                   int32_t* flags, void* workspace, size_t workspace_bytes, void* stream,
                                   uint32_t* order, void* sorted_positions) {
    if ((!order || !sorted_positions) && npos > 0) return PRC_ERR_ARG;
    return assign_cic_impl(mesh, column_sums, nmesh, boxsize, boxcenter, mesh_bytes, positions, pos_bytes, weights,
                           weight_bytes, npos, wrap, accumulate, flags, workspace, workspace_bytes, stream, order,
                           sorted_positions);
}

prc_status_t prc_cic_cell_order(uint32_t* keys_sorted, uint32_t* order, const int32_t nmesh[3], const double boxsize[3],
                                const double boxcenter[3], int mesh_bytes, const void* positions, int pos_bytes,
                                int64_t npos, int wrap, int32_t* flags, void* workspace, size_t workspace_bytes,
                                void* stream) {
    if (!keys_sorted || !order || !valid_nmesh(nmesh) || !boxsize || !boxcenter || !flags || npos < 0) return PRC_ERR_ARG;
    if (npos >= ((int64_t)1 << 32) || (npos > 0 && !positions)) return PRC_ERR_ARG;
    if ((mesh_bytes != 4 && mesh_bytes != 8) || (pos_bytes != 4 && pos_bytes != 8)) return PRC_ERR_ARG;
    if (workspace_bytes < prc_assign_cic_workspace_bytes(nmesh, npos, mesh_bytes) || !workspace) return PRC_ERR_WORKSPACE;
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemsetAsync(flags, 0, sizeof(int32_t), st) != cudaSuccess) return PRC_ERR_CUDA;
    if (npos == 0) return PRC_OK;
    PaintWs ws;
    paint_layout(nmesh, npos, mesh_bytes, (char*)workspace, &ws);
    BoxGeom g = make_geom(nmesh, boxsize, boxcenter);
    uint32_t *k = nullptr, *v = nullptr;
    int s;
    if (pos_bytes == 4 && mesh_bytes == 4) s = paint_sort<float, float, float>((const float*)positions, nullptr, npos, g, wrap, ws, flags, &k, &v, st);
    else if (pos_bytes == 4) s = paint_sort<float, double, double>((const float*)positions, nullptr, npos, g, wrap, ws, flags, &k, &v, st);
    else if (mesh_bytes == 4) s = paint_sort<double, float, float>((const double*)positions, nullptr, npos, g, wrap, ws, flags, &k, &v, st);
    else s = paint_sort<double, double, double>((const double*)positions, nullptr, npos, g, wrap, ws, flags, &k, &v, st);
    if (s != PRC_OK) return s;
    if (cudaMemcpyAsync(keys_sorted, k, (size_t)npos * 4, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return PRC_ERR_CUDA;
    if (cudaMemcpyAsync(order, v, (size_t)npos * 4, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return PRC_ERR_CUDA;
    return PRC_OK;
}

size_t prc_sum_workspace_bytes(int64_t n) {
    (void)n;
    return SUM_BLOCKS * sizeof(double);
}

prc_status_t prc_sum_f64(const double* x, int64_t n, double* out, void* workspace, size_t workspace_bytes, void* stream) {
    if (!out || n < 0 || (n > 0 && !x)) return PRC_ERR_ARG;
    if (!workspace || workspace_bytes < prc_sum_workspace_bytes(n)) return PRC_ERR_WORKSPACE;
    cudaStream_t st = (cudaStream_t)stream;
    PRC_LAUNCH("sum", st, sum_partials<double><<<SUM_BLOCKS, SUM_THREADS, 0, st>>>(x, n, (double*)workspace));
    PRC_LAUNCH("sum", st, sum_final<<<1, SUM_THREADS, 0, st>>>((const double*)workspace, out));
    PRC_CHECK_LAUNCH();
    return PRC_OK;
}

prc_status_t prc_sum_f32(const float* x, int64_t n, double* out, void* workspace, size_t workspace_bytes, void* stream) {
    if (!out || n < 0 || (n > 0 && !x)) return PRC_ERR_ARG;
    if (!workspace || workspace_bytes < prc_sum_workspace_bytes(n)) return PRC_ERR_WORKSPACE;
    cudaStream_t st = (cudaStream_t)stream;
    PRC_LAUNCH("sum", st, sum_partials<float><<<SUM_BLOCKS, SUM_THREADS, 0, st>>>(x, n, (double*)workspace));
    PRC_LAUNCH("sum", st, sum_final<<<1, SUM_THREADS, 0, st>>>((const double*)workspace, out));
    PRC_CHECK_LAUNCH();
    return PRC_OK;
}

#define READ_CIC_IMPL(NAME, F)                                                                                     \
    prc_status_t NAME(const F* mesh, const int32_t nmesh[3], const double boxsize[3], const double boxcenter[3],   \
                      const void* positions, int pos_bytes, int64_t npos, int wrap, void* out, int32_t* flags,      \
                      void* stream) {                                                                              \
        if (!mesh || !valid_nmesh(nmesh) || !boxsize || !boxcenter || !flags || npos < 0) return PRC_ERR_ARG;    \
        if (npos > 0 && (!positions || !out)) return PRC_ERR_ARG;                                                  \
        if (pos_bytes != 4 && pos_bytes != 8) return PRC_ERR_ARG;                                                  \
        cudaStream_t st = (cudaStream_t)stream;                                                                    \
        if (cudaMemsetAsync(flags, 0, sizeof(int32_t), st) != cudaSuccess) return PRC_ERR_CUDA;                   \
        if (npos == 0) return PRC_OK;                                                                              \
        BoxGeom g = make_geom(nmesh, boxsize, boxcenter);                                                          \
        if (pos_bytes == 4)                                                                                        \
            PRC_LAUNCH("read_cic", st, read_cic_kernel<float, F><<<particle_grid(npos), 256, 0, st>>>(             \
                                           mesh, g, (const float*)positions, npos, wrap, (float*)out, flags));      \
        else                                                                                                       \
            PRC_LAUNCH("read_cic", st, read_cic_kernel<double, F><<<particle_grid(npos), 256, 0, st>>>(            \
                                           mesh, g, (const double*)positions, npos, wrap, (double*)out, flags));    \
        PRC_CHECK_LAUNCH();                                                                                        \
        return PRC_OK;                                                                                             \
    }

READ_CIC_IMPL(prc_read_cic_f32, float)
READ_CIC_IMPL(prc_read_cic_f64, double)

#define READ_FD_IMPL(NAME, F)                                                                                      \
    prc_status_t NAME(const F* mesh, const int32_t nmesh[3], const double boxsize[3], const double boxcenter[3],   \
                      const void* positions, int pos_bytes, int64_t npos, int wrap, void* out, int32_t* flags,      \
                      void* stream) {                                                                              \
        if (!mesh || !valid_nmesh(nmesh) || !boxsize || !boxcenter || !flags || npos < 0) return PRC_ERR_ARG;    \
        if (npos > 0 && (!positions || !out)) return PRC_ERR_ARG;                                                  \
        if (pos_bytes != 4 && pos_bytes != 8) return PRC_ERR_ARG;                                                  \
        cudaStream_t st = (cudaStream_t)stream;                                                                    \
        if (cudaMemsetAsync(flags, 0, sizeof(int32_t), st) != cudaSuccess) return PRC_ERR_CUDA;                   \
        if (npos == 0) return PRC_OK;                                                                              \
        BoxGeom g = make_geom(nmesh, boxsize, boxcenter);                                                          \
        F tc[3];                                                                                                   \
        twocell_of(g, tc);                                                                                         \
        if (pos_bytes == 4)                                                                                        \
            PRC_LAUNCH("read_fd_cic", st, read_fd_kernel<float, F><<<particle_grid(npos), 256, 0, st>>>(           \
                                              mesh, g, tc[0], tc[1], tc[2], (const float*)positions, npos, wrap,   \
                                              (float*)out, flags));                                                \
        else                                                                                                       \
            PRC_LAUNCH("read_fd_cic", st, read_fd_kernel<double, F><<<particle_grid(npos), 256, 0, st>>>(          \
                                              mesh, g, tc[0], tc[1], tc[2], (const double*)positions, npos, wrap,  \
                                              (double*)out, flags));                                               \
        PRC_CHECK_LAUNCH();                                                                                        \
        return PRC_OK;                                                                                             \
    }

READ_FD_IMPL(prc_read_finite_difference_cic_f32, float)
READ_FD_IMPL(prc_read_finite_difference_cic_f64, double)

#define READ_SHIFTS_IMPL(NAME, F, PHI, ARGS, M0, M1, M2, STRIDE)                                                           \
    prc_status_t NAME ARGS {                                                                                       \
        if (!M0 || !M1 || !M2 || !valid_nmesh(nmesh) || !boxsize || !boxcenter || !flags || npos < 0)             \
            return PRC_ERR_ARG;                                                                                    \
        if (npos > 0 && (!positions || !out)) return PRC_ERR_ARG;                                                  \
        if ((pos_bytes != 4 && pos_bytes != 8) || (out_bytes != 4 && out_bytes != 8)) return PRC_ERR_ARG;        \
        if (field < PRC_FIELD_DISP || field > PRC_FIELD_DISP_RSD) return PRC_ERR_ARG;                             \
        cudaStream_t st = (cudaStream_t)stream;                                                                    \
        if (cudaMemsetAsync(flags, 0, sizeof(int32_t), st) != cudaSuccess) return PRC_ERR_CUDA;                   \
        if (npos == 0) return PRC_OK;                                                                              \
        BoxGeom g = make_geom(nmesh, boxsize, boxcenter);                                                          \
        if (pos_bytes == 4)                                                                                        \
            return read_shifts_launch<float, F>(M0, M1, M2, STRIDE, PHI, g, positions, npos, order, f, los, field,  \
                                                shifted, wrap, out, out_bytes, flags, st, sorted_positions);      \
        return read_shifts_launch<double, F>(M0, M1, M2, STRIDE, PHI, g, positions, npos, order, f, los, field,   \
                                             shifted, wrap, out, out_bytes, flags, st, sorted_positions);         \
    }

READ_SHIFTS_IMPL(prc_read_shifts_psi_f32, float, false,
                 (const float* psi_x, const float* psi_y, const float* psi_z, int psi_stride, const int32_t nmesh[3],
                  const double boxsize[3], const double boxcenter[3], const void* positions, int pos_bytes,
                  int64_t npos, const uint32_t* order, double f, const double* los, int field, int shifted, int wrap, void* out,
                  int out_bytes, int32_t* flags, void* stream, const void* sorted_positions),
                 psi_x, psi_y, psi_z, psi_stride)
READ_SHIFTS_IMPL(prc_read_shifts_psi_f64, double, false,
                 (const double* psi_x, const double* psi_y, const double* psi_z, int psi_stride, const int32_t nmesh[3],
                  const double boxsize[3], const double boxcenter[3], const void* positions, int pos_bytes,
                  int64_t npos, const uint32_t* order, double f, const double* los, int field, int shifted, int wrap, void* out,
                  int out_bytes, int32_t* flags, void* stream, const void* sorted_positions),
                 psi_x, psi_y, psi_z, psi_stride)
READ_SHIFTS_IMPL(prc_read_shifts_phi_f32, float, true,
                 (const float* phi, const int32_t nmesh[3], const double boxsize[3], const double boxcenter[3],
                  const void* positions, int pos_bytes, int64_t npos, const uint32_t* order, double f,
                  const double* los, int field, int shifted, int wrap, void* out, int out_bytes, int32_t* flags,
                  void* stream, const void* sorted_positions),
                 phi, phi, phi, 1)
READ_SHIFTS_IMPL(prc_read_shifts_phi_f64, double, true,
                 (const double* phi, const int32_t nmesh[3], const double boxsize[3], const double boxcenter[3],
                  const void* positions, int pos_bytes, int64_t npos, const uint32_t* order, double f,
                  const double* los, int field, int shifted, int wrap, void* out, int out_bytes, int32_t* flags,
                  void* stream, const void* sorted_positions),
                 phi, phi, phi, 1)


// ---- IterativeFFTParticleReconstruction ----

#define DELTA_MESHES_IMPL(NAME, T)                                                                                    \
    prc_status_t NAME(const void* mesh_data, const void* mesh_randoms, int in_bytes, const double* sums,            \
                      const int32_t nmesh[3], double bias, double ran_min, double size_randoms, T* delta,           \
                      void* stream) {                                                                             \
        if (!mesh_data || !sums || !delta || !valid_nmesh(nmesh) || (in_bytes != 4 && in_bytes != 8))             \
            return PRC_ERR_ARG;                                                                                   \
        cudaStream_t st = (cudaStream_t)stream;                                                                   \
        const int64_t n = (int64_t)nmesh[0] * nmesh[1] * nmesh[2];                                                \
        const int grid = particle_grid(n);                                                                        \
        const double bytes = (double)n * (in_bytes * (mesh_randoms ? 2 : 1) + sizeof(T));                         \
        if (in_bytes == 8)                                                                                        \
            PRC_LAUNCH_B("delta_meshes", st, bytes, delta_meshes_kernel<double, T><<<grid, 256, 0, st>>>(          \
                (const double*)mesh_data, (const double*)mesh_randoms, sums, n, bias, ran_min, size_randoms, delta)); \
        else                                                                                                      \
            PRC_LAUNCH_B("delta_meshes", st, bytes, delta_meshes_kernel<float, T><<<grid, 256, 0, st>>>(           \
                (const float*)mesh_data, (const float*)mesh_randoms, sums, n, bias, ran_min, size_randoms, delta));  \
        PRC_CHECK_LAUNCH();                                                                                       \
        return PRC_OK;                                                                                            \
    }
DELTA_MESHES_IMPL(prc_delta_from_meshes_f32, float)
DELTA_MESHES_IMPL(prc_delta_from_meshes_f64, double)

static int ifftp_args_ok(const void* psi4, size_t fsize, const int32_t nmesh[3], const double* boxsize,
                         const double* boxcenter, const int32_t* flags, int pos_bytes, int64_t npos) {
    if (!psi4 || !valid_nmesh(nmesh) || !boxsize || !boxcenter || !flags || npos < 0) return PRC_ERR_ARG;
    if (pos_bytes != 4 && pos_bytes != 8) return PRC_ERR_ARG;
    if (((uintptr_t)psi4 % (4 * fsize)) != 0) return PRC_ERR_ARG;
    return PRC_OK;
}

#define IFFTP_UPDATE_IMPL(NAME, F)                                                                                    \
    prc_status_t NAME(const F* psi4, const int32_t nmesh[3], const double boxsize[3], const double boxcenter[3],     \
                      const void* pos_data, void* pos_rec, int pos_bytes, int64_t npos, double f, double beta,       \
                      int first, const double* los, int wrap_data, int32_t* flags, void* stream) {                   \
        PRC_TRY(ifftp_args_ok(psi4, sizeof(F), nmesh, boxsize, boxcenter, flags, pos_bytes, npos));                         \
        if (npos > 0 && (!pos_data || !pos_rec)) return PRC_ERR_ARG;                                              \
        cudaStream_t st = (cudaStream_t)stream;                                                                   \
        if (cudaMemsetAsync(flags, 0, sizeof(int32_t), st) != cudaSuccess) return PRC_ERR_CUDA;                  \
        if (npos == 0) return PRC_OK;                                                                             \
        BoxGeom g = make_geom(nmesh, boxsize, boxcenter);                                                         \
        double l[3] = {0, 0, 0};                                                                                  \
        if (los)                                                                                                  \
            for (int a = 0; a < 3; a++) l[a] = (double)(F)los[a];                                                 \
        typedef typename vec4_of<F>::type V4;                                                                     \
        const double bytes = (double)npos * 9 * pos_bytes + 8.0 * npos * 4 * sizeof(F);                           \
        if (pos_bytes == 4)                                                                                       \
            PRC_LAUNCH_B("ifftp_update", st, bytes, ifftp_update_kernel<float, F><<<particle_grid(npos), 256, 0, st>>>( \
                (const V4*)psi4, g, (const float*)pos_data, (float*)pos_rec, npos, f, beta, first, los != nullptr,  \
                l[0], l[1], l[2], wrap_data, flags));                                                             \
        else                                                                                                      \
            PRC_LAUNCH_B("ifftp_update", st, bytes, ifftp_update_kernel<double, F><<<particle_grid(npos), 256, 0, st>>>( \
                (const V4*)psi4, g, (const double*)pos_data, (double*)pos_rec, npos, f, beta, first,               \
                los != nullptr, l[0], l[1], l[2], wrap_data, flags));                                             \
        PRC_CHECK_LAUNCH();                                                                                       \
        return PRC_OK;                                                                                            \
    }
IFFTP_UPDATE_IMPL(prc_ifftp_update_f32, float)
IFFTP_UPDATE_IMPL(prc_ifftp_update_f64, double)

#define IFFTP_READ_IMPL(NAME, F)                                                                                      \
    prc_status_t NAME(const F* psi4, const int32_t nmesh[3], const double boxsize[3], const double boxcenter[3],     \
                      const void* positions, const void* pos_rec, int pos_bytes, int64_t npos, double f,             \
                      const double* los, int field, int shifted, int wrap, void* out, int out_bytes, int32_t* flags, \
                      const uint32_t* order, void* stream) {                                                      \
        PRC_TRY(ifftp_args_ok(psi4, sizeof(F), nmesh, boxsize, boxcenter, flags, pos_bytes, npos));                         \
        if (npos > 0 && (!positions || !out)) return PRC_ERR_ARG;                                                 \
        if ((out_bytes != 4 && out_bytes != 8) || field < PRC_FIELD_DISP || field > PRC_FIELD_DISP_RSD)           \
            return PRC_ERR_ARG;                                                                                   \
        cudaStream_t st = (cudaStream_t)stream;                                                                   \
        if (cudaMemsetAsync(flags, 0, sizeof(int32_t), st) != cudaSuccess) return PRC_ERR_CUDA;                  \
        if (npos == 0) return PRC_OK;                                                                             \
        BoxGeom g = make_geom(nmesh, boxsize, boxcenter);                                                         \
        double l[3] = {0, 0, 0};                                                                                  \
        if (los)                                                                                                  \
            for (int a = 0; a < 3; a++) l[a] = (double)(F)los[a];                                                 \
        typedef typename vec4_of<F>::type V4;                                                                     \
        const int grid = particle_grid(npos);                                                                     \
        const double bytes = (double)npos * (3 * pos_bytes * (pos_rec ? 2 : 1) + 3 * out_bytes) +                 \
                             8.0 * npos * 4 * sizeof(F) * (field == PRC_FIELD_DISP_RSD && !pos_rec ? 2 : 1);     \
        const int gl = los != nullptr;                                                                            \
        if (pos_bytes == 4 && out_bytes == 4)                                                                     \
            PRC_LAUNCH_B("ifftp_read", st, bytes, ifftp_read_kernel<float, F, float><<<grid, 256, 0, st>>>(        \
                (const V4*)psi4, g, (const float*)positions, (const float*)pos_rec, npos, f, gl, l[0], l[1], l[2],  \
                field, shifted, wrap, (float*)out, flags, order));                                                       \
        else if (pos_bytes == 4)                                                                                  \
            PRC_LAUNCH_B("ifftp_read", st, bytes, ifftp_read_kernel<float, F, double><<<grid, 256, 0, st>>>(       \
                (const V4*)psi4, g, (const float*)positions, (const float*)pos_rec, npos, f, gl, l[0], l[1], l[2],  \
                field, shifted, wrap, (double*)out, flags, order));                                                      \
        else if (out_bytes == 4)                                                                                  \
            PRC_LAUNCH_B("ifftp_read", st, bytes, ifftp_read_kernel<double, F, float><<<grid, 256, 0, st>>>(       \
                (const V4*)psi4, g, (const double*)positions, (const double*)pos_rec, npos, f, gl, l[0], l[1],      \
                l[2], field, shifted, wrap, (float*)out, flags, order));                                                 \
        else                                                                                                      \
            PRC_LAUNCH_B("ifftp_read", st, bytes, ifftp_read_kernel<double, F, double><<<grid, 256, 0, st>>>(      \
                (const V4*)psi4, g, (const double*)positions, (const double*)pos_rec, npos, f, gl, l[0], l[1],      \
                l[2], field, shifted, wrap, (double*)out, flags, order));                                                \
        PRC_CHECK_LAUNCH();                                                                                       \
        return PRC_OK;                                                                                            \
    }
IFFTP_READ_IMPL(prc_ifftp_read_f32, float)
IFFTP_READ_IMPL(prc_ifftp_read_f64, double)

}  // extern "C"

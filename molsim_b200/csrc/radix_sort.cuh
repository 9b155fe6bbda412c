// radix_sort.cuh -- stable LSD radix sort of (uint32 key, uint32 value) pairs.
//
// Used by the Verlet-cell rebuild so that the new particle order is a pure
// function of the positions: (cell, previous order), which for rebuilt
// systems is (cell, MOLSIM index).  8-bit digits; each pass is a histogram
// kernel, an exclusive scan of each digit's per-block counts (one block per
// digit) and a stable scatter that adds the digits' bases.  1024 items per block (256 threads x 4 rounds); within a round
// the item order is the thread order, so ranks come from __match_any_sync
// plus per-warp digit counts in shared memory.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace msg {

constexpr int RS_THREADS = 256;
constexpr int RS_ROUNDS = 4;
constexpr int RS_TILE = RS_THREADS * RS_ROUNDS;
constexpr int RS_BINS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;

template <int NB>
__global__ void __launch_bounds__(RS_THREADS) rs_hist(const uint32_t *__restrict__ keys, int n,
                                                      int shift, uint32_t *__restrict__ hist)
{
    __shared__ uint32_t cnt[NB];
    for (int b = threadIdx.x; b < NB; b += RS_THREADS) cnt[b] = 0;
    __syncthreads();
    const int base = blockIdx.x * RS_TILE;
#pragma unroll
    for (int k = 0; k < RS_ROUNDS; ++k) {
        int idx = base + k * RS_THREADS + threadIdx.x;
        if (idx < n) atomicAdd(&cnt[(keys[idx] >> shift) & (NB - 1)], 1u);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < NB; b += RS_THREADS) hist[b * gridDim.x + blockIdx.x] = cnt[b];
}

// Exclusive scan of each digit's row of per-tile counts in place (row d holds
// hist[d * ntile + tile]), one block per digit, 256 consecutive entries at a
// time; the row total goes to tot[d].  The scatter adds the exclusive scan of
// the totals (the digit's base), so the two together give the exclusive scan
// of the whole (digit, tile) table.
__global__ void __launch_bounds__(RS_THREADS) rs_scan(uint32_t *__restrict__ hist, int ntile,
                                                      uint32_t *__restrict__ tot)
{
    __shared__ uint32_t wsum[RS_WARPS];
    uint32_t *row = hist + (size_t)blockIdx.x * ntile;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    uint32_t carry = 0;
    for (int b0 = 0; b0 < ntile; b0 += RS_THREADS) {
        const int i = b0 + t;
        const uint32_t x = i < ntile ? row[i] : 0u;
        uint32_t v = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        if (lane == 31) wsum[w] = v;
        __syncthreads();
        uint32_t before = carry;
        for (int k = 0; k < w; ++k) before += wsum[k];
        uint32_t all = 0;
#pragma unroll
        for (int k = 0; k < RS_WARPS; ++k) all += wsum[k];
        if (i < ntile) row[i] = before + v - x;
        carry += all;
        __syncthreads();
    }
    if (t == 0) tot[blockIdx.x] = carry;
}

template <int NB>
__global__ void __launch_bounds__(RS_THREADS) rs_scatter(const uint32_t *__restrict__ kin,
                                                         const uint32_t *__restrict__ vin,
                                                         uint32_t *__restrict__ kout,
                                                         uint32_t *__restrict__ vout, int n, int shift,
                                                         const uint32_t *__restrict__ offs,
                                                         const uint32_t *__restrict__ tot)
{
    static_assert(NB == RS_THREADS, "one digit per thread");
    __shared__ uint32_t base[NB];
    __shared__ uint32_t wcnt[RS_WARPS][NB];
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    // the digit's base: exclusive scan of the digit totals
    {
        const uint32_t x = tot[t];
        uint32_t v = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        if (lane == 31) wcnt[0][w] = v;
        __syncthreads();
        uint32_t before = 0;
        for (int k = 0; k < w; ++k) before += wcnt[0][k];
        __syncthreads();
        base[t] = before + v - x + offs[t * gridDim.x + blockIdx.x];
#pragma unroll
        for (int ww = 0; ww < RS_WARPS; ++ww) wcnt[ww][t] = 0;
    }
    __syncthreads();
    const int blockbase = blockIdx.x * RS_TILE;
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll 1
    for (int k = 0; k < RS_ROUNDS; ++k) {
        const int idx = blockbase + k * RS_THREADS + t;
        const bool valid = idx < n;
        const uint32_t key = valid ? kin[idx] : 0u;
        const uint32_t val = valid ? vin[idx] : 0u;
        const uint32_t d = valid ? ((key >> shift) & (NB - 1)) : (uint32_t)NB;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int lrank = __popc(peers & lt);
        if (valid && lane == __ffs(peers) - 1) wcnt[w][d] = (uint32_t)__popc(peers);
        __syncthreads();
        if (valid) {
            uint32_t off = 0;
            for (int ww = 0; ww < w; ++ww) off += wcnt[ww][d];
            const uint32_t pos = base[d] + off + (uint32_t)lrank;
            kout[pos] = key;
            vout[pos] = val;
        }
        __syncthreads();
        for (int b = t; b < NB; b += RS_THREADS) {
            uint32_t tot = 0;
#pragma unroll
            for (int ww = 0; ww < RS_WARPS; ++ww) {
                tot += wcnt[ww][b];
                wcnt[ww][b] = 0;
            }
            base[b] += tot;
        }
        __syncthreads();
    }
}

// Sort n pairs by the low `bits` bits of the key in 8-bit passes.  k0/v0 hold
// the input; k1/v1 are scratch of the same size; hist needs 256*ceil(n/1024)
// + 256 entries (the per-tile counts, then the digit totals).  Returns true when the sorted data ended in (k1, v1), false when in
// (k0, v0).  Sets *launches.
inline bool radix_sort_pairs(uint32_t *k0, uint32_t *v0, uint32_t *k1, uint32_t *v1, uint32_t *hist,
                             int n, int bits, cudaStream_t st, int *launches = nullptr)
{
    const int nb = (n + RS_TILE - 1) / RS_TILE;
    if (launches) *launches = 0;
    if (n <= 0) return false;
    bool flip = false;
    for (int shift = 0; shift < bits; shift += 8) {
        uint32_t *ki = flip ? k1 : k0, *vi = flip ? v1 : v0;
        uint32_t *ko = flip ? k0 : k1, *vo = flip ? v0 : v1;
        uint32_t *tot = hist + (size_t)RS_BINS * nb;
        rs_hist<RS_BINS><<<nb, RS_THREADS, 0, st>>>(ki, n, shift, hist);
        rs_scan<<<RS_BINS, RS_THREADS, 0, st>>>(hist, nb, tot);
        rs_scatter<RS_BINS><<<nb, RS_THREADS, 0, st>>>(ki, vi, ko, vo, n, shift, hist, tot);
        if (launches) *launches += 3;
        flip = !flip;
    }
    return flip;
}

}  // namespace msg

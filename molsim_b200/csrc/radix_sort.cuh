// radix_sort.cuh -- stable LSD radix sort of (uint32 key, uint32 value) pairs.
//
// Used by the Verlet-cell rebuild so that the new particle order is a pure
// function of the positions: (cell, previous order), which for rebuilt
// systems is (cell, MOLSIM index).  8-bit digits; each pass is a histogram
// kernel, one exclusive scan over the (digit, block) table and a stable
// scatter.  1024 items per block (256 threads x 4 rounds); within a round
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

// Exclusive scan of len entries in place, one block of 1024 threads.
__global__ void __launch_bounds__(1024) rs_scan(uint32_t *__restrict__ a, int len)
{
    __shared__ uint32_t wsum[32];
    const int t = threadIdx.x, per = (len + 1023) / 1024;
    const int b = t * per, e = min(len, b + per);
    uint32_t s = 0;
    // eight independent loads in flight per thread
    for (int i0 = b; i0 < e; i0 += 8) {
        uint32_t x[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = (i0 + k < e) ? a[i0 + k] : 0u;
#pragma unroll
        for (int k = 0; k < 8; ++k) s += x[k];
    }
    // inclusive warp scan of the per-thread sums
    uint32_t v = s;
    const int lane = t & 31, w = t >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
    }
    if (lane == 31) wsum[w] = v;
    __syncthreads();
    if (w == 0) {
        uint32_t x = wsum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        wsum[lane] = x;
    }
    __syncthreads();
    uint32_t run = v - s + (w > 0 ? wsum[w - 1] : 0u);
    for (int i0 = b; i0 < e; i0 += 8) {
        uint32_t x[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = (i0 + k < e) ? a[i0 + k] : 0u;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (i0 + k < e) a[i0 + k] = run;
            run += x[k];
        }
    }
}

template <int NB>
__global__ void __launch_bounds__(RS_THREADS) rs_scatter(const uint32_t *__restrict__ kin,
                                                         const uint32_t *__restrict__ vin,
                                                         uint32_t *__restrict__ kout,
                                                         uint32_t *__restrict__ vout, int n, int shift,
                                                         const uint32_t *__restrict__ offs)
{
    __shared__ uint32_t base[NB];
    __shared__ uint32_t wcnt[RS_WARPS][NB];
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    for (int b = t; b < NB; b += RS_THREADS) {
        base[b] = offs[b * gridDim.x + blockIdx.x];
#pragma unroll
        for (int ww = 0; ww < RS_WARPS; ++ww) wcnt[ww][b] = 0;
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
// entries.  Returns true when the sorted data ended in (k1, v1), false when in
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
        rs_hist<RS_BINS><<<nb, RS_THREADS, 0, st>>>(ki, n, shift, hist);
        rs_scan<<<1, 1024, 0, st>>>(hist, RS_BINS * nb);
        rs_scatter<RS_BINS><<<nb, RS_THREADS, 0, st>>>(ki, vi, ko, vo, n, shift, hist);
        if (launches) *launches += 3;
        flip = !flip;
    }
    return flip;
}

}  // namespace msg

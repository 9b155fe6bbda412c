// kernels_pair.cuh -- UTwoBodyA (Src/energy.F90:445-544) over the Verlet list.
//
// k_pair (below) serves the FP64 path over a full list; the mixed path runs
// k_pair_h, at the end of this file, over a half list by default (or over a
// full list), and keeps k_pair_m and k_pair<PrecM> as tuning alternatives.
//
// One particle per group of G lanes; the lanes stride over the particle's
// row, so a row is read with coalesced 64-byte segments and every pair is
// evaluated by both of its particles (forces need no atomics and are summed in
// a fixed order).  Each pair's energy and virial are counted once (i < j).
// List entries carry the partner's type in bits 28-29, so the type-pair record
// is found without a load of the partner's type.  A block owns a contiguous
// range of warp tasks (32/G particles each, G lanes per particle chosen per
// system from the row length), keeps the current system's table (coefficient
// rows and bucket starts) in shared memory, and its warps pull tasks from a
// shared counter, so no barrier waits on a long row.  The G lanes of a particle read
// consecutive row entries -- consecutive particles of one cell, so the
// position gathers coalesce -- and in FP32 each lane carries two such entries
// in lockstep, so their loads and polynomial chains overlap.
// Each particle's energy and virial are rounded once to 64-bit fixed point and
// summed as integers, so the totals do not depend on the task layout.
//
// Two precisions share the kernel:
//   PrecD  positions double4, table FP64, forces summed in FP64 registers;
//   PrecM  positions as 32-bit fixed-point box coordinates (exact, wrapping
//          differences converted to FP32), table and pair forces FP32; each
//          lane's partial force (a few pair terms, FP32) is rounded to 64-bit
//          fixed point (2^-32 kJ/(mol A)) and the lanes are combined as
//          integers, so the result does not depend on the combination order.
// Energies and virial are summed in FP64 within a block and added to the
// system's 64-bit fixed-point accumulators (order-independent) in both.
#pragma once

#include "common.cuh"

namespace msg {

constexpr int PAIR_BLOCK = 256;
constexpr int MAXT = 4;
constexpr int NBL_JMASK = (1 << 28) - 1;
constexpr double kFixScale = 4294967296.0;          // 2^32
constexpr double kFixInv = 1.0 / 4294967296.0;

struct PrecD {
    using R = double;
    using V4 = double4;
    static constexpr bool mixed = false;
};
struct PrecM {
    using R = float;
    using V4 = int4;   // fixed-point box coordinates (fx_pos)
    static constexpr bool mixed = true;
};

// Interval of MOLSIM's table (Src/energy.F90:481-486): the reference walks
// ibuf upwards from iubuflow while r2 < zlow.  pair_eval starts the walk at a
// bucket entry chosen on the host to lie at or before the interval the full
// walk finds, then makes the same comparisons, so it ends on the same interval.
__device__ __forceinline__ double pbc_shift(double d, double half, double box)
{
    return (fabs(d) > half) ? d - copysign(box, d) : d;
}

// Warp tasks: 32/G consecutive particles of one system, G lanes each.  send is
// the index one past the last task of the same system (a task run).
struct PairTask { int sys, i0, i1, g, send, pad0, pad1, pad2; };

// Coefficient row of 12 values ([0] = zlow of the interval,
// Src/potential.F90:1192-1207) read with 16-byte loads.
template <typename R> struct Row12;
template <> struct Row12<double> {
    double c[12];
    __device__ __forceinline__ void load(const double *p)
    {
        const double2 *q = reinterpret_cast<const double2 *>(p);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const double2 v = q[k];
            c[2 * k] = v.x;
            c[2 * k + 1] = v.y;
        }
    }
};
template <> struct Row12<float> {
    float c[12];
    __device__ __forceinline__ void load(const float *p)
    {
        const float4 *q = reinterpret_cast<const float4 *>(p);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float4 v = q[k];
            c[4 * k] = v.x;
            c[4 * k + 1] = v.y;
            c[4 * k + 2] = v.z;
            c[4 * k + 3] = v.w;
        }
    }
};

// Row of the half-list kernel's table: 16 floats, [z_hi, z_lo, c1_hi, c1_lo, c2..c6,
// c7_hi, c7_lo, c8..c11, 0], the interval's z_low, u(z_low) and f(z_low) each as an
// FP32 pair whose sum is the FP64 value to 2^-48 (Src/potential.F90:1192-1207 layout
// otherwise).  With them d = r2 - z_low and the two polynomials' leading terms carry
// no FP32 rounding of the table itself.
struct Row16 {
    float c[16];
    __device__ __forceinline__ void load(const float *p)
    {
        const float4 *q = reinterpret_cast<const float4 *>(p);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float4 v = q[k];
            c[4 * k] = v.x;
            c[4 * k + 1] = v.y;
            c[4 * k + 2] = v.z;
            c[4 * k + 3] = v.w;
        }
    }
};
constexpr int ROW16 = 16;
// Rows are laid out 20 floats apart: with a 64-byte stride every row would start in one of
// two 16-byte bank groups, and the 8 lanes of a 16-byte shared load phase, each reading its
// own row, would collide 4 ways; a 80-byte stride spreads row starts over 8 bank groups.
constexpr int ROWST = 20;

// r2 of a pair from its exact fixed-point coordinate differences: in a cubic box
// the exact 64-bit integer sum of squares (each square < 2^62) rounded to FP32 and
// scaled by (box/2^32)^2 in FP32 (two roundings); otherwise in FP64, rounded once.
// Unlike dx^2 + dy^2 + dz^2 from FP32 differences it carries no error of the
// coordinate conversions, whose bias would reach the energy sums.
__device__ __forceinline__ float r2_from_fix(int ax, int ay, int az, const SysDev &S)
{
    if (S.fx_cubic) {
        const unsigned long long q = (unsigned long long)((long long)ax * ax) + (unsigned long long)((long long)ay * ay) +
                                     (unsigned long long)((long long)az * az);
        return __ull2float_rn(q) * S.fx2f;
    }
    const double x = (double)ax * S.fxd[0], y = (double)ay * S.fxd[1], z = (double)az * S.fxd[2];
    return __double2float_rn(fma(x, x, fma(y, y, z * z)));
}

// Shared-memory image of a system's table: coefficient rows, then bucket
// starts.  Sized on the host (pair_smem_bytes); systems whose table does not
// fit read it from global memory through the same generic pointers.
template <typename R>
__host__ __device__ inline size_t pair_smem_bytes(int nk, int nbucket)
{
    return (size_t)nk * 12 * sizeof(R) + (size_t)nbucket * sizeof(unsigned short);
}

// Shared-memory image of a system's table for k_pair_m (12 floats a row) and
// k_pair_h (16): FP32 coefficient rows, then (row, z_low) buckets.
__host__ __device__ inline size_t lean_smem_bytes(int nk, int nbucket, int rowf = 12)
{
    return (size_t)nk * rowf * sizeof(float) + (size_t)nbucket * sizeof(int2);
}

// Lanes per batch: B row segments per lane are in flight together.
#ifndef MSG_PAIR_B32
#define MSG_PAIR_B32 2
#endif
#ifndef MSG_PAIR_MINB
#define MSG_PAIR_MINB 2
#endif
#ifndef MSG_PAIR_MINB_M
#define MSG_PAIR_MINB_M 3
#endif
template <class PR> struct PairBatch { static constexpr int B = PR::mixed ? MSG_PAIR_B32 : 1; };

// NT: particle types per system accounted in registers (2 or 4).
// Block b owns warp tasks [b*ntasks/nb, (b+1)*ntasks/nb); it walks them in runs of
// one system: load that system's table into shared memory, let its warps pull
// tasks from a shared counter, and meet at a barrier only where the run ends.
template <class PR, int NT>
__global__ void __launch_bounds__(PAIR_BLOCK, MSG_PAIR_MINB) k_pair(
    const SysDev *__restrict__ sysv, const PairTask *__restrict__ tasks, int ntasks,
    const typename PR::V4 *__restrict__ pos, const int *__restrict__ typ, const int *__restrict__ nbl,
    const int *__restrict__ nnb, const int *__restrict__ ptmap, const PairTab *__restrict__ ptab,
    const typename PR::R *__restrict__ tz, const typename PR::R *__restrict__ tc,
    const unsigned short *__restrict__ bst, double4 *__restrict__ fsr, long long *__restrict__ eacc, ErrWord *err)
{
    using R = typename PR::R;
    using V4 = typename PR::V4;
    constexpr int B = PairBatch<PR>::B;
    (void)tz;
    extern __shared__ __align__(16) unsigned char dyn[];
    __shared__ PairTab sP[MSG_MAX_NATAT];
    __shared__ int sMap[MAXT * MAXT];
    __shared__ int sNext;
    const int lane = threadIdx.x & 31;
    const int t0 = (int)(((long long)blockIdx.x * ntasks) / gridDim.x);
    const int t1 = (int)(((long long)(blockIdx.x + 1) * ntasks) / gridDim.x);
    // energies by (particle type, partner type) in 64-bit fixed point: each particle's
    // contribution is rounded once, so the sums do not depend on which warp took which task
    long long ue[NT * NT];
    long long vir = 0;
#pragma unroll
    for (int q = 0; q < NT * NT; ++q) ue[q] = 0;
    int loaded = -1;
    const R *Tc = nullptr;
    const unsigned short *Tb = nullptr;
    int kbase = 0, bbase = 0;
    for (int rs = t0; rs < t1;) {
        const PairTask W0 = tasks[rs];
        const int re = min(t1, W0.send);
        __syncthreads();                      // previous run's warps are done with sNext / the table
        if (W0.sys != loaded) {
            const SysDev &Sn = sysv[W0.sys];
            if (threadIdx.x < Sn.natat) sP[threadIdx.x] = ptab[Sn.pt_off + threadIdx.x];
            if (threadIdx.x < Sn.npt * Sn.npt) sMap[threadIdx.x] = ptmap[Sn.ptmap_off + threadIdx.x] - Sn.pt_off;
            kbase = Sn.tab_k0;
            bbase = Sn.tab_b0;
            if (Sn.tab_smem) {
                R *sc = reinterpret_cast<R *>(dyn);
                unsigned short *sb = reinterpret_cast<unsigned short *>(sc + (size_t)12 * Sn.tab_nk);
                const int nc = 12 * Sn.tab_nk, nb = Sn.natat * MSG_NBUCKET;
                for (int k = threadIdx.x; k < nc; k += PAIR_BLOCK) sc[k] = tc[(size_t)12 * Sn.tab_k0 + k];
                for (int k = threadIdx.x; k < nb; k += PAIR_BLOCK) sb[k] = bst[Sn.tab_b0 + k];
                Tc = sc;
                Tb = sb;
            } else {
                Tc = tc + (size_t)12 * Sn.tab_k0;
                Tb = bst + Sn.tab_b0;
            }
            loaded = W0.sys;
        }
        if (threadIdx.x == 0) sNext = rs;
        __syncthreads();
        const SysDev &S = sysv[W0.sys];
        const R rcut2 = (R)S.rcut2;
        const R lowmax = (R)fmax(S.r2umin_max, S.r2atat_max);
        for (;;) {
            int task = 0;
            if (lane == 0) task = atomicAdd(&sNext, 1);
            task = __shfl_sync(0xffffffffu, task, 0);
            if (task >= re) break;
            const PairTask W = tasks[task];
            const int G = W.g;
            const int g = lane & (G - 1);
            const int i = W.i0 + lane / G;
            const bool act = i < W.i1;
            // lane partial sums in R: a lane adds only a few pair terms before the
            // particle's sums are rounded to 64-bit fixed point
            R fx = 0, fy = 0, fz = 0;
            R ut[NT];                                        // energy by partner type
            R vi = 0;
#pragma unroll
            for (int t = 0; t < NT; ++t) ut[t] = 0;
            int ti = 0, n = 0;
            V4 xi;
            const int *row = nbl;
            if (act) {
                xi = pos[i];
                ti = typ[i];
                n = nnb[i];
                row = nbl + S.nbl_off + (long long)(i - S.off) * S.cap;
            }
            for (int kb = g; kb < n; kb += B * G) {
                // B row entries G apart per lane: the particle's G lanes read consecutive entries
                int ee[B];
                bool ok[B];
                V4 xj[B];
#pragma unroll
                for (int u = 0; u < B; ++u) {
                    ok[u] = kb + u * G < n;
                    ee[u] = ok[u] ? __ldg(row + kb + u * G) : 0;
                }
#pragma unroll
                for (int u = 0; u < B; ++u) xj[u] = pos[ok[u] ? (ee[u] & NBL_JMASK) : i];
                R dx[B], dy[B], dz[B], r2[B];
#pragma unroll
                for (int u = 0; u < B; ++u) {
                    if constexpr (PR::mixed) {
                        // exact integer difference, wrapped to the minimum image
                        dx[u] = (float)(int)((unsigned)xi.x - (unsigned)xj[u].x) * S.fxi[0];
                        dy[u] = (float)(int)((unsigned)xi.y - (unsigned)xj[u].y) * S.fxi[1];
                        dz[u] = (float)(int)((unsigned)xi.z - (unsigned)xj[u].z) * S.fxi[2];
                        r2[u] = dx[u] * dx[u] + dy[u] * dy[u] + dz[u] * dz[u];
                    } else {
                        dx[u] = pbc_shift(xi.x - xj[u].x, S.half[0], S.box[0]);
                        dy[u] = pbc_shift(xi.y - xj[u].y, S.half[1], S.box[1]);
                        dz[u] = pbc_shift(xi.z - xj[u].z, S.half[2], S.box[2]);
                        // the reference's rounding: ((dx*dx)+(dy*dy))+(dz*dz), no FMA
                        r2[u] = __dadd_rn(__dadd_rn(__dmul_rn(dx[u], dx[u]), __dmul_rn(dy[u], dy[u])),
                                          __dmul_rn(dz[u], dz[u]));
                    }
                    ok[u] = ok[u] && !(r2[u] > rcut2);
                }
                int tj[B], kk[B], pi[B];
#pragma unroll
                for (int u = 0; u < B; ++u) {
                    tj[u] = (unsigned)ee[u] >> 28;
                    pi[u] = sMap[ti * S.npt + (ok[u] ? tj[u] : 0)];
                    const PairTab &P = sP[pi[u]];
                    const float r2f = (float)r2[u];
                    int k = 0;
                    if (r2f < P.fz_hi) {
                        int bk = (int)((r2f - P.fz_lo) * P.finv_h);
                        bk = bk < 0 ? 0 : (bk >= MSG_NBUCKET ? MSG_NBUCKET - 1 : bk);
                        k = Tb[P.b0 - bbase + bk];
                    }
                    kk[u] = k;
                }
                Row12<R> c[B];
#pragma unroll
                for (int u = 0; u < B; ++u) c[u].load(Tc + (size_t)(sP[pi[u]].k0 - kbase + kk[u]) * 12);
                R usum[B], fsum[B];
#pragma unroll
                for (int u = 0; u < B; ++u) {
                    if (ok[u] && (r2[u] < lowmax || r2[u] < c[u].c[0])) {
                        // rare: below the type pair's lower limits, or the walk goes past the bucket start
                        const PairTab &Q = sP[pi[u]];
                        if (r2[u] < (R)Q.r2atat) {
                            // hard-core overlap: u = 1e10, f = 0 (the reference leaves fsum stale here)
                            c[u].c[0] = r2[u];
                            c[u].c[1] = (R)1e10;
#pragma unroll
                            for (int q = 2; q < 12; ++q) c[u].c[q] = (R)0;
                        } else if (r2[u] < (R)Q.r2umin) {
                            raise_error(err, 1, W.sys, i, ee[u] & NBL_JMASK);
                            ok[u] = false;
                        } else {
                            while (r2[u] < c[u].c[0]) {
                                if (++kk[u] >= Q.nk) {
                                    raise_error(err, 2, W.sys, i, ee[u] & NBL_JMASK);
                                    kk[u] = Q.nk - 1;
                                    c[u].load(Tc + (size_t)(Q.k0 - kbase + kk[u]) * 12);
                                    break;
                                }
                                c[u].load(Tc + (size_t)(Q.k0 - kbase + kk[u]) * 12);
                            }
                        }
                    }
                    const R d = r2[u] - c[u].c[0];
                    usum[u] = c[u].c[1] + d * (c[u].c[2] + d * (c[u].c[3] + d * (c[u].c[4] + d * (c[u].c[5] +
                              d * c[u].c[6]))));
                    fsum[u] = c[u].c[7] + d * (c[u].c[8] + d * (c[u].c[9] + d * (c[u].c[10] + d * c[u].c[11])));
                }
#pragma unroll
                for (int u = 0; u < B; ++u) {
                    if (!ok[u]) continue;
                    const int j = ee[u] & NBL_JMASK;
                    fx += fsum[u] * dx[u];
                    fy += fsum[u] * dy[u];
                    fz += fsum[u] * dz[u];
                    if (i < j) {
#pragma unroll
                        for (int t = 0; t < NT; ++t) ut[t] += (tj[u] == t) ? usum[u] : (R)0;
                        vi -= fsum[u] * r2[u];
                    }
                }
            }
#pragma unroll
            for (int t = 0; t < NT; ++t) {
                const long long v = __double2ll_rn((double)ut[t] * kEFix);
#pragma unroll
                for (int q = 0; q < NT; ++q) ue[q * NT + t] += (q == ti) ? v : 0;
            }
            vir += __double2ll_rn((double)vi * kEFix);
            // reduce the particle's force over its G lanes; in FP32 mode each lane's FP64
            // partial is rounded to 64-bit fixed point first, so the combination is exact
            if constexpr (PR::mixed) {
                long long ax = __double2ll_rn((double)fx * kFixScale), ay = __double2ll_rn((double)fy * kFixScale),
                          az = __double2ll_rn((double)fz * kFixScale);
                for (int o = G >> 1; o > 0; o >>= 1) {
                    ax += __shfl_xor_sync(0xffffffffu, ax, o);
                    ay += __shfl_xor_sync(0xffffffffu, ay, o);
                    az += __shfl_xor_sync(0xffffffffu, az, o);
                }
                if (act && g == 0)
                    fsr[i] = make_double4((double)ax * kFixInv, (double)ay * kFixInv, (double)az * kFixInv, 0.0);
            } else {
                for (int o = G >> 1; o > 0; o >>= 1) {
                    fx += __shfl_xor_sync(0xffffffffu, fx, o);
                    fy += __shfl_xor_sync(0xffffffffu, fy, o);
                    fz += __shfl_xor_sync(0xffffffffu, fz, o);
                }
                if (act && g == 0) fsr[i] = make_double4((double)fx, (double)fy, (double)fz, 0.0);
            }
        }
        // the run's energies: per warp, integer sums into the system's accumulators
#pragma unroll
        for (int q = 0; q < NT * NT; ++q)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) ue[q] += __shfl_xor_sync(0xffffffffu, ue[q], o);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vir += __shfl_xor_sync(0xffffffffu, vir, o);
        long long *ea = eacc + (size_t)W0.sys * EA_N;
        if (lane < S.npt * S.npt) {
            const int ti = lane / S.npt, tj = lane % S.npt;
            // (ti, tj) and (tj, ti) are one type pair: take ti <= tj and add both halves
            if (ti <= tj) {
                long long v = 0;
#pragma unroll
                for (int q = 0; q < NT * NT; ++q)
                    v += (q == ti * NT + tj || (ti != tj && q == tj * NT + ti)) ? ue[q] : 0;
                if (v) atomicAdd(reinterpret_cast<unsigned long long *>(ea + EA_UTWOB + sMap[lane]), (unsigned long long)v);
            }
        }
        if (lane == 31 && vir) atomicAdd(reinterpret_cast<unsigned long long *>(ea + EA_VIRPAIR), (unsigned long long)vir);
#pragma unroll
        for (int q = 0; q < NT * NT; ++q) ue[q] = 0;
        vir = 0;
        rs = re;
    }
}

// ---------------------------------------------------------------------------
// Lean FP32 pair kernel of the mixed-precision path.
//
// Same work split as k_pair (G lanes per particle over the full list, tasks
// pulled from a shared counter, the system's table in shared memory), with
// less work and more memory parallelism per list entry:
//   * one shared record per (particle type, partner type): the FP32 bucket
//     grid (z_lo, 1/h) and the bucket base, read with one 16-byte load;
//   * a bucket holds the interval containing its top, as a row of the system's
//     table, and that interval's z_low; a pair below that z_low takes the next
//     row.  Intervals are wider than buckets except at the shortest distances,
//     so this compare replaces MOLSIM's walk for all but about 2e-4 of the
//     pairs, which still walk (`bkz`, built on the host);
//   * above the table top the clamped last bucket already names the first
//     interval, so there is no separate upper-range test;
//   * every pair is seen from both ends; each end adds half of the pair's
//     energy and virial, so there is no ownership test per entry;
//   * each lane loads U row entries, then their U partner positions, before
//     it uses any of them, so U gathers per lane are in flight together;
//   * each system has a global task counter; a block starts at the system that
//     holds its share of the tasks, its warps pull tasks from that counter
//     until it runs dry, then the block moves on to the next system (the
//     table is reloaded only then), so blocks that draw cheap tasks take more
//     of them; the last block to finish resets the counters for the next launch.
// The interval found is the one MOLSIM's walk ends on (Src/energy.F90:481-486),
// as in k_pair.
// ---------------------------------------------------------------------------

// Unordered type pair (a <= b) of NT types -> 0 .. NT(NT+1)/2-1, a-major.
template <int NT>
__host__ __device__ constexpr int tpair(int a, int b) { return a * (2 * NT - a + 1) / 2 + (b - a); }

// Register budget with two particle types: one entry in flight per lane (U = 1) leaves room
// for 4 blocks of 256 per SM, two entries for 3; otherwise 2 blocks.
template <int NT, int U>
__global__ void __launch_bounds__(PAIR_BLOCK, NT == 2 ? (U == 1 ? 4 : (U == 2 ? MSG_PAIR_MINB_M : 2)) : 2) k_pair_m(
    const SysDev *__restrict__ sysv, const PairTask *__restrict__ tasks, const int2 *__restrict__ srange,
    int nsys, int ntasks, int *__restrict__ sched,
    const int4 *__restrict__ pos, const int *__restrict__ typ, const int *__restrict__ nbl,
    const int *__restrict__ nnb, const int *__restrict__ ptmap, const PairTab *__restrict__ ptab,
    const float *__restrict__ tc, const int2 *__restrict__ bkz, double4 *__restrict__ fsr,
    long long *__restrict__ eacc, ErrWord *err)
{
    extern __shared__ __align__(16) unsigned char dyn[];
    __shared__ PairTab sP[MSG_MAX_NATAT];
    __shared__ float4 sT[MAXT * MAXT];        // (z_lo, 1/h, end row, bucket base), the last two as int bits
    __shared__ int sMap[MAXT * MAXT];
    __shared__ int sNpt, sDrained;
    const int lane = threadIdx.x & 31;
    // energies by unordered type pair and the virial, 64-bit fixed point per lane
    constexpr int NQ = tpair<NT>(NT - 1, NT - 1) + 1;
    long long ue[NQ];
    long long vir = 0;
#pragma unroll
    for (int q = 0; q < NQ; ++q) ue[q] = 0;
    int loaded = -1;
    const float *Tc = nullptr;
    const int2 *Tb = nullptr;
    int kbase = 0;
    // the lanes' energy sums belong to system `held`; they go to its accumulators
    // (one warp-wide sum per lane group) when the block moves to another system
    int held = -1;
    auto flush = [&](int sys) {
#pragma unroll
        for (int q = 0; q < NQ; ++q)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) ue[q] += __shfl_xor_sync(0xffffffffu, ue[q], o);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vir += __shfl_xor_sync(0xffffffffu, vir, o);
        long long *ea = eacc + (size_t)sys * EA_N;
        const int npt = sNpt;
        if (lane < npt * npt) {
            const int ta = lane / npt, tb = lane % npt;
            if (ta <= tb) {
                long long v = 0;
#pragma unroll
                for (int a = 0; a < NT; ++a)
#pragma unroll
                    for (int b = a; b < NT; ++b) v += (a == ta && b == tb) ? ue[tpair<NT>(a, b)] : 0;
                if (v) atomicAdd(reinterpret_cast<unsigned long long *>(ea + EA_UTWOB + sMap[lane]), (unsigned long long)v);
            }
        }
        if (lane == 31 && vir) atomicAdd(reinterpret_cast<unsigned long long *>(ea + EA_VIRPAIR), (unsigned long long)vir);
#pragma unroll
        for (int q = 0; q < NQ; ++q) ue[q] = 0;
        vir = 0;
    };
    // the system holding this block's share of the tasks
    int s0 = 0;
    {
        const int p = (int)(((long long)blockIdx.x * ntasks) / gridDim.x);
        while (s0 + 1 < nsys && srange[s0].y <= p) ++s0;
    }
    for (int visit = 0; visit < nsys; ++visit) {
        const int sys = (s0 + visit) % nsys;
        const int2 R = srange[sys];           // the system's tasks [R.x, R.y)
        if (R.y <= R.x) continue;
        __syncthreads();                      // every warp is done with the previous system
        // skip a system other blocks have drained already (one read, shared by the block)
        if (threadIdx.x == 0) sDrained = atomicAdd(&sched[sys], 0) >= R.y - R.x;
        __syncthreads();
        if (sDrained) continue;
        if (held >= 0) flush(held);
        held = sys;
        if (sys != loaded) {
            __syncthreads();                  // every warp has flushed with the old type map
            const PairTask W0 = tasks[R.x];
            const SysDev &Sn = sysv[W0.sys];
            if (threadIdx.x < Sn.natat) sP[threadIdx.x] = ptab[Sn.pt_off + threadIdx.x];
            if (threadIdx.x < Sn.npt * Sn.npt) {
                const int q = ptmap[Sn.ptmap_off + threadIdx.x] - Sn.pt_off;
                sMap[threadIdx.x] = q;
                const PairTab &P = ptab[Sn.pt_off + q];
                const int a = threadIdx.x / Sn.npt, b = threadIdx.x % Sn.npt;
                sT[a * MAXT + b] = make_float4(P.fz_lo, P.finv_h, __int_as_float(P.k0 - Sn.tab_k0 + P.nk),
                                               __int_as_float(q * MSG_NBUCKET));
            }
            kbase = Sn.tab_k0;
            if (Sn.tab_smem_m) {
                float *sc = reinterpret_cast<float *>(dyn);
                int2 *sb = reinterpret_cast<int2 *>(sc + (size_t)12 * Sn.tab_nk);
                const int nc = 12 * Sn.tab_nk, nb = Sn.natat * MSG_NBUCKET;
                for (int k = threadIdx.x; k < nc; k += PAIR_BLOCK) sc[k] = tc[(size_t)12 * Sn.tab_k0 + k];
                for (int k = threadIdx.x; k < nb; k += PAIR_BLOCK) sb[k] = bkz[Sn.tab_b0 + k];
                Tc = sc;
                Tb = sb;
            } else {
                Tc = tc + (size_t)12 * Sn.tab_k0;
                Tb = bkz + Sn.tab_b0;
            }
            if (threadIdx.x == 0) sNpt = Sn.npt;
            loaded = W0.sys;
        }
        __syncthreads();
        const SysDev &S = sysv[sys];
        const float rcut2 = (float)S.rcut2;
        const float lowmax = (float)fmax(S.r2umin_max, S.r2atat_max);
        const float sx = S.fxi[0], sy = S.fxi[1], sz = S.fxi[2];
        // the next task's index is fetched while this one runs, hiding the atomic's latency
        int nxt = 0;
        if (lane == 0) nxt = R.x + atomicAdd(&sched[sys], 1);
        for (;;) {
            const int task = __shfl_sync(0xffffffffu, nxt, 0);
            if (task >= R.y) break;
            if (lane == 0) nxt = R.x + atomicAdd(&sched[sys], 1);
            const PairTask W = tasks[task];
            const int G = W.g;
            const int g = lane & (G - 1);
            const int i = W.i0 + lane / G;
            const bool act = i < W.i1;
            float fx = 0.0f, fy = 0.0f, fz = 0.0f, vi = 0.0f;
            float ut[NT];
#pragma unroll
            for (int t = 0; t < NT; ++t) ut[t] = 0.0f;
            int ti = 0, n = 0;
            int4 xi = make_int4(0, 0, 0, 0);
            const int *row = nbl;
            if (act) {
                xi = pos[i];
                ti = typ[i];
                n = nnb[i];
                row = nbl + S.nbl_off + (long long)(i - S.off) * S.cap;
            }
            const float4 *sTi = sT + ti * MAXT;
            // U row entries per lane in flight: their indices, then their partners' positions,
            // are loaded before any of them is used
            for (int kb = g; kb < n; kb += U * G) {
                int ee[U];
                int4 xj[U];
#pragma unroll
                for (int u = 0; u < U; ++u) ee[u] = (kb + u * G < n) ? __ldg(row + kb + u * G) : -1;
#pragma unroll
                for (int u = 0; u < U; ++u) xj[u] = pos[ee[u] >= 0 ? (ee[u] & NBL_JMASK) : i];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (ee[u] < 0) continue;
                    const int e = ee[u];
                    const int j = e & NBL_JMASK;
                    const int tj = (unsigned)e >> 28;
                    // exact integer difference, wrapped to the minimum image
                    const float dx = (float)(int)((unsigned)xi.x - (unsigned)xj[u].x) * sx;
                    const float dy = (float)(int)((unsigned)xi.y - (unsigned)xj[u].y) * sy;
                    const float dz = (float)(int)((unsigned)xi.z - (unsigned)xj[u].z) * sz;
                    const float r2 = dx * dx + dy * dy + dz * dz;
                    if (r2 > rcut2) continue;
                    const float4 T = sTi[tj];
                    int bk = __float2int_rz((r2 - T.x) * T.y);
                    bk = min(max(bk, 0), MSG_NBUCKET - 1);
                    const int2 B = Tb[__float_as_int(T.w) + bk];
                    int kk = min(B.x + (r2 < __int_as_float(B.y) ? 1 : 0), __float_as_int(T.z) - 1);
                    Row12<float> c;
                    c.load(Tc + (size_t)kk * 12);
                    bool ok = true;
                    if (r2 < lowmax || r2 < c.c[0]) {
                        // rare: below the type pair's lower limits, or the walk goes past the bucket start
                        const PairTab &Q = sP[sMap[ti * S.npt + tj]];
                        const int kend = Q.k0 - kbase + Q.nk;
                        if (r2 < (float)Q.r2atat) {
                            // hard-core overlap: u = 1e10, f = 0 (the reference leaves fsum stale here)
                            c.c[0] = r2;
                            c.c[1] = 1e10f;
#pragma unroll
                            for (int q = 2; q < 12; ++q) c.c[q] = 0.0f;
                        } else if (r2 < (float)Q.r2umin) {
                            raise_error(err, 1, W.sys, i, j);
                            ok = false;
                        } else {
                            while (r2 < c.c[0]) {
                                if (++kk >= kend) {
                                    raise_error(err, 2, W.sys, i, j);
                                    kk = kend - 1;
                                    c.load(Tc + (size_t)kk * 12);
                                    break;
                                }
                                c.load(Tc + (size_t)kk * 12);
                            }
                        }
                    }
                    if (!ok) continue;
                    const float d = r2 - c.c[0];
                    const float uu = c.c[1] + d * (c.c[2] + d * (c.c[3] + d * (c.c[4] + d * (c.c[5] + d * c.c[6]))));
                    const float f = c.c[7] + d * (c.c[8] + d * (c.c[9] + d * (c.c[10] + d * c.c[11])));
                    fx += f * dx;
                    fy += f * dy;
                    fz += f * dz;
#pragma unroll
                    for (int t = 0; t < NT; ++t) ut[t] += (tj == t) ? uu : 0.0f;
                    vi -= f * r2;
                }
            }
            // each pair was seen from both ends: each end keeps half of its energy and virial
#pragma unroll
            for (int t = 0; t < NT; ++t) {
                const long long v = __double2ll_rn((double)ut[t] * (0.5 * kEFix));
#pragma unroll
                for (int a = 0; a < NT; ++a) ue[tpair<NT>(min(a, t), max(a, t))] += (a == ti) ? v : 0;
            }
            vir += __double2ll_rn((double)vi * (0.5 * kEFix));
            long long ax = __float2ll_rn(fx * 4294967296.0f), ay = __float2ll_rn(fy * 4294967296.0f),
                      az = __float2ll_rn(fz * 4294967296.0f);
            for (int o = G >> 1; o > 0; o >>= 1) {
                ax += __shfl_xor_sync(0xffffffffu, ax, o);
                ay += __shfl_xor_sync(0xffffffffu, ay, o);
                az += __shfl_xor_sync(0xffffffffu, az, o);
            }
            if (act && g == 0)
                fsr[i] = make_double4((double)ax * kFixInv, (double)ay * kFixInv, (double)az * kFixInv, 0.0);
        }
    }
    if (held >= 0) flush(held);
    // the last block to finish resets the task counters for the next launch
    __shared__ bool lastb;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        lastb = atomicAdd(&sched[nsys], 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    if (lastb) {
        for (int k = threadIdx.x; k <= nsys; k += blockDim.x) sched[k] = 0;
        __threadfence();
    }
}


// ---------------------------------------------------------------------------
// FP32 pair kernel of the mixed-precision path with FP64 energy and virial sums.
//
// The work split, the shared-memory table, the bucket lookup and the scheduling
// are k_pair_m's.  Each pair's r2 comes from the exact integer differences of the
// fixed-point coordinates (r2_from_fix), and the table rows carry z_low, c1 and c7
// as FP32 (hi, lo) pairs (Row16), so the per-pair energy and virial carry no
// systematic FP32 error; each lane sums them in FP64 and every particle's share
// is rounded once to 64-bit fixed point.  Forces stay FP32 per pair.
//
// HALF = true: the list holds each unordered pair once (the row half_owner
// names, k_nlist with half = 1), so every pair is evaluated once: half the list
// to stream, half the pair arithmetic.  The row particle's force is summed over
// its G lanes and stored to fsr; the partner's force (minus the same pair term)
// is rounded to 64-bit fixed point (2^-32 kJ/(mol A)) per pair and added with
// one integer atomic per component into fpart (x, y, z blocks of fstride
// entries), which k_finalize adds to fsr and clears for the next step.  Integer
// sums do not depend on their order, so results stay bitwise reproducible and
// identical whether a system runs alone or batched.  Each pair's energy and
// virial count once, in the row particle's lane.
// HALF = false: the full list (each pair from both ends), no atomics; each end
// keeps half of the pair's energy and virial.
// ---------------------------------------------------------------------------
// Register budget with two particle types: three blocks of 256 per SM with one or two row
// entries in flight per lane (two entries spill a few values to L1, and still run faster
// than at two blocks per SM), two blocks with four; two blocks with more types.
template <int NT, int U, bool HALF>
__global__ void __launch_bounds__(PAIR_BLOCK, (NT == 2 && U <= 2) ? 3 : 2) k_pair_h(
    const SysDev *__restrict__ sysv, const int *__restrict__ gsys, const int2 *__restrict__ srange,
    int nsys, int ntasks, int *__restrict__ sched,
    const int4 *__restrict__ pos, const int *__restrict__ typ, const int *__restrict__ nbl,
    const int *__restrict__ nnb, const int *__restrict__ ptmap, const PairTab *__restrict__ ptab,
    const float *__restrict__ tc, const int2 *__restrict__ bkz, double4 *__restrict__ fsr,
    unsigned long long *__restrict__ fpart, int fstride, long long *__restrict__ eacc, ErrWord *err)
{
    extern __shared__ __align__(16) unsigned char dyn[];
    __shared__ PairTab sP[MSG_MAX_NATAT];
    __shared__ float4 sT[MAXT * MAXT];        // (z_lo, 1/h, end row, bucket base), the last two as int bits
    __shared__ int sMap[MAXT * MAXT];
    __shared__ int sNpt, sDrained;
    const int lane = threadIdx.x & 31;
    constexpr int NQ = tpair<NT>(NT - 1, NT - 1) + 1;
    long long ue[NQ];
    long long vir = 0;
#pragma unroll
    for (int q = 0; q < NQ; ++q) ue[q] = 0;
    int loaded = -1;
    const float *Tc = nullptr;
    const int2 *Tb = nullptr;
    int kbase = 0;
    int held = -1;
    auto flush = [&](int sys) {
#pragma unroll
        for (int q = 0; q < NQ; ++q)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) ue[q] += __shfl_xor_sync(0xffffffffu, ue[q], o);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vir += __shfl_xor_sync(0xffffffffu, vir, o);
        long long *ea = eacc + (size_t)sys * EA_N;
        const int npt = sNpt;
        if (lane < npt * npt) {
            const int ta = lane / npt, tb = lane % npt;
            if (ta <= tb) {
                long long v = 0;
#pragma unroll
                for (int a = 0; a < NT; ++a)
#pragma unroll
                    for (int b = a; b < NT; ++b) v += (a == ta && b == tb) ? ue[tpair<NT>(a, b)] : 0;
                if (v) atomicAdd(reinterpret_cast<unsigned long long *>(ea + EA_UTWOB + sMap[lane]), (unsigned long long)v);
            }
        }
        if (lane == 31 && vir) atomicAdd(reinterpret_cast<unsigned long long *>(ea + EA_VIRPAIR), (unsigned long long)vir);
#pragma unroll
        for (int q = 0; q < NQ; ++q) ue[q] = 0;
        vir = 0;
    };
    unsigned long long *fpx = fpart, *fpy = fpart + fstride, *fpz = fpart + 2 * (size_t)fstride;
    int s0 = 0;
    {
        const int p = (int)(((long long)blockIdx.x * ntasks) / gridDim.x);
        while (s0 + 1 < nsys && srange[s0].y <= p) ++s0;
    }
    for (int visit = 0; visit < nsys; ++visit) {
        const int sys = (s0 + visit) % nsys;
        const int2 R = srange[sys];
        if (R.y <= R.x) continue;
        __syncthreads();
        if (threadIdx.x == 0) sDrained = atomicAdd(&sched[sys], 0) >= R.y - R.x;
        __syncthreads();
        if (sDrained) continue;
        if (held >= 0) flush(held);
        held = sys;
        if (sys != loaded) {
            __syncthreads();
            const SysDev &Sn = sysv[sys];
            if (threadIdx.x < Sn.natat) sP[threadIdx.x] = ptab[Sn.pt_off + threadIdx.x];
            if (threadIdx.x < Sn.npt * Sn.npt) {
                const int q = ptmap[Sn.ptmap_off + threadIdx.x] - Sn.pt_off;
                sMap[threadIdx.x] = q;
                const PairTab &P = ptab[Sn.pt_off + q];
                const int a = threadIdx.x / Sn.npt, b = threadIdx.x % Sn.npt;
                sT[a * MAXT + b] = make_float4(P.fz_lo, P.finv_h, __int_as_float(P.k0 - Sn.tab_k0 + P.nk),
                                               __int_as_float(q * MSG_NBUCKET));
            }
            kbase = Sn.tab_k0;
            if (Sn.tab_smem_h) {
                float *sc = reinterpret_cast<float *>(dyn);
                int2 *sb = reinterpret_cast<int2 *>(sc + (size_t)ROWST * Sn.tab_nk);
                const int nc = ROWST * Sn.tab_nk, nb = Sn.natat * MSG_NBUCKET;
                for (int k = threadIdx.x; k < nc; k += PAIR_BLOCK) sc[k] = tc[(size_t)ROWST * Sn.tab_k0 + k];
                for (int k = threadIdx.x; k < nb; k += PAIR_BLOCK) sb[k] = bkz[Sn.tab_b0 + k];
                Tc = sc;
                Tb = sb;
            } else {
                Tc = tc + (size_t)ROWST * Sn.tab_k0;
                Tb = bkz + Sn.tab_b0;
            }
            if (threadIdx.x == 0) sNpt = Sn.npt;
            loaded = sys;
        }
        __syncthreads();
        const SysDev &S = sysv[sys];
        const float rcut2 = (float)S.rcut2;
        const float lowmax = (float)fmax(S.r2umin_max, S.r2atat_max);
        const float sx = S.fxi[0], sy = S.fxi[1], sz = S.fxi[2];
        // a task is 32/G consecutive particles of the system, G lanes each (G per system)
        const int G = gsys[sys];
        const int per = 32 / G, g = lane & (G - 1);
        int nxt = 0;
        if (lane == 0) nxt = R.x + atomicAdd(&sched[sys], 1);
        for (;;) {
            const int task = __shfl_sync(0xffffffffu, nxt, 0);
            if (task >= R.y) break;
            if (lane == 0) nxt = R.x + atomicAdd(&sched[sys], 1);
            const int li = (task - R.x) * per + lane / G;
            const bool act = li < S.n;
            const int i = S.off + (act ? li : 0);
            // forces in FP32; energies and virial of the lane's pairs in FP64
            float fx = 0.0f, fy = 0.0f, fz = 0.0f;
            double vi = 0.0;
            double ut[NT];
#pragma unroll
            for (int t = 0; t < NT; ++t) ut[t] = 0.0;
            // the particle's own data and its first row entries are loaded together: the
            // entries' addresses need only i, and entries past the row's end are masked
            // once its length has arrived
            const int *row = nbl + S.nbl_off + (long long)(i - S.off) * S.cap;
            int ee[U];
#pragma unroll
            for (int u = 0; u < U; ++u) ee[u] = (g + u * G < S.cap) ? __ldg(row + g + u * G) : -1;
            const int4 xi = pos[i];
            const int ti = typ[i];
            const int n = act ? nnb[i] : 0;
            const float4 *sTi = sT + ti * MAXT;
            for (int kb = g; kb < n; kb += U * G) {
                int4 xj[U];
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (kb + u * G >= n) ee[u] = -1;
#pragma unroll
                for (int u = 0; u < U; ++u) xj[u] = pos[ee[u] >= 0 ? (ee[u] & NBL_JMASK) : i];
                // the next batch's entries go out before this batch is evaluated
                int en[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int kn = kb + U * G + u * G;
                    en[u] = (kn < n) ? __ldg(row + kn) : -1;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (ee[u] < 0) continue;
                    const int e = ee[u];
                    const int j = e & NBL_JMASK;
                    const int tj = (unsigned)e >> 28;
                    // exact integer differences, wrapped to the minimum image
                    const int ax = (int)((unsigned)xi.x - (unsigned)xj[u].x);
                    const int ay = (int)((unsigned)xi.y - (unsigned)xj[u].y);
                    const int az = (int)((unsigned)xi.z - (unsigned)xj[u].z);
                    const float r2 = r2_from_fix(ax, ay, az, S);
                    if (r2 > rcut2) continue;
                    const float dx = (float)ax * sx, dy = (float)ay * sy, dz = (float)az * sz;
                    const float4 T = sTi[tj];
                    int bk = __float2int_rz((r2 - T.x) * T.y);
                    bk = min(max(bk, 0), MSG_NBUCKET - 1);
                    const int2 B = Tb[__float_as_int(T.w) + bk];
                    int kk = min(B.x + (r2 < __int_as_float(B.y) ? 1 : 0), __float_as_int(T.z) - 1);
                    Row16 c;
                    c.load(Tc + (size_t)kk * ROWST);
                    bool ok = true;
                    if (r2 < lowmax || r2 < c.c[0]) {
                        const PairTab &Q = sP[sMap[ti * S.npt + tj]];
                        const int kend = Q.k0 - kbase + Q.nk;
                        if (r2 < (float)Q.r2atat) {
                            // hard-core overlap: u = 1e10, f = 0 (the reference leaves fsum stale here)
#pragma unroll
                            for (int q = 0; q < ROW16; ++q) c.c[q] = 0.0f;
                            c.c[0] = r2;
                            c.c[2] = 1e10f;
                        } else if (r2 < (float)Q.r2umin) {
                            raise_error(err, 1, sys, i, j);
                            ok = false;
                        } else {
                            while (r2 < c.c[0]) {
                                if (++kk >= kend) {
                                    raise_error(err, 2, sys, i, j);
                                    kk = kend - 1;
                                    c.load(Tc + (size_t)kk * ROWST);
                                    break;
                                }
                                c.load(Tc + (size_t)kk * ROWST);
                            }
                        }
                    }
                    if (!ok) continue;
                    // d = r2 - z_low with z_low's low part; the leading coefficients' low parts
                    // join the polynomials, so u and f round once each, without bias
                    const float d = (r2 - c.c[0]) - c.c[1];
                    const float ulo = c.c[3] + d * (c.c[4] + d * (c.c[5] + d * (c.c[6] + d * (c.c[7] + d * c.c[8]))));
                    const float flo = c.c[10] + d * (c.c[11] + d * (c.c[12] + d * (c.c[13] + d * c.c[14])));
                    const float f = c.c[9] + flo;
                    const double uu = (double)(c.c[2] + ulo);
                    const float px = f * dx, py = f * dy, pz = f * dz;
                    fx += px;
                    fy += py;
                    fz += pz;
                    if constexpr (HALF) {
                        // the partner's share: -f d, rounded once to 2^-32 and added as an integer
                        atomicAdd(fpx + j, (unsigned long long)__float2ll_rn(px * -4294967296.0f));
                        atomicAdd(fpy + j, (unsigned long long)__float2ll_rn(py * -4294967296.0f));
                        atomicAdd(fpz + j, (unsigned long long)__float2ll_rn(pz * -4294967296.0f));
                    }
#pragma unroll
                    for (int t = 0; t < NT; ++t)
                        if (tj == t) ut[t] += uu;
                    vi -= (double)(f * r2);
                }
#pragma unroll
                for (int u = 0; u < U; ++u) ee[u] = en[u];
            }
            // a full list sees each pair from both ends: each end keeps half of it
            constexpr double ef = HALF ? kEFix : 0.5 * kEFix;
#pragma unroll
            for (int t = 0; t < NT; ++t) {
                const long long v = __double2ll_rn(ut[t] * ef);
#pragma unroll
                for (int a = 0; a < NT; ++a) ue[tpair<NT>(min(a, t), max(a, t))] += (a == ti) ? v : 0;
            }
            vir += __double2ll_rn(vi * ef);
            long long ax = __float2ll_rn(fx * 4294967296.0f), ay = __float2ll_rn(fy * 4294967296.0f),
                      az = __float2ll_rn(fz * 4294967296.0f);
            for (int o = G >> 1; o > 0; o >>= 1) {
                ax += __shfl_xor_sync(0xffffffffu, ax, o);
                ay += __shfl_xor_sync(0xffffffffu, ay, o);
                az += __shfl_xor_sync(0xffffffffu, az, o);
            }
            if (act && g == 0)
                fsr[i] = make_double4((double)ax * kFixInv, (double)ay * kFixInv, (double)az * kFixInv, 0.0);
        }
    }
    if (held >= 0) flush(held);
    __shared__ bool lastb;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        lastb = atomicAdd(&sched[nsys], 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    if (lastb) {
        for (int k = threadIdx.x; k <= nsys; k += blockDim.x) sched[k] = 0;
        __threadfence();
    }
}

}  // namespace msg

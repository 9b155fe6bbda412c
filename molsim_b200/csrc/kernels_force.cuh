// kernels_force.cuh -- pair table force, SPME and per-step reductions.
#pragma once

#include "common.cuh"

namespace msg {

constexpr int PAIR_G = 8;                 // lanes per particle in the pair kernel
constexpr int PAIR_THREADS = 256;         // 32 particles per block (tile of 32)
constexpr int NPART_PAIR = MSG_MAX_NATAT + 1;
constexpr int MAXT = 4;                   // particle types per system (natat <= 10)

// Interval of MOLSIM's table (Src/energy.F90:481-486).  The reference walks
// ibuf upwards from iubuflow while r2 < zlow; the walk here starts at a bucket
// entry bstart[b] chosen on the host to lie at or before the interval the full
// walk would find, and then performs the same comparisons, so it ends on the
// same interval.
template <typename Z>
__device__ __forceinline__ int table_interval(const PairTab &P, const Z *__restrict__ tz,
                                              const unsigned short *__restrict__ bst, Z r2, bool &bad)
{
    int k = 0;
    if (r2 < (Z)P.z_hi) {
        int b = (int)((r2 - (Z)P.z_lo) * (Z)P.inv_h);
        b = b < 0 ? 0 : (b >= MSG_NBUCKET ? MSG_NBUCKET - 1 : b);
        k = bst[P.b0 + b];
    }
    const Z *z = tz + P.k0;
    while (r2 < __ldg(z + k)) {
        if (++k >= P.nk) { bad = true; k = P.nk - 1; break; }
    }
    return k;
}

// ---------------------------------------------------------------------------
// UTwoBodyA (Src/energy.F90:445-544) over a full Verlet list, FP64.
// PAIR_G lanes per particle; forces of particle i are summed in registers in
// a fixed order (no atomics).  Each pair's energy and virial are counted once
// (i < j); per-tile partial sums go to ppart[tile][type pair | virial].
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(PAIR_THREADS) k_pair_fp64(
    const SysDev *__restrict__ sysv, const Tile *__restrict__ tiles, const double4 *__restrict__ pos,
    const int *__restrict__ typ, const int *__restrict__ nbl, const int *__restrict__ nnb,
    const int *__restrict__ ptmap, const PairTab *__restrict__ ptab, const double *__restrict__ tz,
    const double *__restrict__ tc, const unsigned short *__restrict__ bst, double4 *__restrict__ fsr,
    double *__restrict__ ppart, ErrWord *err)
{
    __shared__ double red[PAIR_THREADS / PAIR_G][NPART_PAIR];
    const Tile T = tiles[blockIdx.x];
    const SysDev &S = sysv[T.sys];
    const int li = threadIdx.x / PAIR_G, g = threadIdx.x % PAIR_G;
    const int i = T.i0 + li;
    double fx = 0.0, fy = 0.0, fz = 0.0, vir = 0.0;
    double ut[MAXT] = {0.0, 0.0, 0.0, 0.0};
    int ti = 0;
    if (i < T.i1) {
        const double4 xi = pos[i];
        ti = typ[i];
        const int n = nnb[i];
        const int *row = nbl + S.nbl_off + (long long)(i - S.off) * S.cap;
        for (int k = g; k < n; k += PAIR_G) {
            const int j = __ldg(row + k);
            const double4 xj = pos[j];
            double dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
            const double r2 = pbcr2_exact(dx, dy, dz, S);
            if (r2 > S.rcut2) continue;
            const int tj = typ[j];
            const PairTab &P = ptab[pair_of(ptmap, S, ti, tj)];
            double usum, fsum;
            if (r2 < P.r2atat) {
                usum = 1e10;   // hard-core overlap (the reference leaves fsum stale here)
                fsum = 0.0;
            } else if (r2 < P.r2umin) {
                raise_error(err, 1, T.sys, i, j);
                continue;
            } else {
                bool bad = false;
                const int kk = table_interval(P, tz, bst, r2, bad);
                if (bad) raise_error(err, 2, T.sys, i, j);
                const double *c = tc + (size_t)(P.k0 + kk) * 12;
                const double d = r2 - c[0];
                usum = c[1] + d * (c[2] + d * (c[3] + d * (c[4] + d * (c[5] + d * c[6]))));
                fsum = c[7] + d * (c[8] + d * (c[9] + d * (c[10] + d * c[11])));
            }
            fx += fsum * dx;
            fy += fsum * dy;
            fz += fsum * dz;
            if (i < j) {
#pragma unroll
                for (int t = 0; t < MAXT; ++t) ut[t] += (tj == t) ? usum : 0.0;
                vir -= fsum * r2;
            }
        }
    }
#pragma unroll
    for (int o = PAIR_G / 2; o > 0; o >>= 1) {
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
        vir += __shfl_xor_sync(0xffffffffu, vir, o);
#pragma unroll
        for (int t = 0; t < MAXT; ++t) ut[t] += __shfl_xor_sync(0xffffffffu, ut[t], o);
    }
    if (g == 0) {
        if (i < T.i1) fsr[i] = make_double4(fx, fy, fz, 0.0);
#pragma unroll
        for (int p = 0; p < NPART_PAIR; ++p) red[li][p] = 0.0;
        if (i < T.i1) {
            for (int t = 0; t < S.npt; ++t) red[li][pair_of(ptmap, S, ti, t) - S.pt_off] += ut[t];
            red[li][MSG_MAX_NATAT] = vir;
        }
    }
    __syncthreads();
    if (threadIdx.x < NPART_PAIR) {
        double s = 0.0;
        for (int l = 0; l < PAIR_THREADS / PAIR_G; ++l) s += red[l][threadIdx.x];
        ppart[(size_t)blockIdx.x * NPART_PAIR + threadIdx.x] = s;
    }
}

// ---------------------------------------------------------------------------
// SPME charge spreading (Src/energy.F90:1226-1245): Q(k - i) += q*Mx*My*Mz.
// ---------------------------------------------------------------------------
// Also writes the per-tile dipole sums sum(q r) of the surface term
// (UEwaldSurf, Src/energy.F90:1354-1357) from the same final positions.
__device__ __forceinline__ void tile_dipole(const SysDev &S, double qx, double qy, double qz,
                                            double *__restrict__ psurf)
{
    __shared__ double red[3][4];
    qx = warp_sum(qx);
    qy = warp_sum(qy);
    qz = warp_sum(qz);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { red[0][w] = qx; red[1][w] = qy; red[2][w] = qz; }
    __syncthreads();
    if (threadIdx.x < 3) {
        double s = 0.0;
        for (int k = 0; k < 4; ++k) s += red[threadIdx.x][k];
        psurf[blockIdx.x * 4 + threadIdx.x] = s;
    }
}

template <int P>
__global__ void __launch_bounds__(128) k_spread_fp64(const SysDev *__restrict__ sysv, const Tile *__restrict__ tiles,
                                                    const double4 *__restrict__ pos, double *__restrict__ grid,
                                                    double *__restrict__ psurf)
{
    const Tile T = tiles[blockIdx.x];
    const SysDev &S = sysv[T.sys];
    if (!S.lewald) return;
    const int i = T.i0 + threadIdx.x;
    double4 x = make_double4(0.0, 0.0, 0.0, 0.0);
    if (i < T.i1) {
        x = pos[i];
        const int s = S.s;
        double th[3][P], dth[3][P];
        int km[3];
        const double xc[3] = {x.x, x.y, x.z};
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            int k = bspline<P>(S.dkdr[m] * xc[m], th[m], dth[m]);
            k %= s;
            km[m] = k < 0 ? k + s : k;
        }
        double *G = grid + S.grid_off;
#pragma unroll
        for (int iz = 0; iz < P; ++iz) {
            int nz = km[2] - iz;
            nz += (nz < 0) ? s : 0;
            const double qz = x.w * th[2][iz];
#pragma unroll
            for (int iy = 0; iy < P; ++iy) {
                int ny = km[1] - iy;
                ny += (ny < 0) ? s : 0;
                const double qyz = qz * th[1][iy];
                double *rowp = G + ((size_t)nz * s + ny) * s;
#pragma unroll
                for (int ix = 0; ix < P; ++ix) {
                    int nx = km[0] - ix;
                    nx += (nx < 0) ? s : 0;
                    atomicAdd(rowp + nx, qyz * th[0][ix]);
                }
            }
        }
    }
    if (S.lsurf) tile_dipole(S, x.w * x.x, x.w * x.y, x.w * x.z, psurf);
}

// ---------------------------------------------------------------------------
// Reciprocal-space multiply of SPMFFTRec (Src/energy.F90:6550-6578) over every
// entry of the r2c half spectrum: F *= meshfac, E += |F|^2 * emf,
// W -= |F|^2 * vmf, where emf/vmf carry the reference's halving at kx=0, s/2
// and the mirror double counts in y and z are already resolved.
// ---------------------------------------------------------------------------
constexpr int INFL_THREADS = 256, INFL_ITEMS = 4;
constexpr int INFL_TILE = INFL_THREADS * INFL_ITEMS;

__global__ void __launch_bounds__(INFL_THREADS) k_influence_fp64(
    const SysDev *__restrict__ sysv, const int4 *__restrict__ items, double2 *__restrict__ cg,
    const double *__restrict__ mfac, const double *__restrict__ emf, const double *__restrict__ vmf,
    double *__restrict__ ipart)
{
    __shared__ double red[2][INFL_THREADS / 32];
    const int4 W = items[blockIdx.x];   // sys, first complex index, end
    const SysDev &S = sysv[W.x];
    const int s = S.s, h = s / 2 + 1;
    double e = 0.0, v = 0.0;
    double2 *F = cg + S.cgrid_off;
    for (int c = W.y + threadIdx.x; c < W.z; c += INFL_THREADS) {
        const int kx = c % h, r = c / h, ky = r % s, kz = r / s;
        const int fy = ky <= s / 2 ? ky : s - ky, fz = kz <= s / 2 ? kz : s - kz;
        const size_t f = S.fac_off + kx + (size_t)h * (fy + (size_t)h * fz);
        double2 q = F[c];
        const double q2 = q.x * q.x + q.y * q.y;
        e += q2 * emf[f];
        v -= q2 * vmf[f];
        const double m = mfac[f];
        q.x *= m;
        q.y *= m;
        F[c] = q;
    }
    e = warp_sum(e);
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { red[0][w] = e; red[1][w] = v; }
    __syncthreads();
    if (threadIdx.x < 2) {
        double sacc = 0.0;
        for (int k = 0; k < INFL_THREADS / 32; ++k) sacc += red[threadIdx.x][k];
        ipart[(size_t)blockIdx.x * 2 + threadIdx.x] = sacc;
    }
}

// ---------------------------------------------------------------------------
// Finalize: SPME force gather (Src/energy.F90:1258-1285), surface term
// (Src/energy.F90:1349-1371), bonds (UBond, Src/energy.F90:5335-5387), the
// UTotal unit conversion into forceo (Src/energy.F90:405-419) and, for MD,
// the velocity half of VelVer with GetLinAcc (Src/md.F90:349-358, 601-617)
// and the kinetic-energy partial sum of GetKinEnergy.
// mode 0: forces only; 1: + velocity Verlet update.
// ---------------------------------------------------------------------------
constexpr int NPART_FIN = 4;    // ubond, virbond, ekin, spare

template <int P>
__global__ void __launch_bounds__(128) k_finalize_fp64(
    const SysDev *__restrict__ sysv, const Tile *__restrict__ tiles, const double4 *__restrict__ pos,
    const int *__restrict__ typ, const int *__restrict__ orig, const int *__restrict__ inv,
    const double *__restrict__ grid, const double4 *__restrict__ fsr, const double *__restrict__ psurf,
    const int *__restrict__ bptr, const int *__restrict__ bpart, const double *__restrict__ bk,
    const double *__restrict__ beq, const int *__restrict__ bpw, const double *__restrict__ massip,
    const double *__restrict__ massp, double4 *__restrict__ ftot, double4 *__restrict__ forceo,
    double4 *__restrict__ vel, double4 *__restrict__ acc, double *__restrict__ fpart, int mode,
    ErrWord *err)
{
    __shared__ double sq[3];
    __shared__ double red[3][4];
    const Tile T = tiles[blockIdx.x];
    const SysDev &S = sysv[T.sys];
    const int i = T.i0 + threadIdx.x;
    if (S.lsurf) {
        if (threadIdx.x < 3) {
            double a = 0.0;
            for (int k = 0; k < S.ntile128; ++k) a += psurf[(size_t)(S.tile128_off + k) * 4 + threadIdx.x];
            sq[threadIdx.x] = a;
        }
        __syncthreads();
    }
    double ub = 0.0, vb = 0.0, ek = 0.0;
    if (i < T.i1) {
        const double4 x = pos[i];
        const double4 f0 = fsr[i];
        double Fx = f0.x, Fy = f0.y, Fz = f0.z;
        if (S.lewald) {
            const int s = S.s;
            double th[3][P], dth[3][P];
            int km[3];
            const double xc[3] = {x.x, x.y, x.z};
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                int k = bspline<P>(S.dkdr[m] * xc[m], th[m], dth[m]);
                k %= s;
                km[m] = k < 0 ? k + s : k;
            }
            const double *G = grid + S.grid_off;
            double e0 = 0.0, e1 = 0.0, e2 = 0.0;
#pragma unroll
            for (int iz = 0; iz < P; ++iz) {
                int nz = km[2] - iz;
                nz += (nz < 0) ? s : 0;
#pragma unroll
                for (int iy = 0; iy < P; ++iy) {
                    int ny = km[1] - iy;
                    ny += (ny < 0) ? s : 0;
                    const double *rowp = G + ((size_t)nz * s + ny) * s;
#pragma unroll
                    for (int ix = 0; ix < P; ++ix) {
                        int nx = km[0] - ix;
                        nx += (nx < 0) ? s : 0;
                        const double Q = rowp[nx];
                        e0 += dth[0][ix] * th[1][iy] * th[2][iz] * Q;
                        e1 += th[0][ix] * dth[1][iy] * th[2][iz] * Q;
                        e2 += th[0][ix] * th[1][iy] * dth[2][iz] * Q;
                    }
                }
            }
            Fx -= x.w * e0 * S.dkdr[0] * S.epsfp;
            Fy -= x.w * e1 * S.dkdr[1] * S.epsfp;
            Fz -= x.w * e2 * S.dkdr[2] * S.epsfp;
            if (S.lsurf) {
                const double fac = 2.0 * 3.1415926535897932 / (3.0 * S.vol);
                Fx -= S.epsfp * (2.0 * fac) * x.w * sq[0];
                Fy -= S.epsfp * (2.0 * fac) * x.w * sq[1];
                Fz -= S.epsfp * (2.0 * fac) * x.w * sq[2];
            }
        }
        // bonds of this particle (both ends of a bond compute it; counted once)
        const int o = orig[i];
        const int b1 = bptr[S.off + o + 1];
        for (int b = bptr[S.off + o]; b < b1; ++b) {
            const int po = bpart[b];
            const double4 xj = pos[inv[S.off + po]];
            double dx = x.x - xj.x, dy = x.y - xj.y, dz = x.z - xj.z;
            const double r2 = pbcr2_exact(dx, dy, dz, S), r1 = sqrt(r2);
            const double term = r1 - beq[b];
            const int pw = bpw[b];
            double tp = 1.0;
            for (int k = 0; k < pw - 1; ++k) tp *= term;
            double fac = bk[b] * tp;
            const double u = fac * term;
            fac = -(pw * fac / r1);
            Fx += fac * dx;
            Fy += fac * dy;
            Fz += fac * dz;
            if (o < po) {
                ub += u;
                vb -= fac * r2;
            }
        }
        if (!isfinite(Fx) || !isfinite(Fy) || !isfinite(Fz)) raise_error(err, 7, T.sys, i, 0);
        ftot[i] = make_double4(Fx, Fy, Fz, 0.0);
        const double4 fo = make_double4(Fx * kForceFac, Fy * kForceFac, Fz * kForceFac, 0.0);
        forceo[i] = fo;
        if (mode == 1) {
            const int t = S.type_off + typ[i];
            const double mi = massip[t], hdt = 0.5 * S.dt;
            const double4 ao = acc[i];
            const double4 an = make_double4(mi * fo.x, mi * fo.y, mi * fo.z, 0.0);
            double4 v = vel[i];
            v.x = __dadd_rn(v.x, __dmul_rn(hdt, __dadd_rn(an.x, ao.x)));
            v.y = __dadd_rn(v.y, __dmul_rn(hdt, __dadd_rn(an.y, ao.y)));
            v.z = __dadd_rn(v.z, __dmul_rn(hdt, __dadd_rn(an.z, ao.z)));
            vel[i] = v;
            acc[i] = an;
            ek = 0.5 * massp[t] * (v.x * v.x + v.y * v.y + v.z * v.z);
        }
    }
    ub = warp_sum(ub);
    vb = warp_sum(vb);
    ek = warp_sum(ek);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { red[0][w] = ub; red[1][w] = vb; red[2][w] = ek; }
    __syncthreads();
    if (threadIdx.x < 3) {
        double a = 0.0;
        for (int k = 0; k < 4; ++k) a += red[threadIdx.x][k];
        fpart[(size_t)blockIdx.x * NPART_FIN + threadIdx.x] = a;
    }
}

// ---------------------------------------------------------------------------
// Per-system totals (UTotal/UEwald bookkeeping, Src/energy.F90:395-430, 948-952),
// summed in a fixed order.  Record layout (ESZ doubles):
//   0 utot, 1 utwob(0), 2..11 utwob(1..10), 12 urec, 13 ubond, 14 virial, 15 ekin
// ---------------------------------------------------------------------------
constexpr int ESZ = 16;

__device__ double block_sum_fixed(double v, double *sm)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sm[w] = v;
    __syncthreads();
    double r = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r += sm[k];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(256) k_reduce(const SysDev *__restrict__ sysv, const double *__restrict__ ppart,
                                               const double *__restrict__ ipart, const double *__restrict__ fpart,
                                               const double *__restrict__ psurf, double *__restrict__ esys,
                                               double *__restrict__ hist, int hist_cap,
                                               unsigned long long *__restrict__ stepctr,
                                               unsigned long long *__restrict__ sstep,
                                               unsigned *__restrict__ done, int nsys)
{
    __shared__ double sm[8];
    __shared__ unsigned long long step;
    const int s = blockIdx.x;
    const SysDev &S = sysv[s];
    if (threadIdx.x == 0) step = *stepctr;
    double acc[NPART_PAIR];
    for (int p = 0; p < NPART_PAIR; ++p) {
        double a = 0.0;
        for (int k = threadIdx.x; k < S.ntile32; k += blockDim.x)
            a += ppart[(size_t)(S.tile32_off + k) * NPART_PAIR + p];
        acc[p] = block_sum_fixed(a, sm);
    }
    double fin[3];
    for (int p = 0; p < 3; ++p) {
        double a = 0.0;
        for (int k = threadIdx.x; k < S.ntile128; k += blockDim.x)
            a += fpart[(size_t)(S.tile128_off + k) * NPART_FIN + p];
        fin[p] = block_sum_fixed(a, sm);
    }
    double rec[2] = {0.0, 0.0};
    if (S.lewald) {
        for (int p = 0; p < 2; ++p) {
            double a = 0.0;
            for (int k = threadIdx.x; k < S.ninfl; k += blockDim.x) a += ipart[(size_t)(S.infl_off + k) * 2 + p];
            rec[p] = block_sum_fixed(a, sm);
        }
    }
    double sq[3] = {0.0, 0.0, 0.0};
    if (S.lsurf) {
        for (int p = 0; p < 3; ++p) {
            double a = 0.0;
            for (int k = threadIdx.x; k < S.ntile128; k += blockDim.x) a += psurf[(size_t)(S.tile128_off + k) * 4 + p];
            sq[p] = block_sum_fixed(a, sm);
        }
    }
    if (threadIdx.x == 0) {
        double e[ESZ];
        for (int k = 0; k < ESZ; ++k) e[k] = 0.0;
        double u0 = 0.0;
        for (int p = 0; p < S.natat; ++p) {
            e[2 + p] = acc[p];
            u0 += acc[p];
        }
        e[1] = u0;
        double urec = 0.0, virrec = 0.0;
        if (S.lewald) {
            urec = rec[0] + S.uself;
            virrec = rec[1];
            if (S.lsurf) {
                const double fac = 2.0 * 3.1415926535897932 / (3.0 * S.vol);
                const double term = fac * (sq[0] * sq[0] + sq[1] * sq[1] + sq[2] * sq[2]);
                urec += term;
                virrec -= term;
            }
            urec *= S.epsfp;
        }
        e[12] = urec;
        e[13] = fin[0];
        e[0] = u0 + urec + fin[0];
        e[14] = acc[MSG_MAX_NATAT] + S.epsfp * virrec + fin[1];
        e[15] = fin[2] * kEkinFac;
        for (int k = 0; k < ESZ; ++k) esys[(size_t)s * ESZ + k] = e[k];
        sstep[s] += 1;
        if (hist && step < (unsigned long long)hist_cap)
            for (int k = 0; k < ESZ; ++k) hist[((size_t)step * nsys + s) * ESZ + k] = e[k];
        __threadfence();
        if (atomicAdd(done, 1u) == (unsigned)(nsys - 1)) {
            *done = 0u;
            *stepctr = step + 1;
        }
    }
}

}  // namespace msg

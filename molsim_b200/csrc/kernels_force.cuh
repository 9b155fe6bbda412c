// kernels_force.cuh -- SPME (spread, influence, gather) and the per-step finalize.
#pragma once

#include "common.cuh"
#include "kernels_pair.cuh"

namespace msg {

constexpr double kGridFix = 1099511627776.0;       // 2^40: fixed-point scale of the mixed charge grid
constexpr double kGridFixInv = 1.0 / 1099511627776.0;

// Block dipole sums sum(q r) of the surface term (UEwaldSurf,
// Src/energy.F90:1354-1357) from the final positions of the step, added to the
// system's fixed-point accumulators.
__device__ __forceinline__ void block_dipole(double qx, double qy, double qz, long long *__restrict__ ea)
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
        acc_add(ea + EA_DIP + threadIdx.x, s);
    }
}

// ---------------------------------------------------------------------------
// SPME charge spreading (Src/energy.F90:1226-1245): Q(k - i) += q*Mx*My*Mz.
// PrecD: FP64 atomics into the FP64 grid.  PrecM: FP32 splines, each
// contribution rounded to 2^-40 and added as a 64-bit integer, so the grid is
// the same whatever order the atomics land in.
// ---------------------------------------------------------------------------
template <int P, class PR>
__global__ void __launch_bounds__(128) k_spread(const SysDev *__restrict__ sysv, const Tile *__restrict__ tiles,
                                               const double4 *__restrict__ pos, double *__restrict__ grid, unsigned long long *__restrict__ igrid,
                                               long long *__restrict__ eacc)
{
    using R = typename PR::R;
    const Tile T = tiles[blockIdx.x];
    const SysDev &S = sysv[T.sys];
    if (!S.lewald) return;
    const int i = T.i0 + threadIdx.x;
    double4 x = make_double4(0.0, 0.0, 0.0, 0.0);
    if (i < T.i1) {
        x = pos[i];
        const double xc[3] = {x.x, x.y, x.z};
        const int s = S.s;
        R th[3][P], dth[3][P];
        int km[3];
#pragma unroll
        for (int m = 0; m < 3; ++m) km[m] = bspline_at<P, R>(S.dkdr[m] * xc[m], s, th[m], dth[m]);
        const R q = (R)x.w;
#pragma unroll
        for (int iz = 0; iz < P; ++iz) {
            int nz = km[2] - iz;
            nz += (nz < 0) ? s : 0;
            const R qz = q * th[2][iz];
#pragma unroll
            for (int iy = 0; iy < P; ++iy) {
                int ny = km[1] - iy;
                ny += (ny < 0) ? s : 0;
                const R qyz = qz * th[1][iy];
                const size_t rowo = S.grid_off + ((size_t)nz * s + ny) * s;
#pragma unroll
                for (int ix = 0; ix < P; ++ix) {
                    int nx = km[0] - ix;
                    nx += (nx < 0) ? s : 0;
                    if (PR::mixed)
                        atomicAdd(igrid + rowo + nx,
                                  (unsigned long long)__double2ll_rn((double)(qyz * th[0][ix]) * kGridFix));
                    else
                        atomicAdd(grid + rowo + nx, (double)(qyz * th[0][ix]));
                }
            }
        }
    }
    if (S.lsurf) block_dipole(x.w * x.x, x.w * x.y, x.w * x.z, eacc + (size_t)T.sys * EA_N);
}

// Mixed path: fixed-point grid -> FP32 grid for the FP32 FFT, clearing the
// fixed-point grid for the next step.
__global__ void k_grid_to_f32(unsigned long long *__restrict__ igrid, float *__restrict__ g, long long n)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) {
        g[k] = (float)((double)(long long)igrid[k] * kGridFixInv);
        igrid[k] = 0ull;
    }
}

// ---------------------------------------------------------------------------
// Reciprocal-space multiply of SPMFFTRec (Src/energy.F90:6550-6578) over every
// entry of the r2c half spectrum: F *= meshfac, E += |F|^2 * emf,
// W -= |F|^2 * vmf, where emf/vmf carry the reference's halving at kx=0, s/2
// and the mirror double counts in y and z are already resolved.
// ---------------------------------------------------------------------------
constexpr int INFL_THREADS = 256;
constexpr int INFL_TILE = 512;

template <class PR>
__global__ void __launch_bounds__(INFL_THREADS) k_influence(const SysDev *__restrict__ sysv, const int4 *__restrict__ items,
                                                           double2 *__restrict__ cg, float2 *__restrict__ cg32,
                                                           const double *__restrict__ mfac, const double *__restrict__ emf,
                                                           const double *__restrict__ vmf, long long *__restrict__ eacc)
{
    __shared__ double red[2][INFL_THREADS / 32];
    const int4 W = items[blockIdx.x];   // sys, first complex index, end
    const SysDev &S = sysv[W.x];
    const int s = S.s, h = s / 2 + 1;
    double e = 0.0, v = 0.0;
    for (int c = W.y + threadIdx.x; c < W.z; c += INFL_THREADS) {
        const int kx = c % h, r = c / h, ky = r % s, kz = r / s;
        const int fy = ky <= s / 2 ? ky : s - ky, fz = kz <= s / 2 ? kz : s - kz;
        const size_t f = S.fac_off + kx + (size_t)h * (fy + (size_t)h * fz);
        const double m = mfac[f];
        double q2;
        if (PR::mixed) {
            float2 q = cg32[S.cgrid_off + c];
            q2 = (double)(q.x * q.x + q.y * q.y);
            q.x *= (float)m;
            q.y *= (float)m;
            cg32[S.cgrid_off + c] = q;
        } else {
            double2 q = cg[S.cgrid_off + c];
            q2 = q.x * q.x + q.y * q.y;
            q.x *= m;
            q.y *= m;
            cg[S.cgrid_off + c] = q;
        }
        e += q2 * emf[f];
        v -= q2 * vmf[f];
    }
    e = warp_sum(e);
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { red[0][w] = e; red[1][w] = v; }
    __syncthreads();
    if (threadIdx.x < 2) {
        double sacc = 0.0;
        for (int k = 0; k < INFL_THREADS / 32; ++k) sacc += red[threadIdx.x][k];
        acc_add(eacc + (size_t)W.x * EA_N + EA_UREC + threadIdx.x, sacc);
    }
}

// ---------------------------------------------------------------------------
// Finalize: SPME force gather (Src/energy.F90:1258-1285), surface term
// (Src/energy.F90:1349-1371), bonds (UBond, Src/energy.F90:5335-5387), the
// UTotal unit conversion into forceo (Src/energy.F90:405-419) and, for MD,
// the velocity half of VelVer with GetLinAcc (Src/md.F90:349-358, 601-617)
// and GetKinEnergy's partial sum.  The last block of each system then sums
// the system's partials in a fixed order into its energy record
// (UTotal/UEwald bookkeeping, Src/energy.F90:395-430, 948-952):
//   0 utot, 1 utwob(0), 2..11 utwob(1..10), 12 urec, 13 ubond, 14 virial, 15 ekin
// mode 0: forces only; 1: + velocity Verlet update.
// ---------------------------------------------------------------------------
constexpr int NPART_FIN = 4;    // ubond, virbond, ekin, spare
constexpr int ESZ = 16;
constexpr int FIN_THREADS = 128;

struct FinOut {
    double *esys, *hist;
    int hist_cap, nsys;
    unsigned long long *stepctr, *sstep;
    unsigned *fdone, *alldone;
};

template <int P, class PR>
__global__ void __launch_bounds__(FIN_THREADS) k_finalize(
    const SysDev *__restrict__ sysv, const Tile *__restrict__ tiles, const double4 *__restrict__ pos,
    const int *__restrict__ typ, const int *__restrict__ orig,
    const int *__restrict__ inv, const double *__restrict__ grid, const float *__restrict__ grid32,
    const double4 *__restrict__ fsr, long long *__restrict__ eacc, const int *__restrict__ bptr,
    const int *__restrict__ bpart,
    const double *__restrict__ bk, const double *__restrict__ beq, const int *__restrict__ bpw,
    const double *__restrict__ massip, const double *__restrict__ massp, double4 *__restrict__ ftot,
    double4 *__restrict__ forceo, double4 *__restrict__ vel, double4 *__restrict__ acc, int mode, FinOut out,
    ErrWord *err)
{
    using R = typename PR::R;
    __shared__ double sq[3];
    __shared__ double red[3][FIN_THREADS / 32];
    __shared__ bool last;
    const Tile T = tiles[blockIdx.x];
    const SysDev &S = sysv[T.sys];
    const int i = T.i0 + threadIdx.x;
    long long *ea = eacc + (size_t)T.sys * EA_N;
    if (S.lsurf) {
        if (threadIdx.x < 3) sq[threadIdx.x] = acc_get(ea + EA_DIP + threadIdx.x);
        __syncthreads();
    }
    double ub = 0.0, vb = 0.0, ek = 0.0;
    if (i < T.i1) {
        const double4 x = pos[i];
        const double4 f0 = fsr[i];
        double Fx = f0.x, Fy = f0.y, Fz = f0.z;
        if (S.lewald) {
            const int s = S.s;
            const double xc[3] = {x.x, x.y, x.z};
            R th[3][P], dth[3][P];
            int km[3];
#pragma unroll
            for (int m = 0; m < 3; ++m) km[m] = bspline_at<P, R>(S.dkdr[m] * xc[m], s, th[m], dth[m]);
            R e0 = 0, e1 = 0, e2 = 0;
#pragma unroll
            for (int iz = 0; iz < P; ++iz) {
                int nz = km[2] - iz;
                nz += (nz < 0) ? s : 0;
#pragma unroll
                for (int iy = 0; iy < P; ++iy) {
                    int ny = km[1] - iy;
                    ny += (ny < 0) ? s : 0;
                    const size_t rowo = S.grid_off + ((size_t)nz * s + ny) * s;
#pragma unroll
                    for (int ix = 0; ix < P; ++ix) {
                        int nx = km[0] - ix;
                        nx += (nx < 0) ? s : 0;
                        const R Q = PR::mixed ? (R)grid32[rowo + nx] : (R)grid[rowo + nx];
                        e0 += dth[0][ix] * th[1][iy] * th[2][iz] * Q;
                        e1 += th[0][ix] * dth[1][iy] * th[2][iz] * Q;
                        e2 += th[0][ix] * th[1][iy] * dth[2][iz] * Q;
                    }
                }
            }
            Fx -= x.w * (double)e0 * S.dkdr[0] * S.epsfp;
            Fy -= x.w * (double)e1 * S.dkdr[1] * S.epsfp;
            Fz -= x.w * (double)e2 * S.dkdr[2] * S.epsfp;
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
        for (int k = 0; k < FIN_THREADS / 32; ++k) a += red[threadIdx.x][k];
        acc_add(ea + EA_UBOND + threadIdx.x, a);
    }
    // ---- the last block of the system forms the system's totals ----
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(&out.fdone[T.sys], 1u) == (unsigned)(S.ntile128 - 1));
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x == 0) {
        double a[EA_N];
        for (int p = 0; p < EA_N; ++p) a[p] = acc_get(ea + p);
        for (int p = 0; p < EA_N; ++p) ea[p] = 0;   // ready for the next step
        const unsigned long long step = *((volatile unsigned long long *)out.stepctr);
        double e[ESZ];
        for (int k = 0; k < ESZ; ++k) e[k] = 0.0;
        double u0 = 0.0;
        for (int p = 0; p < S.natat; ++p) {
            e[2 + p] = a[EA_UTWOB + p];
            u0 += a[EA_UTWOB + p];
        }
        e[1] = u0;
        double urec = 0.0, virrec = 0.0;
        if (S.lewald) {
            urec = a[EA_UREC] + S.uself;
            virrec = a[EA_VIRREC];
            if (S.lsurf) {
                const double fac = 2.0 * 3.1415926535897932 / (3.0 * S.vol);
                const double term =
                    fac * (a[EA_DIP] * a[EA_DIP] + a[EA_DIP + 1] * a[EA_DIP + 1] + a[EA_DIP + 2] * a[EA_DIP + 2]);
                urec += term;
                virrec -= term;
            }
            urec *= S.epsfp;
        }
        e[12] = urec;
        e[13] = a[EA_UBOND];
        e[0] = u0 + urec + a[EA_UBOND];
        e[14] = a[EA_VIRPAIR] + S.epsfp * virrec + a[EA_VIRBOND];
        e[15] = a[EA_EKIN] * kEkinFac;
        for (int k = 0; k < ESZ; ++k) out.esys[(size_t)T.sys * ESZ + k] = e[k];
        if (out.hist && step < (unsigned long long)out.hist_cap)
            for (int k = 0; k < ESZ; ++k) out.hist[((size_t)step * out.nsys + T.sys) * ESZ + k] = e[k];
        out.sstep[T.sys] += 1;
        out.fdone[T.sys] = 0u;
        __threadfence();
        if (atomicAdd(out.alldone, 1u) == (unsigned)(out.nsys - 1)) {
            *out.alldone = 0u;
            *out.stepctr = step + 1;
        }
    }
}

}  // namespace msg

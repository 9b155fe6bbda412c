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
    __shared__ double red[3][32];
    qx = warp_sum(qx);
    qy = warp_sum(qy);
    qz = warp_sum(qz);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (lane == 0) { red[0][w] = qx; red[1][w] = qy; red[2][w] = qz; }
    __syncthreads();
    if (threadIdx.x < 3) {
        double s = 0.0;
        for (int k = 0; k < nw; ++k) s += red[threadIdx.x][k];
        acc_add(ea + EA_DIP + threadIdx.x, s);
    }
}

// ---------------------------------------------------------------------------
// SPME charge spreading (Src/energy.F90:1226-1245): Q(k - i) += q*Mx*My*Mz.
// Each contribution is rounded to 2^-40 e and added as a 64-bit integer, so the
// grid is the same whatever order the atomics land in (results repeat bit for
// bit, alone or batched).  The splines are FP64 in both precisions: the charge
// grid feeds the reciprocal energy and virial, which stay FP64.  A conversion
// kernel then turns the integer grid into the FP64 input of the forward FFT and
// clears it (the convolution kernel of kernels_spme.cuh, where a handle uses it,
// reads and clears the integer grid itself).
// A block takes SPREAD_PART particles: one thread per particle forms the
// splines into shared memory, then the block walks the particles' P^3
// contributions x-fastest, so the lanes of a warp add into runs of P
// consecutive grid points (fewer L2 sectors per atomic instruction than one
// particle per lane).
// ---------------------------------------------------------------------------
constexpr int SPREAD_PART = 32;
constexpr int SPREAD_THREADS = 128;

template <int P, class PR>
__global__ void __launch_bounds__(SPREAD_THREADS) k_spread(const SysDev *__restrict__ sysv, const Tile *__restrict__ tiles,
                                                           const double4 *__restrict__ pos, double *__restrict__ grid,
                                                           unsigned long long *__restrict__ igrid, long long *__restrict__ eacc)
{
    using R = double;
    __shared__ R sth[SPREAD_PART][3][P];
    __shared__ int skm[SPREAD_PART][3];
    __shared__ R sq[SPREAD_PART];
    const Tile T = tiles[blockIdx.x / (128 / SPREAD_PART)];
    const SysDev &S = sysv[T.sys];
    if (!S.lewald || S.recstd) return;
    const int p0 = T.i0 + (int)(blockIdx.x % (128 / SPREAD_PART)) * SPREAD_PART;
    const int np = max(0, min(SPREAD_PART, T.i1 - p0));
    const int s = S.s;
    double4 x = make_double4(0.0, 0.0, 0.0, 0.0);
    if ((int)threadIdx.x < np) {
        x = pos[p0 + threadIdx.x];
        const double xc[3] = {x.x, x.y, x.z};
        R th[3][P], dth[3][P];
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            skm[threadIdx.x][m] = bspline_at<P, R>(S.dkdr[m] * xc[m], s, th[m], dth[m]);
#pragma unroll
            for (int k = 0; k < P; ++k) sth[threadIdx.x][m][k] = th[m][k];
        }
        sq[threadIdx.x] = (R)x.w;
    }
    __syncthreads();
    const int ncon = np * P * P * P;
    for (int c = threadIdx.x; c < ncon; c += SPREAD_THREADS) {
        const int ix = c % P, r1 = c / P, iy = r1 % P, r2 = r1 / P, iz = r2 % P, pp = r2 / P;
        int nx = skm[pp][0] - ix, ny = skm[pp][1] - iy, nz = skm[pp][2] - iz;
        nx += (nx < 0) ? s : 0;
        ny += (ny < 0) ? s : 0;
        nz += (nz < 0) ? s : 0;
        const R v = sq[pp] * sth[pp][2][iz] * sth[pp][1][iy] * sth[pp][0][ix];
        const size_t at = S.grid_off + ((size_t)nz * s + ny) * s + nx;
        atomicAdd(igrid + at, (unsigned long long)__double2ll_rn((double)v * kGridFix));
    }
    (void)grid;
    if (S.lsurf) block_dipole(x.w * x.x, x.w * x.y, x.w * x.z, eacc + (size_t)T.sys * EA_N);
}

// Fixed-point grid -> FP64 grid for the forward FFT, clearing the fixed-point
// grid for the next step.
__global__ void k_grid_to_f64(unsigned long long *__restrict__ igrid, double *__restrict__ g, long long n)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) {
        g[k] = (double)(long long)igrid[k] * kGridFixInv;
        igrid[k] = 0ull;
    }
}

// ---------------------------------------------------------------------------
// Reciprocal-space multiply of SPMFFTRec (Src/energy.F90:6550-6578) over every
// entry of the r2c half spectrum: F *= meshfac, E += |F|^2 * emf,
// W -= |F|^2 * vmf, where emf/vmf carry the reference's halving at kx=0, s/2
// and the mirror double counts in y and z are already resolved.  The forward
// transform is FP64 in both precisions, so E and W are FP64 sums of FP64
// terms; the mixed path writes F * meshfac in FP32 for its FP32 backward
// transform (the grid forces), the FP64 path in place.
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
        double2 q = cg[S.cgrid_off + c];
        const double q2 = q.x * q.x + q.y * q.y;
        q.x *= m;
        q.y *= m;
        if (PR::mixed)
            cg32[S.cgrid_off + c] = make_float2((float)q.x, (float)q.y);
        else
            cg[S.cgrid_off + c] = q;
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
// (Src/energy.F90:1349-1371) on top of the pair and bond forces, the
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
constexpr int FIN_LANES = 4;                      // lanes per particle in the grid gather
constexpr int FIN_PART = 64;                      // particles per block: half a 128-particle tile
constexpr int FIN_SPLIT = 128 / FIN_PART;         // blocks per tile
constexpr int FIN_THREADS = FIN_PART * FIN_LANES;

struct FinOut {
    double *esys, *hist;
    int hist_cap, nsys;
    unsigned long long *stepctr, *sstep;
    unsigned *fdone, *alldone;
};

// Bonds of every system (CSR over MOLSIM indices; bptr null: no bonds in the handle).
struct FinBonds {
    const int *orig, *inv, *bptr, *bpart, *bpw;
    const double *bk, *beq;
    const int4 *tab;   // per-particle bond table in internal order, or null (CSR walk)
};

// Bond table entry flag: this end counts the bond's energy and virial (UBond's o < po).
constexpr int BT_COUNT = 1 << 30;

// Per-particle bond table for systems whose particles have at most two bonds: entry
// k of particle i = (internal index of its k-th partner, CSR slot of the bond |
// BT_COUNT when this end counts its energy), partner -1 when absent.  Written for
// the rebuilt systems after their particles are re-ordered, so that the finalize
// reads a particle's bonds with one load and its partners' positions with one more.
__global__ void __launch_bounds__(128) k_bond_table(const SysDev *__restrict__ sysv, const Tile *__restrict__ tiles,
                                                   const int *__restrict__ flag, const int *__restrict__ orig,
                                                   const int *__restrict__ inv, const int *__restrict__ bptr,
                                                   const int *__restrict__ bpart, int4 *__restrict__ tab)
{
    const Tile T = tiles[blockIdx.x];
    if (!flag[T.sys]) return;
    const int i = T.i0 + threadIdx.x;
    if (i >= T.i1) return;
    const SysDev &S = sysv[T.sys];
    const int o = orig[i];
    const int b0 = bptr[S.off + o], b1 = bptr[S.off + o + 1];
    int4 e = make_int4(-1, 0, -1, 0);
    if (b0 < b1) {
        const int po = bpart[b0];
        e.x = inv[S.off + po];
        e.y = b0 | (o < po ? BT_COUNT : 0);
    }
    if (b0 + 1 < b1) {
        const int po = bpart[b0 + 1];
        e.z = inv[S.off + po];
        e.w = (b0 + 1) | (o < po ? BT_COUNT : 0);
    }
    tab[i] = e;
}

// One bond of particle i (position x) with its partner at xj: its force added to F;
// its energy and virial counted when this end counts them.
__device__ __forceinline__ void bond_term(const FinBonds &bd, const SysDev &S, const double4 &x, const double4 &xj,
                                          int b, bool count, double &Fx, double &Fy, double &Fz, double &ub,
                                          double &vb)
{
    double dx = x.x - xj.x, dy = x.y - xj.y, dz = x.z - xj.z;
    const double r2 = pbcr2_exact(dx, dy, dz, S), r1 = sqrt(r2);
    const double term = r1 - bd.beq[b];
    const int pw = bd.bpw[b];
    double tp = 1.0;
    for (int k = 0; k < pw - 1; ++k) tp *= term;
    double fac = bd.bk[b] * tp;
    const double u = fac * term;
    fac = -(pw * fac / r1);
    Fx += fac * dx;
    Fy += fac * dy;
    Fz += fac * dz;
    if (count) {
        ub += u;
        vb -= fac * r2;
    }
}

// UBond (Src/energy.F90:5335-5387) for particle i: the forces of its bonds (both ends of
// a bond compute it) added to F; each bond's energy and virial counted once (o < po).
// Bonds in CSR order, from the bond table when there is one.
__device__ __forceinline__ void bond_forces(const FinBonds &bd, const SysDev &S, const double4 *__restrict__ pos,
                                            int i, const double4 &x, double &Fx, double &Fy, double &Fz,
                                            double &ub, double &vb)
{
    if (bd.tab) {
        const int4 e = bd.tab[i];
        if (e.x >= 0) bond_term(bd, S, x, pos[e.x], e.y & (BT_COUNT - 1), (e.y & BT_COUNT) != 0, Fx, Fy, Fz, ub, vb);
        if (e.z >= 0) bond_term(bd, S, x, pos[e.z], e.w & (BT_COUNT - 1), (e.w & BT_COUNT) != 0, Fx, Fy, Fz, ub, vb);
        return;
    }
    const int o = bd.orig[i];
    const int b0 = bd.bptr[S.off + o], b1 = bd.bptr[S.off + o + 1];
    for (int b = b0; b < b1; ++b) {
        const int po = bd.bpart[b];
        bond_term(bd, S, x, pos[bd.inv[S.off + po]], b, o < po, Fx, Fy, Fz, ub, vb);
    }
}

template <int P, class PR>
__global__ void __launch_bounds__(FIN_THREADS) k_finalize(
    const SysDev *__restrict__ sysv, const Tile *__restrict__ tiles, const double4 *__restrict__ pos,
    const int *__restrict__ typ, const double *__restrict__ grid, const float *__restrict__ grid32,
    const double4 *__restrict__ fsr, unsigned long long *__restrict__ fpart, int fstride, FinBonds bd,
    const double4 *__restrict__ fks, long long *__restrict__ eacc,
    const double *__restrict__ massip, const double *__restrict__ massp, double4 *__restrict__ ftot,
    double4 *__restrict__ forceo, double4 *__restrict__ vel, double4 *__restrict__ acc, int mode, FinOut out,
    ErrWord *err)
{
    using R = typename PR::R;
    __shared__ double sq[3];
    __shared__ double red[3][FIN_THREADS / 32];
    __shared__ bool last;
    const Tile T = tiles[blockIdx.x / FIN_SPLIT];
    const SysDev &S = sysv[T.sys];
    // FIN_LANES lanes per particle share the gather; the group's first lane does the rest
    const int g = threadIdx.x & (FIN_LANES - 1);
    const int i = T.i0 + (int)(blockIdx.x % FIN_SPLIT) * FIN_PART + (int)threadIdx.x / FIN_LANES;
    long long *ea = eacc + (size_t)T.sys * EA_N;
    if (S.lsurf) {
        if (threadIdx.x < 3) sq[threadIdx.x] = acc_get(ea + EA_DIP + threadIdx.x);
        __syncthreads();
    }
    double ub = 0.0, vb = 0.0, ek = 0.0;
    R e0 = 0, e1 = 0, e2 = 0;
    double4 x = make_double4(0.0, 0.0, 0.0, 0.0);
    // the particle's own loads go out before the gather so that their latencies overlap
    double4 f0 = make_double4(0.0, 0.0, 0.0, 0.0), vold = f0, aold = f0;
    int tyi = 0;
    if (i < T.i1) {
        x = pos[i];
        if (g == 0) {
            f0 = fsr[i];
            if (fpart) {
                // partner shares of the half-list pair kernel (2^-32 fixed point), cleared for the next step
                unsigned long long *px = fpart + i, *py = px + fstride, *pz = py + fstride;
                f0.x += (double)(long long)*px * 2.3283064365386962890625e-10;
                f0.y += (double)(long long)*py * 2.3283064365386962890625e-10;
                f0.z += (double)(long long)*pz * 2.3283064365386962890625e-10;
                *px = 0ull;
                *py = 0ull;
                *pz = 0ull;
            }
            // the particle's bonds, before the gather, so that their registers are free again
            if (bd.bptr) bond_forces(bd, S, pos, i, x, f0.x, f0.y, f0.z, ub, vb);
        }
    }
    if (S.lewald && !S.recstd) {
        // the y and z spline values of the block's particles, read by whichever lane takes a line
        __shared__ R sTy[FIN_PART][P], sDy[FIN_PART][P], sTz[FIN_PART][P], sDz[FIN_PART][P];
        const int pl = (int)threadIdx.x / FIN_LANES;
        const int s = S.s;
        R th0[P], dth0[P];
        int km[3] = {0, 0, 0};
        if (i < T.i1) {
            const double xc[3] = {x.x, x.y, x.z};
            R th[3][P], dth[3][P];
#pragma unroll
            for (int m = 0; m < 3; ++m) km[m] = bspline_at<P, R>(S.dkdr[m] * xc[m], s, th[m], dth[m]);
#pragma unroll
            for (int k = 0; k < P; ++k) {
                th0[k] = th[0][k];
                dth0[k] = dth[0][k];
            }
            if (g == 0) {
#pragma unroll
                for (int k = 0; k < P; ++k) {
                    sTy[pl][k] = th[1][k];
                    sDy[pl][k] = dth[1][k];
                    sTz[pl][k] = th[2][k];
                    sDz[pl][k] = dth[2][k];
                }
            }
        }
        __syncwarp();
        if (i < T.i1) {
            int nxs[P];
#pragma unroll
            for (int ix = 0; ix < P; ++ix) {
                const int nx = km[0] - ix;
                nxs[ix] = nx + ((nx < 0) ? s : 0);
            }
            // the P*P (iy, iz) grid lines of the particle, dealt round the group's lanes;
            // unrolled so that the lane's grid loads go out together
#pragma unroll
            for (int t = 0; t < (P * P + FIN_LANES - 1) / FIN_LANES; ++t) {
                const int l = g + t * FIN_LANES;
                if (l >= P * P) break;
                const int iy = l % P, iz = l / P;
                int nz = km[2] - iz;
                nz += (nz < 0) ? s : 0;
                int ny = km[1] - iy;
                ny += (ny < 0) ? s : 0;
                const R ty = sTy[pl][iy], dty = sDy[pl][iy], tz = sTz[pl][iz], dtz = sDz[pl][iz];
                const size_t rowo = S.grid_off + ((size_t)nz * s + ny) * s;
                R a0 = 0, a1 = 0;
#pragma unroll
                for (int ix = 0; ix < P; ++ix) {
                    const R Q = PR::mixed ? (R)grid32[rowo + nxs[ix]] : (R)grid[rowo + nxs[ix]];
                    a0 += dth0[ix] * Q;
                    a1 += th0[ix] * Q;
                }
                e0 += a0 * ty * tz;
                e1 += a1 * dty * tz;
                e2 += a1 * ty * dtz;
            }
        }
    }
#pragma unroll
    for (int m = FIN_LANES >> 1; m > 0; m >>= 1) {
        e0 += __shfl_xor_sync(0xffffffffu, e0, m);
        e1 += __shfl_xor_sync(0xffffffffu, e1, m);
        e2 += __shfl_xor_sync(0xffffffffu, e2, m);
    }
    if (i < T.i1 && g == 0) {
        double Fx = f0.x, Fy = f0.y, Fz = f0.z;
        if (S.lewald) {
            if (S.recstd) {
                // standard Ewald: the k-vector slices of k_ew_force, in slice order
                for (int k = 0; k < S.ew_nks + S.elc; ++k) {
                    const double4 f = fks[S.ew_fks_off + (size_t)k * S.n + (i - S.off)];
                    Fx += f.x;
                    Fy += f.y;
                    Fz += f.z;
                }
            } else {
                Fx -= x.w * (double)e0 * S.dkdr[0] * S.epsfp;
                Fy -= x.w * (double)e1 * S.dkdr[1] * S.epsfp;
                Fz -= x.w * (double)e2 * S.dkdr[2] * S.epsfp;
            }
            if (S.lsurf && S.elc) {
                // 2d-periodic form (Src/energy.F90:1362-1369): the z dipole only
                const double fac = 2.0 * 3.1415926535897932 / S.vol;
                Fz -= S.epsfp * (2.0 * fac) * x.w * sq[2];
            } else if (S.lsurf) {
                const double fac = 2.0 * 3.1415926535897932 / (3.0 * S.vol);
                Fx -= S.epsfp * (2.0 * fac) * x.w * sq[0];
                Fy -= S.epsfp * (2.0 * fac) * x.w * sq[1];
                Fz -= S.epsfp * (2.0 * fac) * x.w * sq[2];
            }
        }
        if (mode == 1) {
            // read after the gather: held across it they would cost the block its occupancy
            tyi = typ[i];
            vold = vel[i];
            aold = acc[i];
        }
        if (!isfinite(Fx) || !isfinite(Fy) || !isfinite(Fz)) raise_error(err, 7, T.sys, i, 0);
        ftot[i] = make_double4(Fx, Fy, Fz, 0.0);
        const double4 fo = make_double4(Fx * kForceFac, Fy * kForceFac, Fz * kForceFac, 0.0);
        forceo[i] = fo;
        if (mode == 1) {
            const int t = S.type_off + tyi;
            const double mi = massip[t], hdt = 0.5 * S.dt;
            const double4 ao = aold;
            const double4 an = make_double4(mi * fo.x, mi * fo.y, mi * fo.z, 0.0);
            double4 v = vold;
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
    // (the block's energy atomics above are ordered before its count by the barrier
    // and one thread's fence)
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = (atomicAdd(&out.fdone[T.sys], 1u) == (unsigned)(FIN_SPLIT * S.ntile128 - 1));
    }
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
                const double fac = S.elc ? 2.0 * 3.1415926535897932 / S.vol : 2.0 * 3.1415926535897932 / (3.0 * S.vol);
                const double term = S.elc ? fac * (a[EA_DIP + 2] * a[EA_DIP + 2])
                                          : fac * (a[EA_DIP] * a[EA_DIP] + a[EA_DIP + 1] * a[EA_DIP + 1] +
                                                   a[EA_DIP + 2] * a[EA_DIP + 2]);
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

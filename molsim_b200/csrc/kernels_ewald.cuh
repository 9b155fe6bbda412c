// kernels_ewald.cuh -- the standard Ewald reciprocal sum (txewaldrec 'std',
// UEwaldRecStd with EwaldSetArray, Src/energy.F90:964-1104, 1401-1426).
//
// The reference visits the k-vectors n = (nx, ny, nz), 0 <= n_i <= ncut, in the
// order nz, ny, nx (the kfac order of EwaldSetup, Src/energy.F90:6762-6782), and
// for each forms four structure factors, one per sign pattern (-x-y, -x+y, +x-y,
// +x+y) over the half space nz >= 0.  Here:
//   k_ew_eik    per particle: exp(i 2pi n x / L) for n = 0..ncut by the reference's
//               recurrence e(n) = e(n-1) e(1), the x table scaled by the charge
//               (az * eikx), and the block sums of q r for the surface term;
//   k_ew_sk     k-vectors across threads, the particles of one chunk staged through
//               shared memory: partial structure factors per (chunk, k); the last
//               chunk of each k tile sums the chunks in a fixed order into S(k) and
//               adds the energy kfac |S|^2 and virial -(1 - k^2/2alpha^2) kfac |S|^2
//               to the system's fixed-point accumulators;
//   k_ew_force  particles across threads, k-vectors in the reference's order with
//               the exponentials advanced by the same recurrence: each particle's
//               reciprocal force over one slice of the k-vectors.  The slices are
//               summed by the finalize kernel.
// Every sum has a fixed order, so results repeat bit for bit.  The whole chain is
// FP64 in both precision modes.
#pragma once

#include "common.cuh"
#include "kernels_force.cuh"

namespace msg {

constexpr int EW_MAXCUT = 100;      // largest ncut accepted
constexpr int EWK_THREADS = 128;    // k-vectors per structure-factor block
constexpr int EW_SUB = 16;          // particles staged per shared-memory round of k_ew_sk
constexpr int EWF_THREADS = 128;    // particles per force block
constexpr int EWF_TILE = 256;       // k-vectors staged per shared-memory round of k_ew_force

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// exp(i 2pi x / L) of the three coordinates (EwaldSetArray's e(1)).
__device__ __forceinline__ void ew_base(const SysDev &S, double4 x, double2 e1[3])
{
    const double xc[3] = {x.x, x.y, x.z};
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        double sn, cs;
        sincos(2.0 * 3.1415926535897932 * S.boxi[m] * xc[m], &sn, &cs);
        e1[m] = make_double2(cs, sn);
    }
}

// Tables eik[particle][3][ncut+1] of one step (x row scaled by the charge), and the
// dipole sums of the surface term.
__global__ void __launch_bounds__(128) k_ew_eik(const SysDev *__restrict__ sysv, const Tile *__restrict__ tiles,
                                                const double4 *__restrict__ pos, double2 *__restrict__ eik,
                                                long long *__restrict__ eacc)
{
    const Tile T = tiles[blockIdx.x];
    const SysDev &S = sysv[T.sys];
    if (!S.recstd) return;
    const int i = T.i0 + threadIdx.x;
    double4 x = make_double4(0.0, 0.0, 0.0, 0.0);
    if (i < T.i1) {
        x = pos[i];
        const int w = S.ew_ncut + 1;
        double2 *row = eik + S.ew_eik_off + (size_t)(i - S.off) * 3 * w;
        double2 e1[3];
        ew_base(S, x, e1);
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            double2 e = make_double2(1.0, 0.0);
            double2 *r = row + m * w;
            const double sc = (m == 0) ? x.w : 1.0;
            r[0] = make_double2(sc * e.x, sc * e.y);
            for (int n = 1; n < w; ++n) {
                e = (n == 1) ? e1[m] : cmul(e, e1[m]);
                r[n] = make_double2(sc * e.x, sc * e.y);
            }
        }
    }
    if (S.lsurf) block_dipole(x.w * x.x, x.w * x.y, x.w * x.z, eacc + (size_t)T.sys * EA_N);
}

// Partial structure factors of one (k tile, particle chunk): item = {sys, first k,
// chunk, tile}.  Dynamic shared memory: EW_SUB particles' tables, EW_SUB*3*(ncut+1)
// double2, for the largest ncut of the handle.  The last chunk of a tile to finish
// sums the tile's partials in chunk order into S(k) and adds the energy
// kfac |S|^2 and virial -(1 - k^2/2alpha^2) kfac |S|^2 to the system's fixed-point
// accumulators; it then clears the tile's counter for the next step.
__global__ void __launch_bounds__(EWK_THREADS) k_ew_sk(const SysDev *__restrict__ sysv, const int4 *__restrict__ items,
                                                       const int4 *__restrict__ kv, const double *__restrict__ kfac,
                                                       const double2 *__restrict__ eik, double2 *__restrict__ part,
                                                       double2 *__restrict__ sk, unsigned *__restrict__ tiledone,
                                                       long long *__restrict__ eacc)
{
    extern __shared__ double2 stab[];
    __shared__ double red[2][EWK_THREADS / 32];
    __shared__ bool last;
    const int4 W = items[blockIdx.x];
    const SysDev &S = sysv[W.x];
    const int kn = W.y + threadIdx.x;
    const bool on = kn < S.ew_nkv;
    const int4 n = on ? kv[S.ew_kv_off + kn] : make_int4(0, 0, 0, 0);
    const int w = S.ew_ncut + 1;
    const int p0 = W.z * S.ew_clen, p1 = min(S.n, p0 + S.ew_clen);
    double2 a[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) a[c] = make_double2(0.0, 0.0);
    for (int q0 = p0; q0 < p1; q0 += EW_SUB) {
        const int np = min(EW_SUB, p1 - q0);
        const double2 *src = eik + S.ew_eik_off + (size_t)q0 * 3 * w;
        __syncthreads();
        for (int e = threadIdx.x; e < np * 3 * w; e += EWK_THREADS) stab[e] = src[e];
        __syncthreads();
        if (on) {
            for (int p = 0; p < np; ++p) {
                const double2 *t = stab + (size_t)p * 3 * w;
                const double2 qx = t[n.x], ey = t[w + n.y], ez = t[2 * w + n.z];
                const double2 yzm = cmul(cconj(ey), ez), yzp = cmul(ey, ez);
                const double2 qxc = cconj(qx);
                const double2 r0 = cmul(qxc, yzm), r1 = cmul(qxc, yzp), r2 = cmul(qx, yzm), r3 = cmul(qx, yzp);
                a[0].x += r0.x; a[0].y += r0.y;
                a[1].x += r1.x; a[1].y += r1.y;
                a[2].x += r2.x; a[2].y += r2.y;
                a[3].x += r3.x; a[3].y += r3.y;
            }
        }
    }
    if (on) {
        double2 *o = part + (S.ew_part_off + (size_t)W.z * S.ew_nkv + kn) * 4;
#pragma unroll
        for (int c = 0; c < 4; ++c) o[c] = a[c];
    }
    // ---- the tile's last chunk: S(k), energy and virial ----
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&tiledone[W.w], 1u) == (unsigned)(S.ew_nchunk - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    double e = 0.0, v = 0.0;
    if (on) {
#pragma unroll
        for (int c = 0; c < 4; ++c) a[c] = make_double2(0.0, 0.0);
#pragma unroll 4
        for (int ch = 0; ch < S.ew_nchunk; ++ch) {
            const double2 *p = part + (S.ew_part_off + (size_t)ch * S.ew_nkv + kn) * 4;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const double2 q = __ldcg(p + c);
                a[c].x += q.x;
                a[c].y += q.y;
            }
        }
        double t = 0.0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            sk[((size_t)S.ew_kv_off + kn) * 4 + c] = a[c];
            t = t + (a[c].x * a[c].x + a[c].y * a[c].y);
        }
        t = kfac[S.ew_kv_off + kn] * t;
        const double tp = 2.0 * 3.1415926535897932;
        const double kx = n.x * (tp * S.boxi[0]), ky = n.y * (tp * S.boxi[1]), kz = n.z * (tp * S.boxi[2]);
        const double k2 = kx * kx + ky * ky + kz * kz;
        e = t;
        v = -((1.0 - k2 / (2.0 * (S.alpha * S.alpha))) * t);
    }
    e = warp_sum(e);
    v = warp_sum(v);
    const int wi = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { red[0][wi] = e; red[1][wi] = v; }
    __syncthreads();
    if (threadIdx.x < 2) {
        double s = 0.0;
        for (int k = 0; k < EWK_THREADS / 32; ++k) s += red[threadIdx.x][k];
        acc_add(eacc + (size_t)W.x * EA_N + EA_UREC + threadIdx.x, s);
    }
    if (threadIdx.x == 0) tiledone[W.w] = 0u;
}

// Reciprocal forces of up to EWF_THREADS particles over one slice of the
// k-vectors: item = {sys, first particle, end particle, slice}.  Output
// fks[slice][particle] (the system's particles in internal order).
__global__ void __launch_bounds__(EWF_THREADS) k_ew_force(const SysDev *__restrict__ sysv, const int4 *__restrict__ items,
                                                          const double4 *__restrict__ pos, const int4 *__restrict__ kv,
                                                          const double *__restrict__ kfac, const double2 *__restrict__ sk,
                                                          double4 *__restrict__ fks)
{
    __shared__ int4 skv[EWF_TILE];
    __shared__ double2 ssk[EWF_TILE][4];
    __shared__ double skf[EWF_TILE];
    const int4 W = items[blockIdx.x];
    const SysDev &S = sysv[W.x];
    const int i = W.y + threadIdx.x;
    const bool on = i < W.z;
    const int k0 = W.w * S.ew_klen, k1 = min(S.ew_nkv, k0 + S.ew_klen);
    double4 x = make_double4(0.0, 0.0, 0.0, 0.0);
    if (on) x = pos[i];
    double2 e1[3];
    ew_base(S, x, e1);
    const double q = x.w;
    const double tp = 2.0 * 3.1415926535897932;
    const double tpb[3] = {tp * S.boxi[0], tp * S.boxi[1], tp * S.boxi[2]};
    // running exponentials: e(n) = e(n-1) e(1) from e(0) = 1, as EwaldSetArray builds them
    double2 ex = make_double2(1.0, 0.0), ey = ex, ez = ex, yzm = ex, yzp = ex;
    int cx = 0, cy = 0, cz = 0, row = -1;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int t0 = k0; t0 < k1; t0 += EWF_TILE) {
        const int nt = min(EWF_TILE, k1 - t0);
        __syncthreads();
        for (int e = threadIdx.x; e < nt; e += EWF_THREADS) {
            const size_t g = (size_t)S.ew_kv_off + t0 + e;
            skv[e] = kv[g];
            skf[e] = kfac[g];
#pragma unroll
            for (int c = 0; c < 4; ++c) ssk[e][c] = sk[g * 4 + c];
        }
        __syncthreads();
        for (int e = 0; e < nt; ++e) {
            const int4 n = skv[e];
            const int key = n.z * (EW_MAXCUT + 1) + n.y;
            if (key != row) {
                if (n.z != cz) {
                    while (cz < n.z) { ez = (cz == 0) ? e1[2] : cmul(ez, e1[2]); ++cz; }
                    ey = make_double2(1.0, 0.0);
                    cy = 0;
                }
                while (cy < n.y) { ey = (cy == 0) ? e1[1] : cmul(ey, e1[1]); ++cy; }
                yzm = cmul(cconj(ey), ez);
                yzp = cmul(ey, ez);
                ex = make_double2(1.0, 0.0);
                cx = 0;
                row = key;
            }
            while (cx < n.x) { ex = (cx == 0) ? e1[0] : cmul(ex, e1[0]); ++cx; }
            const double2 qx = make_double2(q * ex.x, q * ex.y), qxc = cconj(qx);
            const double2 r0 = cmul(qxc, yzm), r1 = cmul(qxc, yzp), r2 = cmul(qx, yzm), r3 = cmul(qx, yzp);
            const double2 s0 = ssk[e][0], s1 = ssk[e][1], s2 = ssk[e][2], s3 = ssk[e][3];
            const double fmm = -r0.x * s0.y + r0.y * s0.x;
            const double fmp = -r1.x * s1.y + r1.y * s1.x;
            const double fpm = -r2.x * s2.y + r2.y * s2.x;
            const double fpp = -r3.x * s3.y + r3.y * s3.x;
            const double kf2 = S.epsfp * 2.0 * skf[e];
            fx += (kf2 * n.x * tpb[0]) * (-fmm - fmp + fpm + fpp);
            fy += (kf2 * n.y * tpb[1]) * (-fmm + fmp - fpm + fpp);
            fz += (kf2 * n.z * tpb[2]) * (fmm + fmp + fpm + fpp);
        }
    }
    if (on) fks[S.ew_fks_off + (size_t)W.w * S.n + (i - S.off)] = make_double4(fx, fy, fz, 0.0);
}

// ---------------------------------------------------------------------------
// 2D layer correction (UEwaldRecStd2dlc with EwaldSetArray2d, Src/energy.F90:1106-1203,
// 1435-1463).  2D k-vectors kv2 = {nx, ny, system, 0} in the reference's order (ny outer)
// with kfac2d.  The trigonometric tables follow the reference: sin and cos of n = 1 from
// the coordinate, higher n by the angle-sum recurrence, and sin(0) = cos(0) = 1.
// ---------------------------------------------------------------------------
constexpr int ELC_THREADS = 128;

// sin, cos of n 2pi x / L by the recurrence from e1 = (cos, sin) of n = 1; n = 0 gives (1, 1).
__device__ __forceinline__ void elc_trig(int n, double2 e1, double &sn, double &cs)
{
    if (n == 0) {
        sn = 1.0;
        cs = 1.0;
        return;
    }
    double2 e = e1;
    for (int k = 2; k <= n; ++k) e = cmul(e, e1);
    sn = e.y;
    cs = e.x;
}

// One 2D k-vector per block: the eight sums over the system's particles (fixed partition
// over the threads, then a fixed-order reduction), stored in st2[k][8]; the energy term
// kfac2d (-S1^2 - S2^2 - S3^2 - S4^2 + S5^2 + S6^2 + S7^2 + S8^2) is added to u%rec.
__global__ void __launch_bounds__(ELC_THREADS) k_elc_sum(const SysDev *__restrict__ sysv, const int4 *__restrict__ kv2,
                                                         const double *__restrict__ kfac2,
                                                         const double4 *__restrict__ pos, double *__restrict__ st2,
                                                         long long *__restrict__ eacc)
{
    __shared__ double red[8][ELC_THREADS / 32];
    const int4 K = kv2[blockIdx.x];
    const SysDev &S = sysv[K.z];
    const double tp = 2.0 * 3.1415926535897932;
    const double tpx = tp * S.boxi[0], tpy = tp * S.boxi[1];
    const double kx = K.x * tpx, ky = K.y * tpy, kp = sqrt(kx * kx + ky * ky);
    double a[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) a[c] = 0.0;
    for (int i = S.off + threadIdx.x; i < S.off + S.n; i += ELC_THREADS) {
        const double4 x = pos[i];
        double s1, c1, sx, cx, sy, cy;
        sincos(tpx * x.x, &s1, &c1);
        elc_trig(K.x, make_double2(c1, s1), sx, cx);
        sincos(tpy * x.y, &s1, &c1);
        elc_trig(K.y, make_double2(c1, s1), sy, cy);
        const double e = exp(kp * x.z), ei = 1.0 / e;
        const double sh = 0.5 * (e - ei), ch = 0.5 * (e + ei), q = x.w;
        a[0] = a[0] + q * sx * sy * sh;
        a[1] = a[1] + q * cx * sy * sh;
        a[2] = a[2] + q * sx * cy * sh;
        a[3] = a[3] + q * cx * cy * sh;
        a[4] = a[4] + q * sx * sy * ch;
        a[5] = a[5] + q * cx * sy * ch;
        a[6] = a[6] + q * sx * cy * ch;
        a[7] = a[7] + q * cx * cy * ch;
    }
    const int wi = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const double v = warp_sum(a[c]);
        if (lane == 0) red[c][wi] = v;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        double t = 0.0;
        for (int k = 0; k < ELC_THREADS / 32; ++k) t += red[threadIdx.x][k];
        st2[(size_t)blockIdx.x * 8 + threadIdx.x] = t;
        red[threadIdx.x][0] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const double *q = &red[0][0];
        const int ld = ELC_THREADS / 32;
        const double term = kfac2[blockIdx.x] * (-q[0] * q[0] - q[ld] * q[ld] - q[2 * ld] * q[2 * ld] -
                                                 q[3 * ld] * q[3 * ld] + q[4 * ld] * q[4 * ld] +
                                                 q[5 * ld] * q[5 * ld] + q[6 * ld] * q[6 * ld] +
                                                 q[7 * ld] * q[7 * ld]);
        acc_add(eacc + (size_t)K.z * EA_N + EA_UREC, term);
    }
}

// The layer correction's force on every particle of a system with elc, over the system's 2D
// k-vectors in order, as the reference forms it per k (Src/energy.F90:1170-1197); written
// as the force slice after the standard sum's slices.
__global__ void __launch_bounds__(128) k_elc_force(const SysDev *__restrict__ sysv, const Tile *__restrict__ tiles,
                                                   const double4 *__restrict__ pos, const int4 *__restrict__ kv2,
                                                   const double *__restrict__ kfac2, const double *__restrict__ st2,
                                                   double4 *__restrict__ fks)
{
    const Tile T = tiles[blockIdx.x];
    const SysDev &S = sysv[T.sys];
    if (!S.elc || !S.recstd) return;
    const int i = T.i0 + threadIdx.x;
    if (i >= T.i1) return;
    const double4 x = pos[i];
    const double tp = 2.0 * 3.1415926535897932;
    const double tpx = tp * S.boxi[0], tpy = tp * S.boxi[1];
    double s1, c1;
    sincos(tpx * x.x, &s1, &c1);
    const double2 e1x = make_double2(c1, s1);
    sincos(tpy * x.y, &s1, &c1);
    const double2 e1y = make_double2(c1, s1);
    const double q = x.w;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    // running exponentials along the reference's (ny outer, nx inner) order
    double2 ex = make_double2(1.0, 0.0), ey = ex;
    int cxn = 0, cyn = 0;
    for (int k = S.elc_kv_off; k < S.elc_kv_off + S.elc_nkv; ++k) {
        const int4 K = kv2[k];
        if (K.y != cyn) {
            while (cyn < K.y) { ey = (cyn == 0) ? e1y : cmul(ey, e1y); ++cyn; }
            ex = make_double2(1.0, 0.0);
            cxn = 0;
        }
        while (cxn < K.x) { ex = (cxn == 0) ? e1x : cmul(ex, e1x); ++cxn; }
        const double sx = K.x ? ex.y : 1.0, cx = K.x ? ex.x : 1.0;
        const double sy = K.y ? ey.y : 1.0, cy = K.y ? ey.x : 1.0;
        const double kx = K.x * tpx, ky = K.y * tpy, kp = sqrt(kx * kx + ky * ky);
        const double e = exp(kp * x.z), ei = 1.0 / e;
        const double sh = 0.5 * (e - ei), ch = 0.5 * (e + ei);
        const double *t = st2 + (size_t)k * 8;
        const double kf2 = S.epsfp * 2.0 * kfac2[k];
        const double kxx = kf2 * kx, kyy = kf2 * ky, kpp = kf2 * kp;
        fx = fx - kxx * q * (-(cx) * (sy) * sh * t[0] - (-sx) * (sy) * sh * t[1] - (cx) * (cy) * sh * t[2] -
                             (-sx) * (cy) * sh * t[3] + (cx) * (sy) * ch * t[4] + (-sx) * (sy) * ch * t[5] +
                             (cx) * (cy) * ch * t[6] + (-sx) * (cy) * ch * t[7]);
        fy = fy - kyy * q * (-(sx) * (cy) * sh * t[0] - (cx) * (cy) * sh * t[1] - (sx) * (-sy) * sh * t[2] -
                             (cx) * (-sy) * sh * t[3] + (sx) * (cy) * ch * t[4] + (cx) * (cy) * ch * t[5] +
                             (sx) * (-sy) * ch * t[6] + (cx) * (-sy) * ch * t[7]);
        fz = fz - kpp * q * (-(sx) * (sy) * ch * t[0] - (cx) * (sy) * ch * t[1] - (sx) * (cy) * ch * t[2] -
                             (cx) * (cy) * ch * t[3] + (sx) * (sy) * sh * t[4] + (cx) * (sy) * sh * t[5] +
                             (sx) * (cy) * sh * t[6] + (cx) * (cy) * sh * t[7]);
    }
    fks[S.ew_fks_off + (size_t)S.ew_nks * S.n + (i - S.off)] = make_double4(fx, fy, fz, 0.0);
}

}  // namespace msg

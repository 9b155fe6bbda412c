// kernels_mc.cuh -- Monte Carlo single-particle translations (MCPass with
// SPartMove, Src/mc.F90:1470-1755): trial position (GetRandomTrialPos, :4527-4580;
// CheckPartBCTM with PBC, :4810-4858), energy difference (DUTotal,
// Src/denergy.F90:110-230: DUTwoBody over every partner inside rcut as the
// cell-list routines see them, :728-912; DUTwoBodyEwald 'std' and surface,
// :1240-1335, 1504-1536; DUBond, :2893-2957), Metropolis (Src/mc.F90:5135-5175)
// and MCUpdate (:5203-5236).
//
// A Metropolis chain is sequential, so one block runs one system's chain and
// spreads each trial's work over its threads: the pair differences over the
// system's particles, the structure-factor update over its k-vectors.  Thread 0
// draws the reference's random numbers (Random, Src/mollib.F90:2689-2708) in the
// reference's order and decides.  Every reduction has a fixed order: a system's
// chain is the same alone or beside others.  FP64 throughout.
#pragma once

#include "common.cuh"
#include "kernels_ewald.cuh"

namespace msg {

constexpr int MC_THREADS = 256;

// Per-system parameters of a sweep.
struct McPar {
    double beta;        // 1/kT in mol/kJ
    int isamp;          // 0: particles in order, 1: a random particle per trial
    int pad;
};

// Random (Src/mollib.F90:2689-2708): xorshift (13, 17, 5) combined with Park-Miller
// by Schrage's method, masked to a nonzero 31-bit integer, times
// am = (1 - 2^-24) 2^-31 (nearest(1.0,-1.0)/im in single precision).
__device__ __forceinline__ double mc_random(int2 &st)
{
    unsigned x = (unsigned)st.x;
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    st.x = (int)x;
    int iy = st.y;
    const int k = iy / 127773;
    iy = 16807 * (iy - k * 127773) - 2836 * k;
    if (iy < 0) iy += 2147483647;
    st.y = iy;
    const double am = (1.0 - 5.9604644775390625e-08) * 4.656612873077392578125e-10;
    return __dmul_rn(am, (double)((2147483647 & (st.x ^ st.y)) | 1));
}

// u(r2) of one type pair: the reference's table walk (the lookup of
// UTwoBodyANewCellList, Src/denergy.F90:779-785), entered at the bucket start, which
// only skips intervals the walk from the pair's first interval would pass.
// tc/bst are the handle's arrays (koff = boff = 0) or the system's slices staged in
// shared memory (koff = its first interval, boff = its first bucket).
__device__ __forceinline__ double mc_tab_u(const PairTab &T, const double *__restrict__ tc,
                                           const unsigned short *__restrict__ bst, int koff, int boff, double r2)
{
    int k = 0;
    const float r2f = (float)r2;
    if (r2f < T.fz_hi) {
        int b = (int)((r2f - T.fz_lo) * T.finv_h);
        b = b < 0 ? 0 : (b >= MSG_NBUCKET ? MSG_NBUCKET - 1 : b);
        k = bst[T.b0 - boff + b];
    }
    k += T.k0 - koff;
    // column 0 of a row is its z_low; the walk never leaves the pair's own rows (a pair
    // below the table minimum would, and the old configuration is not checked for one)
    const int kend = T.k0 - koff + T.nk - 1;
    while (k < kend && r2 < tc[(size_t)12 * k]) ++k;
    const double *c = tc + (size_t)12 * k;
    const double d = r2 - c[0];
    return c[1] + d * (c[2] + d * (c[3] + d * (c[4] + d * (c[5] + d * c[6]))));
}

// Block sum of v into slot `slot` of red (thread 0 reads the result after the
// next barrier).
__device__ __forceinline__ void mc_block_add(double v, double (*red)[MC_THREADS / 32], int slot)
{
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) red[slot][threadIdx.x >> 5] = v;
}

// Cardinal B-spline values M_P(x + i), i = 0..order-1, of the mesh coordinate u
// (CardinalBSpline, Src/mollib.F90:1629-1683) for a run-time order <= MSG_MAX_ORDER;
// returns floor(u) wrapped into [0, s).
__device__ __forceinline__ int mc_bspline(int order, double u, int s, double *v)
{
    const double fl = floor(u), x = u - fl;
    double last[MSG_MAX_ORDER];
    v[0] = x;
    v[1] = 1.0 - x;
    for (int n = 3; n <= order; ++n) {
        for (int i = 0; i < n - 1; ++i) last[i] = v[i];
        const double nm1 = (double)(n - 1);
        v[0] = x * last[0] / nm1;
        for (int i = 1; i <= n - 2; ++i) {
            const double a = (double)i + x;
            v[i] = (a * last[i] + ((double)n - a) * last[i - 1]) / nm1;
        }
        v[n - 1] = (1.0 - x) * last[n - 2] / nm1;
    }
    int k = (int)fl % s;
    return k < 0 ? k + s : k;
}

// The charge mesh of an SPME system for a Monte Carlo pass: q Mx My Mz spread as 64-bit
// fixed point (2^-40), one thread per particle, at the system's grid offset.
__global__ void k_mc_spread(const SysDev *__restrict__ sysv, const Tile *__restrict__ tiles,
                            const double4 *__restrict__ pos, unsigned long long *__restrict__ ig)
{
    const Tile T = tiles[blockIdx.x];
    const SysDev &S = sysv[T.sys];
    if (!S.lewald || S.recstd) return;
    const int i = T.i0 + threadIdx.x;
    if (i >= T.i1) return;
    const double4 x = pos[i];
    const int s = S.s, P = S.order;
    const double xc[3] = {x.x, x.y, x.z};
    double th[3][MSG_MAX_ORDER];
    int km[3];
    for (int m = 0; m < 3; ++m) km[m] = mc_bspline(P, S.dkdr[m] * xc[m], s, th[m]);
    for (int iz = 0; iz < P; ++iz) {
        int nz = km[2] - iz;
        nz += (nz < 0) ? s : 0;
        const double qz = x.w * th[2][iz];
        for (int iy = 0; iy < P; ++iy) {
            int ny = km[1] - iy;
            ny += (ny < 0) ? s : 0;
            const double qyz = qz * th[1][iy];
            for (int ix = 0; ix < P; ++ix) {
                int nx = km[0] - ix;
                nx += (nx < 0) ? s : 0;
                atomicAdd(ig + S.grid_off + ((size_t)nz * s + ny) * s + nx,
                          (unsigned long long)__double2ll_rn(qyz * th[0][ix] * kGridFix));
            }
        }
    }
}

__global__ void k_mc_mesh_f64(long long n, unsigned long long *__restrict__ ig, double *__restrict__ g)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) {
        g[k] = (double)(long long)ig[k] * kGridFixInv;
        ig[k] = 0ull;
    }
}

// The transform of one particle's stencil along one dimension,
// B(k) = sum_i M(i) exp(-2 pi i k (km - i) / s), from the twiddles tw[m] = exp(-2 pi i m / s).
__device__ __forceinline__ double2 mc_stencil_ft(int order, double u, int s, int k, const double2 *tw)
{
    double v[MSG_MAX_ORDER];
    const int km = mc_bspline(order, u, s, v);
    double2 b = make_double2(0.0, 0.0);
    for (int i = 0; i < order; ++i) {
        int n = km - i;
        n += (n < 0) ? s : 0;
        const double2 e = tw[(int)(((long long)k * n) % s)];
        b.x += v[i] * e.x;
        b.y += v[i] * e.y;
    }
    return b;
}

// npass sweeps of one system per block.  Dynamic shared memory: six rows of
// wmax double2 (new and old exp(i k x) of the moved particle, standard Ewald), then,
// when `cache` is set, the system's positions and types, its table rows and its
// bucket starts, staged once so that the pair differences read shared memory.
__host__ __device__ inline size_t mc_cache_bytes(int n, int nk, int natat)
{
    return ((36 * (size_t)n + 15) / 16) * 16 + 96 * (size_t)nk + 2 * (size_t)natat * MSG_NBUCKET;
}

// FEAT: the features compiled in (1: SPME systems, 2: the 2D layer correction), so that a
// handle without them runs a kernel without their registers.
template <int FEAT>
__global__ void __launch_bounds__(MC_THREADS) k_mc_pass(
    const SysDev *__restrict__ sysv, double4 *__restrict__ pos, const int *__restrict__ typ,
    const int *__restrict__ inv, const int *__restrict__ ptmap, const PairTab *__restrict__ ptab,
    const double *__restrict__ tc, const unsigned short *__restrict__ bst, const int4 *__restrict__ kv,
    const double *__restrict__ kfac, double2 *__restrict__ sk, double2 *__restrict__ sktm,
    const int *__restrict__ bptr, const int *__restrict__ bpart, const double *__restrict__ bk,
    const double *__restrict__ beq, const int *__restrict__ bpw, const McPar *__restrict__ par,
    const double *__restrict__ dtr, int2 *__restrict__ rng, double *__restrict__ mcu,
    long long *__restrict__ cnt, int npass, int cache, int wmax, const int4 *__restrict__ kv2,
    const double *__restrict__ kfac2, double *__restrict__ st2, double *__restrict__ st2tm,
    double2 *__restrict__ mcF, const double *__restrict__ emf, int etabn)
{
    // etabn double2: standard Ewald [6][ncut+1] (new x, y, z; old x, y, z); SPME the twiddles
    // [s] and the stencil transforms [2][3][s] (trial, current)
    extern __shared__ double2 etab[];
    constexpr int NSLOT = 10 + 4;              // type pairs, reciprocal, dipole x, y, z
    __shared__ double red[NSLOT][MC_THREADS / 32];
    __shared__ double srt[3], sro[3], sq;
    __shared__ int si, sip, sty, sover, sacc;
    const int sys = blockIdx.x;
    const SysDev &S = sysv[sys];
    const int t = threadIdx.x;
    const bool spm = (FEAT & 1) && S.lewald && !S.recstd;
    const int natat = S.natat, w = S.ew_ncut + 1;
    const McPar P = par[sys];
    int2 st = rng[sys];                        // used by thread 0 only
    double *u = mcu + (size_t)sys * ESZ;
    long long nacc = 0, nhs = 0;
    const double tp = 2.0 * 3.1415926535897932;
    const long long ntrial = (long long)npass * S.n;
    // where the system's particles and table rows are read from
    const double4 *P4 = pos;
    const int *PT = typ;
    const double *TC = tc;
    const unsigned short *BS = bst;
    int poff = 0, koff = 0, boff = 0;
    double4 *cpos = nullptr;
    if (cache) {
        unsigned char *base = reinterpret_cast<unsigned char *>(etab + etabn);
        cpos = reinterpret_cast<double4 *>(base);
        int *ctyp = reinterpret_cast<int *>(cpos + S.n);
        double *ctc = reinterpret_cast<double *>(base + ((36 * (size_t)S.n + 15) / 16) * 16);
        unsigned short *cbst = reinterpret_cast<unsigned short *>(ctc + (size_t)12 * S.tab_nk);
        for (int e = t; e < S.n; e += MC_THREADS) {
            cpos[e] = pos[S.off + e];
            ctyp[e] = typ[S.off + e];
        }
        for (int e = t; e < 12 * S.tab_nk; e += MC_THREADS) ctc[e] = tc[(size_t)12 * S.tab_k0 + e];
        for (int e = t; e < S.natat * MSG_NBUCKET; e += MC_THREADS) cbst[e] = bst[S.tab_b0 + e];
        P4 = cpos;
        PT = ctyp;
        TC = ctc;
        BS = cbst;
        poff = S.off;
        koff = S.tab_k0;
        boff = S.tab_b0;
        __syncthreads();
    }
    if (spm) {
        for (int m = t; m < S.s; m += MC_THREADS) {
            double sn, cs;
            sincospi(2.0 * (double)m / (double)S.s, &sn, &cs);
            etab[m] = make_double2(cs, -sn);
        }
        __syncthreads();
    }
    // Thread 0 sets up a trial: particle, displacement, periodic wrap.
    auto setup = [&](int ipass) {
        int ip = (P.isamp == 0) ? ipass + 1 : 1 + (int)(S.n * mc_random(st));
        ip = max(1, min(ip, S.n)) - 1;
        const int i = inv[S.off + ip];
        const int ty = PT[i - poff];
        const double dt = dtr[S.type_off + ty];
        double d[3];
        if (dt >= 0.0) {
            for (int m = 0; m < 3; ++m) d[m] = __dmul_rn(mc_random(st) - 0.5, dt);
        } else {
            for (;;) {
                for (int m = 0; m < 3; ++m) d[m] = mc_random(st) - 0.5;
                if (__dadd_rn(__dadd_rn(__dmul_rn(d[0], d[0]), __dmul_rn(d[1], d[1])), __dmul_rn(d[2], d[2])) < 0.25)
                    break;
            }
            for (int m = 0; m < 3; ++m) d[m] = __dmul_rn(d[m], fabs(dt));
        }
        const double4 x = P4[i - poff];
        const double xo[3] = {x.x, x.y, x.z};
        for (int m = 0; m < 3; ++m) {
            sro[m] = xo[m];
            srt[m] = pbc_wrap(__dadd_rn(xo[m], d[m]), S.half[m], S.box[m], S.boxi[m]);
        }
        sq = x.w;
        si = i;
        sip = ip;
        sty = ty;
        sover = 0;
    };
    // the structure factors in use and the trial's, swapped when a move is accepted (and the
    // layer correction's eight sums per 2D k-vector, the same way)
    double2 *scur = sk, *stry = sktm;
    double *ecur = st2, *etry = st2tm;
    if (t == 0 && ntrial > 0) setup(0);
    __syncthreads();
    for (long long m = 0; m < ntrial; ++m) {
        const int i = si, ty = sty;
        const double q = sq;
        const double rt[3] = {srt[0], srt[1], srt[2]}, r0[3] = {sro[0], sro[1], sro[2]};
        // ---- exp(i 2pi n x / L) of the trial and the current position (standard Ewald) ----
        if (S.recstd && t < 6) {
            const int c3 = t % 3;
            const double xm = (t < 3) ? rt[c3] : r0[c3];
            double sn, cs;
            sincos(tp * S.boxi[c3] * xm, &sn, &cs);
            const double2 e1 = make_double2(cs, sn);
            double2 *row = etab + t * w;
            double2 e = make_double2(1.0, 0.0);
            row[0] = e;
            for (int n = 1; n < w; ++n) {
                e = (n == 1) ? e1 : cmul(e, e1);
                row[n] = e;
            }
        }
        // ---- SPME: transforms of the trial's and the current stencil along each dimension ----
        if (spm) {
            const int sm = S.s;
            for (int e = t; e < 6 * sm; e += MC_THREADS) {
                const int set = e / (3 * sm), d = (e / sm) % 3, k = e % sm;
                const double xm = set == 0 ? rt[d] : r0[d];
                etab[sm + e] = mc_stencil_ft(S.order, S.dkdr[d] * xm, sm, k, etab);
            }
        }
        // ---- pair differences (and the dipole sum of the surface term) ----
        double du[10];
#pragma unroll
        for (int p = 0; p < 10; ++p) du[p] = 0.0;
        double dip0 = 0.0, dip1 = 0.0, dip2 = 0.0;
        bool over = false;
        for (int j = S.off + t; j < S.off + S.n; j += MC_THREADS) {
            const double4 xj = P4[j - poff];
            if (S.lsurf) {
                dip0 += xj.w * xj.x;
                dip1 += xj.w * xj.y;
                dip2 += xj.w * xj.z;
            }
            if (j == i) continue;
            const int pg = pair_of(ptmap, S, ty, PT[j - poff]);
            const PairTab &T = ptab[pg];
            const int pl = pg - S.pt_off;
            double dx = rt[0] - xj.x, dy = rt[1] - xj.y, dz = rt[2] - xj.z;
            const double r2n = pbcr2_exact(dx, dy, dz, S);
            double v = 0.0;
            if (r2n < S.rcut2) {
                if (r2n < T.r2atat || r2n < T.r2umin)
                    over = true;
                else
                    v += mc_tab_u(T, TC, BS, koff, boff, r2n);
            }
            dx = r0[0] - xj.x;
            dy = r0[1] - xj.y;
            dz = r0[2] - xj.z;
            const double r2o = pbcr2_exact(dx, dy, dz, S);
            if (r2o < S.rcut2) v -= mc_tab_u(T, TC, BS, koff, boff, r2o);
#pragma unroll
            for (int p = 0; p < 10; ++p)
                if (p == pl) du[p] += v;
        }
        if (over) sover = 1;
        __syncthreads();                       // tables ready, overlap flag final
        // ---- structure factors of the trial (standard Ewald) ----
        double dr = 0.0;
        if (S.recstd) {
            const double2 *tx = etab, *ty_ = etab + w, *tzn = etab + 2 * w;
            const double2 *ox = etab + 3 * w, *oy = etab + 4 * w, *oz = etab + 5 * w;
            for (int kn = t; kn < S.ew_nkv; kn += MC_THREADS) {
                const size_t g = (size_t)S.ew_kv_off + kn;
                const int4 n = kv[g];
                const double2 yzm = cmul(cconj(oy[n.y]), oz[n.z]), yzp = cmul(oy[n.y], oz[n.z]);
                const double2 yzmt = cmul(cconj(ty_[n.y]), tzn[n.z]), yzpt = cmul(ty_[n.y], tzn[n.z]);
                const double2 xo = ox[n.x], xt = tx[n.x];
                const double2 nw[4] = {cmul(cconj(xt), yzmt), cmul(cconj(xt), yzpt), cmul(xt, yzmt), cmul(xt, yzpt)};
                const double2 od[4] = {cmul(cconj(xo), yzm), cmul(cconj(xo), yzp), cmul(xo, yzm), cmul(xo, yzp)};
                double tnew = 0.0, told = 0.0;
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const double2 s0 = scur[g * 4 + c];
                    const double2 s1 = make_double2(s0.x + q * (nw[c].x - od[c].x), s0.y + q * (nw[c].y - od[c].y));
                    stry[g * 4 + c] = s1;
                    tnew = tnew + (s1.x * s1.x + s1.y * s1.y);
                    told = told + (s0.x * s0.x + s0.y * s0.y);
                }
                dr = dr + kfac[g] * (tnew - told);
            }
        }
        // ---- SPME: u%rec(trial mesh) - u%rec(mesh) (DUTwoBodyEwaldRecSPM, Src/denergy.F90:1413-1495)
        //      from the spectrum F and the stencils' transform dF = q (Bx By Bz - Bx' By' Bz'):
        //      sum emf (2 Re(conj F dF) + |dF|^2) over the r2c half spectrum ----
        if (spm) {
            const int sm = S.s, h = sm / 2 + 1;
            const double2 *Bn = etab + sm, *Bo = etab + 4 * sm;
            const int nc = sm * sm * h;
            // unrolled so that a warp keeps several of its spectrum loads in flight
#pragma unroll 4
            for (int c = t; c < nc; c += MC_THREADS) {
                const int kx = c % h, rr = c / h, ky = rr % sm, kz = rr / sm;
                const double2 pn = cmul(cmul(Bn[kx], Bn[sm + ky]), Bn[2 * sm + kz]);
                const double2 po = cmul(cmul(Bo[kx], Bo[sm + ky]), Bo[2 * sm + kz]);
                const double2 dF = make_double2(q * (pn.x - po.x), q * (pn.y - po.y));
                const double2 F = mcF[S.cgrid_off + c];
                const int fy = ky <= sm / 2 ? ky : sm - ky, fz = kz <= sm / 2 ? kz : sm - kz;
                const double wgt = emf[S.fac_off + kx + (size_t)h * (fy + (size_t)h * fz)];
                dr = dr + wgt * (2.0 * (F.x * dF.x + F.y * dF.y) + (dF.x * dF.x + dF.y * dF.y));
            }
        }
        // ---- the layer correction's sums of the trial (DUTwoBodyEwaldRec2dlc,
        //      Src/denergy.F90:1339-1409; the old values by the same recurrence as the
        //      tables the reference keeps) ----
        if ((FEAT & 2) && S.elc && S.recstd) {
            const double tpx = tp * S.boxi[0], tpy = tp * S.boxi[1];
            double s1, c1;
            sincos(tpx * rt[0], &s1, &c1);
            const double2 etx = make_double2(c1, s1);
            sincos(tpy * rt[1], &s1, &c1);
            const double2 ety = make_double2(c1, s1);
            sincos(tpx * r0[0], &s1, &c1);
            const double2 eox = make_double2(c1, s1);
            sincos(tpy * r0[1], &s1, &c1);
            const double2 eoy = make_double2(c1, s1);
            for (int kn = t; kn < S.elc_nkv; kn += MC_THREADS) {
                const size_t g = (size_t)S.elc_kv_off + kn;
                const int4 K = kv2[g];
                double sxt, cxt, syt, cyt, sxo, cxo, syo, cyo;
                elc_trig(K.x, etx, sxt, cxt);
                elc_trig(K.y, ety, syt, cyt);
                elc_trig(K.x, eox, sxo, cxo);
                elc_trig(K.y, eoy, syo, cyo);
                const double kx = K.x * tpx, ky = K.y * tpy, kp = sqrt(kx * kx + ky * ky);
                double e = exp(kp * rt[2]), ei = 1.0 / e;
                const double sht = 0.5 * (e - ei), cht = 0.5 * (e + ei);
                e = exp(kp * r0[2]);
                ei = 1.0 / e;
                const double sho = 0.5 * (e - ei), cho = 0.5 * (e + ei);
                const double *so = ecur + g * 8;
                double *sn = etry + g * 8;
                sn[0] = so[0] + q * (sxt * syt * sht - sxo * syo * sho);
                sn[1] = so[1] + q * (cxt * syt * sht - cxo * syo * sho);
                sn[2] = so[2] + q * (sxt * cyt * sht - sxo * cyo * sho);
                sn[3] = so[3] + q * (cxt * cyt * sht - cxo * cyo * sho);
                sn[4] = so[4] + q * (sxt * syt * cht - sxo * syo * cho);
                sn[5] = so[5] + q * (cxt * syt * cht - cxo * syo * cho);
                sn[6] = so[6] + q * (sxt * cyt * cht - sxo * cyo * cho);
                sn[7] = so[7] + q * (cxt * cyt * cht - cxo * cyo * cho);
                const double tn = -sn[0] * sn[0] - sn[1] * sn[1] - sn[2] * sn[2] - sn[3] * sn[3] + sn[4] * sn[4] +
                                  sn[5] * sn[5] + sn[6] * sn[6] + sn[7] * sn[7];
                const double to = -so[0] * so[0] - so[1] * so[1] - so[2] * so[2] - so[3] * so[3] + so[4] * so[4] +
                                  so[5] * so[5] + so[6] * so[6] + so[7] * so[7];
                dr = dr + kfac2[g] * (tn - to);
            }
        }
#pragma unroll
        for (int p = 0; p < 10; ++p)
            if (p < natat) mc_block_add(du[p], red, p);
        mc_block_add(dr, red, 10);
        if (S.lsurf) {
            mc_block_add(dip0, red, 11);
            mc_block_add(dip1, red, 12);
            mc_block_add(dip2, red, 13);
        }
        __syncthreads();
        // ---- DUTotal's sum, bonds, surface, Metropolis; then the next trial (thread 0) ----
        if (t == 0) {
            int acc = 0;
            double dtw[10], dutot = 0.0, durec = 0.0, dubond = 0.0;
            if (sover) {
                ++nhs;                         // Metropolis: hard-core reject, no random number
            } else {
                double d0 = 0.0;
                for (int p = 0; p < natat; ++p) {
                    double a = 0.0;
                    for (int k = 0; k < MC_THREADS / 32; ++k) a += red[p][k];
                    dtw[p] = a;
                    d0 += a;
                }
                dutot = d0;
                if (S.lewald) {
                    for (int k = 0; k < MC_THREADS / 32; ++k) durec += red[10][k];
                    if (S.lsurf) {
                        double m0 = 0.0, m1 = 0.0, m2 = 0.0;
                        for (int k = 0; k < MC_THREADS / 32; ++k) {
                            m0 += red[11][k];
                            m1 += red[12][k];
                            m2 += red[13][k];
                        }
                        if (S.elc) {
                            // DUTwoBodyEwaldSurf, 2d-periodic form (Src/denergy.F90:1527-1536)
                            const double fac = tp / S.vol;
                            const double a2 = m2 + q * (rt[2] - r0[2]);
                            durec += fac * (a2 * a2 - m2 * m2);
                        } else {
                            const double fac = tp / (3.0 * S.vol);
                            const double a0 = m0 + q * (rt[0] - r0[0]), a1 = m1 + q * (rt[1] - r0[1]),
                                         a2 = m2 + q * (rt[2] - r0[2]);
                            durec += fac * ((a0 * a0 + a1 * a1 + a2 * a2) - (m0 * m0 + m1 * m1 + m2 * m2));
                        }
                    }
                    durec = S.epsfp * durec;
                    dutot += durec;
                }
                const int ip = sip;
                for (int b = bptr ? bptr[S.off + ip] : 0; bptr && b < bptr[S.off + ip + 1]; ++b) {
                    const double4 xb = P4[inv[S.off + bpart[b]] - poff];
                    double dx = rt[0] - xb.x, dy = rt[1] - xb.y, dz = rt[2] - xb.z;
                    const double r2n = pbcr2_exact(dx, dy, dz, S);
                    dx = r0[0] - xb.x;
                    dy = r0[1] - xb.y;
                    dz = r0[2] - xb.z;
                    const double r2o = pbcr2_exact(dx, dy, dz, S);
                    const double xn = sqrt(r2n) - beq[b], xo = sqrt(r2o) - beq[b];
                    double pn = 1.0, po = 1.0;
                    for (int e = 0; e < bpw[b]; ++e) {
                        pn *= xn;
                        po *= xo;
                    }
                    dubond += bk[b] * (pn - po);
                }
                dutot += dubond;
                const double dured = dutot * P.beta;
                if (dured > 87.0)
                    acc = 0;
                else if (dured < -87.0)
                    acc = 1;
                else {
                    const double fac = exp(-dured);
                    acc = (fac > 1.0) ? 1 : (fac > mc_random(st) ? 1 : 0);
                }
                if (acc) {
                    ++nacc;
                    u[0] += dutot;
                    u[1] += d0;
                    for (int p = 0; p < natat; ++p) u[2 + p] += dtw[p];
                    if (S.lewald) u[12] += durec;
                    u[13] += dubond;
                    double4 x = P4[i - poff];
                    x.x = rt[0];
                    x.y = rt[1];
                    x.z = rt[2];
                    pos[i] = x;
                    if (cpos) cpos[i - poff] = x;
                }
            }
            sacc = acc;
            if (m + 1 < ntrial) setup((int)((m + 1) % S.n));
        }
        __syncthreads();                       // decision and the next trial's set-up
        if (sacc) {
            double2 *tmp = scur;
            scur = stry;
            stry = tmp;
            double *etmp = ecur;
            ecur = etry;
            etry = etmp;
        }
        if (spm) {
            // MCUpdate: the spectrum follows the accepted move; the stencil transforms are
            // read before the next trial overwrites them
            if (sacc) {
                const int sm = S.s, h = sm / 2 + 1;
                const double2 *Bn = etab + sm, *Bo = etab + 4 * sm;
                const int nc = sm * sm * h;
#pragma unroll 4
                for (int c = t; c < nc; c += MC_THREADS) {
                    const int kx = c % h, rr = c / h, ky = rr % sm, kz = rr / sm;
                    const double2 pn = cmul(cmul(Bn[kx], Bn[sm + ky]), Bn[2 * sm + kz]);
                    const double2 po = cmul(cmul(Bo[kx], Bo[sm + ky]), Bo[2 * sm + kz]);
                    double2 F = mcF[S.cgrid_off + c];
                    F.x += q * (pn.x - po.x);
                    F.y += q * (pn.y - po.y);
                    mcF[S.cgrid_off + c] = F;
                }
            }
            __syncthreads();
        }
    }
    if ((FEAT & 2) && S.elc && S.recstd && ecur != st2)
        for (int e = t; e < 8 * S.elc_nkv; e += MC_THREADS) st2[(size_t)8 * S.elc_kv_off + e] = ecur[(size_t)8 * S.elc_kv_off + e];
    // the structure factors end where the last accepted move left them: back into sk
    if (S.recstd && scur != sk)
        for (int kn = t; kn < S.ew_nkv; kn += MC_THREADS) {
            const size_t g = (size_t)S.ew_kv_off + kn;
#pragma unroll
            for (int c = 0; c < 4; ++c) sk[g * 4 + c] = scur[g * 4 + c];
        }
    if (t == 0) {
        rng[sys] = st;
        cnt[2 * (size_t)sys] += nacc;
        cnt[2 * (size_t)sys + 1] += nhs;
    }
}

// ---------------------------------------------------------------------------
// MCAllPass (Src/mc.F90:4024-4178): every particle displaced at once, one UTotal of
// the trial configuration, Metropolis on du%tot.  The reference draws, per particle
// in order, three displacements and the two numbers of GetRandomTrialOri
// (Src/mc.F90:4583-4622); here each particle's thread draws its own five from the
// right place in the stream by jumping the generator ahead: the xorshift part is linear
// over GF(2) (a 32x32 bit matrix, squared once per bit of the jump), the Park-Miller
// part multiplicative mod 2^31 - 1 (a power of 16807), so the draws are the sequential
// ones exactly.
// ---------------------------------------------------------------------------
struct McJump {
    unsigned xs[32][32];            // [b][j]: column j of the xorshift map raised to 2^b
    unsigned long long pm[32];      // 16807^(2^b) mod (2^31 - 1)
};

__host__ __device__ inline unsigned mc_xs_apply(const unsigned *col, unsigned v)
{
    unsigned r = 0u;
    for (int j = 0; j < 32; ++j)
        if ((v >> j) & 1u) r ^= col[j];
    return r;
}

// The generator state after k further draws.
__host__ __device__ inline int2 mc_jump(const McJump &J, int2 st, unsigned k)
{
    unsigned x = (unsigned)st.x;
    unsigned long long y = (unsigned long long)(unsigned)st.y;
    for (int b = 0; b < 32; ++b)
        if ((k >> b) & 1u) {
            x = mc_xs_apply(J.xs[b], x);
            y = (y * J.pm[b]) % 2147483647ull;
        }
    return make_int2((int)x, (int)y);
}

// Positions of every particle in MOLSIM order into psave, and the energies into esave.
__global__ void k_mcall_save(long long ntot, const double4 *__restrict__ pos, const int *__restrict__ inv,
                             double4 *__restrict__ psave, int nsys, const double *__restrict__ esys,
                             double *__restrict__ esave)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g < ntot) psave[g] = pos[inv[g]];
    if (g < (long long)nsys * ESZ) esave[g] = esys[g];
}

// The trial configuration: particle ip of system s draws Random numbers 5 ip + 1 .. 5 ip + 5
// of its chain; the first three displace it by (r - 1/2) dtranall(ipt), then PBC
// (CheckPartBCTM, txbc 'xyz').
// The step is added to the particle's displacement since the last list build (dsum) and
// kept in step[g] (MOLSIM order) for a rejection; the fixed-point mirror follows (mixed path).
__global__ void k_mcall_trial(const SysDev *__restrict__ sysv, long long ntot, const int *__restrict__ sysid,
                              const int *__restrict__ inv, const int *__restrict__ typ, double4 *__restrict__ pos,
                              const int2 *__restrict__ rng, const McJump *__restrict__ J,
                              const double *__restrict__ dtr, double4 *__restrict__ dsum,
                              double4 *__restrict__ step, int4 *__restrict__ posfx)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ntot) return;
    const int s = sysid[g];
    const SysDev &S = sysv[s];
    const int ip = (int)(g - S.off);
    int2 st = mc_jump(*J, rng[s], 5u * (unsigned)ip);
    double d[3];
    for (int m = 0; m < 3; ++m) d[m] = mc_random(st) - 0.5;
    mc_random(st);                    // GetRandomTrialOri: the axis
    mc_random(st);                    // and the angle
    const int i = inv[g];
    const double dt = dtr[S.type_off + typ[i]];
    const double4 dd = make_double4(__dmul_rn(d[0], dt), __dmul_rn(d[1], dt), __dmul_rn(d[2], dt), 0.0);
    double4 x = pos[i];
    x.x = pbc_wrap(__dadd_rn(x.x, dd.x), S.half[0], S.box[0], S.boxi[0]);
    x.y = pbc_wrap(__dadd_rn(x.y, dd.y), S.half[1], S.box[1], S.boxi[1]);
    x.z = pbc_wrap(__dadd_rn(x.z, dd.z), S.half[2], S.box[2], S.boxi[2]);
    pos[i] = x;
    if (posfx) posfx[i] = fx_pos(x, S);
    double4 ds = dsum[i];
    ds.x += dd.x;
    ds.y += dd.y;
    ds.z += dd.z;
    dsum[i] = ds;
    step[g] = dd;
}

// NList's decision per system (Src/nlist.F90:600-615) on the displacements since the last
// build, with the true two largest (never less conservative than the reference's scan):
// flag[s] = 1 when they sum to more than drnlist.
__global__ void __launch_bounds__(256) k_mcall_skin(const SysDev *__restrict__ sysv, const double4 *__restrict__ dsum,
                                                    int *__restrict__ flag)
{
    __shared__ double r1[8], r2[8];
    const SysDev &S = sysv[blockIdx.x];
    double a1 = 0.0, a2 = 0.0;
    for (int i = S.off + threadIdx.x; i < S.off + S.n; i += 256) {
        const double4 d = dsum[i];
        const double r = sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
        if (r > a1) {
            a2 = a1;
            a1 = r;
        } else if (r > a2) {
            a2 = r;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double b1 = __shfl_xor_sync(0xffffffffu, a1, o), b2 = __shfl_xor_sync(0xffffffffu, a2, o);
        const double m1 = fmax(a1, b1), m2 = fmax(fmin(a1, b1), fmax(a2, b2));
        a1 = m1;
        a2 = m2;
    }
    if ((threadIdx.x & 31) == 0) {
        r1[threadIdx.x >> 5] = a1;
        r2[threadIdx.x >> 5] = a2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double m1 = 0.0, m2 = 0.0;
        for (int w = 0; w < 8; ++w) {
            const double n1 = fmax(m1, r1[w]), n2 = fmax(fmin(m1, r1[w]), fmax(m2, r2[w]));
            m1 = n1;
            m2 = n2;
        }
        flag[blockIdx.x] = (m1 + m2 > S.drnlist) ? 1 : 0;
    }
}

// Metropolis on du%tot = u%tot(trial) - u%tot(saved) per system, after the chain's 5 np
// draws (Src/mc.F90:5135-5175); a rejected system gets its saved energies back.
__global__ void k_mcall_decide(const SysDev *__restrict__ sysv, int nsys, int2 *__restrict__ rng,
                               const McJump *__restrict__ J, const double *__restrict__ beta,
                               double *__restrict__ esys, const double *__restrict__ esave,
                               int *__restrict__ accf, long long *__restrict__ cnt)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    int2 st = mc_jump(*J, rng[s], 5u * (unsigned)sysv[s].n);
    const double dured = (esys[(size_t)s * ESZ] - esave[(size_t)s * ESZ]) * beta[s];
    int acc;
    if (dured > 87.0)
        acc = 0;
    else if (dured < -87.0)
        acc = 1;
    else {
        const double fac = exp(-dured);
        acc = (fac > 1.0) ? 1 : (fac > mc_random(st) ? 1 : 0);
    }
    rng[s] = st;
    accf[s] = acc;
    cnt[2 * (size_t)s] += acc;
    if (!acc)
        for (int k = 0; k < ESZ; ++k) esys[(size_t)s * ESZ + k] = esave[(size_t)s * ESZ + k];
}

// A rejected system's particles back to their saved positions (MOLSIM order to internal),
// their steps taken back out of the displacements since the build, the mirror restored.
__global__ void k_mcall_restore(const SysDev *__restrict__ sysv, long long ntot, const int *__restrict__ sysid,
                                const int *__restrict__ inv, const int *__restrict__ accf,
                                const double4 *__restrict__ psave, double4 *__restrict__ pos,
                                double4 *__restrict__ dsum, const double4 *__restrict__ step,
                                int4 *__restrict__ posfx)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ntot) return;
    const int s = sysid[g];
    if (accf[s]) return;
    const int i = inv[g];
    const double4 x = psave[g];
    pos[i] = x;
    if (posfx) posfx[i] = fx_pos(x, sysv[s]);
    const double4 dd = step[g];
    double4 ds = dsum[i];
    ds.x -= dd.x;
    ds.y -= dd.y;
    ds.z -= dd.z;
    dsum[i] = ds;
}

}  // namespace msg

// polyatomic.cu -- UTwoBodyP (Src/energy.F90:786-896): the site-site pair energy,
// forces and virial of polyatomic particles, as UTotal calls it for molecules.
//
// The particle list (MOLSIM's nneighpn/jpnlist over particle centres) decides the
// pairs: a pair interacts when its centres are within rcut after the box shift of
// PBC2 (Src/molaux.F90:193-210); then every site of one particle meets every site
// of the other through the atom-type table, shifted by the centres' box shift.
//
// One warp per particle (four per block), one lane per list entry.  A lane walks the two
// particles' sites; the forces on both sites, the energy of the particle-type pair
// and the virial are added as 64-bit fixed point (2^-40 of the unit), so the sums do
// not depend on the order the threads land in.  FP64 throughout.
//
// The entry point takes the caller's host arrays in MOLSIM's layout (1-based
// indices), copies them to the device, runs, and copies the results back.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <utility>
#include <vector>

#include <cufft.h>

#include "../../include/molsim_gpu.h"
#include "common.cuh"
#include "setup.h"

namespace {

constexpr int kPThreads = 128;             // four warps: one particle's list row per warp
constexpr int kPWarps = kPThreads / 32;
constexpr int kPBuckets = 1024;            // bucket starts per atom-type pair of the site table
constexpr int kPMaxType = 4;               // particle types (their energies ride in registers)
constexpr int kPMaxPair = kPMaxType * (kPMaxType + 1) / 2;
// 64-bit fixed point at 2^-40 of the unit: |force|, |energy| and |virial| sums up to
// 8e6 (kJ/(mol A), kJ/mol) fit, far above what a tabulated pair potential produces.
constexpr double kPFix = 1099511627776.0;       // 2^40
constexpr double kPFixInv = 1.0 / 1099511627776.0;

// 1-based enumeration of unordered type pairs (MOLSIM's iptpt / iatat order:
// (1,1), (1,2), ..., (1,n), (2,2), ...), returned 0-based.
__host__ __device__ inline int type_pair(int n, int a, int b)
{
    const int lo = a < b ? a : b, hi = a < b ? b : a;   // 1-based
    return (lo - 1) * n - (lo - 1) * (lo - 2) / 2 + (hi - lo);
}

// Bucket grid of one atom-type pair's table: z_lo = r2umin, z_hi = the top interval's z_low.
struct SiteBuckets {
    double z_lo, z_hi, inv_h, pad;
};

__global__ void __launch_bounds__(kPThreads) k_utwobody_p(
    int np, int npt, int nat, double3 box, double rcut2, const double *__restrict__ ro,
    const double *__restrict__ r, const int *__restrict__ iptpn, const int *__restrict__ ianpn,
    const int *__restrict__ napt, const int *__restrict__ iatan, const int *__restrict__ nneighpn,
    const int *__restrict__ jpnlist, int maxnneigh, const double *__restrict__ ubuf, int nbuf,
    const int *__restrict__ iubuflow, const double *__restrict__ r2umin, const SiteBuckets *__restrict__ sb,
    const int *__restrict__ bstart, int maxsite, unsigned long long *__restrict__ ffix,
    unsigned long long *__restrict__ ufix, unsigned long long *__restrict__ vfix, int *__restrict__ err)
{
    // per warp: the row particle's site forces, summed in shared memory before one
    // global add per component (every lane of the warp adds to the same sites)
    extern __shared__ unsigned long long sfi[];
    const int warp = (int)(threadIdx.x >> 5), lane = threadIdx.x & 31;
    const int ip = blockIdx.x * kPWarps + warp;
    if (ip >= np) return;                      // a whole warp: only warp-level syncs below
    unsigned long long *fi_w = sfi + (size_t)warp * 3 * maxsite;
    const double half[3] = {0.5 * box.x, 0.5 * box.y, 0.5 * box.z}, len[3] = {box.x, box.y, box.z};
    const int ipt = iptpn[ip], ialow = ianpn[ip] - 1, nsi = napt[ipt - 1];
    for (int k = lane; k < 3 * nsi; k += 32) fi_w[k] = 0ull;
    __syncwarp();
    long long vir = 0;
    long long ue[kPMaxPair];                   // energy by particle-type pair, this lane's entries
#pragma unroll
    for (int q = 0; q < kPMaxPair; ++q) ue[q] = 0;
    for (int jploc = lane; jploc < nneighpn[ip]; jploc += 32) {
        const int jp = jpnlist[(size_t)ip * maxnneigh + jploc] - 1;
        const int jpt = iptpn[jp];
        const int jalow = ianpn[jp] - 1, jaupp = jalow + napt[jpt - 1] - 1;
        double d[3], sh[3];
        for (int m = 0; m < 3; ++m) {
            d[m] = ro[3 * (size_t)ip + m] - ro[3 * (size_t)jp + m];
            sh[m] = fabs(d[m]) > half[m] ? copysign(len[m], d[m]) : 0.0;
            d[m] = __dsub_rn(d[m], sh[m]);
        }
        const double rr = __dadd_rn(__dadd_rn(__dmul_rn(d[0], d[0]), __dmul_rn(d[1], d[1])), __dmul_rn(d[2], d[2]));
        if (rr > rcut2) continue;
        double usum = 0.0;
        for (int il = 0; il < nsi; ++il) {
            const int ia = ialow + il;
            const int iat = iatan[ia];
            double fi[3] = {0.0, 0.0, 0.0};
            for (int ja = jalow; ja <= jaupp; ++ja) {
                const int q = type_pair(nat, iat, iatan[ja]);
                const double dx = __dsub_rn(__dsub_rn(r[3 * (size_t)ia], r[3 * (size_t)ja]), sh[0]);
                const double dy = __dsub_rn(__dsub_rn(r[3 * (size_t)ia + 1], r[3 * (size_t)ja + 1]), sh[1]);
                const double dz = __dsub_rn(__dsub_rn(r[3 * (size_t)ia + 2], r[3 * (size_t)ja + 2]), sh[2]);
                const double a2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
                if (a2 < r2umin[q]) {
                    atomicCAS(err, 0, 1);      // StopUTwoBodyP: below the table
                    continue;
                }
                // the walk starts at the bucket's start, which never passes the interval sought
                const SiteBuckets B = sb[q];
                int ib = iubuflow[q] - 1;
                if (a2 < B.z_hi) {
                    int bk = (int)((a2 - B.z_lo) * B.inv_h);
                    bk = bk < 0 ? 0 : (bk >= kPBuckets ? kPBuckets - 1 : bk);
                    ib += 12 * bstart[q * kPBuckets + bk];
                }
                bool bad = false;
                while (a2 < ubuf[ib]) {
                    ib += 12;
                    if (ib + 12 > nbuf) {
                        bad = true;
                        break;
                    }
                }
                if (bad) {
                    atomicCAS(err, 0, 2);      // table overrun
                    continue;
                }
                const double *c = ubuf + ib;
                const double dd = a2 - c[0];
                usum += c[1] + dd * (c[2] + dd * (c[3] + dd * (c[4] + dd * (c[5] + dd * c[6]))));
                const double fs = c[7] + dd * (c[8] + dd * (c[9] + dd * (c[10] + dd * c[11])));
                fi[0] += fs * dx;
                fi[1] += fs * dy;
                fi[2] += fs * dz;
                unsigned long long *fj = ffix + 3 * (size_t)ja;
                atomicAdd(fj, (unsigned long long)__double2ll_rn(-(fs * dx) * kPFix));
                atomicAdd(fj + 1, (unsigned long long)__double2ll_rn(-(fs * dy) * kPFix));
                atomicAdd(fj + 2, (unsigned long long)__double2ll_rn(-(fs * dz) * kPFix));
                vir += __double2ll_rn(-(fs * a2) * kPFix);
            }
            atomicAdd(fi_w + 3 * il, (unsigned long long)__double2ll_rn(fi[0] * kPFix));
            atomicAdd(fi_w + 3 * il + 1, (unsigned long long)__double2ll_rn(fi[1] * kPFix));
            atomicAdd(fi_w + 3 * il + 2, (unsigned long long)__double2ll_rn(fi[2] * kPFix));
        }
        const long long uq = __double2ll_rn(usum * kPFix);
        const int pq = type_pair(npt, ipt, jpt);
#pragma unroll
        for (int q = 0; q < kPMaxPair; ++q) ue[q] += (q == pq) ? uq : 0;
    }
    // warp sums (integers: exact, order-free), then one global add each
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) vir += __shfl_xor_sync(0xffffffffu, vir, o);
#pragma unroll
    for (int q = 0; q < kPMaxPair; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ue[q] += __shfl_xor_sync(0xffffffffu, ue[q], o);
    __syncwarp();
    for (int k = lane; k < 3 * nsi; k += 32)
        if (fi_w[k]) atomicAdd(ffix + 3 * (size_t)ialow + k, fi_w[k]);
    if (lane == 0) {
        if (vir) atomicAdd(vfix, (unsigned long long)vir);
        const int nptpt = npt * (npt + 1) / 2;
#pragma unroll
        for (int q = 0; q < kPMaxPair; ++q)
            if (q < nptpt && ue[q]) atomicAdd(ufix + q, (unsigned long long)ue[q]);
    }
}

__global__ void k_utwobody_p_out(int na, int nptpt, const unsigned long long *__restrict__ ffix,
                                 const unsigned long long *__restrict__ ufix,
                                 const unsigned long long *__restrict__ vfix, double *__restrict__ force,
                                 double *__restrict__ uv)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < 3 * na) force[k] = (double)(long long)ffix[k] * kPFixInv;
    if (k == 0) {
        double u0 = 0.0;
        for (int q = 0; q < nptpt; ++q) {
            const double v = (double)(long long)ufix[q] * kPFixInv;
            uv[1 + q] = v;
            u0 += v;
        }
        uv[0] = u0;
        uv[1 + nptpt] = (double)(long long)vfix[0] * kPFixInv;
    }
}

// ---------------------------------------------------------------------------
// Rigid-body velocity Verlet (VelVer with lpolyatom, Src/md.F90:252-410).
// ---------------------------------------------------------------------------
struct RigidArgs {
    int np, nvvite;
    double tstep, tvvite, fac;          // fac = dt^2 / 2
    double box[3], half[3], boxi[3];
    int maxsite;
    double ffac;                        // (sclene / scllen) / sclfor: kJ/(mol A) -> internal force units
};

// Position and quaternion update, QuaNorm, QuaToOri, PBC of the centre, SetAtomPos
// (Src/md.F90:290-318, Src/mollib.F90:2221-2255, 2594-2612, Src/molaux.F90:526-545),
// in the reference's operation order.
__global__ void k_rigid_move(RigidArgs A, double *__restrict__ ro, const double *__restrict__ rod,
                             const double *__restrict__ rodd, double *__restrict__ qua,
                             const double *__restrict__ quad, const double *__restrict__ quadd,
                             double *__restrict__ ori, double *__restrict__ r, const int *__restrict__ iptpn,
                             const int *__restrict__ ianpn, const int *__restrict__ napt, const double *__restrict__ ra)
{
    const int ip = blockIdx.x * blockDim.x + threadIdx.x;
    if (ip >= A.np) return;
    double x[3];
    for (int m = 0; m < 3; ++m) {
        const double d = __dadd_rn(__dmul_rn(A.tstep, rod[3 * ip + m]), __dmul_rn(A.fac, rodd[3 * ip + m]));
        double v = __dadd_rn(ro[3 * ip + m], d);
        if (fabs(v) > A.half[m]) v = __dsub_rn(v, __dmul_rn(A.box[m], round(__dmul_rn(v, A.boxi[m]))));
        ro[3 * ip + m] = v;
        x[m] = v;
    }
    double q[4];
    for (int k = 0; k < 4; ++k)
        q[k] = __dadd_rn(__dadd_rn(qua[4 * ip + k], __dmul_rn(A.tstep, quad[4 * ip + k])),
                         __dmul_rn(A.fac, quadd[4 * ip + k]));
    const double nn = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(q[0], q[0]), __dmul_rn(q[1], q[1])), __dmul_rn(q[2], q[2])),
                                __dmul_rn(q[3], q[3]));
    const double norm = 1.0 / sqrt(nn);
    for (int k = 0; k < 4; ++k) {
        q[k] = __dmul_rn(q[k], norm);
        qua[4 * ip + k] = q[k];
    }
    const double q00 = __dmul_rn(q[0], q[0]), q11 = __dmul_rn(q[1], q[1]), q22 = __dmul_rn(q[2], q[2]),
                 q33 = __dmul_rn(q[3], q[3]), q01 = __dmul_rn(q[0], q[1]), q02 = __dmul_rn(q[0], q[2]),
                 q03 = __dmul_rn(q[0], q[3]), q12 = __dmul_rn(q[1], q[2]), q13 = __dmul_rn(q[1], q[3]),
                 q23 = __dmul_rn(q[2], q[3]);
    double o[9];
    o[0] = __dadd_rn(__dsub_rn(__dadd_rn(-q22, q11), q33), q00);
    o[3] = __dmul_rn(2.0, __dsub_rn(q03, q12));
    o[6] = __dmul_rn(2.0, __dadd_rn(q13, q02));
    o[1] = -__dmul_rn(2.0, __dadd_rn(q12, q03));
    o[4] = __dadd_rn(__dsub_rn(__dsub_rn(q22, q11), q33), q00);
    o[7] = __dmul_rn(2.0, __dsub_rn(q01, q23));
    o[2] = __dmul_rn(2.0, __dsub_rn(q13, q02));
    o[5] = -__dmul_rn(2.0, __dadd_rn(q23, q01));
    o[8] = __dadd_rn(__dadd_rn(__dsub_rn(-q22, q11), q33), q00);
    for (int k = 0; k < 9; ++k) ori[9 * (size_t)ip + k] = o[k];
    const int ipt = iptpn[ip] - 1, ia0 = ianpn[ip] - 1;
    for (int a = 0; a < napt[ipt]; ++a) {
        const double *s = ra + 3 * ((size_t)ipt * A.maxsite + a);
        for (int m = 0; m < 3; ++m)
            r[3 * (size_t)(ia0 + a) + m] =
                __dadd_rn(__dadd_rn(__dadd_rn(x[m], __dmul_rn(o[3 * m], s[0])), __dmul_rn(o[3 * m + 1], s[1])),
                          __dmul_rn(o[3 * m + 2], s[2]));
    }
}

// UTotal's forces, torques and molecular virial (Src/energy.F90:403-426), GetLinAcc and the
// half-kick, then the quaternion velocities: nvvite rounds of QuaVelToAngVel and GetAngAcc
// (Src/md.F90:360-402, 628-663; Src/mollib.F90:2651-2669).  One thread per particle; the
// sites' forces come from k_utwobody_p_out in kJ/(mol A).
__global__ void k_rigid_kick(RigidArgs A, const double *__restrict__ ro, double *__restrict__ rod,
                             double *__restrict__ rodd, const double *__restrict__ qua, double *__restrict__ quad,
                             double *__restrict__ quadd, const double *__restrict__ ori, const double *__restrict__ r,
                             const double *__restrict__ force, const int *__restrict__ iptpn,
                             const int *__restrict__ ianpn, const int *__restrict__ napt,
                             const double *__restrict__ masspt, const double *__restrict__ momp,
                             unsigned long long *__restrict__ vmfix)
{
    const int ip = blockIdx.x * blockDim.x + threadIdx.x;
    if (ip >= A.np) return;
    const int ipt = iptpn[ip] - 1, ia0 = ianpn[ip] - 1;
    double fo[3] = {0.0, 0.0, 0.0}, to[3] = {0.0, 0.0, 0.0}, vm = 0.0;
    for (int a = 0; a < napt[ipt]; ++a) {
        const size_t ia = (size_t)(ia0 + a);
        const double dx = __dsub_rn(r[3 * ia], ro[3 * ip]), dy = __dsub_rn(r[3 * ia + 1], ro[3 * ip + 1]),
                     dz = __dsub_rn(r[3 * ia + 2], ro[3 * ip + 2]);
        double f0 = force[3 * ia], f1 = force[3 * ia + 1], f2 = force[3 * ia + 2];
        vm = __dadd_rn(__dadd_rn(__dadd_rn(vm, __dmul_rn(dx, f0)), __dmul_rn(dy, f1)), __dmul_rn(dz, f2));
        f0 = __dmul_rn(f0, A.ffac);
        f1 = __dmul_rn(f1, A.ffac);
        f2 = __dmul_rn(f2, A.ffac);
        fo[0] = __dadd_rn(fo[0], f0);
        fo[1] = __dadd_rn(fo[1], f1);
        fo[2] = __dadd_rn(fo[2], f2);
        // torqueo + dy f3 - dz f2, left to right as the reference writes it
        to[0] = __dsub_rn(__dadd_rn(to[0], __dmul_rn(dy, f2)), __dmul_rn(dz, f1));
        to[1] = __dsub_rn(__dadd_rn(to[1], __dmul_rn(dz, f0)), __dmul_rn(dx, f2));
        to[2] = __dsub_rn(__dadd_rn(to[2], __dmul_rn(dx, f1)), __dmul_rn(dy, f0));
    }
    atomicAdd(vmfix, (unsigned long long)__double2ll_rn(vm * kPFix));
    const double mi = 1.0 / masspt[ipt];
    for (int m = 0; m < 3; ++m) {
        const double ao = rodd[3 * ip + m];
        const double an = __dmul_rn(fo[m], mi);
        rodd[3 * ip + m] = an;
        rod[3 * ip + m] = __dadd_rn(rod[3 * ip + m], __dmul_rn(__dmul_rn(0.5, A.tstep), __dadd_rn(an, ao)));
    }
    const double *o = ori + 9 * (size_t)ip, *mp = momp + 3 * ipt;
    double q[4], qd[4], qdo[4], qddo[4], qdd[4];
    for (int k = 0; k < 4; ++k) {
        q[k] = qua[4 * ip + k];
        qddo[k] = quadd[4 * ip + k];
        qdo[k] = quad[4 * ip + k];
        qd[k] = __dadd_rn(qdo[k], __dmul_rn(__dmul_rn(A.tvvite, A.tstep), qddo[k]));
        qdd[k] = qddo[k];
    }
    const double t1 = __dadd_rn(__dadd_rn(__dmul_rn(to[0], o[0]), __dmul_rn(to[1], o[3])), __dmul_rn(to[2], o[6]));
    const double t2 = __dadd_rn(__dadd_rn(__dmul_rn(to[0], o[1]), __dmul_rn(to[1], o[4])), __dmul_rn(to[2], o[7]));
    const double t3 = __dadd_rn(__dadd_rn(__dmul_rn(to[0], o[2]), __dmul_rn(to[1], o[5])), __dmul_rn(to[2], o[8]));
    const double mi1 = 1.0 / mp[0], mi2 = 1.0 / mp[1], mi3 = 1.0 / mp[2];
    for (int it = 0; it < A.nvvite; ++it) {
        // QuaVelToAngVel
        const double w1 = __dmul_rn(2.0, __dsub_rn(__dadd_rn(__dadd_rn(-__dmul_rn(q[3], qd[2]), __dmul_rn(q[0], qd[1])),
                                                             __dmul_rn(q[2], qd[3])), __dmul_rn(q[1], qd[0])));
        const double w2 = __dmul_rn(2.0, __dadd_rn(__dadd_rn(__dsub_rn(-__dmul_rn(q[0], qd[2]), __dmul_rn(q[3], qd[1])),
                                                             __dmul_rn(q[1], qd[3])), __dmul_rn(q[2], qd[0])));
        const double w3 = __dmul_rn(2.0, __dsub_rn(__dadd_rn(__dsub_rn(__dmul_rn(q[1], qd[2]), __dmul_rn(q[2], qd[1])),
                                                             __dmul_rn(q[0], qd[3])), __dmul_rn(q[3], qd[0])));
        // GetAngAcc
        const double a1 = __dmul_rn(__dadd_rn(t1, __dmul_rn(__dmul_rn(w2, w3), __dsub_rn(mp[1], mp[2]))), mi1);
        const double a2 = __dmul_rn(__dadd_rn(t2, __dmul_rn(__dmul_rn(w3, w1), __dsub_rn(mp[2], mp[0]))), mi2);
        const double a3 = __dmul_rn(__dadd_rn(t3, __dmul_rn(__dmul_rn(w1, w2), __dsub_rn(mp[0], mp[1]))), mi3);
        const double fq = __dmul_rn(-2.0, __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(qd[2], qd[2]), __dmul_rn(qd[1], qd[1])),
                                                              __dmul_rn(qd[3], qd[3])), __dmul_rn(qd[0], qd[0])));
        qdd[0] = __dmul_rn(0.5, __dadd_rn(__dsub_rn(__dadd_rn(-__dmul_rn(q[1], a1), __dmul_rn(q[2], a2)),
                                                    __dmul_rn(q[3], a3)), __dmul_rn(q[0], fq)));
        qdd[1] = __dmul_rn(0.5, __dadd_rn(__dsub_rn(__dsub_rn(__dmul_rn(q[0], a1), __dmul_rn(q[3], a2)),
                                                    __dmul_rn(q[2], a3)), __dmul_rn(q[1], fq)));
        qdd[2] = __dmul_rn(0.5, __dadd_rn(__dadd_rn(__dsub_rn(-__dmul_rn(q[3], a1), __dmul_rn(q[0], a2)),
                                                    __dmul_rn(q[1], a3)), __dmul_rn(q[2], fq)));
        qdd[3] = __dmul_rn(0.5, __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(q[2], a1), __dmul_rn(q[1], a2)),
                                                    __dmul_rn(q[0], a3)), __dmul_rn(q[3], fq)));
        for (int k = 0; k < 4; ++k)
            qd[k] = __dadd_rn(qdo[k], __dmul_rn(__dmul_rn(0.5, A.tstep), __dadd_rn(qdd[k], qddo[k])));
    }
    for (int k = 0; k < 4; ++k) {
        quad[4 * ip + k] = qd[k];
        quadd[4 * ip + k] = qdd[k];
    }
}

// The site table's bucket grid and starts, per atom-type pair q: buckets over
// [r2umin, top interval's z_low); a bucket's start is the interval where the reference's
// walk from the top stops for z = z_lo + (b + 2) h, one bucket above b's top, so it never
// passes the interval of any r2 in the bucket (the stop only moves down as z grows).
void site_buckets(int natat, const double *ubuf, int nbuf, const int32_t *iubuflow, const double *r2umin,
                  std::vector<SiteBuckets> &sb, std::vector<int> &bs)
{
    sb.assign(natat, SiteBuckets{0.0, 0.0, 1.0, 0.0});
    bs.assign((size_t)natat * kPBuckets, 0);
    for (int q = 0; q < natat; ++q) {
        const int first = iubuflow[q] - 1;
        const double z_lo = r2umin[q], z_top = ubuf[first];
        int nk = 0;
        while (first + 12 * (nk + 1) <= nbuf) {
            ++nk;
            if (ubuf[first + 12 * (nk - 1)] <= z_lo) break;
        }
        const double h = (z_top > z_lo) ? (z_top - z_lo) / kPBuckets : 1.0;
        sb[q] = SiteBuckets{z_lo, z_top, 1.0 / h, 0.0};
        int kk = 0;
        for (int b = kPBuckets - 1; b >= 0; --b) {
            const double zq = z_lo + (b + 2.0) * h;
            while (kk < nk - 1 && zq < ubuf[first + 12 * kk]) ++kk;
            bs[(size_t)q * kPBuckets + b] = kk;
        }
    }
}

int max_sites(int npt, const int32_t *napt)
{
    int m = 1;
    for (int t = 0; t < npt; ++t) m = std::max(m, (int)napt[t]);
    return m;
}

// shared memory of k_utwobody_p: each warp's row-particle site forces
size_t site_smem(int npt, const int32_t *napt)
{
    return (size_t)kPWarps * 3 * max_sites(npt, napt) * sizeof(unsigned long long);
}

// Device memory of the stateless entry points: a per-thread, per-device arena of blocks kept
// across calls (cudaMalloc and cudaFree per call would dominate a call: cudaFree waits for
// the whole device).  An entry point's ArenaScope hands everything back when it returns;
// every entry point ends with a synchronous copy, so nothing in flight still uses it.
struct Arena {
    std::vector<std::pair<char *, size_t>> blocks;
    size_t bi = 0, off = 0;
    int depth = 0;
};

Arena &arena()
{
    static thread_local std::map<int, Arena> per_device;
    int dev = 0;
    cudaGetDevice(&dev);
    return per_device[dev];
}

template <class T>
cudaError_t pmalloc(T **p, size_t bytes)
{
    Arena &A = arena();
    bytes = (std::max<size_t>(bytes, 1) + 255) & ~(size_t)255;
    while (A.bi < A.blocks.size()) {
        if (A.off + bytes <= A.blocks[A.bi].second) {
            *p = reinterpret_cast<T *>(A.blocks[A.bi].first + A.off);
            A.off += bytes;
            return cudaSuccess;
        }
        ++A.bi;
        A.off = 0;
    }
    const size_t cap = std::max(bytes, (size_t)64 << 20);
    char *q = nullptr;
    const cudaError_t e = cudaMalloc(&q, cap);
    if (e != cudaSuccess) return e;
    A.blocks.push_back({q, cap});
    A.bi = A.blocks.size() - 1;
    A.off = bytes;
    *p = reinterpret_cast<T *>(q);
    return cudaSuccess;
}

inline void pfree(void *) {}          // arena memory returns with its entry point's scope

struct ArenaScope {
    ArenaScope() { ++arena().depth; }
    ~ArenaScope()
    {
        Arena &A = arena();
        if (--A.depth == 0) {
            A.bi = 0;
            A.off = 0;
        }
    }
};

// cuFFT plans of the SPME site sum, per thread, device and mesh edge (D2Z, Z2D).
bool spm_plans(int nmesh, cufftHandle &pf, cufftHandle &pb)
{
    static thread_local std::map<std::pair<int, int>, std::pair<cufftHandle, cufftHandle>> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    auto it = cache.find({dev, nmesh});
    if (it == cache.end()) {
        cufftHandle f = 0, b = 0;
        if (cufftPlan3d(&f, nmesh, nmesh, nmesh, CUFFT_D2Z) != CUFFT_SUCCESS) return false;
        if (cufftPlan3d(&b, nmesh, nmesh, nmesh, CUFFT_Z2D) != CUFFT_SUCCESS) {
            cufftDestroy(f);
            return false;
        }
        it = cache.emplace(std::make_pair(dev, nmesh), std::make_pair(f, b)).first;
    }
    pf = it->second.first;
    pb = it->second.second;
    return true;
}

template <class T>
T *dev_copy(const T *h, size_t n, cudaError_t &e)
{
    T *d = nullptr;
    if (e == cudaSuccess) e = pmalloc(&d, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess && n) e = cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice);
    return d;
}

}  // namespace

extern "C" int msg_utwobody_p(int32_t np, int32_t na, int32_t npt, int32_t nat, const double boxlen[3], double rcut,
                              const double *ro, const double *r, const int32_t *iptpn, const int32_t *ianpn,
                              const int32_t *napt, const int32_t *iatan, const int32_t *nneighpn,
                              const int32_t *jpnlist, int32_t maxnneigh, const double *ubuf, int32_t nbuf,
                              const int32_t *iubuflow, const double *r2umin, double *force, double *utwob,
                              double *virial, float *kernel_ms)
{
    ArenaScope scope;
    if (np < 1 || na < 1 || npt < 1 || npt > kPMaxType || nat < 1 || maxnneigh < 1 || nbuf < 12 || !boxlen || !ro ||
        !r || !iptpn ||
        !ianpn || !napt || !iatan || !nneighpn || !jpnlist || !ubuf || !iubuflow || !r2umin || !force || !utwob ||
        !virial)
        return MSG_ERR_ARG;
    // host-side checks of the indices the kernel follows
    for (int t = 0; t < npt; ++t)
        if (napt[t] < 1 || napt[t] > 256) return MSG_ERR_ARG;
    for (int i = 0; i < np; ++i) {
        if (iptpn[i] < 1 || iptpn[i] > npt || ianpn[i] < 1 || ianpn[i] - 1 + napt[iptpn[i] - 1] > na)
            return MSG_ERR_ARG;
        if (nneighpn[i] < 0 || nneighpn[i] > maxnneigh) return MSG_ERR_ARG;
        for (int k = 0; k < nneighpn[i]; ++k) {
            const int j = jpnlist[(size_t)i * maxnneigh + k];
            if (j < 1 || j > np) return MSG_ERR_ARG;
        }
    }
    const int natat = nat * (nat + 1) / 2, nptpt = npt * (npt + 1) / 2;
    for (int a = 0; a < na; ++a)
        if (iatan[a] < 1 || iatan[a] > nat) return MSG_ERR_ARG;
    for (int q = 0; q < natat; ++q)
        if (iubuflow[q] < 1 || iubuflow[q] + 11 > nbuf) return MSG_ERR_ARG;
    cudaError_t e = cudaSuccess;
    double *dro = dev_copy(ro, 3 * (size_t)np, e), *dr = dev_copy(r, 3 * (size_t)na, e);
    int *dipt = dev_copy(iptpn, (size_t)np, e), *dian = dev_copy(ianpn, (size_t)np, e);
    int *dnapt = dev_copy(napt, (size_t)npt, e), *diat = dev_copy(iatan, (size_t)na, e);
    int *dnn = dev_copy(nneighpn, (size_t)np, e), *djp = dev_copy(jpnlist, (size_t)np * maxnneigh, e);
    double *dub = dev_copy(ubuf, (size_t)nbuf, e), *dr2 = dev_copy(r2umin, (size_t)natat, e);
    int *diub = dev_copy(iubuflow, (size_t)natat, e);
    std::vector<SiteBuckets> hsb;
    std::vector<int> hbs;
    site_buckets(natat, ubuf, nbuf, iubuflow, r2umin, hsb, hbs);
    SiteBuckets *dsb = dev_copy(hsb.data(), hsb.size(), e);
    int *dbs = dev_copy(hbs.data(), hbs.size(), e);
    unsigned long long *ffix = nullptr, *ufix = nullptr;
    double *dforce = nullptr, *duv = nullptr;
    int *derr = nullptr;
    const size_t nfix = 3 * (size_t)na + nptpt + 1;
    if (e == cudaSuccess) e = pmalloc(&ffix, nfix * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(ffix, 0, nfix * sizeof(unsigned long long));
    ufix = ffix ? ffix + 3 * (size_t)na : nullptr;
    if (e == cudaSuccess) e = pmalloc(&dforce, 3 * (size_t)na * sizeof(double));
    if (e == cudaSuccess) e = pmalloc(&duv, (nptpt + 2) * sizeof(double));
    if (e == cudaSuccess) e = pmalloc(&derr, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(derr, 0, sizeof(int));
    int herr = 0;
    if (e == cudaSuccess) {
        cudaEvent_t a = nullptr, b = nullptr;
        if (kernel_ms) {
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            cudaEventRecord(a, 0);
        }
        k_utwobody_p<<<(np + kPWarps - 1) / kPWarps, kPThreads, site_smem(npt, napt)>>>(
            np, npt, nat, make_double3(boxlen[0], boxlen[1], boxlen[2]), rcut * rcut, dro, dr, dipt, dian, dnapt, diat,
            dnn, djp, maxnneigh, dub, nbuf, diub, dr2, dsb, dbs, max_sites(npt, napt), ffix, ufix, ufix + nptpt, derr);
        k_utwobody_p_out<<<(int)((3 * (size_t)na + 255) / 256), 256>>>(na, nptpt, ffix, ufix, ufix + nptpt, dforce,
                                                                        duv);
        if (kernel_ms) {
            cudaEventRecord(b, 0);
            cudaEventSynchronize(b);
            cudaEventElapsedTime(kernel_ms, a, b);
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
        std::vector<double> uv(nptpt + 2);
        if (e == cudaSuccess && !herr) e = cudaMemcpy(force, dforce, 3 * (size_t)na * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && !herr) e = cudaMemcpy(uv.data(), duv, uv.size() * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && !herr) {
            for (int q = 0; q <= nptpt; ++q) utwob[q] = uv[q];
            *virial = uv[nptpt + 1];
        }
    }
    for (void *p : {(void *)dro, (void *)dr, (void *)dipt, (void *)dian, (void *)dnapt, (void *)diat, (void *)dnn,
                    (void *)djp, (void *)dub, (void *)dr2, (void *)diub, (void *)dsb, (void *)dbs, (void *)ffix,
                    (void *)dforce, (void *)duv, (void *)derr})
        if (p) pfree(p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return MSG_ERR_CUDA;
    }
    if (herr == 1) return MSG_ERR_TABLE_MIN;
    if (herr == 2) return MSG_ERR_TABLE_RANGE;
    return MSG_OK;
}

// ---------------------------------------------------------------------------
// UEwald over the sites of polyatomic particles (Src/energy.F90:905-958 with the
// standard reciprocal sum, UEwaldRecStd :964-1104, and UEwaldSelf's atomic and
// molecular terms, :1301-1345).
// ---------------------------------------------------------------------------
namespace {

constexpr int kSK = 128;                  // k-vectors per structure-factor block
constexpr int kSF = 128;                  // sites per force block
constexpr int kSFTile = 256;              // k-vectors staged per shared-memory round of k_site_force
constexpr int kSMaxCut = 100;             // largest ncut accepted
constexpr int kSSmem = 48 * 1024;         // k_site_sk's staged tables stay within the default limit
// the dipole sum of the surface term in 64-bit fixed point at 2^-32: |sum q r| up to 2e9
constexpr double kDipFix = 4294967296.0;
constexpr double kDipFixInv = 1.0 / 4294967296.0;

__device__ __forceinline__ double2 zmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 zconj(double2 a) { return make_double2(a.x, -a.y); }

// exp(i 2pi n x / L), n = 0..ncut, by EwaldSetArray's recurrence (Src/energy.F90:1401-1426);
// the x row is scaled by the site's charge (az * eikx).
__global__ void k_site_eik(int na, int w, double3 tpbi, const double *__restrict__ r, const double *__restrict__ az,
                           double2 *__restrict__ eik)
{
    const int ia = blockIdx.x * blockDim.x + threadIdx.x;
    if (ia >= na) return;
    const double t[3] = {tpbi.x, tpbi.y, tpbi.z};
    for (int m = 0; m < 3; ++m) {
        double sn, cs;
        sincos(t[m] * r[3 * (size_t)ia + m], &sn, &cs);
        const double2 e1 = make_double2(cs, sn);
        const double sc = (m == 0) ? az[ia] : 1.0;
        double2 *row = eik + ((size_t)ia * 3 + m) * w;
        double2 e = make_double2(1.0, 0.0);
        row[0] = make_double2(sc, 0.0);
        for (int n = 1; n < w; ++n) {
            e = (n == 1) ? e1 : zmul(e, e1);
            row[n] = make_double2(sc * e.x, sc * e.y);
        }
    }
}

// Partial structure factors of (k tile blockIdx.x, site chunk blockIdx.y): part[chunk][k][4].
// The chunk's sites pass through shared memory `sub` at a time (their tables, sub*3*w double2).
__global__ void __launch_bounds__(kSK) k_site_sk(int na, int nkv, int w, int clen, int sub,
                                                 const int4 *__restrict__ kv, const double2 *__restrict__ eik,
                                                 double2 *__restrict__ part)
{
    extern __shared__ double2 stab[];
    const int kn = blockIdx.x * kSK + threadIdx.x;
    const bool on = kn < nkv;
    const int4 n = on ? kv[kn] : make_int4(0, 0, 0, 0);
    const int a0 = blockIdx.y * clen, a1 = min(na, a0 + clen);
    double2 s[4];
    for (int c = 0; c < 4; ++c) s[c] = make_double2(0.0, 0.0);
    for (int q0 = a0; q0 < a1; q0 += sub) {
        const int nq = min(sub, a1 - q0);
        const double2 *src = eik + (size_t)q0 * 3 * w;
        __syncthreads();
        for (int e = threadIdx.x; e < nq * 3 * w; e += kSK) stab[e] = src[e];
        __syncthreads();
        if (on)
            for (int p = 0; p < nq; ++p) {
                const double2 *t = stab + (size_t)p * 3 * w;
                const double2 qx = t[n.x], ey = t[w + n.y], ez = t[2 * w + n.z];
                const double2 yzm = zmul(zconj(ey), ez), yzp = zmul(ey, ez), qxc = zconj(qx);
                const double2 v0 = zmul(qxc, yzm), v1 = zmul(qxc, yzp), v2 = zmul(qx, yzm), v3 = zmul(qx, yzp);
                s[0].x += v0.x; s[0].y += v0.y;
                s[1].x += v1.x; s[1].y += v1.y;
                s[2].x += v2.x; s[2].y += v2.y;
                s[3].x += v3.x; s[3].y += v3.y;
            }
    }
    if (on) {
        double2 *o = part + ((size_t)blockIdx.y * nkv + kn) * 4;
        for (int c = 0; c < 4; ++c) o[c] = s[c];
    }
}

// S(k) = the chunks in order; energy kfac |S|^2 and virial -(1 - k^2/2alpha^2) kfac |S|^2
// in 64-bit fixed point (2^-40).
__global__ void __launch_bounds__(kSK) k_site_reduce(int nkv, int nchunk, double alpha2, double3 tpbi,
                                                     const int4 *__restrict__ kv, const double *__restrict__ kfac,
                                                     const double2 *__restrict__ part, double2 *__restrict__ sk,
                                                     unsigned long long *__restrict__ efix)
{
    const int kn = blockIdx.x * kSK + threadIdx.x;
    long long e = 0, v = 0;
    if (kn < nkv) {
        double2 s[4];
        for (int c = 0; c < 4; ++c) s[c] = make_double2(0.0, 0.0);
        for (int ch = 0; ch < nchunk; ++ch)
            for (int c = 0; c < 4; ++c) {
                const double2 p = part[((size_t)ch * nkv + kn) * 4 + c];
                s[c].x += p.x;
                s[c].y += p.y;
            }
        double t = 0.0;
        for (int c = 0; c < 4; ++c) {
            sk[(size_t)kn * 4 + c] = s[c];
            t = t + (s[c].x * s[c].x + s[c].y * s[c].y);
        }
        t = kfac[kn] * t;
        const int4 n = kv[kn];
        const double kx = n.x * tpbi.x, ky = n.y * tpbi.y, kz = n.z * tpbi.z;
        const double k2 = kx * kx + ky * ky + kz * kz;
        e = __double2ll_rn(t * kPFix);
        v = __double2ll_rn(-((1.0 - k2 / (2.0 * alpha2)) * t) * kPFix);
    }
    for (int o = 16; o > 0; o >>= 1) {
        e += __shfl_xor_sync(0xffffffffu, e, o);
        v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (e) atomicAdd(efix, (unsigned long long)e);
        if (v) atomicAdd(efix + 1, (unsigned long long)v);
    }
}

// Reciprocal force of the sites of block blockIdx.x over the k-vector slice blockIdx.y
// (klen k-vectors), in the reference's order (Src/energy.F90:1078-1092):
// F += kfac2 k (combinations of Im(eikr conj S)).  The k-vectors, kfac and S(k) pass
// through shared memory a tile at a time; each site advances its exponentials by
// EwaldSetArray's recurrence e(n) = e(n-1) e(1), so they equal the tables' entries.
// Output fks[slice][site][3]; k_site_fsum adds the slices in order.
__global__ void __launch_bounds__(kSF) k_site_force(int na, int nkv, int klen, double epsfp, double3 tpbi,
                                                    const double *__restrict__ r, const double *__restrict__ az,
                                                    const int4 *__restrict__ kv, const double *__restrict__ kfac,
                                                    const double2 *__restrict__ sk, double *__restrict__ fks)
{
    __shared__ int4 skv[kSFTile];
    __shared__ double2 ssk[kSFTile][4];
    __shared__ double3 skk[kSFTile];        // kfac2 n 2pi/L per component, as the reference forms it
    const int ia = blockIdx.x * kSF + threadIdx.x;
    const bool on = ia < na;
    const int k0 = blockIdx.y * klen, k1 = min(nkv, k0 + klen);
    double x[3] = {0.0, 0.0, 0.0}, q = 0.0;
    if (on) {
        for (int m = 0; m < 3; ++m) x[m] = r[3 * (size_t)ia + m];
        q = az[ia];
    }
    const double tp[3] = {tpbi.x, tpbi.y, tpbi.z};
    double2 e1[3];
    for (int m = 0; m < 3; ++m) {
        double sn, cs;
        sincos(tp[m] * x[m], &sn, &cs);
        e1[m] = make_double2(cs, sn);
    }
    double2 ex = make_double2(1.0, 0.0), ey = ex, ez = ex, yzm = ex, yzp = ex;
    int cx = 0, cy = 0, cz = 0, row = -1;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int t0 = k0; t0 < k1; t0 += kSFTile) {
        const int nt = min(kSFTile, k1 - t0);
        __syncthreads();
        for (int e = threadIdx.x; e < nt; e += kSF) {
            const size_t g = (size_t)t0 + e;
            const int4 n = kv[g];
            const double kf2 = epsfp * 2.0 * kfac[g];
            skv[e] = n;
            skk[e] = make_double3(kf2 * n.x * tp[0], kf2 * n.y * tp[1], kf2 * n.z * tp[2]);
            for (int c = 0; c < 4; ++c) ssk[e][c] = sk[g * 4 + c];
        }
        __syncthreads();
        // one k-vector's terms, added to the site's force in k order
        auto term = [&](int e, double2 exv, double &gx, double &gy, double &gz) {
            const double2 qx = make_double2(q * exv.x, q * exv.y), qxc = zconj(qx);
            const double2 r0 = zmul(qxc, yzm), r1 = zmul(qxc, yzp), r2 = zmul(qx, yzm), r3 = zmul(qx, yzp);
            const double2 s0 = ssk[e][0], s1 = ssk[e][1], s2 = ssk[e][2], s3 = ssk[e][3];
            const double fmm = -r0.x * s0.y + r0.y * s0.x, fmp = -r1.x * s1.y + r1.y * s1.x;
            const double fpm = -r2.x * s2.y + r2.y * s2.x, fpp = -r3.x * s3.y + r3.y * s3.x;
            const double3 K = skk[e];
            gx = K.x * (-fmm - fmp + fpm + fpp);
            gy = K.y * (-fmm + fmp - fpm + fpp);
            gz = K.z * (fmm + fmp + fpm + fpp);
        };
        for (int e = 0; e < nt;) {
            const int4 n = skv[e];
            const int key = n.z * (kSMaxCut + 1) + n.y;
            if (key != row) {
                if (n.z != cz) {
                    while (cz < n.z) { ez = (cz == 0) ? e1[2] : zmul(ez, e1[2]); ++cz; }
                    ey = make_double2(1.0, 0.0);
                    cy = 0;
                }
                while (cy < n.y) { ey = (cy == 0) ? e1[1] : zmul(ey, e1[1]); ++cy; }
                yzm = zmul(zconj(ey), ez);
                yzp = zmul(ey, ez);
                ex = make_double2(1.0, 0.0);
                cx = 0;
                row = key;
            }
            while (cx < n.x) { ex = (cx == 0) ? e1[0] : zmul(ex, e1[0]); ++cx; }
            // two k-vectors at a time when the next one is the same row's next nx (the common
            // case): their terms are independent work for the scheduler; the sums keep k order
            if (e + 1 < nt && skv[e + 1].x == n.x + 1 && skv[e + 1].y == n.y && skv[e + 1].z == n.z) {
                const double2 ex2 = (cx == 0) ? e1[0] : zmul(ex, e1[0]);
                double ax, ay, az_, bx, by, bz;
                term(e, ex, ax, ay, az_);
                term(e + 1, ex2, bx, by, bz);
                fx += ax;
                fy += ay;
                fz += az_;
                fx += bx;
                fy += by;
                fz += bz;
                ex = ex2;
                ++cx;
                e += 2;
            } else {
                double ax, ay, az_;
                term(e, ex, ax, ay, az_);
                fx += ax;
                fy += ay;
                fz += az_;
                ++e;
            }
        }
    }
    if (on) {
        double *o = fks + ((size_t)blockIdx.y * na + ia) * 3;
        o[0] = fx;
        o[1] = fy;
        o[2] = fz;
    }
}

// The sites' dipole sum q r of the surface term, in 64-bit fixed point (2^-32) at efix[3..5].
__global__ void k_site_dipole(int na, const double *__restrict__ r, const double *__restrict__ az,
                              unsigned long long *__restrict__ efix)
{
    const int ia = blockIdx.x * blockDim.x + threadIdx.x;
    long long m[3] = {0, 0, 0};
    if (ia < na)
        for (int c = 0; c < 3; ++c) m[c] = __double2ll_rn(az[ia] * r[3 * (size_t)ia + c] * kDipFix);
    for (int o = 16; o > 0; o >>= 1)
        for (int c = 0; c < 3; ++c) m[c] += __shfl_xor_sync(0xffffffffu, m[c], o);
    if ((threadIdx.x & 31) == 0)
        for (int c = 0; c < 3; ++c)
            if (m[c]) atomicAdd(efix + 3 + c, (unsigned long long)m[c]);
}

// The sites' reciprocal force: the k slices added in slice order, less the surface term's
// force epsfp 2 fac q M (UEwaldSurf, Src/energy.F90:1349-1371) when sfac = 2 fac is not 0;
// stored, or added to the force already there when add is set.
__global__ void k_site_fsum(int na, int nks, int add, double epsfp, double sfac, const double *__restrict__ az,
                            const unsigned long long *__restrict__ efix, const double *__restrict__ fks,
                            double *__restrict__ force)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * na) return;
    double f = 0.0;
    for (int k = 0; k < nks; ++k) f += fks[(size_t)k * 3 * na + i];
    if (sfac != 0.0) {
        const double M = (double)(long long)efix[3 + i % 3] * kDipFixInv;
        f = f - epsfp * sfac * az[i / 3] * M;
    }
    force[i] = add ? force[i] + f : f;
}

// UEwaldSelf's molecular term (Src/energy.F90:1315-1343): every site pair inside a
// particle subtracts q q erf(alpha r)/r; its forces are added into `force`.
__global__ void k_site_self(int np, double alpha, double ewaldfac1, double epsfp, const double *__restrict__ r,
                            const double *__restrict__ az, const int *__restrict__ iptpn,
                            const int *__restrict__ ianpn, const int *__restrict__ napt, double *__restrict__ force,
                            unsigned long long *__restrict__ efix)
{
    const int ip = blockIdx.x * blockDim.x + threadIdx.x;
    long long eu = 0;
    if (ip < np) {
        const int ialow = ianpn[ip] - 1, iaupp = ialow + napt[iptpn[ip] - 1] - 1;
        for (int i = ialow; i <= iaupp; ++i)
            for (int j = i + 1; j <= iaupp; ++j) {
                const double dx = r[3 * (size_t)i] - r[3 * (size_t)j], dy = r[3 * (size_t)i + 1] - r[3 * (size_t)j + 1],
                             dz = r[3 * (size_t)i + 2] - r[3 * (size_t)j + 2];
                const double r2 = dx * dx + dy * dy + dz * dz, r1 = sqrt(r2);
                double r1i = 1.0 / r1;
                const double r2i = r1i * r1i, ex = exp(-(alpha * alpha) * r2);
                r1i = r1i * erf(alpha * r1);
                const double r3i = r2i * (r1i - ewaldfac1 * ex);
                eu += __double2ll_rn(-(az[i] * az[j] * r1i) * kPFix);
                const double fac = epsfp * az[i] * az[j] * r3i;
                // the particle's own sites: this thread is the only writer
                force[3 * (size_t)i] -= fac * dx;
                force[3 * (size_t)i + 1] -= fac * dy;
                force[3 * (size_t)i + 2] -= fac * dz;
                force[3 * (size_t)j] += fac * dx;
                force[3 * (size_t)j + 1] += fac * dy;
                force[3 * (size_t)j + 2] += fac * dz;
            }
    }
    for (int o = 16; o > 0; o >>= 1) eu += __shfl_xor_sync(0xffffffffu, eu, o);
    if ((threadIdx.x & 31) == 0 && eu) atomicAdd(efix + 2, (unsigned long long)eu);
}

// ---- SPME over the sites (UEwaldRecSPM + SPMFFTRec, Src/energy.F90:1207-1297, 6525-6587) ----
// the charge mesh in 64-bit fixed point at 2^-40 while it is spread, so it repeats bit for bit
constexpr double kGFix = 1099511627776.0;
constexpr double kGFixInv = 1.0 / 1099511627776.0;

// Q(k - i) += q Mx My Mz over the site's order^3 mesh points (Src/energy.F90:1226-1245).
template <int P>
__global__ void k_sspm_spread(int na, int s, double3 dkdr, const double *__restrict__ r,
                              const double *__restrict__ az, unsigned long long *__restrict__ igrid)
{
    const int ia = blockIdx.x * blockDim.x + threadIdx.x;
    if (ia >= na) return;
    const double dk[3] = {dkdr.x, dkdr.y, dkdr.z};
    double th[3][P], dth[3][P];
    int km[3];
    for (int m = 0; m < 3; ++m) km[m] = msg::bspline_at<P, double>(dk[m] * r[3 * (size_t)ia + m], s, th[m], dth[m]);
    const double q = az[ia];
    for (int iz = 0; iz < P; ++iz) {
        int nz = km[2] - iz;
        nz += (nz < 0) ? s : 0;
        const double qz = q * th[2][iz];
        for (int iy = 0; iy < P; ++iy) {
            int ny = km[1] - iy;
            ny += (ny < 0) ? s : 0;
            const double qyz = qz * th[1][iy];
            for (int ix = 0; ix < P; ++ix) {
                int nx = km[0] - ix;
                nx += (nx < 0) ? s : 0;
                const double v = qyz * th[0][ix];
                atomicAdd(igrid + ((size_t)nz * s + ny) * s + nx, (unsigned long long)__double2ll_rn(v * kGFix));
            }
        }
    }
}

// The fixed-point mesh to FP64 for the transform, cleared for the next spread.
__global__ void k_sspm_to_f64(size_t n, unsigned long long *__restrict__ igrid, double *__restrict__ grid)
{
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) {
        grid[k] = (double)(long long)igrid[k] * kGFixInv;
        igrid[k] = 0ull;
    }
}

// F *= meshfac; energy |F|^2 emf and virial -|F|^2 vmf over the r2c half spectrum (the
// reference's mirror loop resolved into per-entry weights; Src/energy.F90:6550-6578), summed
// in 64-bit fixed point (2^-40).
__global__ void __launch_bounds__(256) k_sspm_influence(int s, double2 *__restrict__ cg, const double *__restrict__ mfac,
                                                        const double *__restrict__ emf, const double *__restrict__ vmf,
                                                        unsigned long long *__restrict__ efix)
{
    const int h = s / 2 + 1;
    const size_t n = (size_t)s * s * h;
    const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    long long e = 0, v = 0;
    if (c < n) {
        const int kx = (int)(c % h), rr = (int)(c / h), ky = rr % s, kz = rr / s;
        const int fy = ky <= s / 2 ? ky : s - ky, fz = kz <= s / 2 ? kz : s - kz;
        const size_t f = kx + (size_t)h * (fy + (size_t)h * fz);
        double2 q = cg[c];
        const double q2 = q.x * q.x + q.y * q.y, m = mfac[f];
        q.x *= m;
        q.y *= m;
        cg[c] = q;
        e = __double2ll_rn(q2 * emf[f] * kPFix);
        v = __double2ll_rn(-(q2 * vmf[f]) * kPFix);
    }
    for (int o = 16; o > 0; o >>= 1) {
        e += __shfl_xor_sync(0xffffffffu, e, o);
        v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (e) atomicAdd(efix, (unsigned long long)e);
        if (v) atomicAdd(efix + 1, (unsigned long long)v);
    }
}

// The sites' reciprocal forces from the convolved mesh (Src/energy.F90:1258-1285), less the
// surface term's force when sfac = 2 fac is not 0; stored, or added when add is set.
template <int P>
__global__ void k_sspm_gather(int na, int s, double3 dkdr, int add, double epsfp, double sfac,
                              const double *__restrict__ r, const double *__restrict__ az,
                              const double *__restrict__ grid, const unsigned long long *__restrict__ efix,
                              double *__restrict__ force)
{
    const int ia = blockIdx.x * blockDim.x + threadIdx.x;
    if (ia >= na) return;
    const double dk[3] = {dkdr.x, dkdr.y, dkdr.z};
    double th[3][P], dth[3][P];
    int km[3];
    for (int m = 0; m < 3; ++m) km[m] = msg::bspline_at<P, double>(dk[m] * r[3 * (size_t)ia + m], s, th[m], dth[m]);
    double es[3] = {0.0, 0.0, 0.0};
    for (int iz = 0; iz < P; ++iz) {
        int nz = km[2] - iz;
        nz += (nz < 0) ? s : 0;
        for (int iy = 0; iy < P; ++iy) {
            int ny = km[1] - iy;
            ny += (ny < 0) ? s : 0;
            const double *row = grid + ((size_t)nz * s + ny) * s;
            for (int ix = 0; ix < P; ++ix) {
                int nx = km[0] - ix;
                nx += (nx < 0) ? s : 0;
                const double Q = row[nx];
                es[0] = es[0] + dth[0][ix] * th[1][iy] * th[2][iz] * Q;
                es[1] = es[1] + th[0][ix] * dth[1][iy] * th[2][iz] * Q;
                es[2] = es[2] + th[0][ix] * th[1][iy] * dth[2][iz] * Q;
            }
        }
    }
    const double q = az[ia];
    for (int m = 0; m < 3; ++m) {
        double f = -(q * es[m] * dk[m] * epsfp);
        if (sfac != 0.0) f = f - epsfp * sfac * q * ((double)(long long)efix[3 + m] * kDipFixInv);
        double *o = force + 3 * (size_t)ia + m;
        *o = add ? *o + f : f;
    }
}

// The site Ewald sum of one system: set-up on the host (k-vectors, kfac, launch shapes,
// device buffers) and a launch sequence on the caller's device arrays, so one set-up
// serves every step of a run.  Device accumulators efix: reciprocal energy, its virial,
// the molecular self energy (2^-40) and the dipole sum (2^-32).
struct SiteEwald {
    int lewald = 0;                 // 1: SPME over the sites, 2: standard Ewald
    int na = 0, np = 0, lsurf = 0;
    double alpha = 0.0, epsfp = 0.0, vol = 0.0, q2 = 0.0, ewaldfac1 = 0.0;
    double *daz = nullptr;
    unsigned long long *efix = nullptr;
    // standard Ewald
    int nkv = 0, w = 0, ktiles = 0, ptiles = 0, clen = 0, nchunk = 0, klen = 0, nks = 0, sub = 0;
    double3 tpbi = make_double3(0.0, 0.0, 0.0);
    double *dkf = nullptr, *fks = nullptr;
    int4 *dkv = nullptr;
    double2 *eik = nullptr, *part = nullptr, *sk = nullptr;
    // SPME
    int smesh = 0, order = 0;
    double3 dkdr = make_double3(0.0, 0.0, 0.0);
    unsigned long long *igrid = nullptr;
    double *grid = nullptr, *mfac = nullptr, *emf = nullptr, *vmf = nullptr;
    double2 *cgrid = nullptr;
    cufftHandle pf = 0, pb = 0;       // from the per-thread plan cache

    static constexpr double kPi = 3.1415926535897932;

    // Checks and the parts both methods share.  MSG_ERR_ARG for arguments outside what the
    // reference accepts, else the CUDA status.
    int common(int32_t na_, const double boxlen[3], double ualpha, int32_t lsurf_, double epsfp_, const double *az,
               int32_t np_, const int32_t *iptpn, const int32_t *ianpn, const int32_t *napt, int32_t npt)
    {
        if (na_ < 1 || np_ < 1 || npt < 1 || !(ualpha > 0.0) || !boxlen || !az || !iptpn || !ianpn || !napt)
            return MSG_ERR_ARG;
        for (int t = 0; t < npt; ++t)
            if (napt[t] < 1) return MSG_ERR_ARG;
        for (int i = 0; i < np_; ++i)
            if (iptpn[i] < 1 || iptpn[i] > npt || ianpn[i] < 1 || ianpn[i] - 1 + napt[iptpn[i] - 1] > na_)
                return MSG_ERR_ARG;
        na = na_;
        np = np_;
        lsurf = lsurf_ ? 1 : 0;
        alpha = ualpha;
        epsfp = epsfp_;
        vol = boxlen[0] * boxlen[1] * boxlen[2];
        ewaldfac1 = (1.0 / (std::sqrt(kPi) * ualpha)) * 2.0 * (ualpha * ualpha);
        q2 = 0.0;
        for (int a = 0; a < na; ++a) q2 += az[a] * az[a];
        cudaError_t e = cudaSuccess;
        daz = dev_copy(az, (size_t)na, e);
        if (e == cudaSuccess) e = pmalloc(&efix, 6 * sizeof(unsigned long long));
        return e == cudaSuccess ? MSG_OK : MSG_ERR_CUDA;
    }

    // Standard Ewald (txewaldrec 'std'): ncut 1..100, ncutregion 0 sphere / 1 cube.
    int setup(int32_t na_, const double boxlen[3], double ualpha, int32_t ncut, int32_t ncutregion, int32_t lsurf_,
              double epsfp_, const double *az, int32_t np_, const int32_t *iptpn, const int32_t *ianpn,
              const int32_t *napt, int32_t npt)
    {
        if (ncut < 1 || ncut > kSMaxCut || ncutregion < 0 || ncutregion > 1) return MSG_ERR_ARG;
        const int rc = common(na_, boxlen, ualpha, lsurf_, epsfp_, az, np_, iptpn, ianpn, napt, npt);
        if (rc != MSG_OK) return rc;
        lewald = 2;
        tpbi = make_double3(2.0 * kPi * (1.0 / boxlen[0]), 2.0 * kPi * (1.0 / boxlen[1]), 2.0 * kPi * (1.0 / boxlen[2]));
        // k-vectors and kfac in the order of EwaldSetup 'std' (Src/energy.F90:6762-6782)
        std::vector<int4> kv;
        std::vector<double> kf;
        const int ncut2 = ncutregion ? 3 * ncut * ncut : ncut * ncut;
        for (int nz = 0; nz <= ncut; ++nz)
            for (int ny = 0; ny <= ncut; ++ny)
                for (int nx = 0; nx <= ncut; ++nx) {
                    if (nx * nx + ny * ny + nz * nz > ncut2 || (nx == 0 && ny == 0 && nz == 0)) continue;
                    const double facz = nz == 0 ? 1.0 : 2.0, facy = ny == 0 ? 0.5 : 1.0, facx = nx == 0 ? 0.5 : 1.0;
                    const double kx = nx * tpbi.x, ky = ny * tpbi.y, kz = nz * tpbi.z, k2 = kx * kx + ky * ky + kz * kz;
                    kf.push_back(2.0 * kPi / vol * facz * facy * facx * std::exp(-k2 / (4.0 * (ualpha * ualpha))) / k2);
                    kv.push_back(make_int4(nx, ny, nz, 0));
                }
        nkv = (int)kv.size();
        w = ncut + 1;
        // site chunks of the structure-factor sum (about eight blocks per SM of a 148-SM B200, a
        // chunk at least 128 sites) and k slices of the force sum (about four blocks per SM, a
        // slice at least 16 k-vectors): from the system's sizes only, so the sums repeat bit for bit
        ktiles = (nkv + kSK - 1) / kSK;
        ptiles = (na + kSF - 1) / kSF;
        const int nch = std::max(1, std::min((8 * 148 + ktiles - 1) / ktiles, (na + 127) / 128));
        clen = (na + nch - 1) / nch;
        nchunk = (na + clen - 1) / clen;
        const int nks0 = std::max(1, std::min((4 * 148 + ptiles - 1) / ptiles, std::max(1, nkv / 16)));
        klen = (nkv + nks0 - 1) / nks0;
        nks = (nkv + klen - 1) / klen;
        sub = std::max(1, std::min(16, kSSmem / (3 * w * (int)sizeof(double2))));
        cudaError_t e = cudaSuccess;
        dkf = dev_copy(kf.data(), kf.size(), e);
        dkv = dev_copy(kv.data(), kv.size(), e);
        if (e == cudaSuccess) e = pmalloc(&eik, (size_t)na * 3 * w * sizeof(double2));
        if (e == cudaSuccess) e = pmalloc(&part, (size_t)nchunk * nkv * 4 * sizeof(double2));
        if (e == cudaSuccess) e = pmalloc(&sk, (size_t)nkv * 4 * sizeof(double2));
        if (e == cudaSuccess) e = pmalloc(&fks, (size_t)nks * 3 * na * sizeof(double));
        return e == cudaSuccess ? MSG_OK : MSG_ERR_CUDA;
    }

    // SPME (txewaldrec 'spm'): order 4..8, nmesh even, 8..1024 (EwaldSetup SPM branch,
    // Src/energy.F90:6980-7018, for the mesh factors).
    int setup_spm(int32_t na_, const double boxlen[3], double ualpha, int32_t order_, int32_t nmesh, int32_t lsurf_,
                  double epsfp_, const double *az, int32_t np_, const int32_t *iptpn, const int32_t *ianpn,
                  const int32_t *napt, int32_t npt)
    {
        if (order_ < 4 || order_ > 8 || nmesh < 8 || nmesh > 1024 || (nmesh & 1)) return MSG_ERR_ARG;
        const int rc = common(na_, boxlen, ualpha, lsurf_, epsfp_, az, np_, iptpn, ianpn, napt, npt);
        if (rc != MSG_OK) return rc;
        lewald = 1;
        smesh = nmesh;
        order = order_;
        dkdr = make_double3(nmesh / boxlen[0], nmesh / boxlen[1], nmesh / boxlen[2]);
        const int h = nmesh / 2 + 1;
        const size_t nf = (size_t)h * h * h, ng = (size_t)nmesh * nmesh * nmesh, nc = (size_t)nmesh * nmesh * h;
        std::vector<double> hm(nf), he(nf), hv(nf);
        msg::spme_factors(nmesh, order, ualpha, boxlen, hm.data(), he.data(), hv.data());
        cudaError_t e = cudaSuccess;
        mfac = dev_copy(hm.data(), nf, e);
        emf = dev_copy(he.data(), nf, e);
        vmf = dev_copy(hv.data(), nf, e);
        if (e == cudaSuccess) e = pmalloc(&igrid, ng * sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMemset(igrid, 0, ng * sizeof(unsigned long long));
        if (e == cudaSuccess) e = pmalloc(&grid, ng * sizeof(double));
        if (e == cudaSuccess) e = pmalloc(&cgrid, nc * sizeof(double2));
        if (e != cudaSuccess) return MSG_ERR_CUDA;
        if (!spm_plans(nmesh, pf, pb)) return MSG_ERR_CUDA;
        return MSG_OK;
    }

    template <int P>
    void launch_spm(const double *dr, double *dforce, int add, double sfac, cudaStream_t st) const
    {
        const size_t ng = (size_t)smesh * smesh * smesh, nc = (size_t)smesh * smesh * (smesh / 2 + 1);
        k_sspm_spread<P><<<(na + 127) / 128, 128, 0, st>>>(na, smesh, dkdr, dr, daz, igrid);
        k_sspm_to_f64<<<(unsigned)((ng + 255) / 256), 256, 0, st>>>(ng, igrid, grid);
        cufftSetStream(pf, st);
        cufftExecD2Z(pf, grid, reinterpret_cast<cufftDoubleComplex *>(cgrid));
        k_sspm_influence<<<(unsigned)((nc + 255) / 256), 256, 0, st>>>(smesh, cgrid, mfac, emf, vmf, efix);
        cufftSetStream(pb, st);
        cufftExecZ2D(pb, reinterpret_cast<cufftDoubleComplex *>(cgrid), grid);
        k_sspm_gather<P><<<(na + 127) / 128, 128, 0, st>>>(na, smesh, dkdr, add, epsfp, sfac, dr, daz, grid, efix,
                                                           dforce);
    }

    // One evaluation at the sites dr: the Ewald forces stored into dforce (add = 0) or added
    // to it (add = 1); the accumulators restart.
    void launch(const double *dr, const int *dipt, const int *dian, const int *dnapt, double *dforce, int add,
                cudaStream_t st) const
    {
        cudaMemsetAsync(efix, 0, 6 * sizeof(unsigned long long), st);
        double sfac = 0.0;
        if (lsurf) {
            k_site_dipole<<<(na + 127) / 128, 128, 0, st>>>(na, dr, daz, efix);
            sfac = 2.0 * (2.0 * kPi / (3.0 * vol));
        }
        if (lewald == 2) {
            k_site_eik<<<(na + 127) / 128, 128, 0, st>>>(na, w, tpbi, dr, daz, eik);
            k_site_sk<<<dim3(ktiles, nchunk), kSK, (size_t)sub * 3 * w * sizeof(double2), st>>>(na, nkv, w, clen, sub,
                                                                                              dkv, eik, part);
            k_site_reduce<<<ktiles, kSK, 0, st>>>(nkv, nchunk, alpha * alpha, tpbi, dkv, dkf, part, sk, efix);
            k_site_force<<<dim3(ptiles, nks), kSF, 0, st>>>(na, nkv, klen, epsfp, tpbi, dr, daz, dkv, dkf, sk, fks);
            k_site_fsum<<<(3 * na + 255) / 256, 256, 0, st>>>(na, nks, add, epsfp, sfac, daz, efix, fks, dforce);
        } else {
            switch (order) {
            case 4: launch_spm<4>(dr, dforce, add, sfac, st); break;
            case 5: launch_spm<5>(dr, dforce, add, sfac, st); break;
            case 6: launch_spm<6>(dr, dforce, add, sfac, st); break;
            case 7: launch_spm<7>(dr, dforce, add, sfac, st); break;
            default: launch_spm<8>(dr, dforce, add, sfac, st); break;
            }
        }
        k_site_self<<<(np + 127) / 128, 128, 0, st>>>(np, alpha, ewaldfac1, epsfp, dr, daz, dipt, dian, dnapt, dforce,
                                                      efix);
    }

    // u%rec and its virial (scaled by EpsiFourPi as UEwald does) of the last launch.
    cudaError_t energies(double &urec, double &virrec) const
    {
        unsigned long long h[6];
        const cudaError_t e = cudaMemcpy(h, efix, sizeof(h), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return e;
        double u = (double)(long long)h[0] * kPFixInv - alpha / std::sqrt(kPi) * q2 + (double)(long long)h[2] * kPFixInv;
        double vr = (double)(long long)h[1] * kPFixInv;
        if (lsurf) {
            const double fac = 2.0 * kPi / (3.0 * vol);
            double M[3];
            for (int c = 0; c < 3; ++c) M[c] = (double)(long long)h[3 + c] * kDipFixInv;
            const double term = fac * (M[0] * M[0] + M[1] * M[1] + M[2] * M[2]);
            u += term;
            vr -= term;
        }
        urec = epsfp * u;
        virrec = epsfp * vr;
        return cudaSuccess;
    }

    ~SiteEwald()
    {
        for (void *p : {(void *)daz, (void *)efix, (void *)dkf, (void *)dkv, (void *)eik, (void *)part, (void *)sk,
                        (void *)fks, (void *)igrid, (void *)grid, (void *)cgrid, (void *)mfac, (void *)emf,
                        (void *)vmf})
            if (p) pfree(p);
    }
};

}  // namespace

// One site Ewald evaluation of host arrays through a set-up SiteEwald.
static int uewald_sites_call(const SiteEwald &E, int32_t na, const double *r, int32_t np, const int32_t *iptpn,
                             const int32_t *ianpn, const int32_t *napt, int32_t npt, double *force, double *urec,
                             double *virrec, float *kernel_ms)
{
    cudaError_t e = cudaSuccess;
    double *dr = dev_copy(r, 3 * (size_t)na, e), *dforce = nullptr;
    int *dipt = dev_copy(iptpn, (size_t)np, e), *dian = dev_copy(ianpn, (size_t)np, e), *dnapt = dev_copy(napt, (size_t)npt, e);
    if (e == cudaSuccess) e = pmalloc(&dforce, 3 * (size_t)na * sizeof(double));
    if (e == cudaSuccess) {
        cudaEvent_t a = nullptr, b = nullptr;
        if (kernel_ms) {
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            cudaEventRecord(a, 0);
        }
        E.launch(dr, dipt, dian, dnapt, dforce, 0, 0);
        if (kernel_ms) {
            cudaEventRecord(b, 0);
            cudaEventSynchronize(b);
            cudaEventElapsedTime(kernel_ms, a, b);
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpy(force, dforce, 3 * (size_t)na * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = E.energies(*urec, *virrec);
    }
    for (void *p : {(void *)dr, (void *)dipt, (void *)dian, (void *)dnapt, (void *)dforce})
        if (p) pfree(p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return MSG_ERR_CUDA;
    }
    return MSG_OK;
}

extern "C" int msg_uewald_sites(int32_t na, const double boxlen[3], double ualpha, int32_t ncut, int32_t ncutregion,
                                int32_t lsurf, double epsfp, const double *r, const double *az, int32_t np,
                                const int32_t *iptpn, const int32_t *ianpn, const int32_t *napt, int32_t npt,
                                double *force, double *urec, double *virrec, float *kernel_ms)
{
    ArenaScope scope;
    if (!r || !force || !urec || !virrec) return MSG_ERR_ARG;
    SiteEwald E;
    const int rc = E.setup(na, boxlen, ualpha, ncut, ncutregion, lsurf, epsfp, az, np, iptpn, ianpn, napt, npt);
    if (rc != MSG_OK) {
        cudaGetLastError();
        return rc;
    }
    return uewald_sites_call(E, na, r, np, iptpn, ianpn, napt, npt, force, urec, virrec, kernel_ms);
}

extern "C" int msg_uewald_sites_spm(int32_t na, const double boxlen[3], double ualpha, int32_t order, int32_t nmesh,
                                    int32_t lsurf, double epsfp, const double *r, const double *az, int32_t np,
                                    const int32_t *iptpn, const int32_t *ianpn, const int32_t *napt, int32_t npt,
                                    double *force, double *urec, double *virrec, float *kernel_ms)
{
    ArenaScope scope;
    if (!r || !force || !urec || !virrec) return MSG_ERR_ARG;
    SiteEwald E;
    const int rc = E.setup_spm(na, boxlen, ualpha, order, nmesh, lsurf, epsfp, az, np, iptpn, ianpn, napt, npt);
    if (rc != MSG_OK) {
        cudaGetLastError();
        return rc;
    }
    return uewald_sites_call(E, na, r, np, iptpn, ianpn, napt, npt, force, urec, virrec, kernel_ms);
}

// The rigid-body MD steps of msg_velver_p and msg_velver_p_ewald: ew (optional) adds the
// site Ewald sum to the site forces of every step before the kick, and its reciprocal
// virial to the returned virial; urec receives u%rec of the last step.
static int velver_p_run(const SiteEwald *ew, double *urec, int32_t nsteps, int32_t np, int32_t na, int32_t npt,
                        int32_t nat, const double boxlen[3], double rcut, double tstep, int32_t nvvite, double tvvite,
                        double *ro, double *rod, double *rodd, double *qua, double *quad, double *quadd, double *r,
                        const int32_t *iptpn, const int32_t *ianpn, const int32_t *napt, const int32_t *iatan,
                        const double *ra, int32_t maxsite, const double *masspt, const double *momp,
                        const int32_t *nneighpn, const int32_t *jpnlist, int32_t maxnneigh, const double *ubuf,
                        int32_t nbuf, const int32_t *iubuflow, const double *r2umin, double *utwob, double *virial,
                        float *kernel_ms)
{
    if (nsteps < 0 || np < 1 || na < 1 || npt < 1 || npt > kPMaxType || nat < 1 || maxsite < 1 || maxsite > 256 ||
        maxnneigh < 1 || nbuf < 12 ||
        nvvite < 0 || !boxlen || !ro || !rod || !rodd || !qua || !quad || !quadd || !r || !iptpn || !ianpn ||
        !napt || !iatan || !ra || !masspt || !momp || !nneighpn || !jpnlist || !ubuf || !iubuflow || !r2umin ||
        !utwob || !virial)
        return MSG_ERR_ARG;
    for (int t = 0; t < npt; ++t)
        if (napt[t] < 1 || napt[t] > maxsite || !(masspt[t] > 0.0) || !(momp[3 * t] > 0.0) || !(momp[3 * t + 1] > 0.0) ||
            !(momp[3 * t + 2] > 0.0))
            return MSG_ERR_ARG;
    for (int i = 0; i < np; ++i) {
        if (iptpn[i] < 1 || iptpn[i] > npt || ianpn[i] < 1 || ianpn[i] - 1 + napt[iptpn[i] - 1] > na)
            return MSG_ERR_ARG;
        if (nneighpn[i] < 0 || nneighpn[i] > maxnneigh) return MSG_ERR_ARG;
        for (int k = 0; k < nneighpn[i]; ++k) {
            const int j = jpnlist[(size_t)i * maxnneigh + k];
            if (j < 1 || j > np) return MSG_ERR_ARG;
        }
    }
    const int natat = nat * (nat + 1) / 2, nptpt = npt * (npt + 1) / 2;
    for (int a = 0; a < na; ++a)
        if (iatan[a] < 1 || iatan[a] > nat) return MSG_ERR_ARG;
    for (int q = 0; q < natat; ++q)
        if (iubuflow[q] < 1 || iubuflow[q] + 11 > nbuf) return MSG_ERR_ARG;
    RigidArgs A;
    A.np = np;
    A.nvvite = nvvite;
    A.tstep = tstep;
    A.tvvite = tvvite;
    A.fac = 0.5 * tstep * tstep;
    for (int m = 0; m < 3; ++m) {
        A.box[m] = boxlen[m];
        A.half[m] = boxlen[m] / 2.0;
        A.boxi[m] = 1.0 / boxlen[m];
    }
    A.maxsite = maxsite;
    {
        // (sclene / scllen) / sclfor with MOLSIM's scales (Src/molsim.F90:786-805)
        const double scllen = 1.0e-10, sclmas = 1.0e-03, scltim = 1.0e-12, sclene = 1.0e+03;
        const double sclvel = scllen / scltim, sclacc = sclvel / scltim;
        A.ffac = (sclene / scllen) / (sclacc * sclmas);
    }
    cudaError_t e = cudaSuccess;
    double *dro = dev_copy(ro, 3 * (size_t)np, e), *drod = dev_copy(rod, 3 * (size_t)np, e),
           *drodd = dev_copy(rodd, 3 * (size_t)np, e), *dqua = dev_copy(qua, 4 * (size_t)np, e),
           *dquad = dev_copy(quad, 4 * (size_t)np, e), *dquadd = dev_copy(quadd, 4 * (size_t)np, e),
           *dr = dev_copy(r, 3 * (size_t)na, e), *dra = dev_copy(ra, 3 * (size_t)npt * maxsite, e),
           *dmass = dev_copy(masspt, (size_t)npt, e), *dmom = dev_copy(momp, 3 * (size_t)npt, e);
    int *dipt = dev_copy(iptpn, (size_t)np, e), *dian = dev_copy(ianpn, (size_t)np, e);
    int *dnapt = dev_copy(napt, (size_t)npt, e), *diat = dev_copy(iatan, (size_t)na, e);
    int *dnn = dev_copy(nneighpn, (size_t)np, e), *djp = dev_copy(jpnlist, (size_t)np * maxnneigh, e);
    double *dub = dev_copy(ubuf, (size_t)nbuf, e), *dr2 = dev_copy(r2umin, (size_t)natat, e);
    int *diub = dev_copy(iubuflow, (size_t)natat, e);
    std::vector<SiteBuckets> hsb;
    std::vector<int> hbs;
    site_buckets(natat, ubuf, nbuf, iubuflow, r2umin, hsb, hbs);
    SiteBuckets *dsb = dev_copy(hsb.data(), hsb.size(), e);
    int *dbs = dev_copy(hbs.data(), hbs.size(), e);
    unsigned long long *ffix = nullptr;
    double *dforce = nullptr, *duv = nullptr, *dori = nullptr;
    int *derr = nullptr;
    const size_t nfix = 3 * (size_t)na + nptpt + 2;           // site forces, energies, pair and molecular virial
    if (e == cudaSuccess) e = pmalloc(&ffix, nfix * sizeof(unsigned long long));
    if (e == cudaSuccess) e = pmalloc(&dforce, 3 * (size_t)na * sizeof(double));
    if (e == cudaSuccess) e = pmalloc(&duv, (nptpt + 2) * sizeof(double));
    if (e == cudaSuccess) e = pmalloc(&dori, 9 * (size_t)np * sizeof(double));
    if (e == cudaSuccess) e = pmalloc(&derr, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(derr, 0, sizeof(int));
    int herr = 0;
    double vmol = 0.0;
    if (e == cudaSuccess && nsteps > 0) {
        unsigned long long *ufix = ffix + 3 * (size_t)na, *vfix = ufix + nptpt, *vmfix = vfix + 1;
        cudaEvent_t a = nullptr, b = nullptr;
        if (kernel_ms) {
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            cudaEventRecord(a, 0);
        }
        const int pb = (np + 127) / 128;
        for (int step = 0; step < nsteps; ++step) {
            cudaMemsetAsync(ffix, 0, nfix * sizeof(unsigned long long), 0);
            k_rigid_move<<<pb, 128>>>(A, dro, drod, drodd, dqua, dquad, dquadd, dori, dr, dipt, dian, dnapt, dra);
            k_utwobody_p<<<(np + kPWarps - 1) / kPWarps, kPThreads, site_smem(npt, napt)>>>(
                np, npt, nat, make_double3(boxlen[0], boxlen[1], boxlen[2]), rcut * rcut, dro, dr, dipt, dian, dnapt,
                diat, dnn, djp, maxnneigh, dub, nbuf, diub, dr2, dsb, dbs, max_sites(npt, napt), ffix, ufix, vfix, derr);
            k_utwobody_p_out<<<(int)((3 * (size_t)na + 255) / 256), 256>>>(na, nptpt, ffix, ufix, vfix, dforce, duv);
            if (ew) ew->launch(dr, dipt, dian, dnapt, dforce, 1, 0);
            k_rigid_kick<<<pb, 128>>>(A, dro, drod, drodd, dqua, dquad, dquadd, dori, dr, dforce, dipt, dian, dnapt,
                                      dmass, dmom, vmfix);
        }
        if (kernel_ms) {
            cudaEventRecord(b, 0);
            cudaEventSynchronize(b);
            cudaEventElapsedTime(kernel_ms, a, b);
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
        unsigned long long vm = 0;
        if (e == cudaSuccess) e = cudaMemcpy(&vm, vmfix, sizeof(vm), cudaMemcpyDeviceToHost);
        vmol = (double)(long long)vm * kPFixInv;
    }
    if (e == cudaSuccess && !herr) {
        std::vector<double> uv(nptpt + 2, 0.0);
        if (nsteps > 0) e = cudaMemcpy(uv.data(), duv, uv.size() * sizeof(double), cudaMemcpyDeviceToHost);
        struct Back { double *h, *d; size_t n; } back[] = {
            {ro, dro, 3 * (size_t)np}, {rod, drod, 3 * (size_t)np}, {rodd, drodd, 3 * (size_t)np},
            {qua, dqua, 4 * (size_t)np}, {quad, dquad, 4 * (size_t)np}, {quadd, dquadd, 4 * (size_t)np},
            {r, dr, 3 * (size_t)na}};
        for (const Back &x : back)
            if (e == cudaSuccess) e = cudaMemcpy(x.h, x.d, x.n * sizeof(double), cudaMemcpyDeviceToHost);
        double ur = 0.0, vr = 0.0;
        if (e == cudaSuccess && nsteps > 0 && ew) e = ew->energies(ur, vr);
        if (e == cudaSuccess && nsteps > 0) {
            for (int q = 0; q <= nptpt; ++q) utwob[q] = uv[q];
            *virial = uv[nptpt + 1] + vr + vmol;
            if (urec) *urec = ur;
        }
    }
    for (void *p : {(void *)dro, (void *)drod, (void *)drodd, (void *)dqua, (void *)dquad, (void *)dquadd, (void *)dr,
                    (void *)dra, (void *)dmass, (void *)dmom, (void *)dipt, (void *)dian, (void *)dnapt, (void *)diat,
                    (void *)dnn, (void *)djp, (void *)dub, (void *)dr2, (void *)diub, (void *)dsb, (void *)dbs,
                    (void *)ffix, (void *)dforce, (void *)duv, (void *)dori, (void *)derr})
        if (p) pfree(p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return MSG_ERR_CUDA;
    }
    if (herr == 1) return MSG_ERR_TABLE_MIN;
    if (herr == 2) return MSG_ERR_TABLE_RANGE;
    return MSG_OK;
}

extern "C" int msg_velver_p(int32_t nsteps, int32_t np, int32_t na, int32_t npt, int32_t nat, const double boxlen[3],
                            double rcut, double tstep, int32_t nvvite, double tvvite, double *ro, double *rod,
                            double *rodd, double *qua, double *quad, double *quadd, double *r, const int32_t *iptpn,
                            const int32_t *ianpn, const int32_t *napt, const int32_t *iatan, const double *ra,
                            int32_t maxsite, const double *masspt, const double *momp, const int32_t *nneighpn,
                            const int32_t *jpnlist, int32_t maxnneigh, const double *ubuf, int32_t nbuf,
                            const int32_t *iubuflow, const double *r2umin, double *utwob, double *virial,
                            float *kernel_ms)
{
    ArenaScope scope;
    return velver_p_run(nullptr, nullptr, nsteps, np, na, npt, nat, boxlen, rcut, tstep, nvvite, tvvite, ro, rod, rodd,
                        qua, quad, quadd, r, iptpn, ianpn, napt, iatan, ra, maxsite, masspt, momp, nneighpn, jpnlist,
                        maxnneigh, ubuf, nbuf, iubuflow, r2umin, utwob, virial, kernel_ms);
}

extern "C" int msg_velver_p_ewald(int32_t nsteps, int32_t np, int32_t na, int32_t npt, int32_t nat,
                                  const double boxlen[3], double rcut, double tstep, int32_t nvvite, double tvvite,
                                  double *ro, double *rod, double *rodd, double *qua, double *quad, double *quadd,
                                  double *r, const int32_t *iptpn, const int32_t *ianpn, const int32_t *napt,
                                  const int32_t *iatan, const double *ra, int32_t maxsite, const double *masspt,
                                  const double *momp, const int32_t *nneighpn, const int32_t *jpnlist,
                                  int32_t maxnneigh, const double *ubuf, int32_t nbuf, const int32_t *iubuflow,
                                  const double *r2umin, const msg_site_ewald *ew, double *utwob, double *urec,
                                  double *virial, float *kernel_ms)
{
    ArenaScope scope;
    if (!urec || !ew || (ew->lewald != 1 && ew->lewald != 2)) return MSG_ERR_ARG;
    SiteEwald E;
    const int rc = ew->lewald == 2
                       ? E.setup(na, boxlen, ew->ualpha, ew->ncut, ew->ncutregion, ew->lsurf, ew->epsi_four_pi, ew->az,
                                 np, iptpn, ianpn, napt, npt)
                       : E.setup_spm(na, boxlen, ew->ualpha, ew->order, ew->nmesh, ew->lsurf, ew->epsi_four_pi,
                                     ew->az, np, iptpn, ianpn, napt, npt);
    if (rc != MSG_OK) {
        cudaGetLastError();
        return rc;
    }
    return velver_p_run(&E, urec, nsteps, np, na, npt, nat, boxlen, rcut, tstep, nvvite, tvvite, ro, rod, rodd, qua,
                        quad, quadd, r, iptpn, ianpn, napt, iatan, ra, maxsite, masspt, momp, nneighpn, jpnlist,
                        maxnneigh, ubuf, nbuf, iubuflow, r2umin, utwob, virial, kernel_ms);
}

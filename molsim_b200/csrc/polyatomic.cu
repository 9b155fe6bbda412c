// polyatomic.cu -- UTwoBodyP (Src/energy.F90:786-896): the site-site pair energy,
// forces and virial of polyatomic particles, as UTotal calls it for molecules.
//
// The particle list (MOLSIM's nneighpn/jpnlist over particle centres) decides the
// pairs: a pair interacts when its centres are within rcut after the box shift of
// PBC2 (Src/molaux.F90:193-210); then every site of one particle meets every site
// of the other through the atom-type table, shifted by the centres' box shift.
//
// One block per particle, one thread per list entry.  A thread walks the two
// particles' sites; the forces on both sites, the energy of the particle-type pair
// and the virial are added as 64-bit fixed point (2^-40 of the unit), so the sums do
// not depend on the order the threads land in.  FP64 throughout.
//
// The entry point takes the caller's host arrays in MOLSIM's layout (1-based
// indices), copies them to the device, runs, and copies the results back.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/molsim_gpu.h"

namespace {

constexpr int kPThreads = 128;
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

__global__ void __launch_bounds__(kPThreads) k_utwobody_p(
    int np, int npt, int nat, double3 box, double rcut2, const double *__restrict__ ro,
    const double *__restrict__ r, const int *__restrict__ iptpn, const int *__restrict__ ianpn,
    const int *__restrict__ napt, const int *__restrict__ iatan, const int *__restrict__ nneighpn,
    const int *__restrict__ jpnlist, int maxnneigh, const double *__restrict__ ubuf, int nbuf,
    const int *__restrict__ iubuflow, const double *__restrict__ r2umin, unsigned long long *__restrict__ ffix,
    unsigned long long *__restrict__ ufix, unsigned long long *__restrict__ vfix, int *__restrict__ err)
{
    const int ip = blockIdx.x;
    const double half[3] = {0.5 * box.x, 0.5 * box.y, 0.5 * box.z}, len[3] = {box.x, box.y, box.z};
    const int ipt = iptpn[ip], ialow = ianpn[ip] - 1, iaupp = ialow + napt[ipt - 1] - 1;
    long long vir = 0;
    for (int jploc = threadIdx.x; jploc < nneighpn[ip]; jploc += kPThreads) {
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
        for (int ia = ialow; ia <= iaupp; ++ia) {
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
                int ib = iubuflow[q] - 1;
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
            unsigned long long *fa = ffix + 3 * (size_t)ia;
            atomicAdd(fa, (unsigned long long)__double2ll_rn(fi[0] * kPFix));
            atomicAdd(fa + 1, (unsigned long long)__double2ll_rn(fi[1] * kPFix));
            atomicAdd(fa + 2, (unsigned long long)__double2ll_rn(fi[2] * kPFix));
        }
        atomicAdd(ufix + type_pair(npt, ipt, jpt), (unsigned long long)__double2ll_rn(usum * kPFix));
    }
    if (vir) atomicAdd(vfix, (unsigned long long)vir);
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

template <class T>
T *dev_copy(const T *h, size_t n, cudaError_t &e)
{
    T *d = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&d, std::max<size_t>(n, 1) * sizeof(T));
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
    if (np < 1 || na < 1 || npt < 1 || nat < 1 || maxnneigh < 1 || nbuf < 12 || !boxlen || !ro || !r || !iptpn ||
        !ianpn || !napt || !iatan || !nneighpn || !jpnlist || !ubuf || !iubuflow || !r2umin || !force || !utwob ||
        !virial)
        return MSG_ERR_ARG;
    // host-side checks of the indices the kernel follows
    for (int t = 0; t < npt; ++t)
        if (napt[t] < 1) return MSG_ERR_ARG;
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
    unsigned long long *ffix = nullptr, *ufix = nullptr;
    double *dforce = nullptr, *duv = nullptr;
    int *derr = nullptr;
    const size_t nfix = 3 * (size_t)na + nptpt + 1;
    if (e == cudaSuccess) e = cudaMalloc(&ffix, nfix * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(ffix, 0, nfix * sizeof(unsigned long long));
    ufix = ffix ? ffix + 3 * (size_t)na : nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&dforce, 3 * (size_t)na * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&duv, (nptpt + 2) * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&derr, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(derr, 0, sizeof(int));
    int herr = 0;
    if (e == cudaSuccess) {
        cudaEvent_t a = nullptr, b = nullptr;
        if (kernel_ms) {
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            cudaEventRecord(a, 0);
        }
        k_utwobody_p<<<np, kPThreads>>>(np, npt, nat, make_double3(boxlen[0], boxlen[1], boxlen[2]), rcut * rcut, dro,
                                        dr, dipt, dian, dnapt, diat, dnn, djp, maxnneigh, dub, nbuf, diub, dr2, ffix,
                                        ufix, ufix + nptpt, derr);
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
                    (void *)djp, (void *)dub, (void *)dr2, (void *)diub, (void *)ffix, (void *)dforce, (void *)duv,
                    (void *)derr})
        if (p) cudaFree(p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return MSG_ERR_CUDA;
    }
    if (herr == 1) return MSG_ERR_TABLE_MIN;
    if (herr == 2) return MSG_ERR_TABLE_RANGE;
    return MSG_OK;
}

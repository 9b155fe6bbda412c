// noalloc.cu -- the pair force/energy of UTwoBodyA evaluated on the caller's own
// MOLSIM arrays without allocating anything.
//
// Who needs it: callers that cannot call cudaMalloc -- a host that hands the
// GPU only buffers it already owns (a Fortran program whose device arrays come
// from its own pool or a framework's caching allocator), code running where a
// new allocation would break a memory budget or a captured stream, and
// embedders that forbid libraries from growing device memory.  The handle API
// (msg_create) allocates its buffers once at creation; this entry point
// instead keeps its only scratch -- per-block energy partials, a completion
// counter and an error word -- in a file-scope static __device__ array that
// every GPU which loads the library holds until the process exits.
//
// Limits and rules:
//   * np <= kNaMaxParticles (262144): one block of 256 list rows per 256
//     particles, at most kNaMaxBlocks (1024) blocks of partials.  Larger np
//     is rejected with MSG_ERR_ARG.
//   * Scratch is 1024 x 11 doubles + 16 bytes (about 88 KiB) per device.
//   * The first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, under a mutex); make that first
//     call before any stream capture.
//   * Every call shares the one array and leaves its contents behind.  The
//     call clears the counter and the error word before use; calls that
//     overlap on the GPU (two streams, two host threads) race on it.
//   * Every call waits for its stream to finish: it reads the status word
//     back into host memory before it returns.
//   * The minimum image is PBCr2's rectangular-box branch (lbcbox); MOLSIM's
//     truncated-octahedron and rhombic-dodecahedron cells are not handled.
//   * lmc = 0 takes a half list (SetVList's MD rows: every pair once);
//     lmc = 1 takes a full list (every pair in both rows, as MOLSIM's Monte
//     Carlo builds it) and skips jp < ip as UTwoBodyA does under lmc.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/molsim_gpu.h"

namespace {

constexpr int kNaThreads = 256;                         // list rows per block
constexpr int kNaMaxBlocks = 1024;
constexpr int kNaMaxParticles = kNaThreads * kNaMaxBlocks;
constexpr int kNaPart = 11;                             // 10 type-pair energies + virial
constexpr size_t kNaPartBytes = sizeof(double) * kNaMaxBlocks * kNaPart;
constexpr size_t kNaScratchBytes = kNaPartBytes + 16;   // + counter, error code, the offending ip and jp

static __device__ __align__(256) unsigned char g_na_scratch[kNaScratchBytes];

struct NaArgs {
    int np, npt, natat, maxnneigh, nbuf, lmc;
    double box[3], half[3];
    double rcut2;
    int iubuflow[10];
    double r2umin[10], r2atat[10];
    int pidx[16];       // (ti, tj) -> 0-based type pair
};

__device__ __forceinline__ unsigned *na_counter(unsigned char *s) { return (unsigned *)(s + kNaPartBytes); }
__device__ __forceinline__ int *na_err(unsigned char *s) { return (int *)(s + kNaPartBytes + 4); }

// The first status raised wins; it keeps the 1-based ip and jp of its pair (0 where none).
__device__ __forceinline__ void na_raise(unsigned char *s, int code, int ip1, int jp1)
{
    if (atomicCAS(na_err(s), 0, code) == 0) {
        na_err(s)[1] = ip1;
        na_err(s)[2] = jp1;
    }
}

__global__ void k_na_clear(double *__restrict__ force, int n3, unsigned char *scratch)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n3) force[k] = 0.0;
    if (k == 0) {
        *na_counter(scratch) = 0u;
        na_err(scratch)[0] = 0;
        na_err(scratch)[1] = 0;
        na_err(scratch)[2] = 0;
    }
}

// One thread per list row ip (MOLSIM's serial layout: iploc == ip); the
// reference's linear interval walk from iubuflow; forces of both partners
// added with FP64 atomics; energies and virial reduced per block into the
// scratch partials and summed in block order by the last block to finish.
__global__ void __launch_bounds__(kNaThreads) k_na_pair(NaArgs A, const double *__restrict__ ro,
                                                        const int *__restrict__ iptpn,
                                                        const int *__restrict__ nneighpn,
                                                        const int *__restrict__ jpnlist,
                                                        const double *__restrict__ ubuf, double *__restrict__ force,
                                                        double *__restrict__ utwob, double *__restrict__ virial,
                                                        unsigned char *scratch)
{
    __shared__ double red[kNaThreads / 32][kNaPart];
    __shared__ bool last;
    double *part = (double *)scratch;
    const int ip = blockIdx.x * kNaThreads + threadIdx.x;
    double ut[4] = {0.0, 0.0, 0.0, 0.0};
    double vir = 0.0;
    int ti = 0;
    if (ip < A.np) {
        ti = iptpn[ip] - 1;
        if (ti < 0 || ti >= A.npt) {
            na_raise(scratch, MSG_ERR_ARG, ip + 1, 0);
            ti = 0;
        }
        const double xi = ro[3 * ip], yi = ro[3 * ip + 1], zi = ro[3 * ip + 2];
        double fx = 0.0, fy = 0.0, fz = 0.0;
        int n = nneighpn[ip];
        if (n < 0 || n > A.maxnneigh) {
            // a row longer than jpnlist holds: SetVListMD would have stopped (Src/nlist.F90:752)
            na_raise(scratch, MSG_ERR_ARG, ip + 1, 0);
            n = 0;
        }
        const int *row = jpnlist + (size_t)ip * A.maxnneigh;
        for (int k = 0; k < n; ++k) {
            const int jp = row[k] - 1;
            if (jp < 0 || jp >= A.np) {
                na_raise(scratch, MSG_ERR_ARG, ip + 1, jp + 1);
                continue;
            }
            if (A.lmc && jp < ip) continue;     // full list: each pair once (Src/energy.F90:466-468)
            double dx = xi - ro[3 * jp], dy = yi - ro[3 * jp + 1], dz = zi - ro[3 * jp + 2];
            if (fabs(dx) > A.half[0]) dx = __dsub_rn(dx, copysign(A.box[0], dx));
            if (fabs(dy) > A.half[1]) dy = __dsub_rn(dy, copysign(A.box[1], dy));
            if (fabs(dz) > A.half[2]) dz = __dsub_rn(dz, copysign(A.box[2], dz));
            const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
            if (r2 > A.rcut2) continue;
            const int tj = iptpn[jp] - 1;
            if (tj < 0 || tj >= A.npt) {
                na_raise(scratch, MSG_ERR_ARG, ip + 1, jp + 1);
                continue;
            }
            const int p = A.pidx[ti * 4 + tj];
            double usum, fsum = 0.0;
            if (r2 < A.r2atat[p]) {
                usum = 1e10;
            } else if (r2 < A.r2umin[p]) {
                na_raise(scratch, MSG_ERR_TABLE_MIN, ip + 1, jp + 1);     // StopUTwoBodyA
                continue;
            } else {
                int ib = A.iubuflow[p];
                bool bad = false;
                while (r2 < ubuf[ib - 1]) {
                    ib += 12;
                    if (ib + 11 > A.nbuf) { bad = true; break; }
                }
                if (bad) {
                    na_raise(scratch, MSG_ERR_TABLE_RANGE, ip + 1, jp + 1);   // StopIbuf
                    continue;
                }
                const double *c = ubuf + ib - 1;
                const double d = r2 - c[0];
                usum = c[1] + d * (c[2] + d * (c[3] + d * (c[4] + d * (c[5] + d * c[6]))));
                fsum = c[7] + d * (c[8] + d * (c[9] + d * (c[10] + d * c[11])));
            }
#pragma unroll
            for (int t = 0; t < 4; ++t) ut[t] += (tj == t) ? usum : 0.0;
            fx += fsum * dx;
            fy += fsum * dy;
            fz += fsum * dz;
            atomicAdd(force + 3 * jp, -(fsum * dx));
            atomicAdd(force + 3 * jp + 1, -(fsum * dy));
            atomicAdd(force + 3 * jp + 2, -(fsum * dz));
            vir -= fsum * r2;
        }
        atomicAdd(force + 3 * ip, fx);
        atomicAdd(force + 3 * ip + 1, fy);
        atomicAdd(force + 3 * ip + 2, fz);
    }
    // per-block partials, fixed order
    double e[kNaPart];
#pragma unroll
    for (int q = 0; q < kNaPart; ++q) e[q] = 0.0;
    if (ip < A.np)
        for (int t = 0; t < A.npt; ++t) e[A.pidx[ti * 4 + t]] += ut[t];
    e[kNaPart - 1] = vir;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kNaPart; ++q) {
        double v = e[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[w][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < kNaPart) {
        double v = 0.0;
        for (int k = 0; k < kNaThreads / 32; ++k) v += red[k][threadIdx.x];
        part[(size_t)blockIdx.x * kNaPart + threadIdx.x] = v;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(na_counter(scratch), 1u) == gridDim.x - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x < kNaPart) {
        double v = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) v += __ldcg(part + (size_t)b * kNaPart + threadIdx.x);
        red[0][threadIdx.x] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double u0 = 0.0;
        for (int p = 0; p < A.natat; ++p) {
            utwob[1 + p] = red[0][p];
            u0 += red[0][p];
        }
        utwob[0] = u0;
        *virial = red[0][kNaPart - 1];
        *na_counter(scratch) = 0u;
    }
}

std::mutex g_na_mutex;
unsigned char *g_na_ptr[64] = {};

// Device address of the scratch array on the current device, looked up once.
cudaError_t na_scratch(unsigned char **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_na_scratch);
        if (e != cudaSuccess) return e;
        g_na_ptr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_na_ptr[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" int msg_utwobody_noalloc(int32_t np, int32_t npt, const double boxlen[3], double rcut,
                                    const double *ro, const int32_t *iptpn, const int32_t *nneighpn,
                                    const int32_t *jpnlist, int32_t maxnneigh, int32_t lmc, const double *ubuf,
                                    int32_t nbuf, const int32_t *iubuflow, const double *r2umin,
                                    const double *r2atat, double *force, double *utwob, double *virial,
                                    int32_t *stop_ipjp, void *stream)
{
    if (stop_ipjp) stop_ipjp[0] = stop_ipjp[1] = 0;
    if (np < 1 || np > kNaMaxParticles || npt < 1 || npt > 4 || maxnneigh < 1 || nbuf < 12 || !boxlen || !ro ||
        !iptpn || !nneighpn || !jpnlist || !ubuf || !iubuflow || !r2umin || !force || !utwob || !virial ||
        (lmc != 0 && lmc != 1))
        return MSG_ERR_ARG;
    NaArgs A = {};
    A.np = np;
    A.npt = npt;
    A.natat = npt * (npt + 1) / 2;
    A.maxnneigh = maxnneigh;
    A.nbuf = nbuf;
    A.lmc = lmc;
    for (int d = 0; d < 3; ++d) {
        A.box[d] = boxlen[d];
        A.half[d] = boxlen[d] / 2.0;
    }
    A.rcut2 = rcut * rcut;
    for (int p = 0; p < A.natat; ++p) {
        if (iubuflow[p] < 1 || iubuflow[p] + 11 > nbuf) return MSG_ERR_ARG;
        A.iubuflow[p] = iubuflow[p];
        A.r2umin[p] = r2umin[p];
        A.r2atat[p] = r2atat ? r2atat[p] : 0.0;
    }
    for (int i = 0, p = 0; i < npt; ++i)
        for (int j = i; j < npt; ++j, ++p) {
            A.pidx[i * 4 + j] = p;
            A.pidx[j * 4 + i] = p;
        }
    unsigned char *scratch = nullptr;
    if (na_scratch(&scratch) != cudaSuccess) return MSG_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int n3 = 3 * np;
    k_na_clear<<<(n3 + 255) / 256, 256, 0, st>>>(force, n3, scratch);
    const int blocks = (np + kNaThreads - 1) / kNaThreads;
    k_na_pair<<<blocks, kNaThreads, 0, st>>>(A, ro, iptpn, nneighpn, jpnlist, ubuf, force, utwob, virial, scratch);
    if (cudaGetLastError() != cudaSuccess) return MSG_ERR_CUDA;
    int err[3] = {0, 0, 0};
    if (cudaMemcpyAsync(err, scratch + kNaPartBytes + 4, sizeof(err), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return MSG_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return MSG_ERR_CUDA;
    if (stop_ipjp && err[0]) {
        stop_ipjp[0] = err[1];
        stop_ipjp[1] = err[2];
    }
    return err[0];
}

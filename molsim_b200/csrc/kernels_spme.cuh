// kernels_spme.cuh -- the SPME reciprocal-space convolution (SPMFFTRec,
// Src/energy.F90:6530-6590) as one persistent kernel: forward 3D real-to-complex
// transform of the charge grid, the influence multiply with the reciprocal
// energy and virial, and the backward complex-to-real transform, for every
// system of a handle in one launch.
//
// Work is a list of tasks in stage order:
//   FWD   (system, z):  read plane z of the 64-bit fixed-point charge grid (and
//                       clear it), real-to-complex transform along x, then
//                       complex along y; write the plane of the half spectrum.
//   ZSLAB (system, ky): the ky slab of the half spectrum: forward transform along
//                       z, F *= meshfac with E += |F|^2 emf and W -= |F|^2 vmf,
//                       backward transform along z.
//   BWD   (system, z):  backward transform along y, then complex-to-real along x;
//                       write plane z of the real grid the gather reads.
// Blocks take tasks from one counter in list order and a task waits only for
// tasks earlier in the list (a ZSLAB for all FWD planes of its system, a BWD for
// all ZSLABs), so some running block always holds the earliest unfinished task
// and the launch cannot deadlock whatever number of blocks is resident.  Every
// wait is bounded: past the limit the kernel raises MSG_ERR_TIMEOUT, sets an
// abort flag that ends every other wait, and returns.  The last block out
// clears the counters for the next launch.
//
// Transforms of length N run in shared memory as Stockham passes of radix 8,
// 5, 4, 3 and 2 (N = 2^a 3^b 5^c, at most four passes).  Two real lines travel
// as one complex line and are separated after the forward pass (and joined
// before the backward pass), so the x transforms cost half a complex
// transform each.  The forward transform and the influence multiply are FP64
// in both precisions (the reciprocal energy and virial are FP64 sums); the
// backward transform after the influence multiply is FP64 along z, then FP32
// along y and x in the mixed path (the grid forces), FP64 in the FP64 path.
// Each task's energy and virial are summed in a fixed order and added as
// 64-bit fixed point, so results repeat bit for bit, alone or batched.
//
// A handle uses this kernel when created with MSG_SPME_CONV=1 (every edge it
// supports; the others stay on cuFFT).  The default is the cuFFT chain: on one
// 64^3 grid a stage holds only 64 tasks, each latency-bound at 8 warps per SM,
// and the launch takes as long as the chain it replaces (42 against 43 us).
#pragma once

#include "kernels_force.cuh"

namespace msg {

constexpr int CONV_THREADS = 256;
constexpr unsigned CONV_SPIN_LIMIT = 1u << 22;
constexpr int CONV_MAX_EDGE = 128;
constexpr int CONV_MAX_SMEM = 200 * 1024;   // the two plane buffers of the largest edge taken

// Dynamic shared memory of a launch whose largest plane holds cap complex entries.
inline size_t conv_smem_bytes(int cap) { return 2 * (size_t)cap * sizeof(double2) + CONV_MAX_EDGE * sizeof(double2); }
// counter block: take-counter, blocks out, abort flag, spare; then two
// completion counters per system (FWD planes, ZSLABs)
enum { CONV_HEAD = 0, CONV_EXITED = 1, CONV_ABORT = 2, CONV_HDR = 4 };
enum { CONV_FWD = 0, CONV_ZSLAB = 1, CONV_BWD = 2 };

template <typename T2> struct CplxOf;
template <> struct CplxOf<double2> { using R = double; };
template <> struct CplxOf<float2> { using R = float; };

template <typename T2>
__device__ __forceinline__ T2 cx(typename CplxOf<T2>::R re, typename CplxOf<T2>::R im)
{
    T2 r;
    r.x = re;
    r.y = im;
    return r;
}
template <typename T2> __device__ __forceinline__ T2 cadd(T2 a, T2 b) { return cx<T2>(a.x + b.x, a.y + b.y); }
template <typename T2> __device__ __forceinline__ T2 csub(T2 a, T2 b) { return cx<T2>(a.x - b.x, a.y - b.y); }
template <typename T2> __device__ __forceinline__ T2 cscale(T2 a, typename CplxOf<T2>::R s) { return cx<T2>(a.x * s, a.y * s); }
template <typename T2> __device__ __forceinline__ T2 cmul(T2 a, T2 b)
{
    return cx<T2>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * (SG i): SG = -1 for the forward transform (exp(-2 pi i jk/N)), +1 backward
template <int SG, typename T2> __device__ __forceinline__ T2 crot(T2 a)
{
    return SG < 0 ? cx<T2>(a.y, -a.x) : cx<T2>(-a.y, a.x);
}

// In-register DFTs of length R in natural order.  The constants are cos and sin
// of multiples of 2 pi / R.
template <int R, int SG, typename T2>
__device__ __forceinline__ void dft_small(T2 (&v)[R])
{
    using F = typename CplxOf<T2>::R;
    if constexpr (R == 2) {
        const T2 a = v[0];
        v[0] = cadd(a, v[1]);
        v[1] = csub(a, v[1]);
    } else if constexpr (R == 3) {
        const F s3 = F(0.86602540378443864676);
        const T2 t = cadd(v[1], v[2]), d = csub(v[1], v[2]);
        const T2 m = csub(v[0], cscale(t, F(0.5)));
        const T2 b = cscale(crot<SG>(d), s3);
        v[0] = cadd(v[0], t);
        v[1] = cadd(m, b);
        v[2] = csub(m, b);
    } else if constexpr (R == 4) {
        const T2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
        const T2 t2 = cadd(v[1], v[3]), t3 = crot<SG>(csub(v[1], v[3]));
        v[0] = cadd(t0, t2);
        v[1] = cadd(t1, t3);
        v[2] = csub(t0, t2);
        v[3] = csub(t1, t3);
    } else if constexpr (R == 5) {
        const F c1 = F(0.30901699437494742410), c2 = F(-0.80901699437494742410);
        const F s1 = F(0.95105651629515357212), s2 = F(0.58778525229247312917);
        const T2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        const T2 d1 = csub(v[1], v[4]), d2 = csub(v[2], v[3]);
        const T2 a1 = cx<T2>(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
        const T2 a2 = cx<T2>(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
        const T2 b1 = crot<SG>(cx<T2>(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y));
        const T2 b2 = crot<SG>(cx<T2>(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y));
        v[0] = cadd(v[0], cadd(t1, t2));
        v[1] = cadd(a1, b1);
        v[4] = csub(a1, b1);
        v[2] = cadd(a2, b2);
        v[3] = csub(a2, b2);
    } else if constexpr (R == 8) {
        const F h2 = F(0.70710678118654752440);
        T2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
        dft_small<4, SG>(e);
        dft_small<4, SG>(o);
        // o[k] *= exp(SG 2 pi i k / 8)
        o[1] = cscale(cadd(o[1], crot<SG>(o[1])), h2);
        o[2] = crot<SG>(o[2]);
        o[3] = cscale(csub(crot<SG>(o[3]), o[3]), h2);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            v[k] = cadd(e[k], o[k]);
            v[k + 4] = csub(e[k], o[k]);
        }
    }
}

// One Stockham pass of radix R over nl lines of length N held in x; element p
// of line l sits at x[l*ls + p*ps].  Ns is the product of the radices of the
// earlier passes.  tw[m] = exp(-2 pi i m / N).  Output in natural order after
// the last pass.
template <int R, int SG, typename T2>
__device__ __forceinline__ void conv_pass(const T2 *__restrict__ x, T2 *__restrict__ y, int N, int Ns, int nl, int ls,
                                          int ps, const T2 *tw)
{
    const int T = N / R, st = N / (Ns * R), tot = nl * T;
    const bool lfast = ls == 1;   // lines interleaved: consecutive threads take consecutive lines
    for (int w = threadIdx.x; w < tot; w += CONV_THREADS) {
        int l, j;
        if (lfast) {
            j = w / nl;
            l = w - j * nl;
        } else {
            l = w / T;
            j = w - l * T;
        }
        const T2 *xl = x + l * ls;
        T2 *yl = y + l * ls;
        T2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = xl[(j + r * T) * ps];
        const int k = j % Ns;
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                T2 w8 = tw[r * k * st];   // r*k*st < R*Ns*st = N
                if (SG > 0) w8.y = -w8.y;
                v[r] = cmul(v[r], w8);
            }
        }
        dft_small<R, SG>(v);
        const int base = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) yl[(base + r * Ns) * ps] = v[r];
    }
}

// All passes of a length-N transform over nl lines, ping-ponging between a and
// b; returns the buffer holding the result.  rad packs the pass count in its
// low 4 bits and the radices in the 4-bit fields above.
template <int SG, typename T2>
__device__ T2 *conv_lines(T2 *a, T2 *b, int N, int rad, int nl, int ls, int ps, const T2 *tw)
{
    const int np = rad & 15;
    int Ns = 1;
    for (int p = 0; p < np; ++p) {
        const int R = (rad >> (4 + 4 * p)) & 15;
        switch (R) {
        case 8: conv_pass<8, SG>(a, b, N, Ns, nl, ls, ps, tw); break;
        case 5: conv_pass<5, SG>(a, b, N, Ns, nl, ls, ps, tw); break;
        case 4: conv_pass<4, SG>(a, b, N, Ns, nl, ls, ps, tw); break;
        case 3: conv_pass<3, SG>(a, b, N, Ns, nl, ls, ps, tw); break;
        default: conv_pass<2, SG>(a, b, N, Ns, nl, ls, ps, tw); break;
        }
        __syncthreads();
        T2 *t = a;
        a = b;
        b = t;
        Ns *= R;
    }
    return a;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// 16-byte asynchronous copy global -> shared, cached in L2 only (data written by
// other blocks of the launch is read from L2, never from a stale L1 line).  Both
// addresses are 16-byte aligned: every plane, row and table the kernel copies
// starts at an even offset of 8-byte elements or at a 16-byte element.
__device__ __forceinline__ void cp16(void *dst_smem, const void *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// The edge's twiddle table (N entries of T2) into shared memory.
template <typename T2>
__device__ __forceinline__ void cp_twiddles(T2 *dst, const T2 *__restrict__ src, int N)
{
    const int nc = N * (int)sizeof(T2) / 16;
    for (int c = threadIdx.x; c < nc; c += CONV_THREADS)
        cp16(reinterpret_cast<char *>(dst) + 16 * c, reinterpret_cast<const char *>(src) + 16 * c);
}

// Bounded wait of one thread for a completion counter.  Returns 0 when the
// launch is aborting (this wait gave up, or another one did).
__device__ int conv_wait(const unsigned *c, unsigned target, unsigned *abortf, ErrWord *err, int sys)
{
    for (unsigned it = 0; it < CONV_SPIN_LIMIT; ++it) {
        if (ld_acquire_u32(c) >= target) return 1;
        if (ld_acquire_u32(abortf)) return 0;
        __nanosleep(64);
    }
    atomicExch(abortf, 1u);
    raise_error(err, 5, sys, -1, -1);   // MSG_ERR_TIMEOUT
    return 0;
}

// FWD: plane z of the fixed-point charge grid -> plane z of the half spectrum
// (x and y transformed), the fixed-point plane cleared for the next step.
__device__ void conv_fwd_plane(const SysDev &S, int z, unsigned long long *__restrict__ igrid, double2 *cg,
                               const double2 *__restrict__ tw, double2 *A, double2 *B, double2 *W)
{
    const int N = S.s, h = N / 2 + 1, half = N / 2;
    unsigned long long *g = igrid + S.grid_off + (size_t)z * N * N;
    // the raw plane (N*N 64-bit integers) into B, the twiddles into W
    for (int c = threadIdx.x; c < half * N; c += CONV_THREADS)
        cp16(reinterpret_cast<char *>(B) + 16 * c, reinterpret_cast<const char *>(g) + 16 * c);
    cp_twiddles(W, tw, N);
    cp_wait_all();
    __syncthreads();
    // rows 2*y2 and 2*y2+1 as the real and imaginary parts of packed line y2
    const long long *Bi = reinterpret_cast<const long long *>(B);
    for (int e = threadIdx.x; e < half * N; e += CONV_THREADS) {
        const int y2 = e / N, x = e - y2 * N;
        A[e] = make_double2((double)Bi[(2 * y2) * N + x] * kGridFixInv, (double)Bi[(2 * y2 + 1) * N + x] * kGridFixInv);
    }
    ulonglong2 *gz = reinterpret_cast<ulonglong2 *>(g);
    for (int c = threadIdx.x; c < half * N; c += CONV_THREADS) gz[c] = make_ulonglong2(0ull, 0ull);
    __syncthreads();
    double2 *P = conv_lines<-1>(A, B, N, S.fft_rad, half, N, 1, W);
    double2 *Q = P == A ? B : A;
    // separate the two real lines' spectra: X1 = (Z[k] + conj Z[N-k]) / 2, X2 = (Z[k] - conj Z[N-k]) / 2i
    for (int e = threadIdx.x; e < half * h; e += CONV_THREADS) {
        const int y2 = e / h, k = e - y2 * h;
        const double2 zk = P[y2 * N + k], zm = P[y2 * N + (k ? N - k : 0)];
        Q[(2 * y2) * h + k] = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
        Q[(2 * y2 + 1) * h + k] = make_double2(0.5 * (zk.y + zm.y), -0.5 * (zk.x - zm.x));
    }
    __syncthreads();
    double2 *Y = conv_lines<-1>(Q, P, N, S.fft_rad, h, 1, h, W);
    double2 *out = cg + S.cgrid_off + (size_t)z * N * h;
    for (int e = threadIdx.x; e < N * h; e += CONV_THREADS) __stcg(out + e, Y[e]);
}

// ZSLAB: forward z transform of slab ky, influence multiply, backward z
// transform.  Adds this thread's energy and virial terms to (ea, va).
template <class PR>
__device__ void conv_zslab(const SysDev &S, int ky, double2 *cg, float2 *cg32, const double2 *__restrict__ tw,
                           const double *__restrict__ mfac, const double *__restrict__ emf,
                           const double *__restrict__ vmf, double2 *A, double2 *B, double2 *W, double &ea, double &va)
{
    const int N = S.s, h = N / 2 + 1;
    const double2 *in = cg + S.cgrid_off + (size_t)ky * h;   // (kz, ky, kx) at in[kz*N*h + kx]
    for (int e = threadIdx.x; e < N * h; e += CONV_THREADS) {
        const int kz = e / h, kx = e - kz * h;
        cp16(A + e, in + (size_t)kz * N * h + kx);
    }
    cp_twiddles(W, tw, N);
    cp_wait_all();
    __syncthreads();
    double2 *P = conv_lines<-1>(A, B, N, S.fft_rad, h, 1, h, W);
    double2 *Q = P == A ? B : A;
    const int fy = ky <= N / 2 ? ky : N - ky;
    // four entries per thread at a time, their table loads issued together
    constexpr int UI = 4;
    for (int e0 = threadIdx.x; e0 < N * h; e0 += UI * CONV_THREADS) {
        double m[UI], ef[UI], vf[UI];
#pragma unroll
        for (int u = 0; u < UI; ++u) {
            const int e = e0 + u * CONV_THREADS;
            m[u] = ef[u] = vf[u] = 0.0;
            if (e < N * h) {
                const int kz = e / h, kx = e - kz * h;
                const int fz = kz <= N / 2 ? kz : N - kz;
                const size_t f = S.fac_off + kx + (size_t)h * (fy + (size_t)h * fz);
                m[u] = __ldg(mfac + f);
                ef[u] = __ldg(emf + f);
                vf[u] = __ldg(vmf + f);
            }
        }
#pragma unroll
        for (int u = 0; u < UI; ++u) {
            const int e = e0 + u * CONV_THREADS;
            if (e < N * h) {
                double2 q = P[e];
                const double q2 = q.x * q.x + q.y * q.y;
                ea += q2 * ef[u];
                va -= q2 * vf[u];
                q.x *= m[u];
                q.y *= m[u];
                P[e] = q;
            }
        }
    }
    __syncthreads();
    double2 *Y = conv_lines<1>(P, Q, N, S.fft_rad, h, 1, h, W);
    for (int e = threadIdx.x; e < N * h; e += CONV_THREADS) {
        const int kz = e / h, kx = e - kz * h;
        const size_t at = S.cgrid_off + kx + (size_t)h * (ky + (size_t)N * kz);
        if (PR::mixed)
            __stcg(cg32 + at, make_float2((float)Y[e].x, (float)Y[e].y));
        else
            __stcg(cg + at, Y[e]);
    }
}

// BWD: plane z of the half spectrum (z transformed) -> plane z of the real grid.
template <typename T2, typename RT>
__device__ void conv_bwd_plane(const SysDev &S, int z, const T2 *cgt, RT *__restrict__ rg, const T2 *__restrict__ tw,
                               T2 *A, T2 *B, T2 *W)
{
    const int N = S.s, h = N / 2 + 1, half = N / 2;
    const T2 *in = cgt + S.cgrid_off + (size_t)z * N * h;
    const int nc = N * h * (int)sizeof(T2) / 16;
    for (int c = threadIdx.x; c < nc; c += CONV_THREADS)
        cp16(reinterpret_cast<char *>(A) + 16 * c, reinterpret_cast<const char *>(in) + 16 * c);
    cp_twiddles(W, tw, N);
    cp_wait_all();
    __syncthreads();
    T2 *P = conv_lines<1>(A, B, N, S.fft_rad, h, 1, h, W);
    T2 *Q = P == A ? B : A;
    // join rows 2*y2 and 2*y2+1 (Hermitian extension to N entries, the imaginary
    // parts at k = 0 and N/2 dropped) as X1 + i X2
    for (int e = threadIdx.x; e < half * N; e += CONV_THREADS) {
        const int y2 = e / N, k = e - y2 * N;
        T2 x1, x2;
        if (k < h) {
            x1 = P[(2 * y2) * h + k];
            x2 = P[(2 * y2 + 1) * h + k];
        } else {
            x1 = P[(2 * y2) * h + N - k];
            x2 = P[(2 * y2 + 1) * h + N - k];
            x1.y = -x1.y;
            x2.y = -x2.y;
        }
        if (k == 0 || 2 * k == N) {
            x1.y = 0;
            x2.y = 0;
        }
        Q[e] = cx<T2>(x1.x - x2.y, x1.y + x2.x);
    }
    __syncthreads();
    T2 *Y = conv_lines<1>(Q, P, N, S.fft_rad, half, N, 1, W);
    RT *out = rg + S.grid_off + (size_t)z * N * N;
    for (int e = threadIdx.x; e < half * N; e += CONV_THREADS) {
        const int y2 = e / N, x = e - y2 * N;
        out[(size_t)(2 * y2) * N + x] = Y[e].x;
        out[(size_t)(2 * y2 + 1) * N + x] = Y[e].y;
    }
}

// The persistent convolution kernel (see the top of this file).  Dynamic shared
// memory: two buffers of cap FP64 complex entries, cap = max N*(N/2+1), then the
// twiddle table of the task's edge (at most CONV_MAX_EDGE FP64 complex entries).
template <class PR>
__global__ void __maxnreg__(96) k_spme_conv(
    const SysDev *__restrict__ sysv, const int4 *__restrict__ tasks, int ntasks, int cap,
    unsigned long long *__restrict__ igrid, double2 *cg, float2 *cg32, double *__restrict__ rg,
    float *__restrict__ rg32, const double2 *__restrict__ tw, const float2 *__restrict__ tw32,
    const double *__restrict__ mfac, const double *__restrict__ emf, const double *__restrict__ vmf,
    long long *__restrict__ eacc, unsigned *ctr, int nctr, ErrWord *err)
{
    extern __shared__ __align__(16) unsigned char conv_smem[];
    __shared__ int s_t, s_ok, s_last;
    __shared__ double red[2][CONV_THREADS / 32];
    double2 *A = reinterpret_cast<double2 *>(conv_smem), *B = A + cap, *W = B + cap;
    for (;;) {
        if (threadIdx.x == 0) {
            const int t = (int)atomicAdd(ctr + CONV_HEAD, 1u);
            int ok = 1;
            if (t < ntasks) {
                const int4 T = tasks[t];
                if (T.y != CONV_FWD) {
                    ok = conv_wait(ctr + CONV_HDR + 2 * T.x + (T.y - 1), (unsigned)sysv[T.x].s, ctr + CONV_ABORT, err,
                                   T.x);
                    __threadfence();
                }
            }
            s_t = t;
            s_ok = ok;
        }
        __syncthreads();
        const int t = s_t;
        if (t >= ntasks) break;
        if (s_ok) {
            const int4 T = tasks[t];
            const SysDev &S = sysv[T.x];
            if (T.y == CONV_FWD) {
                conv_fwd_plane(S, T.z, igrid, cg, tw + S.fft_tw, A, B, W);
            } else if (T.y == CONV_ZSLAB) {
                double ea = 0.0, va = 0.0;
                conv_zslab<PR>(S, T.z, cg, cg32, tw + S.fft_tw, mfac, emf, vmf, A, B, W, ea, va);
                ea = warp_sum(ea);
                va = warp_sum(va);
                const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
                if (lane == 0) {
                    red[0][w] = ea;
                    red[1][w] = va;
                }
                __syncthreads();
                if (threadIdx.x < 2) {
                    double sacc = 0.0;
                    for (int k = 0; k < CONV_THREADS / 32; ++k) sacc += red[threadIdx.x][k];
                    acc_add(eacc + (size_t)T.x * EA_N + EA_UREC + threadIdx.x, sacc);
                }
            } else if (PR::mixed) {
                float2 *Af = reinterpret_cast<float2 *>(conv_smem);
                conv_bwd_plane<float2, float>(S, T.z, cg32, rg32, tw32 + S.fft_tw, Af, Af + cap,
                                              reinterpret_cast<float2 *>(W));
            } else {
                conv_bwd_plane<double2, double>(S, T.z, cg, rg, tw + S.fft_tw, A, B, W);
            }
            // the task's stores are visible device-wide before its completion is counted
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0 && T.y != CONV_BWD) {
                __threadfence();
                atomicAdd(ctr + CONV_HDR + 2 * T.x + T.y, 1u);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(ctr + CONV_EXITED, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    // every block has taken its last task, so every task is finished: clear the
    // counters for the next launch
    if (s_last)
        for (int k = threadIdx.x; k < nctr; k += CONV_THREADS) ctr[k] = 0u;
}

}  // namespace msg

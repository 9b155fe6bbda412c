// kernels_md.cuh -- integrator, skin test, list rebuild and API-boundary kernels.
#pragma once

#include "common.cuh"

namespace msg {

// Philox4x32-10 (Salmon et al., SC'11) counter-based generator.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += W0;
        k.y += W1;
    }
    return c;
}

// Three FP32 standard normals for (seed, particle, step) by Box-Muller.
__device__ __forceinline__ float3 gauss3(uint64_t seed, uint32_t particle, uint32_t step)
{
    const uint4 r = philox4x32_10(make_uint4(particle, step, 0x4d4f4c53u, 0u),
                                  make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
    const float inv = 2.3283064365386963e-10f;   // 2^-32
    const float u1 = ((float)r.x + 1.0f) * inv, u2 = (float)r.y * inv;
    const float u3 = ((float)r.z + 1.0f) * inv, u4 = (float)r.w * inv;
    const float m1 = sqrtf(-2.0f * logf(u1)), m2 = sqrtf(-2.0f * logf(u3));
    float s1, c1, s2, c2;
    sincospif(2.0f * u2, &s1, &c1);
    sincospif(2.0f * u4, &s2, &c2);
    return make_float3(m1 * c1, m1 * s1, m2 * c2);
}

// ---------------------------------------------------------------------------
// Skin test of NList (Src/nlist.F90:600-613), reproduced exactly including its
// running "second maximum": r2max2 only collects values that were not a new
// running maximum when visited in MOLSIM order.  Chunks of SK_CHUNK MOLSIM
// indices are summarised in parallel by the position update (block max B,
// non-record max A, the chunk's record values); k_skin_combine then walks a
// system's chunks in order: a chunk record R counts towards r2max2 iff R <= the
// prefix maximum P before the chunk, so the chunk contributes max(A, max{R <= P}).
// ---------------------------------------------------------------------------
// 128 MOLSIM indices per chunk, one per thread: a 16000-particle system spreads
// over 125 blocks.
constexpr int SK_THREADS = 128, SK_PER = 1, SK_CHUNK = SK_THREADS * SK_PER, SK_REC = 32;
struct SkinChunk {
    double bmax, amax;
    int nrec, pad;
    double rec[SK_REC];
};

// Block-wide exclusive prefix max over the block's threads (values >= 0).
__device__ __forceinline__ double block_excl_max(double v, double *sm)
{
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    double inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        double y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc = fmax(inc, y);
    }
    if (lane == 31) sm[w] = inc;
    __syncthreads();
    double pre = 0.0;
    for (int k = 0; k < w; ++k) pre = fmax(pre, sm[k]);
    double exc = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane == 0) exc = 0.0;
    __syncthreads();
    return fmax(pre, exc);
}

__device__ __forceinline__ double block_max(double v, double *sm)
{
    v = warp_max(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sm[w] = v;
    __syncthreads();
    double r = 0.0;
    for (int k = 0; k < SK_THREADS / 32; ++k) r = fmax(r, sm[k]);
    __syncthreads();
    return r;
}

__device__ __forceinline__ int block_excl_sum_int(int v, int *sm, int *total)
{
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    int inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) sm[w] = inc;
    __syncthreads();
    int pre = 0, tot = 0;
    for (int k = 0; k < SK_THREADS / 32; ++k) {
        if (k < w) pre += sm[k];
        tot += sm[k];
    }
    __syncthreads();
    *total = tot;
    return pre + inc - v;
}

// Contribution of one chunk to r2max2 given the prefix max P before it; all
// threads of the block call this with the same arguments.
__device__ double chunk_nonrecord_max(const double *r2, int o0, int o1, double P, double *smd)
{
    const int t = threadIdx.x;
    double v[SK_PER], run = 0.0, tmax = 0.0;
#pragma unroll
    for (int k = 0; k < SK_PER; ++k) {
        int o = o0 + SK_PER * t + k;
        v[k] = (o < o1) ? r2[o] : 0.0;
        tmax = fmax(tmax, v[k]);
    }
    double pre = fmax(P, block_excl_max(tmax, smd));
    double best = 0.0;
    run = pre;
#pragma unroll
    for (int k = 0; k < SK_PER; ++k) {
        int o = o0 + SK_PER * t + k;
        if (o < o1) {
            if (v[k] > run) run = v[k];
            else best = fmax(best, v[k]);
        }
    }
    return block_max(best, smd);
}

// Chunk summary of SK_PER consecutive MOLSIM-order skin values per thread.
__device__ void skin_chunk(int chunk, const double v[SK_PER], int o0, int o1, SkinChunk *__restrict__ sc)
{
    __shared__ double smd[SK_THREADS / 32];
    __shared__ int smi[SK_THREADS / 32];
    const int t = threadIdx.x;
    double tmax = 0.0;
#pragma unroll
    for (int k = 0; k < SK_PER; ++k) tmax = fmax(tmax, v[k]);
    double run = block_excl_max(tmax, smd);
    double amax = 0.0;
    int nrec = 0;
    double recv[SK_PER];
#pragma unroll
    for (int k = 0; k < SK_PER; ++k) {
        const int o = o0 + SK_PER * t + k;
        if (o < o1) {
            if (v[k] > run) { run = v[k]; recv[nrec++] = v[k]; }
            else amax = fmax(amax, v[k]);
        }
    }
    int total;
    const int roff = block_excl_sum_int(nrec, smi, &total);
    SkinChunk &out = sc[chunk];
    for (int k = 0; k < nrec; ++k)
        if (roff + k < SK_REC) out.rec[roff + k] = recv[k];
    const double bm = block_max(tmax, smd);
    const double am = block_max(amax, smd);
    if (t == 0) {
        out.bmax = bm;
        out.amax = am;
        out.nrec = total;
    }
}

// The combination of a system's chunk summaries in MOLSIM order and the rebuild
// decision (NList, Src/nlist.F90:600-613): one block per system, launched after
// the position update.  Only the rebuild at the end of the step needs it, so in
// the step graph it runs beside the force computation.
__global__ void __launch_bounds__(SK_THREADS) k_skin_combine(
    const SysDev *__restrict__ sysv, const double *__restrict__ r2o, const SkinChunk *__restrict__ sc,
    int *__restrict__ flag, long long *__restrict__ nrebuild, double *__restrict__ skinout,
    cudaGraphConditionalHandle cond, int use_cond, unsigned *__restrict__ istep2)
{
    __shared__ double smd[SK_THREADS / 32];
    const int s = blockIdx.x, t = threadIdx.x;
    const SysDev &S = sysv[s];
    if (S.inlist > 0) {
        // regular update interval: rebuild when mod(istep2, inlist) == 0 (Src/nlist.F90:616-617)
        if (t == 0) {
            const unsigned c = istep2[s] + 1u;
            istep2[s] = c;
            const int rebuild = (c % (unsigned)S.inlist) == 0u ? 1 : 0;
            flag[s] = rebuild;
            if (rebuild) {
                nrebuild[s] += 1;
                if (use_cond) cudaGraphSetConditional(cond, 1u);
            }
            if (skinout) { skinout[2 * s] = 0.0; skinout[2 * s + 1] = 0.0; }
        }
        return;
    }
    // Combine the system's chunks in MOLSIM order, SK_THREADS chunks per pass.
    const int c0 = S.chunk_off;
    double carry = 0.0, m2 = 0.0;
    __shared__ int novf;
    for (int cb = 0; cb < S.nchunk; cb += SK_THREADS) {
        const int c = cb + t;
        double bmx = 0.0;
        if (c < S.nchunk) bmx = __ldcg(&sc[c0 + c].bmax);
        const double P = fmax(carry, block_excl_max(bmx, smd));
        double contrib = 0.0;
        bool ovf = false;
        if (c < S.nchunk) {
            const int nr = __ldcg(&sc[c0 + c].nrec);
            if (nr > SK_REC) {
                ovf = true;
            } else {
                contrib = __ldcg(&sc[c0 + c].amax);
                for (int k = 0; k < nr; ++k) {
                    const double R = __ldcg(&sc[c0 + c].rec[k]);
                    if (R <= P) contrib = fmax(contrib, R);
                }
            }
        }
        m2 = fmax(m2, block_max(contrib, smd));
        // chunks with more records than stored are re-scanned by the whole block
        if (t == 0) novf = 0;
        __syncthreads();
        if (ovf) atomicAdd(&novf, 1);
        __syncthreads();
        if (novf) {
            for (int k = 0; k < SK_THREADS && cb + k < S.nchunk; ++k) {
                __shared__ int isovf;
                __shared__ double Pk;
                if (t == k) { isovf = ovf ? 1 : 0; Pk = P; }
                __syncthreads();
                if (isovf) {
                    const int q0 = S.off + (cb + k) * SK_CHUNK, q1 = min(S.off + S.n, q0 + SK_CHUNK);
                    m2 = fmax(m2, chunk_nonrecord_max(r2o, q0, q1, Pk, smd));
                }
                __syncthreads();
            }
        }
        carry = fmax(carry, block_max(bmx, smd));
    }
    if (t == 0) {
        istep2[s] += 1u;
        const int rebuild = (sqrt(carry) + sqrt(m2) > S.drnlist) ? 1 : 0;
        flag[s] = rebuild;
        if (rebuild) {
            nrebuild[s] += 1;
            // inside a CUDA graph: open the conditional rebuild node of this step
            if (use_cond) cudaGraphSetConditional(cond, 1u);
        }
        if (skinout) { skinout[2 * s] = carry; skinout[2 * s + 1] = m2; }
    }
}

// ---------------------------------------------------------------------------
// Velocity Verlet, position half (Src/md.F90:286-298) fused with NList's skin
// test: drostep = dt*rod + (dt*dt/2)*rodd; ro += drostep; PBC(ro);
// drosum += drostep (Src/nlist.F90:603-604).  Each block is one skin chunk of
// SK_CHUNK consecutive MOLSIM indices, so the skin values arrive in MOLSIM order;
// particles are reached through inv[].  Products and sums round separately
// (no FMA) so positions follow MOLSIM's arithmetic.  Also refreshes the FP32
// position mirror used by the mixed-precision kernels.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(SK_THREADS) k_vv_skin(
    const SysDev *__restrict__ sysv, const int4 *__restrict__ chunks, const int *__restrict__ inv,
    double4 *__restrict__ pos, const double4 *__restrict__ vel, const double4 *__restrict__ acc,
    double4 *__restrict__ dsum, int4 *__restrict__ posfx, double *__restrict__ r2o, SkinChunk *__restrict__ sc)
{
    const int4 C = chunks[blockIdx.x];
    const SysDev &S = sysv[C.x];
    const double dt = S.dt, fac = __dmul_rn(0.5, __dmul_rn(dt, dt));
    double v[SK_PER];
#pragma unroll
    for (int k = 0; k < SK_PER; ++k) {
        const int o = C.y + SK_PER * threadIdx.x + k;
        v[k] = 0.0;
        if (o < C.z) {
            const int i = inv[o];
            double4 x = pos[i];
            const double4 u = vel[i], a = acc[i];
            double4 d = dsum[i];
            const double sx = __dadd_rn(__dmul_rn(dt, u.x), __dmul_rn(fac, a.x));
            const double sy = __dadd_rn(__dmul_rn(dt, u.y), __dmul_rn(fac, a.y));
            const double sz = __dadd_rn(__dmul_rn(dt, u.z), __dmul_rn(fac, a.z));
            x.x = pbc_wrap(__dadd_rn(x.x, sx), S.half[0], S.box[0], S.boxi[0]);
            x.y = pbc_wrap(__dadd_rn(x.y, sy), S.half[1], S.box[1], S.boxi[1]);
            x.z = pbc_wrap(__dadd_rn(x.z, sz), S.half[2], S.box[2], S.boxi[2]);
            pos[i] = x;
            if (posfx) posfx[i] = fx_pos(x, S);
            if (S.inlist <= 0) {
                // drosum += drostep only under the skin test (Src/nlist.F90:603-604)
                d.x = __dadd_rn(d.x, sx);
                d.y = __dadd_rn(d.y, sy);
                d.z = __dadd_rn(d.z, sz);
                dsum[i] = d;
            }
            v[k] = __dadd_rn(__dadd_rn(__dmul_rn(d.x, d.x), __dmul_rn(d.y, d.y)), __dmul_rn(d.z, d.z));
            r2o[o] = v[k];
        }
    }
    skin_chunk(blockIdx.x, v, C.y, C.z, sc);
}

// Ermak-McCammon step (Src/bd.F90:142-152) fused with the skin test:
// drostep = fac1*forceo + fac2*xi, ro += drostep, PBC.  xi is caller noise in
// MOLSIM order (xin) or FP32 Philox noise keyed by (seed, particle, step).
__global__ void __launch_bounds__(SK_THREADS) k_bd_skin(
    const SysDev *__restrict__ sysv, const int4 *__restrict__ chunks, const int *__restrict__ inv,
    double4 *__restrict__ pos, const double4 *__restrict__ forceo, double4 *__restrict__ dsum,
    const int *__restrict__ typ, const double *__restrict__ fac1, const double *__restrict__ fac2,
    const double *__restrict__ xin, double *__restrict__ xout, uint64_t seed,
    const unsigned long long *__restrict__ sstep, int4 *__restrict__ posfx, double *__restrict__ r2o,
    SkinChunk *__restrict__ sc)
{
    const int4 C = chunks[blockIdx.x];
    const SysDev &S = sysv[C.x];
    double v[SK_PER];
#pragma unroll
    for (int k = 0; k < SK_PER; ++k) {
        const int o = C.y + SK_PER * threadIdx.x + k;
        v[k] = 0.0;
        if (o < C.z) {
            const int i = inv[o];
            const int t = S.type_off + typ[i];
            double xi0, xi1, xi2;
            if (xin) {
                xi0 = xin[3 * (size_t)o];
                xi1 = xin[3 * (size_t)o + 1];
                xi2 = xin[3 * (size_t)o + 2];
            } else {
                const float3 z = gauss3(seed ^ S.seed, (uint32_t)(o - S.off), (uint32_t)sstep[C.x]);
                xi0 = z.x;
                xi1 = z.y;
                xi2 = z.z;
            }
            if (xout) {
                xout[3 * (size_t)o] = xi0;
                xout[3 * (size_t)o + 1] = xi1;
                xout[3 * (size_t)o + 2] = xi2;
            }
            const double f1 = fac1[t], f2 = fac2[t];
            const double4 f = forceo[i];
            double4 x = pos[i], d = dsum[i];
            const double sx = __dadd_rn(__dmul_rn(f1, f.x), __dmul_rn(f2, xi0));
            const double sy = __dadd_rn(__dmul_rn(f1, f.y), __dmul_rn(f2, xi1));
            const double sz = __dadd_rn(__dmul_rn(f1, f.z), __dmul_rn(f2, xi2));
            x.x = pbc_wrap(__dadd_rn(x.x, sx), S.half[0], S.box[0], S.boxi[0]);
            x.y = pbc_wrap(__dadd_rn(x.y, sy), S.half[1], S.box[1], S.boxi[1]);
            x.z = pbc_wrap(__dadd_rn(x.z, sz), S.half[2], S.box[2], S.boxi[2]);
            pos[i] = x;
            if (posfx) posfx[i] = fx_pos(x, S);
            if (S.inlist <= 0) {
                // drosum += drostep only under the skin test (Src/nlist.F90:603-604)
                d.x = __dadd_rn(d.x, sx);
                d.y = __dadd_rn(d.y, sy);
                d.z = __dadd_rn(d.z, sz);
                dsum[i] = d;
            }
            v[k] = __dadd_rn(__dadd_rn(__dmul_rn(d.x, d.x), __dmul_rn(d.y, d.y)), __dmul_rn(d.z, d.z));
            r2o[o] = v[k];
        }
    }
    skin_chunk(blockIdx.x, v, C.y, C.z, sc);
}

// ---------------------------------------------------------------------------
// Verlet-cell rebuild.  Keys are global cell ids; rebuilt systems enter the
// stable sort in MOLSIM order, other systems in their current order with their
// current cell ids, so the sort leaves them in place.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int cell_coord(double x, double half, double boxi, int nc)
{
    int c = (int)floor((x + half) * boxi * (double)nc);
    return c < 0 ? 0 : (c >= nc ? nc - 1 : c);
}

// Also empties every cell range (k_permute refills those of rebuilt systems).
__global__ void __launch_bounds__(128) k_rb_keys(const SysDev *__restrict__ sysv, const Tile *__restrict__ tiles,
                                                const int *__restrict__ flag, const double4 *__restrict__ pos,
                                                const int *__restrict__ orig, const int *__restrict__ cellid,
                                                uint32_t *__restrict__ key, uint32_t *__restrict__ val,
                                                int *__restrict__ cstart, int *__restrict__ cend, int ncell)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
        cstart[c] = 0;
        cend[c] = 0;
    }
    const Tile T = tiles[blockIdx.x];
    const SysDev &S = sysv[T.sys];
    const int i = T.i0 + threadIdx.x;
    if (i >= T.i1) return;
    if (flag[T.sys]) {
        const double4 x = pos[i];
        const int cx = cell_coord(x.x, S.half[0], S.boxi[0], S.ncell[0]);
        const int cy = cell_coord(x.y, S.half[1], S.boxi[1], S.ncell[1]);
        const int cz = cell_coord(x.z, S.half[2], S.boxi[2], S.ncell[2]);
        const int q = S.off + orig[i];
        key[q] = (uint32_t)(S.cell_off + (cz * S.ncell[1] + cy) * S.ncell[0] + cx);
        val[q] = (uint32_t)i;
    } else {
        key[i] = (uint32_t)cellid[i];
        val[i] = (uint32_t)i;
    }
}

// Gather the per-particle arrays of rebuilt systems into the sorted order
// (into scratch buffers; k_copyback moves them home) and mark where each of
// their cells starts and ends in it.  Systems that are not rebuilt keep their
// order, so their particles are not touched.
__global__ void __launch_bounds__(128) k_permute(const SysDev *__restrict__ sysv, const Tile *__restrict__ tiles,
                                                const int *__restrict__ flag, const uint32_t *__restrict__ skey,
                                                const uint32_t *__restrict__ sval,
                                                const double4 *__restrict__ pos0, double4 *__restrict__ pos1,
                                                const double4 *__restrict__ vel0, double4 *__restrict__ vel1,
                                                const double4 *__restrict__ acc0, double4 *__restrict__ acc1,
                                                const double4 *__restrict__ fo0, double4 *__restrict__ fo1,
                                                const int *__restrict__ typ0, int *__restrict__ typ1,
                                                const int *__restrict__ orig0, int *__restrict__ orig1,
                                                int *__restrict__ cellid, int *__restrict__ inv,
                                                int *__restrict__ cstart, int *__restrict__ cend, int n)
{
    const Tile T = tiles[blockIdx.x];
    if (!flag[T.sys]) return;
    const SysDev &S = sysv[T.sys];
    const int j = T.i0 + threadIdx.x;
    if (j >= T.i1) return;
    const int c = (int)skey[j];
    if (j == 0 || (int)skey[j - 1] != c) cstart[c] = j;
    if (j == n - 1 || (int)skey[j + 1] != c) cend[c] = j + 1;
    const int i = (int)sval[j];
    pos1[j] = pos0[i];
    vel1[j] = vel0[i];
    acc1[j] = acc0[i];
    fo1[j] = fo0[i];
    typ1[j] = typ0[i];
    const int o = orig0[i];
    orig1[j] = o;
    cellid[j] = (int)skey[j];
    inv[S.off + o] = j;
}

// Home the permuted arrays, reset drosum (NList: drosum = Zero at a rebuild)
// and refresh the fixed-point mirror of the moved positions.
__global__ void __launch_bounds__(128) k_copyback(const SysDev *__restrict__ sysv, const Tile *__restrict__ tiles,
                                                 const int *__restrict__ flag,
                                                 double4 *__restrict__ pos0, const double4 *__restrict__ pos1,
                                                 double4 *__restrict__ vel0, const double4 *__restrict__ vel1,
                                                 double4 *__restrict__ acc0, const double4 *__restrict__ acc1,
                                                 double4 *__restrict__ fo0, const double4 *__restrict__ fo1,
                                                 int *__restrict__ typ0, const int *__restrict__ typ1,
                                                 int *__restrict__ orig0, const int *__restrict__ orig1,
                                                 double4 *__restrict__ dsum, int4 *__restrict__ posfx)
{
    const Tile T = tiles[blockIdx.x];
    if (!flag[T.sys]) return;
    const int j = T.i0 + threadIdx.x;
    if (j >= T.i1) return;
    const double4 x = pos1[j];
    pos0[j] = x;
    posfx[j] = fx_pos(x, sysv[T.sys]);
    vel0[j] = vel1[j];
    acc0[j] = acc1[j];
    fo0[j] = fo1[j];
    typ0[j] = typ1[j];
    orig0[j] = orig1[j];
    dsum[j] = make_double4(0.0, 0.0, 0.0, 0.0);
}

// Stencil of neighbour cells along one dimension: the three cells c-1, c, c+1
// (periodic) when there are at least three, otherwise every cell once.
__device__ __forceinline__ int stencil1(int c, int nc, int *out)
{
    if (nc >= 3) {
        out[0] = (c + nc - 1) % nc;
        out[1] = c;
        out[2] = (c + 1) % nc;
        return 3;
    }
    for (int k = 0; k < nc; ++k) out[k] = k;
    return nc;
}

// Pair (i, j) of internal indices belongs to row i of a half list: SetVListMD's
// parity rule (Src/nlist.F90:741-744) applied to the internal order, so each
// unordered pair is stored once and rows are balanced.
__device__ __forceinline__ bool half_owner(int i, int j) { return (i < j) == (((i + j) & 1) != 0); }

// ---------------------------------------------------------------------------
// SetLList / SetNCell (Src/nlist.F90:1168-1260) for systems with lvlistllist.
// Per particle: its linked-list cell (ix, iy, iz) = aint((ro + boxlen2) celli)
// and, per dimension, the cells of SetNCell's probe points ro - rcut, ro,
// ro + rcut after PBC.  The probes' 27 cells are the product of the three
// per-dimension sets, so a particle j lies in a cell SetNCell marks for i iff
// each of j's cell indices is in i's set of that dimension.  Packed 10 bits per
// index (a grid has at most 1000 cells): x = cell, y/z/w = the x/y/z sets.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int llist_index(double r, double half, double celli, int nd)
{
    int c = (int)__dmul_rn(__dadd_rn(r, half), celli);
    return min(max(c, 0), nd - 1);     // r = +boxlen2 exactly lies outside the reference's grid
}

__global__ void __launch_bounds__(128) k_llist_info(const SysDev *__restrict__ sysv, const Tile *__restrict__ tiles,
                                                   const int *__restrict__ flag, const double4 *__restrict__ pos,
                                                   int4 *__restrict__ info)
{
    const Tile T = tiles[blockIdx.x];
    const SysDev &S = sysv[T.sys];
    if (!flag[T.sys] || !S.llist) return;
    const int j = T.i0 + threadIdx.x;
    if (j >= T.i1) return;
    const double4 x = pos[j];
    const double xc[3] = {x.x, x.y, x.z};
    int own = 0, set[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        own |= llist_index(xc[d], S.half[d], S.lcelli[d], S.lnd[d]) << (10 * d);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            // rr + idx*distance, idx = -1, 0, 1; then PBC (Src/nlist.F90:1248-1252)
            const double q = pbc_wrap(__dadd_rn(xc[d], (double)(a - 1) * S.lrcut), S.half[d], S.box[d], S.boxi[d]);
            set[d] |= llist_index(q, S.half[d], S.lcelli[d], S.lnd[d]) << (10 * a);
        }
    }
    info[j] = make_int4(own, set[0], set[1], set[2]);
}

// Is cell `c` (packed as info.x) among the cells SetNCell marks for the particle with info A?
__device__ __forceinline__ bool llist_marked(const int4 &A, int c)
{
    const int cs[3] = {A.y, A.z, A.w};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int v = (c >> (10 * d)) & 1023;
        const int q = cs[d];
        if (v != (q & 1023) && v != ((q >> 10) & 1023) && v != ((q >> 20) & 1023)) return false;
    }
    return true;
}

// SetVListMDLList's row rule (Src/nlist.F90:790-792) on 1-based MOLSIM indices: the
// opposite rows from SetVListMD's.
__device__ __forceinline__ bool llist_owner(int ip, int jp)
{
    const bool odd = ((ip + jp) & 1) != 0;
    return ip != jp && (ip > jp ? odd : !odd);
}

// Verlet list, one warp per particle: every j != i in the stencil with
// r2 < (rcut+drnlist)^2 (SetVListMD's test, Src/nlist.F90:746-751), compacted
// with a warp ballot.  Rows are ordered by stencil cell, then by MOLSIM index.
// half = 0: full list (each pair in both rows); half = 1: each pair once, in the
// row half_owner names (only those candidates are read: every other index on
// either side of i).  With lvlistllist a pair also needs its MOLSIM row owner
// (SetVListMDLList's rule) to reach the partner's cell with SetNCell's probes, so
// the list holds SetVListMDLList's pair set (which can leave out skin pairs).
__global__ void __launch_bounds__(256) k_nlist(const SysDev *__restrict__ sysv, const int *__restrict__ sys,
                                              const int *__restrict__ flag, const double4 *__restrict__ pos,
                                              const int *__restrict__ typ,
                                              const int *__restrict__ cellid, const int *__restrict__ cstart,
                                              const int *__restrict__ cend, int *__restrict__ nbl,
                                              int *__restrict__ nnb, int ntot, int *__restrict__ nmaxrow,
                                              ErrWord *err, int half, const int *__restrict__ orig,
                                              const int4 *__restrict__ llinfo)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= ntot) return;
    const int s = sys[i];
    if (!flag[s]) return;
    const SysDev &S = sysv[s];
    const double4 xi = pos[i];
    const int c = cellid[i] - S.cell_off;
    const int cx = c % S.ncell[0], cy = (c / S.ncell[0]) % S.ncell[1], cz = c / (S.ncell[0] * S.ncell[1]);
    int sx[3], sy[3], sz[3];
    const int nx = stencil1(cx, S.ncell[0], sx), ny = stencil1(cy, S.ncell[1], sy), nz = stencil1(cz, S.ncell[2], sz);
    int *row = nbl + S.nbl_off + (long long)(i - S.off) * S.cap;
    int count = 0;
    const unsigned lt = (1u << lane) - 1u;
    const bool ll = S.llist != 0;
    int4 li = make_int4(0, 0, 0, 0);
    int ip = 0;
    if (ll) {
        li = llinfo[i];
        ip = orig[i] + 1;
    }
    // the pair test of candidates a, a+step, ... below b, 32 at a time, compacted into the row
    auto scan = [&](int a, int b, int step) {
        for (int jb = a; jb < b; jb += 32 * step) {
            const int j = jb + lane * step;
            bool ok = false;
            if (j < b && j != i) {
                const double4 xj = pos[j];
                double dx = __dsub_rn(xi.x, xj.x), dy = __dsub_rn(xi.y, xj.y), dz = __dsub_rn(xi.z, xj.z);
                ok = pbcr2_exact(dx, dy, dz, S) < S.rs2cut;
                if (ok && ll) {
                    const int4 lj = llinfo[j];
                    ok = llist_owner(ip, orig[j] + 1) ? llist_marked(li, lj.x) : llist_marked(lj, li.x);
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, ok);
            if (ok) {
                const int slot = count + __popc(bal & lt);
                // entry: partner index, partner type in bits 28-29
                if (slot < S.cap) row[slot] = j | (typ[j] << 28);
            }
            count += __popc(bal);
        }
    };
    for (int a = 0; a < nz; ++a)
        for (int b = 0; b < ny; ++b)
            for (int e = 0; e < nx; ++e) {
                const int cc = S.cell_off + (sz[a] * S.ncell[1] + sy[b]) * S.ncell[0] + sx[e];
                const int j0 = cstart[cc], j1 = cend[cc];
                if (half) {
                    // the partners half_owner gives row i: below i those of i's parity,
                    // above i those of the other parity (every other index, in order)
                    scan(j0 + ((j0 ^ i) & 1), min(j1, i), 2);
                    int jb = max(j0, i + 1);
                    jb += ((jb + i) & 1) ^ 1;
                    scan(jb, j1, 2);
                } else {
                    scan(j0, j1, 1);
                }
            }
    if (lane == 0) {
        nnb[i] = min(count, S.cap);
        atomicMax(nmaxrow + s, count);
        if (count > S.cap) raise_error(err, 3, s, i, count);
    }
}

// MOLSIM-layout export of one system's list, pass 1: every unordered pair once
// (every entry of a half list; the i < j entries of a full list) goes to the row
// that MOLSIM's rule gives it -- SetVListMD's parity rule (Src/nlist.F90:741-744),
// or SetVListMDLList's (:790-792) with lvlistllist -- at a slot taken from that
// row's counter (nneigh_out, zeroed by the caller).  The slot holds a sort key:
// the partner's 1-based index, preceded (high word) by its linked-list cell
// number with lvlistllist, whose rows run cell by cell.  One warp per row.
__device__ __forceinline__ long long export_key(const SysDev &S, int jp, const int4 *llinfo, int j)
{
    if (!S.llist) return (long long)jp;
    const int c = llinfo[j].x;
    const long long cell = (c & 1023) + (long long)S.lnd[0] * (((c >> 10) & 1023) + (long long)S.lnd[1] * ((c >> 20) & 1023));
    return (cell << 32) | (long long)jp;
}

__global__ void k_export_scatter(const SysDev *__restrict__ sysv, int s, const int *__restrict__ nbl,
                                 const int *__restrict__ nnb, const int *__restrict__ orig, int half,
                                 const int4 *__restrict__ llinfo, int *__restrict__ nneigh_out,
                                 long long *__restrict__ key_out, int maxn, ErrWord *err)
{
    const SysDev &S = sysv[s];
    const int li = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (li >= S.n) return;
    const int i = S.off + li;
    const int ip = orig[i] + 1;
    const int *row = nbl + S.nbl_off + (long long)li * S.cap;
    const int n = nnb[i];
    for (int k = lane; k < n; k += 32) {
        const int j = row[k] & ((1 << 28) - 1);
        if (!half && !(i < j)) continue;
        const int jp = orig[j] + 1;
        bool mine;
        if (S.llist) {
            mine = llist_owner(ip, jp);
        } else {
            const int itemp = (ip + jp) % 2;
            mine = (ip < jp && itemp != 0) || (ip > jp && itemp == 0);
        }
        const int own = mine ? ip : jp, other = mine ? jp : ip;
        const int slot = atomicAdd(nneigh_out + own - 1, 1);
        if (slot < maxn)
            key_out[(long long)(own - 1) * maxn + slot] = export_key(S, other, llinfo, mine ? j : i);
        else
            raise_error(err, 3, s, own, slot + 1);
    }
}

// Pass 2: each MOLSIM row in ascending key order (rank sort, one warp per row):
// ascending jp for SetVListMD's rows, cell by cell then ascending jp for
// SetVListMDLList's.
__global__ void k_export_sort(int n, const int *__restrict__ nneigh, const long long *__restrict__ key_in,
                              int *__restrict__ jp_out, int maxn)
{
    const int r = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= n) return;
    const int cnt = min(nneigh[r], maxn);
    const long long *in = key_in + (long long)r * maxn;
    int *out = jp_out + (long long)r * maxn;
    for (int k = lane; k < cnt; k += 32) {
        const long long v = in[k];
        int q = 0;
        for (int m = 0; m < cnt; ++m) q += (in[m] < v);
        out[q] = (int)(v & 0xffffffffLL);
    }
}

// ---------------------------------------------------------------------------
// API boundary: MOLSIM order <-> internal order.
// ---------------------------------------------------------------------------
__global__ void k_to_molsim(const double4 *__restrict__ src, double *__restrict__ dst, const int *__restrict__ inv,
                            int off, int n, double scale)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    const double4 v = src[inv[off + o]];
    dst[3 * o] = v.x * scale;
    dst[3 * o + 1] = v.y * scale;
    dst[3 * o + 2] = v.z * scale;
}

// Particles one block of k_state_in / k_state_out converts.
constexpr int STATE_BLOCK = 256;

// Positions, velocities and accelerations of one system from MOLSIM layout
// ([n][3] arrays; a null one is skipped) into the internal order, with the
// fixed-point mirror of the positions: one launch per state.  The arrays are read
// through shared memory so that every warp load covers contiguous doubles: the
// sources may be device staging buffers or the caller's mapped page-locked
// arrays, read straight over the bus.  A non-null zero_ctr is cleared by the
// first thread.
__global__ void __launch_bounds__(STATE_BLOCK) k_state_in(
    const SysDev *__restrict__ sysv, int sys, const double *__restrict__ sro, const double *__restrict__ srod,
    const double *__restrict__ srodd, double4 *__restrict__ pos, double4 *__restrict__ vel,
    double4 *__restrict__ acc, int4 *__restrict__ posfx, const int *__restrict__ inv,
    unsigned long long *__restrict__ zero_ctr)
{
    __shared__ double sb[3][3 * STATE_BLOCK];
    const SysDev &S = sysv[sys];
    const int o0 = blockIdx.x * STATE_BLOCK, t = threadIdx.x;
    if (zero_ctr && blockIdx.x == 0 && t == 0) *zero_ctr = 0ull;
    const int cnt = min(STATE_BLOCK, S.n - o0);
    if (cnt <= 0) return;
    const double *src[3] = {sro, srod, srodd};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (!src[k]) continue;
        const double *p = src[k] + 3 * (size_t)o0;
        for (int e = t; e < 3 * cnt; e += STATE_BLOCK) sb[k][e] = p[e];
    }
    __syncthreads();
    if (t >= cnt) return;
    const int i = inv[S.off + o0 + t];
    if (sro) {
        double4 v = pos[i];                       // .w holds the charge
        v.x = sb[0][3 * t];
        v.y = sb[0][3 * t + 1];
        v.z = sb[0][3 * t + 2];
        pos[i] = v;
        posfx[i] = fx_pos(v, S);
    }
    if (srod) vel[i] = make_double4(sb[1][3 * t], sb[1][3 * t + 1], sb[1][3 * t + 2], 0.0);
    if (srodd) acc[i] = make_double4(sb[2][3 * t], sb[2][3 * t + 1], sb[2][3 * t + 2], 0.0);
}

// The reverse: internal order -> MOLSIM-layout arrays (device staging buffers or
// mapped page-locked host arrays), written through shared memory in contiguous runs.
__global__ void __launch_bounds__(STATE_BLOCK) k_state_out(
    const SysDev *__restrict__ sysv, int sys, const double4 *__restrict__ pos, const double4 *__restrict__ vel,
    const double4 *__restrict__ acc, double *__restrict__ dro, double *__restrict__ drod,
    double *__restrict__ drodd, const int *__restrict__ inv)
{
    __shared__ double sb[3][3 * STATE_BLOCK];
    const SysDev &S = sysv[sys];
    const int o0 = blockIdx.x * STATE_BLOCK, t = threadIdx.x;
    const int cnt = min(STATE_BLOCK, S.n - o0);
    if (cnt <= 0) return;
    const double4 *src[3] = {pos, vel, acc};
    double *dst[3] = {dro, drod, drodd};
    if (t < cnt) {
        const int i = inv[S.off + o0 + t];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (!dst[k]) continue;
            const double4 v = src[k][i];
            sb[k][3 * t] = v.x;
            sb[k][3 * t + 1] = v.y;
            sb[k][3 * t + 2] = v.z;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (!dst[k]) continue;
        double *p = dst[k] + 3 * (size_t)o0;
        for (int e = t; e < 3 * cnt; e += STATE_BLOCK) p[e] = sb[k][e];
    }
}

// End-of-step read-back into the handle's mapped pinned block: the longest row of
// every system, one step of energy history (nh doubles, hist may be null) and the
// error word -- one small launch in place of three copies.
__global__ void k_readback(const int *__restrict__ nmaxrow, int nsys, const double *__restrict__ hist, int nh,
                           const ErrWord *__restrict__ errw, int *__restrict__ prow, double *__restrict__ phist,
                           ErrWord *__restrict__ perr)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
    for (int s = t; s < nsys; s += nt) prow[s] = nmaxrow[s];
    if (hist)
        for (int e = t; e < nh; e += nt) phist[e] = hist[e];
    if (t == 0) *perr = *errw;
}

// rodd = massip * forceo (GetLinAcc, Src/md.F90:601-617)
__global__ void k_linacc(const SysDev *__restrict__ sysv, const Tile *__restrict__ tiles, const double4 *__restrict__ fo,
                         const int *__restrict__ typ, const double *__restrict__ massip, double4 *__restrict__ acc)
{
    const Tile T = tiles[blockIdx.x];
    const SysDev &S = sysv[T.sys];
    const int i = T.i0 + threadIdx.x;
    if (i >= T.i1) return;
    const double mi = massip[S.type_off + typ[i]];
    const double4 f = fo[i];
    acc[i] = make_double4(mi * f.x, mi * f.y, mi * f.z, 0.0);
}

}  // namespace msg

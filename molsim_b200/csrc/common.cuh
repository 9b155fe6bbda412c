// common.cuh -- shared definitions of the B200 force/energy path.
//
// Layout in HBM (all systems of a handle are concatenated; "internal order"
// sorts particles by system, then Verlet cell, then MOLSIM index):
//   pos   double4 [Ntot]   x, y, z (A), charge (e)
//   vel   double4 [Ntot]   rod (A/ps)
//   acc   double4 [Ntot]   rodd (A/ps^2)
//   dsum  double4 [Ntot]   drosum, displacement since the last list build
//   typ   int     [Ntot]   0-based particle type
//   orig  int     [Ntot]   0-based MOLSIM index within the system
//   inv   int     [Ntot]   internal index of (system offset + MOLSIM index)
// Per-system constants live in a SysDev array; pair tables are concatenated.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define MSG_MAX_NATAT 10
#define MSG_MAX_ORDER 8
#define MSG_NBUCKET 1024

namespace msg {

// Unit conversion of UTotal (Src/energy.F90:405): fac = (sclene/scllen)/sclfor
// with scllen=1e-10, sclmas=1e-3, scltim=1e-12, sclene=1e3.
constexpr double kForceFac = 100.0;
// GetKinEnergy (Src/md.F90:1089-1112): ekin * sclmas*sclvel**2/sclene.
constexpr double kEkinFac = 1.0e-3 * (100.0 * 100.0) / 1.0e3;

struct SysDev {
    int n, off;                 // particles and offset into the concatenated arrays
    int npt, natat;             // types and type pairs
    int pt_off;                 // first PairTab of this system
    int lewald, lsurf;
    double box[3], half[3], boxi[3];
    double rcut2, rs2cut, drnlist;
    double vol;
    int ncell[3];               // Verlet cells per dimension
    int cell_off;               // first global cell id
    int cap;                    // neighbour-row capacity
    long long nbl_off;          // first neighbour slot
    int s, order;               // SPME grid edge and spline order
    long long grid_off;         // real grid offset (elements)
    long long cgrid_off;        // complex grid offset (complex elements)
    long long fac_off;          // meshfac/energyfac/virfac offset, (s/2+1)^3 each
    double dkdr[3];
    double epsfp, alpha;
    double uself;               // -alpha/sqrt(pi) * sum q^2 (before the epsfp scale)
    double dt;
    int bond_off;               // CSR offset of this system's per-particle bond rows
    int tile128_off, ntile128;  // tiles of 128 particles
    int chunk_off, nchunk;      // skin chunks of 1024 MOLSIM indices
    int infl_off, ninfl;        // influence work items
    int type_off;               // first entry of this system's per-type arrays
    int ptmap_off;              // first entry of this system's npt*npt type-pair map
    int tab_k0, tab_nk, tab_b0; // this system's slice of the concatenated table (intervals, buckets)
    int tab_smem;               // 1: the slice fits the pair kernel's shared-memory table
    int tab_smem_m;             // 1: the slice fits the lean FP32 pair kernel's shared-memory table
    double r2umin_max;          // largest r2umin / r2atat over the type pairs: pairs at or above
    double r2atat_max;          //   these need no per-pair lower-limit check
    double fxs[3];              // 2^32 / box: fixed-point coordinate scale of the mixed mirror
    float fxi[3];               // box / 2^32
    float pad3;
    uint64_t seed;              // Philox key of this system's Brownian noise
    unsigned long long pad2;
    // standard Ewald (txewaldrec 'std'; lewald = 1 with recstd = 1)
    int recstd;                 // 1: reciprocal space by the standard Ewald sum, not SPME
    int ew_ncut;                // k = 2 pi n / L, 0 <= n_i <= ew_ncut
    int ew_nkv, ew_kv_off;      // k-vectors (n, kfac) of this system and their first entry
    long long ew_eik_off;       // first double2 of this system's exp(i k x) tables
    long long ew_part_off;      // first 4-double2 record of the partial structure factors
    int ew_nchunk, ew_clen;     // particle chunks of the structure-factor sum and their length
    long long ew_fks_off;       // first double4 of the per-slice reciprocal forces
    int ew_nks, ew_klen;        // k-vector slices of the force sum and their length
    // 2D layer correction (lewald2dlc): its forces are one more slice after the ew_nks
    int elc;                    // 1: layer correction (with recstd) and the 2D surface term
    int elc_nkv, elc_kv_off;    // 2D k-vectors (nx, ny) of this system and their first entry
    int inlist;                 // NList: 0 skin test; n > 0 rebuild whenever istep2 % n == 0
    // lvlistllist: SetLList(rcut+drnlist) grid (lnd cells per dimension, lcelli = real(lnd)/boxlen)
    // and SetNCell's probe distance lrcut = rcut
    int llist, lnd[3];
    double lcelli[3], lrcut;
    // precise FP32 pair kernel: r2 from fixed-point differences (fxd = box/2^32 per
    // dimension; cubic boxes use the integer sum of squares times fx2f = fxd^2 in FP32)
    int fx_cubic, tab_smem_h;
    float fx2f, pad4;
    double fxd[3];
    // SPME convolution kernel: radices of the grid edge's transform (pass count in
    // the low 4 bits, radices in the 4-bit fields above; 0 when the edge goes
    // through cuFFT) and the first entry of the edge's twiddle table
    int fft_rad, fft_tw;
};

// One type pair's slice of the concatenated table.
struct PairTab {
    int k0, nk;                 // first interval and count (intervals from high z to low z)
    int b0;                     // first bucket entry
    int pad;
    double z_lo, z_hi, inv_h;   // bucket grid over [z_lo, z_hi)
    double r2umin, r2atat;
    float fz_lo, fz_hi, finv_h; // the bucket grid in FP32 (the bucket index is formed in FP32)
    float pad2;
};

struct Tile { int sys, i0, i1, pad; };

// Mixed-precision position mirror: box coordinates as 32-bit fixed point
// (2^32 units per box length, wrapping), charge bits in .w.  The difference
// of two such coordinates is exact and wraps to the minimum image.
__device__ __forceinline__ int fx_coord(double x, double scale)
{
    return (int)(unsigned)(unsigned long long)__double2ll_rn(x * scale);
}
__device__ __forceinline__ int4 fx_pos(const double4 &x, const SysDev &S)
{
    return make_int4(fx_coord(x.x, S.fxs[0]), fx_coord(x.y, S.fxs[1]), fx_coord(x.z, S.fxs[2]),
                     __float_as_int((float)x.w));
}

// Per-system accumulators of one step, 64-bit fixed point (2^-32 units), added
// with integer atomics: the sums do not depend on the order blocks finish.
enum {
    EA_UTWOB = 0,      // 10 slots: u%twob per type pair
    EA_VIRPAIR = 10,
    EA_UREC = 11,      // reciprocal-space energy and virial before the self term
    EA_VIRREC = 12,
    EA_UBOND = 13,
    EA_VIRBOND = 14,
    EA_EKIN = 15,      // sum of m v^2 / 2 in internal units
    EA_DIP = 16,       // 3 slots: sum of q r for the surface term
    EA_N = 20
};
constexpr double kEFix = 4294967296.0;
constexpr double kEFixInv = 1.0 / 4294967296.0;

__device__ __forceinline__ void acc_add(long long *a, double v)
{
    atomicAdd(reinterpret_cast<unsigned long long *>(a), (unsigned long long)__double2ll_rn(v * kEFix));
}
__device__ __forceinline__ double acc_get(const long long *a) { return (double)__ldcg(a) * kEFixInv; }

// Error word: code, system, and two particle indices of the first error seen.
struct ErrWord { int code, sys, i, j; };

__device__ __forceinline__ void raise_error(ErrWord *e, int code, int sys, int i, int j)
{
    if (atomicCAS(&e->code, 0, code) == 0) {
        e->sys = sys;
        e->i = i;
        e->j = j;
    }
}

// PBCr2 for a box (Src/molaux.F90:149-161): a single sign(dpbc, d) shift per
// component when |d| > L/2, then r2 = dx*dx + dy*dy + dz*dz rounded as
// ((dx*dx) + (dy*dy)) + (dz*dz) with no fused multiply-add.
__device__ __forceinline__ double pbcr2_exact(double &dx, double &dy, double &dz, const SysDev &S)
{
    if (fabs(dx) > S.half[0]) dx = __dsub_rn(dx, copysign(S.box[0], dx));
    if (fabs(dy) > S.half[1]) dy = __dsub_rn(dy, copysign(S.box[1], dy));
    if (fabs(dz) > S.half[2]) dz = __dsub_rn(dz, copysign(S.box[2], dz));
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// PBC for a box (Src/molaux.F90:111-113): d - L*anint(d/L) when |d| > L/2.
__device__ __forceinline__ double pbc_wrap(double d, double half, double len, double leni)
{
    if (fabs(d) > half) d = __dsub_rn(d, __dmul_rn(len, round(__dmul_rn(d, leni))));
    return d;
}

__device__ __forceinline__ int pair_of(const int *ptmap, const SysDev &S, int ti, int tj)
{
    return ptmap[S.ptmap_off + ti * S.npt + tj];
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Cardinal B-spline values and first derivatives (Src/mollib.F90:1629-1683):
// values[i] = M_P(x+i), derivs[i] = M_{P-1}(x+i) - M_{P-1}(x+i-1) for the
// fractional position x in [0, 1).
template <int P, typename R>
__device__ __forceinline__ void bspline_frac(R x, R *values, R *derivs)
{
    R lastv[P];
#pragma unroll
    for (int i = 0; i < P; ++i) lastv[i] = R(0);
    values[0] = x;
    if (P > 1) values[1] = R(1) - x;
#pragma unroll
    for (int n = 3; n <= P; ++n) {
#pragma unroll
        for (int i = 0; i < P; ++i) lastv[i] = values[i];
        const R nm1 = R(n - 1);
        values[0] = x * lastv[0] / nm1;
#pragma unroll
        for (int i = 1; i <= n - 2; ++i) {
            R a = R(i) + x;
            values[i] = (a * lastv[i] + (R(n) - a) * lastv[i - 1]) / nm1;
        }
        values[n - 1] = (R(1) - x) * lastv[n - 2] / nm1;
    }
    derivs[0] = lastv[0];
#pragma unroll
    for (int i = 1; i <= P - 2; ++i) derivs[i] = lastv[i] - lastv[i - 1];
    derivs[P - 1] = -lastv[P - 2];
}

// Splines at the mesh coordinate u = dkdr * r; returns kmax = floor(u) wrapped
// into [0, s).  The fraction is formed in FP64 and then rounded to R.
template <int P, typename R>
__device__ __forceinline__ int bspline_at(double u, int s, R *values, R *derivs)
{
    const double fl = floor(u);
    bspline_frac<P, R>((R)(u - fl), values, derivs);
    int k = (int)fl % s;
    return k < 0 ? k + s : k;
}

}  // namespace msg

// engine.cu -- the B200 force/energy engine behind the C-ABI of molsim_gpu.h.
//
// One handle owns every device buffer of its systems (concatenated), the pair
// tables, the SPME grids with their cuFFT plans, and two CUDA streams: a step
// is a fixed graph of kernels whose pair/bond branch runs on the second stream
// beside the SPME chain.  Each API call enqueues its steps and waits for the
// handle's stream once at the end, reading the device error word back then.
#include <cuda.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <unordered_map>
#include <string>
#include <vector>

#include "../../include/molsim_gpu.h"
#include "common.cuh"
#include "kernels_force.cuh"
#include "kernels_spme.cuh"
#include "kernels_md.cuh"
#include "kernels_ewald.cuh"
#include "kernels_mc.cuh"
#include "radix_sort.cuh"
#include "setup.h"

using namespace msg;

namespace {

struct CudaError {
    int code;
    std::string what;
};

#define CK(x)                                                                                  \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess) throw CudaError{MSG_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)}; \
    } while (0)
#define CKF(x)                                                                                 \
    do {                                                                                       \
        cufftResult r_ = (x);                                                                  \
        if (r_ != CUFFT_SUCCESS) throw CudaError{MSG_ERR_CUDA, std::string(#x) + ": cufft error " + std::to_string((int)r_)}; \
    } while (0)

template <typename T>
void h2d(T *d, const T *h, size_t n, cudaStream_t st)
{
    if (n) CK(cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, st));
}

struct HostSys {
    int n, off, npt, natat, order, s;
    msg_params p;
};

enum { TM_POS, TM_PAIR, TM_SPREAD, TM_FFT, TM_INFL, TM_FINAL, TM_REBUILD, TM_EWSTD, TM_N };
const char *const kTimerNames[TM_N] = {"position_update_skin", "pair", "spread", "fft", "influence",
                                        "gather_finalize", "rebuild", "ewald_std"};

// cuFFT plans are cached process-wide by (edge, batch, type, direction) and
// run on a work area that the owning handle allocates stream-ordered, so
// creating or destroying a handle never frees device memory through cuFFT
// (a free would wait for every stream of the device).  A grid class of
// `count` systems runs as power-of-two sub-batches, which bounds the number
// of distinct plans.
struct PlanKey {
    int s, count, f32, fwd;
    bool operator<(const PlanKey &o) const
    {
        return s != o.s ? s < o.s : count != o.count ? count < o.count : f32 != o.f32 ? f32 < o.f32 : fwd < o.fwd;
    }
};
// Small pinned host blocks for the per-call device-to-host reads (error word,
// longest rows, energy history): with the reads in pinned memory an API call
// waits for its stream once.  The blocks are pooled for the process and never
// freed, because freeing pinned memory would wait for the whole device.
constexpr size_t kPinBytes = 64 * 1024;
std::mutex g_pin_mu;
std::vector<void *> g_pin_free;

void *pin_acquire()
{
    std::lock_guard<std::mutex> lk(g_pin_mu);
    if (!g_pin_free.empty()) {
        void *p = g_pin_free.back();
        g_pin_free.pop_back();
        return p;
    }
    void *p = nullptr;
    if (cudaMallocHost(&p, kPinBytes) != cudaSuccess) return nullptr;
    return p;
}

void pin_release(void *p)
{
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    g_pin_free.push_back(p);
}

std::mutex g_plan_mu;
std::map<PlanKey, std::vector<std::pair<cufftHandle, size_t>>> g_plan_idle;

cufftResult make_plan(const PlanKey &k, cufftHandle *out, size_t *ws)
{
    int dims[3] = {k.s, k.s, k.s};
    const int rdist = k.s * k.s * k.s, cdist = k.s * k.s * (k.s / 2 + 1);
    const cufftType t = k.fwd ? (k.f32 ? CUFFT_R2C : CUFFT_D2Z) : (k.f32 ? CUFFT_C2R : CUFFT_Z2D);
    cufftResult r = cufftCreate(out);
    if (r != CUFFT_SUCCESS) return r;
    r = cufftSetAutoAllocation(*out, 0);
    if (r == CUFFT_SUCCESS)
        r = k.fwd ? cufftMakePlanMany(*out, 3, dims, nullptr, 1, rdist, nullptr, 1, cdist, t, k.count, ws)
                  : cufftMakePlanMany(*out, 3, dims, nullptr, 1, cdist, nullptr, 1, rdist, t, k.count, ws);
    if (r != CUFFT_SUCCESS) cufftDestroy(*out);
    return r;
}

struct FftPart {
    int count;
    long long grid_off, cgrid_off;
    cufftHandle fwd = 0, bwd = 0;
    size_t ws_fwd = 0, ws_bwd = 0;
};

struct FftClass {
    int s, count;
    long long grid_off, cgrid_off;
    int rad = 0;                 // > 0: the edge goes through the convolution kernel, not cuFFT
    std::vector<FftPart> parts;
};

// Radices of the convolution kernel's transform of length s (pass count in the
// low 4 bits, radices above), or 0 when the edge is left to cuFFT: odd, beyond
// four passes of 8, 5, 4, 3 and 2, or with planes too large for shared memory.
int conv_radices(int s)
{
    if (s < 8 || (s & 1) || s > CONV_MAX_EDGE || 32LL * s * (s / 2 + 1) > CONV_MAX_SMEM) return 0;
    int rad = 0, np = 0, n = s;
    for (int r : {8, 4, 5, 3, 2})
        while (n % r == 0 && n > 1) {
            if (np == 4) return 0;
            rad |= r << (4 + 4 * np);
            ++np;
            n /= r;
        }
    return n == 1 ? (rad | np) : 0;
}

}  // namespace

struct msg_handle {
    int nsys = 0, ntot = 0, prec = MSG_PREC_FP64, order = 4;
    std::vector<SysDev> hs;
    std::vector<int> hn;
    std::string err;
    cudaStream_t st = nullptr;
    // second stream of the step: the pair kernel runs there beside the SPME chain
    cudaStream_t st2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // third stream of the host-exchange graph: positions go back to the host while the forces run
    cudaStream_t st3 = nullptr;
    cudaEvent_t ev_io0 = nullptr, ev_io1 = nullptr;
    double *io_ro = nullptr;         // mapped host positions written right after the position update
    int io_ro_sys = -1;
    int overlap = 1;                 // pair kernel concurrent with spread/FFT/influence
    int pair_per_sm = 0;             // pair blocks per SM (0: as many as fit; 2 when overlapped)
    int dev = 0;
    // particles (double-buffered where the rebuild permutes)
    int cur = 0;
    double4 *pos[2] = {}, *vel[2] = {}, *acc[2] = {}, *dsum[2] = {}, *fo[2] = {};
    int *typ[2] = {}, *orig[2] = {};
    int *cellid = nullptr, *inv = nullptr, *sysid = nullptr;
    double4 *fsr = nullptr, *ftot = nullptr;
    // half list (each pair once): the pair kernel adds partner forces here as 2^-32 fixed point,
    // x, y and z blocks of ntot entries; k_finalize adds them to fsr and clears them
    int list_half = 0;
    unsigned long long *fpart = nullptr;
    int4 *posfx = nullptr;
    // rebuild
    uint32_t *k0 = nullptr, *v0 = nullptr, *k1 = nullptr, *v1 = nullptr, *rhist = nullptr;
    int ncell_tot = 0, cell_bits = 1;
    int *cstart = nullptr, *cend = nullptr;
    int *nbl = nullptr, *nnb = nullptr, *nmaxrow = nullptr;
    long long nbl_tot = 0;
    // skin
    double *r2o = nullptr, *skinout = nullptr;
    SkinChunk *sc = nullptr;
    int *flag = nullptr;
    long long *nrebuild = nullptr;
    // work lists
    Tile *t128 = nullptr;
    PairTask *ptask = nullptr;
    int2 *psrange = nullptr;          // lean pair kernel: each system's tasks [first, end)
    int *pgsys = nullptr;             // lanes per particle of each system's tasks
    int *psched = nullptr;            // its per-system task counters and finished-block counter
    int nt128 = 0, nptask = 0, max_npt = 1;
    int4 *chunks = nullptr, *infl = nullptr;
    int nchunk = 0, ninfl = 0;
    long long *eacc = nullptr;
    int pair_grid = 0;
    size_t pair_smem = 0;
    double *esys = nullptr, *hist = nullptr;
    int hist_cap = 0;
    unsigned long long *stepctr = nullptr, *sstep = nullptr;
    unsigned *rdone = nullptr, *fdone = nullptr;
    ErrWord *errw = nullptr;
    // tables
    PairTab *ptab = nullptr;
    int *ptmap = nullptr;
    double *tz = nullptr, *tc = nullptr;
    float *tz32 = nullptr, *tc32 = nullptr;
    unsigned short *bst = nullptr;                    // bucket starts per type pair
    int2 *bkz = nullptr;                              // lean kernel buckets: (absolute row, its z_low)
    size_t pair_smem_m = 0, pair_smem_h = 0;
    float *tch = nullptr;                             // k_pair_h rows (ROW16 floats used of ROWST: hi/lo z_low, c1, c7)
    // mixed path: k_pair_h over a half list (2) or a full list (3), k_pair_m (1) or k_pair (0)
    int pair_lean = 1;
    int pair_unroll = 2;                              // k_pair_m: row entries in flight per lane
    int nsm = 148;
    double *massip = nullptr, *massp = nullptr, *fac1 = nullptr, *fac2 = nullptr;
    int has_bd = 0, has_bonds = 0;
    // bonds
    int *bptr = nullptr, *bpart = nullptr, *bpw = nullptr;
    int4 *btab = nullptr;       // per-particle bond table (every particle with at most two bonds)
    double *bk = nullptr, *beq = nullptr;
    // Ewald sums: any_ewald = any system with one (SPME or standard), any_spme / any_std by method
    int any_ewald = 0, any_spme = 0, any_std = 0;
    // lvlistllist: per-particle linked-list cell and SetNCell probe sets (k_llist_info)
    int any_llist = 0;
    int4 *llinfo = nullptr;
    unsigned *istep2 = nullptr;       // per system: steps since NList(iBeforeMacrostep)
    // standard Ewald: k-vectors, tables, partial and full structure factors, force slices, work items
    int4 *ew_kv = nullptr, *ew_kitems = nullptr, *ew_fitems = nullptr;
    unsigned *ew_tiledone = nullptr;   // per k tile: chunks finished this step
    double *ew_kfac = nullptr;
    double2 *ew_eik = nullptr, *ew_part = nullptr, *ew_sk = nullptr;
    double4 *ew_fks = nullptr;
    int ew_nk = 0, ew_ntile = 0, ew_nf = 0;
    // 2D layer correction: 2D k-vectors {nx, ny, system}, kfac2d, the eight sums per k-vector
    int4 *elc_kv = nullptr;
    double *elc_kfac = nullptr, *elc_st = nullptr, *elc_sttm = nullptr;   // elc_sttm: a Monte Carlo trial's sums
    // Monte Carlo with SPME: the FP64 spectrum of each system's charge mesh (engine's grid
    // offsets), its fixed-point and FP64 meshes, D2Z plans per mesh class
    double2 *mc_F = nullptr;
    double *mc_rg = nullptr;
    unsigned long long *mc_ig = nullptr;
    std::vector<cufftHandle> mc_plans;
    // MCAllPass: jump table of Random, saved positions (MOLSIM order) and energies, decisions
    McJump *mc_jumpt = nullptr;
    double4 *mca_psave = nullptr, *mca_step = nullptr;
    int *mca_flag = nullptr;
    double *mca_esave = nullptr, *mca_beta = nullptr;
    int *mca_acc = nullptr;
    int elc_nk = 0;
    // Monte Carlo: Random's state, running energies, counts (accepted, hard-core rejects),
    // sweep parameters, displacement per type, trial structure factors
    int2 *mc_rng = nullptr;
    double *mc_u = nullptr, *mc_dtr = nullptr;
    long long *mc_cnt = nullptr;
    McPar *mc_par = nullptr;
    double2 *ew_sktm = nullptr;
    int type_tot = 0, ew_nkv_tot = 0, ew_maxw = 0;
    void ensure_mc();
    size_t ew_smem = 0;
    // SPME
    double *rgrid = nullptr, *mfac = nullptr, *emf = nullptr, *vmf = nullptr;
    double2 *cgrid = nullptr;
    float *rgrid32 = nullptr;
    float2 *cgrid32 = nullptr;
    unsigned long long *igrid = nullptr;
    long long grid_tot = 0, cgrid_tot = 0;
    std::vector<FftClass> fft;
    // convolution kernel: tasks, counters, twiddle tables, buffer size, grid
    int4 *conv_tasks = nullptr;
    unsigned *conv_ctr = nullptr;
    double2 *conv_tw = nullptr;
    float2 *conv_tw32 = nullptr;
    int conv_ntasks = 0, conv_nctr = 0, conv_cap = 0, conv_grid = 0;
    int conv_widest = 0, conv_occ = 1;   // tasks of the widest stage; blocks per SM that fit
    void set_conv_grid(int per_sm);
    // staging
    double *stage = nullptr;
    size_t stage_n = 0;
    double *xin = nullptr;
    size_t xin_n = 0;
    SysDev *dsys = nullptr;
    // instrumentation
    long long launches = 0;
    bool timing = false;
    std::vector<cudaEvent_t> evpool;
    std::vector<int> pend_k;
    std::vector<cudaEvent_t> pend_a, pend_b;
    cudaEvent_t open_ev[TM_N] = {};
    double tm_ms[TM_N] = {};
    long long tm_n[TM_N] = {};

    // device memory: stream-ordered from the device's pool; a dry build only counts bytes
    // systems whose positions were given: only these have lists to rebuild after a re-layout
    std::vector<int> placed;
    bool dry = false;
    long long bytes_live = 0;
    size_t alloc_log = 0;       // MSG_ALLOC_LOG=<bytes>: report allocations at least that large
    std::unordered_map<void *, size_t> sizes;
    void *fftwork = nullptr;
    std::vector<cudaEvent_t> inflight;   // one event per asynchronous step batch
    template <typename T>
    T *dalloc(size_t n)
    {
        if (n == 0) n = 1;
        const size_t b = ((n * sizeof(T) + 511) / 512) * 512;
        bytes_live += (long long)b;
        if (alloc_log && b >= alloc_log) std::fprintf(stderr, "msg alloc %zu bytes\n", b);
        if (dry) return reinterpret_cast<T *>((uintptr_t)512);
        void *p = nullptr;
        CK(cudaMallocAsync(&p, b, st));
        CK(cudaMemsetAsync(p, 0, b, st));
        sizes[p] = b;
        return static_cast<T *>(p);
    }
    void dfree(void *p)
    {
        if (!p || dry) return;
        auto it = sizes.find(p);
        if (it != sizes.end()) {
            bytes_live -= (long long)it->second;
            sizes.erase(it);
        }
        cudaFreeAsync(p, st);
    }
    void up(void *d, const void *hsrc, size_t bytes)
    {
        if (dry || !bytes) return;
        CK(cudaMemcpyAsync(d, hsrc, bytes, cudaMemcpyHostToDevice, st));
    }
    void down(void *hdst, const void *d, size_t bytes)
    {
        if (!bytes) return;
        CK(cudaMemcpyAsync(hdst, d, bytes, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    void plan_fft();
    void release_fft();
    // pinned block: [0, 256) error word, [256, 256 + 4 nsys) longest rows, then energy history
    unsigned char *pin = nullptr;
    unsigned char *dpin = nullptr;   // the block's mapped device address (null: not mapped)
    template <class T>
    T *map_host(T *p) const
    {
        return p ? reinterpret_cast<T *>(dpin + (reinterpret_cast<unsigned char *>(p) - pin)) : nullptr;
    }
    ErrWord *pin_err() { return reinterpret_cast<ErrWord *>(pin); }
    int *pin_rows() { return (pin && 256 + 4 * (size_t)nsys <= kPinBytes / 2) ? reinterpret_cast<int *>(pin + 256) : nullptr; }
    double *pin_hist(size_t n)
    {
        const size_t off = ((256 + 4 * (size_t)nsys + 15) / 16) * 16;
        return (pin && off + n * sizeof(double) <= kPinBytes) ? reinterpret_cast<double *>(pin + off) : nullptr;
    }
    int pair_blocks_max = 1, pair_blocks_lean = 1, pair_shift = 0;
    std::vector<PairTask> make_pair_tasks(int shift) const;
    void set_pair_chunks(const std::vector<PairTask> &pt, bool replace);
    void set_pair_lanes(int shift, bool force = false);
    void set_lean_grid(int nsm);

    ~msg_handle();
    cudaEvent_t get_event()
    {
        cudaEvent_t e;
        if (!evpool.empty()) {
            e = evpool.back();
            evpool.pop_back();
        } else {
            CK(cudaEventCreate(&e));
        }
        return e;
    }
    bool capturing = false;
    void rec_event(cudaEvent_t e)
    {
        // under stream capture an external record node keeps the timestamp in the graph
        CK(cudaEventRecordWithFlags(e, st, capturing ? cudaEventRecordExternal : cudaEventRecordDefault));
    }
    void tbeg(int k)
    {
        if (!timing) return;
        open_ev[k] = get_event();
        rec_event(open_ev[k]);
    }
    void tend(int k)
    {
        if (!timing) return;
        cudaEvent_t b = get_event();
        rec_event(b);
        pend_k.push_back(k);
        pend_a.push_back(open_ev[k]);
        pend_b.push_back(b);
    }
    void flush_timers()
    {
        for (size_t q = 0; q < pend_k.size(); ++q) {
            float ms = 0.0f;
            CK(cudaEventElapsedTime(&ms, pend_a[q], pend_b[q]));
            tm_ms[pend_k[q]] += ms;
            tm_n[pend_k[q]] += 1;
            evpool.push_back(pend_a[q]);
            evpool.push_back(pend_b[q]);
        }
        pend_k.clear();
        pend_a.clear();
        pend_b.clear();
    }
    void build(const msg_params *p, int n, int prec);
    void enqueue_rebuild();
    void enqueue_forces(int mode, bool record, bool skin = false);
    void enqueue_md_step(bool record);
    void enqueue_bd_step(uint64_t seed, const double *xin_step, double *xout_step, bool record);
    // CUDA graph of one step; the rebuild sits in an IF node opened by k_skin
    cudaGraphConditionalHandle cond = 0;
    int use_cond = 0;
    struct StepGraph {
        cudaGraphExec_t exec = nullptr;
        int kind = -1;            // 0 MD, 1 BD (Philox noise)
        bool record = false, timing = false;
        uint64_t seed = 0;
        double *hist = nullptr;
        int hist_cap = 0;
        long long launches = 0;
        std::vector<int> tk;
        std::vector<cudaEvent_t> ta, tb;
        // host exchange captured with the step (msg_velver_host on page-locked arrays)
        int io_sys = -1;
        double *io[3] = {nullptr, nullptr, nullptr};
    } graph, iograph;
    bool use_graphs = true;
    void drop_graph();
    void drop_one(StepGraph &gr);
    void ensure_graph(int kind, bool record, uint64_t seed);
    void build_graph(StepGraph &gr, int kind, bool record, uint64_t seed, int io_sys, double *const io[3]);
    void ensure_io_graph(bool record, int io_sys, double *const io[3]);
    void launch_graph();
    void launch_one(StepGraph &gr);
    void ensure_stage(size_t n);
    int check();
    int check_word(const ErrWord &e);
    bool grow_lists(const int *mx_host = nullptr);
    int rebuild_checked(const std::vector<int> &flags);
};

static void free_all(msg_handle *h)
{
    void *ptrs[] = {h->pos[0], h->pos[1], h->vel[0], h->vel[1], h->acc[0], h->acc[1], h->dsum[0], h->dsum[1],
                    h->fo[0], h->fo[1], h->typ[0], h->typ[1], h->orig[0], h->orig[1], h->cellid, h->inv,
                    h->sysid, h->fsr, h->fpart, h->ftot, h->posfx, h->k0, h->v0, h->k1, h->v1, h->rhist, h->cstart,
                    h->cend, h->nbl, h->nnb, h->nmaxrow, h->r2o, h->skinout, h->sc, h->flag, h->nrebuild,
                    h->t128, h->ptask, h->psrange, h->pgsys, h->psched, h->chunks, h->infl, h->eacc, h->esys,
                    h->hist, h->stepctr, h->sstep, h->rdone, h->fdone, h->errw, h->ptab, h->ptmap, h->tz, h->tc,
                    h->bst, h->bkz, h->tz32, h->tc32, h->massip, h->massp, h->fac1, h->fac2, h->bptr, h->bpart, h->bpw, h->bk, h->beq,
                    h->rgrid, h->mfac, h->emf, h->vmf, h->cgrid, h->rgrid32, h->cgrid32, h->igrid, h->stage, h->xin, h->dsys,
                    h->ew_kv, h->ew_kitems, h->ew_tiledone, h->ew_fitems, h->ew_kfac, h->ew_eik, h->ew_part,
                    h->ew_sk, h->ew_fks, h->mc_rng, h->mc_u, h->mc_dtr, h->mc_cnt, h->mc_par, h->ew_sktm,
                    h->elc_kv, h->elc_kfac, h->elc_st, h->elc_sttm, h->mc_F, h->mc_rg, h->mc_ig,
                    h->mc_jumpt, h->mca_psave, h->mca_esave, h->mca_beta, h->mca_acc, h->mca_step,
                    h->mca_flag, h->llinfo, h->istep2, h->tch, h->conv_tasks, h->conv_ctr, h->conv_tw,
                    h->conv_tw32, h->btab};
    if (!h->dry && h->st) {
        for (void *p : ptrs) h->dfree(p);
        h->dfree(h->fftwork);
    }
    h->release_fft();
    pin_release(h->pin);
    h->pin = nullptr;
    h->dpin = nullptr;
    for (cudaEvent_t e : h->inflight) cudaEventDestroy(e);
    h->inflight.clear();
    for (cudaEvent_t e : h->evpool) cudaEventDestroy(e);
    for (cudaEvent_t e : h->pend_a) cudaEventDestroy(e);
    for (cudaEvent_t e : h->pend_b) cudaEventDestroy(e);
    h->evpool.clear();
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    if (h->ev_io0) cudaEventDestroy(h->ev_io0);
    if (h->ev_io1) cudaEventDestroy(h->ev_io1);
    if (h->st3) cudaStreamDestroy(h->st3);
    if (h->st2) cudaStreamDestroy(h->st2);
    if (h->st) cudaStreamDestroy(h->st);
    h->st = h->st2 = h->st3 = nullptr;
    h->ev_fork = h->ev_join = h->ev_io0 = h->ev_io1 = nullptr;
}

msg_handle::~msg_handle()
{
    for (cufftHandle p : mc_plans) cufftDestroy(p);
    drop_graph();
    free_all(this);
}

void msg_handle::ensure_stage(size_t n)
{
    if (n <= stage_n) return;
    if (stage) dfree(stage);
    stage = dalloc<double>(n);
    stage_n = n;
}

// For the buckets b = 0..MSG_NBUCKET-1 at z(b) = z_lo + (b + frac) h: where the
// reference's table walk stops, the first kk with kk == nk-1 or z(b) >= z[kk] (z falls
// with kk).  z(b) grows with b, so the stop never moves up as b grows: one pointer
// walked from the top bucket down gives every stop in O(buckets + intervals).
static void bucket_stops(const double *z, int nk, double z_lo, double h, double frac, int *out)
{
    int kk = 0;
    for (int b = MSG_NBUCKET - 1; b >= 0; --b) {
        const double zq = z_lo + (b + frac) * h;
        while (kk < nk - 1 && zq < z[kk]) ++kk;
        out[b] = kk;
    }
}

// ---------------------------------------------------------------------------
// Set-up of all systems.
// ---------------------------------------------------------------------------
void msg_handle::build(const msg_params *P, int n, int precision)
{
    nsys = n;
    prec = precision;
    // the mixed path streams a half list by default (k_pair_h); the FP64 path a full list
    pair_lean = prec == MSG_PREC_MIXED ? 2 : 1;
    list_half = pair_lean == 2 ? 1 : 0;
    if (!dry) {
        CK(cudaGetDevice(&dev));
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking));
        pin = static_cast<unsigned char *>(pin_acquire());
        void *dp = nullptr;
        if (pin && cudaHostGetDevicePointer(&dp, pin, 0) == cudaSuccess)
            dpin = static_cast<unsigned char *>(dp);
        else
            cudaGetLastError();
        CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
        CK(cudaStreamCreateWithFlags(&st3, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&ev_io0, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ev_io1, cudaEventDisableTiming));
    }
    hs.resize(n);
    hn.resize(n);
    placed.assign(n, 0);
    order = 4;
    for (int s = n - 1; s >= 0; --s)
        if (P[s].lewald == 1) order = P[s].order;   // the spline order of the first SPME system
    std::vector<HostSys> H(n);
    ntot = 0;
    int type_tot = 0, pt_tot = 0, ptmap_tot = 0, cell_tot = 0, t128 = 0, nch = 0;
    long long nbl_acc = 0;
    size_t nbond_tot = 0;
    for (int s = 0; s < n; ++s) {
        const msg_params &p = P[s];
        if (p.np < 1 || p.npt < 1 || p.npt > MAXT) throw CudaError{MSG_ERR_ARG, "np >= 1 and 1 <= npt <= 4 required"};
        if (p.lewald < 0 || p.lewald > 2) throw CudaError{MSG_ERR_ARG, "lewald must be 0, 1 (SPME) or 2 (standard Ewald)"};
        if (p.lewald == 1 && (p.order < 4 || p.order > 6 || p.nmesh < 4 || (p.nmesh & 1)))
            throw CudaError{MSG_ERR_ARG, "SPME needs 4 <= order <= 6 and an even nmesh"};
        if (p.lewald == 1 && p.order != order) throw CudaError{MSG_ERR_ARG, "all SPME systems of a handle share one spline order"};
        if (p.lewald == 2 && (p.ncut < 1 || p.ncut > EW_MAXCUT || p.ncutregion < 0 || p.ncutregion > 1))
            throw CudaError{MSG_ERR_ARG, "standard Ewald needs 1 <= ncut <= 100 and ncutregion 0 (sphere) or 1 (cube)"};
        if (!p.iptpn || !p.az || !p.masspt || !p.ubuf || !p.iubuflow || !p.r2umin)
            throw CudaError{MSG_ERR_ARG, "iptpn, az, masspt, ubuf, iubuflow and r2umin are required"};
        if (p.inlist < 0) throw CudaError{MSG_ERR_ARG, "inlist negative"};   // NList's Stop, Src/nlist.F90:619
        if (p.lvlistllist != 0 && p.lvlistllist != 1) throw CudaError{MSG_ERR_ARG, "lvlistllist must be 0 or 1"};
        SysDev &S = hs[s];
        std::memset(&S, 0, sizeof(S));
        S.inlist = p.inlist;
        if (p.lvlistllist) {
            // SetLList(rcut+drnlist): ndivllist = int(boxlen/distance), celli = real(ndivllist)*boxleni
            const double dist = p.rcut + p.drnlist;
            long long nc = 1;
            for (int d = 0; d < 3; ++d) {
                S.lnd[d] = (int)(p.boxlen[d] / dist);
                S.lcelli[d] = (double)(float)S.lnd[d] * (1.0 / p.boxlen[d]);
                nc *= S.lnd[d];
            }
            if (nc < 1 || nc > 1000)
                throw CudaError{MSG_ERR_ARG, "lvlistllist needs 1 to 1000 linked-list cells (Src/nlist.F90:1195)"};
            S.llist = 1;
            S.lrcut = p.rcut;
            any_llist = 1;
        }
        S.n = p.np;
        S.off = ntot;
        S.npt = p.npt;
        S.natat = p.npt * (p.npt + 1) / 2;
        S.pt_off = pt_tot;
        S.lewald = p.lewald ? 1 : 0;
        S.recstd = p.lewald == 2 ? 1 : 0;
        S.lsurf = (p.lewald && p.lsurf) ? 1 : 0;
        S.elc = (p.lewald && p.lewald2dlc) ? 1 : 0;
        for (int d = 0; d < 3; ++d) {
            S.box[d] = p.boxlen[d];
            S.half[d] = p.boxlen[d] / 2.0;
            S.boxi[d] = 1.0 / p.boxlen[d];
        }
        S.vol = p.boxlen[0] * p.boxlen[1] * p.boxlen[2];
        for (int d = 0; d < 3; ++d) {
            S.fxs[d] = 4294967296.0 / p.boxlen[d];
            S.fxi[d] = (float)(p.boxlen[d] / 4294967296.0);
            S.fxd[d] = p.boxlen[d] / 4294967296.0;
        }
        S.fx_cubic = (p.boxlen[0] == p.boxlen[1] && p.boxlen[0] == p.boxlen[2]) ? 1 : 0;
        S.fx2f = (float)(S.fxd[0] * S.fxd[0]);
        S.rcut2 = p.rcut * p.rcut;
        const double rl = p.rcut + p.drnlist;
        S.rs2cut = rl * rl;
        S.drnlist = p.drnlist;
        for (int d = 0; d < 3; ++d) {
            int nc = (int)std::floor(p.boxlen[d] / (rl * (1.0 + 1e-10)));
            S.ncell[d] = std::max(1, nc);
        }
        S.cell_off = cell_tot;
        cell_tot += S.ncell[0] * S.ncell[1] * S.ncell[2];
        const double dens = p.np / S.vol;
        const double vshell = 4.0 / 3.0 * 3.1415926535897932 * rl * rl * rl;
        int cap = (int)std::ceil((list_half ? 1.0 : 2.0) * dens * vshell) + 64;
        if (p.maxnneigh > 0) cap = std::max(cap, (int)p.maxnneigh);
        cap = std::min(cap, ((p.np + 7) / 8) * 8);
        cap = std::max(cap, 8);
        // rows start on 32-byte boundaries: the pair kernel reads them 16 bytes at a time
        cap = ((cap + 7) / 8) * 8;
        S.cap = cap;
        S.nbl_off = nbl_acc;
        nbl_acc += (long long)cap * p.np;
        S.s = p.lewald == 1 ? p.nmesh : 0;
        S.order = p.order;
        for (int d = 0; d < 3; ++d) S.dkdr[d] = p.lewald == 1 ? (double)p.nmesh / p.boxlen[d] : 0.0;
        S.epsfp = p.epsi_four_pi;
        S.alpha = p.ualpha;
        double q2 = 0.0;
        for (int i = 0; i < p.np; ++i) q2 += p.az[i] * p.az[i];
        S.uself = -(p.ualpha / std::sqrt(3.1415926535897932) * q2);
        S.dt = p.tstep;
        S.type_off = type_tot;
        S.ptmap_off = ptmap_tot;
        S.tile128_off = t128;
        S.ntile128 = (p.np + 127) / 128;
        S.chunk_off = nch;
        S.nchunk = (p.np + SK_CHUNK - 1) / SK_CHUNK;
        S.seed = (uint64_t)s * 0x9E3779B97F4A7C15ull;
        t128 += S.ntile128;
        max_npt = std::max(max_npt, (int)p.npt);
        nch += S.nchunk;
        type_tot += p.npt;
        pt_tot += S.natat;
        ptmap_tot += p.npt * p.npt;
        nbond_tot += (size_t)std::max(0, (int)p.nbond);
        if (p.nbond > 0) has_bonds = 1;
        ntot += p.np;
        hn[s] = p.np;
        H[s].p = p;
        if (p.bd_fac1 && p.bd_fac2) has_bd = 1;
        if (p.lewald) any_ewald = 1;
        if (p.lewald == 1) any_spme = 1;
        if (p.lewald == 2) any_std = 1;
    }
    ncell_tot = cell_tot;
    this->type_tot = type_tot;
    cell_bits = 1;
    while ((1u << cell_bits) <= (unsigned)cell_tot) ++cell_bits;
    nbl_tot = nbl_acc;
    nt128 = t128;
    nchunk = nch;

    // --- SPME grids grouped by edge, one batched cuFFT plan pair per edge ---
    if (any_spme) {
        std::map<int, std::vector<int>> bys;
        for (int s = 0; s < n; ++s)
            if (hs[s].lewald && !hs[s].recstd) bys[hs[s].s].push_back(s);
        long long go = 0, co = 0, fo_acc = 0;
        // MSG_SPME_CONV=1 at handle creation: the convolution kernel takes every edge it
        // supports (the rest stays on cuFFT); the choice depends on the edge alone, so a
        // system's result does not depend on the systems batched with it.  Off by default:
        // on the bench's workloads it runs no faster than the cuFFT chain.
        const char *ev_conv = std::getenv("MSG_SPME_CONV");
        const bool conv_on = ev_conv && std::atoi(ev_conv) != 0;
        std::vector<double2> tw;
        for (auto &kv : bys) {
            const int e = kv.first;
            FftClass fc;
            fc.s = e;
            fc.count = (int)kv.second.size();
            fc.grid_off = go;
            fc.cgrid_off = co;
            fc.rad = conv_on ? conv_radices(e) : 0;
            const int tw_off = (int)tw.size();
            if (fc.rad) {
                // exp(-2 pi i m / e), m = 0..e-1
                for (int m = 0; m < e; ++m) {
                    const long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)e;
                    tw.push_back(make_double2((double)cosl(a), (double)sinl(a)));
                }
                conv_cap = std::max(conv_cap, e * (e / 2 + 1));
            }
            for (int s : kv.second) {
                hs[s].grid_off = go;
                hs[s].cgrid_off = co;
                hs[s].fft_rad = fc.rad;
                hs[s].fft_tw = fc.rad ? tw_off : 0;
                go += (long long)e * e * e;
                co += (long long)e * e * (e / 2 + 1);
            }
            fft.push_back(fc);
        }
        if (!tw.empty()) {
            // tasks in stage order: every FWD plane, then every ZSLAB, then every BWD plane
            std::vector<int4> ct;
            for (int kind = CONV_FWD; kind <= CONV_BWD; ++kind)
                for (int s = 0; s < n; ++s)
                    if (hs[s].lewald && !hs[s].recstd && hs[s].fft_rad)
                        for (int z = 0; z < hs[s].s; ++z) ct.push_back(make_int4(s, kind, z, 0));
            conv_ntasks = (int)ct.size();
            conv_tasks = dalloc<int4>(ct.size());
            up(conv_tasks, ct.data(), ct.size() * sizeof(int4));
            conv_nctr = CONV_HDR + 2 * n;
            conv_ctr = dalloc<unsigned>(conv_nctr);
            std::vector<float2> tw32(tw.size());
            for (size_t k = 0; k < tw.size(); ++k) tw32[k] = make_float2((float)tw[k].x, (float)tw[k].y);
            conv_tw = dalloc<double2>(tw.size());
            conv_tw32 = dalloc<float2>(tw.size());
            up(conv_tw, tw.data(), tw.size() * sizeof(double2));
            up(conv_tw32, tw32.data(), tw32.size() * sizeof(float2));
        }
        for (int s = 0; s < n; ++s)
            if (hs[s].lewald && !hs[s].recstd) {
                const int h = hs[s].s / 2 + 1;
                hs[s].fac_off = fo_acc;
                fo_acc += (long long)h * h * h;
            }
        grid_tot = go;
        cgrid_tot = co;
        // the forward transform is FP64 in both precisions (reciprocal energy and virial);
        // the mixed path transforms back in FP32
        igrid = dalloc<unsigned long long>(grid_tot);
        rgrid = dalloc<double>(grid_tot);
        cgrid = dalloc<double2>(cgrid_tot);
        if (prec == MSG_PREC_MIXED) {
            rgrid32 = dalloc<float>(grid_tot);
            cgrid32 = dalloc<float2>(cgrid_tot);
        }
        std::vector<double> hm(fo_acc), he(fo_acc), hv(fo_acc);
        for (int s = 0; s < n && !dry; ++s)
            if (hs[s].lewald && !hs[s].recstd)
                spme_factors(hs[s].s, hs[s].order, hs[s].alpha, hs[s].box, hm.data() + hs[s].fac_off,
                             he.data() + hs[s].fac_off, hv.data() + hs[s].fac_off);
        mfac = dalloc<double>(fo_acc);
        emf = dalloc<double>(fo_acc);
        vmf = dalloc<double>(fo_acc);
        up(mfac, hm.data(), fo_acc * sizeof(double));
        up(emf, he.data(), fo_acc * sizeof(double));
        up(vmf, hv.data(), fo_acc * sizeof(double));
        plan_fft();
        // influence work items
        std::vector<int4> it;
        for (int s = 0; s < n; ++s) {
            if (!hs[s].lewald || hs[s].recstd || hs[s].fft_rad) continue;
            const int e = hs[s].s;
            const int nc = e * e * (e / 2 + 1);
            hs[s].infl_off = (int)it.size();
            for (int c = 0; c < nc; c += INFL_TILE) it.push_back(make_int4(s, c, std::min(nc, c + INFL_TILE), 0));
            hs[s].ninfl = (int)it.size() - hs[s].infl_off;
        }
        ninfl = (int)it.size();
        infl = dalloc<int4>(ninfl);
        up(infl, it.data(), it.size() * sizeof(int4));
    }


    // --- standard Ewald: k-vectors in the reference's order with kfac, work lists ---
    if (any_std) {
        std::vector<int4> kv, ki, fi, ekv;
        std::vector<double> ekf;
        int ntile = 0;
        std::vector<double> kf;
        long long eik_acc = 0, part_acc = 0, fks_acc = 0;
        int maxw = 0;
        for (int s = 0; s < n; ++s) {
            SysDev &S = hs[s];
            if (!S.recstd) continue;
            const int nc = P[s].ncut;
            const int ncut2 = P[s].ncutregion ? 3 * nc * nc : nc * nc;
            const double tp = 2.0 * 3.1415926535897932, fac0 = tp / S.vol;
            // kfac of EwaldSetup 'std' (Src/energy.F90:6762-6782), in the order the sums visit k
            S.ew_kv_off = (int)kv.size();
            for (int nz = 0; nz <= nc; ++nz) {
                const double facz = nz == 0 ? 1.0 : 2.0;
                for (int ny = 0; ny <= nc; ++ny) {
                    const double facy = ny == 0 ? 0.5 : 1.0;
                    for (int nx = 0; nx <= nc; ++nx) {
                        if (nx * nx + ny * ny + nz * nz > ncut2) continue;
                        if (nx == 0 && ny == 0 && nz == 0) continue;
                        const double facx = nx == 0 ? 0.5 : 1.0;
                        const double kx = nx * (tp * S.boxi[0]), ky = ny * (tp * S.boxi[1]), kz = nz * (tp * S.boxi[2]);
                        const double k2 = kx * kx + ky * ky + kz * kz;
                        kf.push_back(fac0 * facz * facy * facx * std::exp(-k2 / (4.0 * (S.alpha * S.alpha))) / k2);
                        kv.push_back(make_int4(nx, ny, nz, 0));
                    }
                }
            }
            S.ew_nkv = (int)kv.size() - S.ew_kv_off;
            S.ew_ncut = nc;
            maxw = std::max(maxw, nc + 1);
            S.ew_eik_off = eik_acc;
            eik_acc += (long long)S.n * 3 * (nc + 1);
            // chunks of the structure-factor sum (about four blocks per SM of a 148-SM B200) and
            // slices of the force sum (about two): from the system's own sizes only, so a
            // system's sums come out the same whatever else shares the handle
            const int ktiles = (S.ew_nkv + EWK_THREADS - 1) / EWK_THREADS;
            const int nch = std::max(1, std::min((4 * 148 + ktiles - 1) / ktiles, (S.n + 127) / 128));
            S.ew_clen = (S.n + nch - 1) / nch;
            S.ew_nchunk = (S.n + S.ew_clen - 1) / S.ew_clen;
            S.ew_part_off = part_acc;
            part_acc += (long long)S.ew_nchunk * S.ew_nkv;
            for (int kt = 0; kt < ktiles; ++kt, ++ntile)
                for (int c = 0; c < S.ew_nchunk; ++c) ki.push_back(make_int4(s, kt * EWK_THREADS, c, ntile));
            const int ptiles = (S.n + EWF_THREADS - 1) / EWF_THREADS;
            // (a chunk holds at least 128 particles, a slice at least 16 k-vectors; a slice that
            // starts inside a row of n_x first advances its exponentials, at most ncut products)
            const int nks = std::max(1, std::min((2 * 148 + ptiles - 1) / ptiles, std::max(1, S.ew_nkv / 16)));
            S.ew_klen = (S.ew_nkv + nks - 1) / nks;
            S.ew_nks = (S.ew_nkv + S.ew_klen - 1) / S.ew_klen;
            S.ew_fks_off = fks_acc;
            fks_acc += (long long)(S.ew_nks + S.elc) * S.n;     // the layer correction's slice last
            if (S.elc) {
                // EwaldSetup lewald2dlc (Src/energy.F90:6785-6851): ncut2d = ncut, ncut2d2 = ncut2d^2
                // ('sphere') or 2 ncut2d^2 ('cube'); ny outer; kfac2d = -2pi/(Lx Ly) fac /
                // (kp (exp(kp Lz) - 1)) with fac = 4 when nx and ny are both nonzero
                const int c2 = P[s].ncutregion ? 2 * nc * nc : nc * nc;
                const double f0 = tp / (S.box[0] * S.box[1]);
                S.elc_kv_off = (int)ekv.size();
                for (int ny = 0; ny <= nc; ++ny)
                    for (int nx = 0; nx <= nc; ++nx) {
                        if (nx * nx + ny * ny > c2 || (nx == 0 && ny == 0)) continue;
                        const double fac = (nx != 0 && ny != 0) ? 4.0 : 1.0;
                        const double kp = std::sqrt((nx * (tp * S.boxi[0])) * (nx * (tp * S.boxi[0])) +
                                                    (ny * (tp * S.boxi[1])) * (ny * (tp * S.boxi[1])));
                        ekf.push_back(-f0 * fac / (kp * (std::exp(kp * S.box[2]) - 1.0)));
                        ekv.push_back(make_int4(nx, ny, s, 0));
                    }
                S.elc_nkv = (int)ekv.size() - S.elc_kv_off;
            }
            for (int pt = 0; pt < ptiles; ++pt)
                for (int k = 0; k < S.ew_nks; ++k)
                    fi.push_back(make_int4(s, S.off + pt * EWF_THREADS, S.off + std::min(S.n, (pt + 1) * EWF_THREADS), k));
        }
        ew_nk = (int)ki.size();
        ew_ntile = ntile;
        ew_nf = (int)fi.size();
        ew_kv = dalloc<int4>(kv.size());
        ew_kfac = dalloc<double>(kf.size());
        ew_kitems = dalloc<int4>(ki.size());
        ew_tiledone = dalloc<unsigned>(ntile);
        if (!dry) CK(cudaMemsetAsync(ew_tiledone, 0, ntile * sizeof(unsigned), st));
        ew_fitems = dalloc<int4>(fi.size());
        ew_eik = dalloc<double2>(eik_acc);
        ew_part = dalloc<double2>(part_acc * 4);
        ew_sk = dalloc<double2>(kv.size() * 4);
        ew_fks = dalloc<double4>(fks_acc);
        elc_nk = (int)ekv.size();
        if (elc_nk) {
            elc_kv = dalloc<int4>(ekv.size());
            elc_kfac = dalloc<double>(ekf.size());
            elc_st = dalloc<double>(8 * ekv.size());
            up(elc_kv, ekv.data(), ekv.size() * sizeof(int4));
            up(elc_kfac, ekf.data(), ekf.size() * sizeof(double));
        }
        up(ew_kv, kv.data(), kv.size() * sizeof(int4));
        up(ew_kfac, kf.data(), kf.size() * sizeof(double));
        up(ew_kitems, ki.data(), ki.size() * sizeof(int4));
        up(ew_fitems, fi.data(), fi.size() * sizeof(int4));
        ew_smem = (size_t)EW_SUB * 3 * maxw * sizeof(double2);
        ew_nkv_tot = (int)kv.size();
        ew_maxw = maxw;
        if (!dry && ew_smem > 48 * 1024)
            CK(cudaFuncSetAttribute(k_ew_sk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ew_smem));
    }

    // --- pair tables: per type pair, intervals from MOLSIM's ubuf ---
    std::vector<PairTab> pt(pt_tot);
    std::vector<int> pmap(std::max(1, ptmap_tot));
    std::vector<double> vz, vc;
    std::vector<unsigned short> vb;
    std::vector<double> vmassip(type_tot), vmassp(type_tot), vf1(type_tot, 0.0), vf2(type_tot, 0.0);
    for (int s = 0; s < n; ++s) {
        const msg_params &p = P[s];
        SysDev &S = hs[s];
        int pidx = 0;
        for (int it = 0; it < p.npt; ++it)
            for (int jt = it; jt < p.npt; ++jt, ++pidx) {
                pmap[S.ptmap_off + it * p.npt + jt] = S.pt_off + pidx;
                pmap[S.ptmap_off + jt * p.npt + it] = S.pt_off + pidx;
                PairTab &T = pt[S.pt_off + pidx];
                T.k0 = (int)vz.size();
                T.r2umin = p.r2umin[pidx];
                T.r2atat = p.r2atat ? p.r2atat[pidx] : 0.0;
                const int first = p.iubuflow[pidx] - 1;
                if (first < 0 || first + 12 > p.nbuf) throw CudaError{MSG_ERR_ARG, "iubuflow outside ubuf"};
                int k = 0;
                for (;;) {
                    const int b = first + 12 * k;
                    if (b + 12 > p.nbuf) throw CudaError{MSG_ERR_ARG, "pair table does not reach r2umin"};
                    vz.push_back(p.ubuf[b]);
                    for (int c = 0; c < 12; ++c) vc.push_back(p.ubuf[b + c]);
                    ++k;
                    if (p.ubuf[b] <= T.r2umin) break;
                }
                T.nk = k;
                // bucket starts
                const double *z = vz.data() + T.k0;
                T.z_hi = z[0];
                T.z_lo = T.r2umin;
                const double h = (T.z_hi > T.z_lo) ? (T.z_hi - T.z_lo) / MSG_NBUCKET : 1.0;
                T.inv_h = 1.0 / h;
                T.fz_lo = (float)T.z_lo;
                T.fz_hi = (float)T.z_hi;
                T.finv_h = (float)T.inv_h;
                T.b0 = (int)vb.size();
                int stop[MSG_NBUCKET];
                bucket_stops(z, T.nk, T.z_lo, h, 2.0, stop);
                for (int b = 0; b < MSG_NBUCKET; ++b) vb.push_back((unsigned short)stop[b]);
            }
        S.tab_k0 = pt[S.pt_off].k0;
        if ((int)vz.size() - S.tab_k0 > 65535) throw CudaError{MSG_ERR_ARG, "more than 65535 table intervals in one system"};
        S.tab_b0 = pt[S.pt_off].b0;
        S.tab_nk = (int)vz.size() - S.tab_k0;
        {
            const size_t bytes = (prec == MSG_PREC_MIXED) ? pair_smem_bytes<float>(S.tab_nk, S.natat * MSG_NBUCKET)
                                                          : pair_smem_bytes<double>(S.tab_nk, S.natat * MSG_NBUCKET);
            S.tab_smem = bytes <= 96 * 1024 ? 1 : 0;
            if (S.tab_smem) pair_smem = std::max(pair_smem, bytes);
            const size_t bm = lean_smem_bytes(S.tab_nk, S.natat * MSG_NBUCKET);
            S.tab_smem_m = bm <= 96 * 1024 ? 1 : 0;
            if (S.tab_smem_m) pair_smem_m = std::max(pair_smem_m, bm);
            const size_t bh = lean_smem_bytes(S.tab_nk, S.natat * MSG_NBUCKET, ROWST);
            S.tab_smem_h = bh <= 96 * 1024 ? 1 : 0;
            if (S.tab_smem_h) pair_smem_h = std::max(pair_smem_h, bh);
        }
        S.r2umin_max = 0.0;
        S.r2atat_max = 0.0;
        for (int q = 0; q < S.natat; ++q) {
            S.r2umin_max = std::max(S.r2umin_max, pt[S.pt_off + q].r2umin);
            S.r2atat_max = std::max(S.r2atat_max, pt[S.pt_off + q].r2atat);
        }
        for (int t = 0; t < p.npt; ++t) {
            vmassp[S.type_off + t] = p.masspt[t];
            vmassip[S.type_off + t] = p.masspt[t] > 0.0 ? 1.0 / p.masspt[t] : 0.0;
            if (p.bd_fac1) vf1[S.type_off + t] = p.bd_fac1[t];
            if (p.bd_fac2) vf2[S.type_off + t] = p.bd_fac2[t];
        }
    }
    ptab = dalloc<PairTab>(pt.size());
    ptmap = dalloc<int>(pmap.size());
    tz = dalloc<double>(vz.size());
    tc = dalloc<double>(vc.size());
    bst = dalloc<unsigned short>(vb.size());
    bkz = dalloc<int2>(vb.size());
    {
        // lean-kernel buckets: the interval that holds the bucket's top (with 1% of a bucket
        // of slack for the FP32 bucket index), as a row of the system's table, and that
        // interval's z_low in FP32.  A pair below that z_low lies in the next interval unless
        // two interval bounds fall inside one bucket, where the kernel walks as MOLSIM does.
        std::vector<int2> va(vb.size());
        for (int s = 0; s < n; ++s)
            for (int q = 0; q < hs[s].natat; ++q) {
                const PairTab &T = pt[hs[s].pt_off + q];
                const double *z = vz.data() + T.k0;
                const double h = (T.z_hi > T.z_lo) ? (T.z_hi - T.z_lo) / MSG_NBUCKET : 1.0;
                int stop[MSG_NBUCKET];
                bucket_stops(z, T.nk, T.z_lo, h, 1.01, stop);
                for (int b = 0; b < MSG_NBUCKET; ++b) {
                    const int kk = stop[b];
                    float zf = (float)z[kk];
                    int zi;
                    std::memcpy(&zi, &zf, sizeof(zi));
                    va[T.b0 + b] = make_int2(kk + (T.k0 - hs[s].tab_k0), zi);
                }
            }
        up(bkz, va.data(), va.size() * sizeof(int2));
    }
    massip = dalloc<double>(type_tot);
    massp = dalloc<double>(type_tot);
    fac1 = dalloc<double>(type_tot);
    fac2 = dalloc<double>(type_tot);
    up(ptab, pt.data(), pt.size() * sizeof(PairTab));
    up(ptmap, pmap.data(), pmap.size() * sizeof(int));
    up(tz, vz.data(), vz.size() * sizeof(double));
    up(tc, vc.data(), vc.size() * sizeof(double));
    up(bst, vb.data(), vb.size() * sizeof(unsigned short));
    {
        std::vector<float> fz(vz.begin(), vz.end()), fc(vc.begin(), vc.end());
        tz32 = dalloc<float>(fz.size());
        tc32 = dalloc<float>(fc.size());
        up(tz32, fz.data(), fz.size() * sizeof(float));
        up(tc32, fc.data(), fc.size() * sizeof(float));
        if (prec == MSG_PREC_MIXED) {
            // rows of k_pair_h: z_low, c1 and c7 as FP32 (hi, lo) pairs
            const size_t nk = vc.size() / 12;
            std::vector<float> fh(nk * ROWST, 0.0f);
            for (size_t k = 0; k < nk; ++k) {
                const double *c = vc.data() + 12 * k;
                float *o = fh.data() + ROWST * k;
                auto split = [](double v, float *hl) {
                    hl[0] = (float)v;
                    hl[1] = (float)(v - (double)hl[0]);
                };
                split(c[0], o);
                split(c[1], o + 2);
                for (int q = 2; q <= 6; ++q) o[2 + q] = (float)c[q];
                split(c[7], o + 9);
                for (int q = 8; q <= 11; ++q) o[3 + q] = (float)c[q];
            }
            tch = dalloc<float>(fh.size());
            up(tch, fh.data(), fh.size() * sizeof(float));
        }
    }
    up(massip, vmassip.data(), type_tot * sizeof(double));
    up(massp, vmassp.data(), type_tot * sizeof(double));
    up(fac1, vf1.data(), type_tot * sizeof(double));
    up(fac2, vf2.data(), type_tot * sizeof(double));

    // --- bonds: per-particle CSR in MOLSIM order (both ends) ---
    {
        std::vector<int> deg(ntot + 1, 0);
        for (int s = 0; s < n; ++s) {
            const msg_params &p = P[s];
            for (int b = 0; b < p.nbond; ++b) {
                const int a = p.bond_ij[2 * b] - 1, c = p.bond_ij[2 * b + 1] - 1;
                if (a < 0 || c < 0 || a >= p.np || c >= p.np || a == c) throw CudaError{MSG_ERR_ARG, "bad bond"};
                deg[hs[s].off + a + 1]++;
                deg[hs[s].off + c + 1]++;
            }
        }
        for (int i = 0; i < ntot; ++i) deg[i + 1] += deg[i];
        std::vector<int> part(std::max(1, deg[ntot])), pw(std::max(1, deg[ntot]));
        std::vector<double> kk(std::max(1, deg[ntot])), eq(std::max(1, deg[ntot]));
        std::vector<int> fill(deg.begin(), deg.end() - 1);
        for (int s = 0; s < n; ++s) {
            const msg_params &p = P[s];
            for (int b = 0; b < p.nbond; ++b) {
                const int a = p.bond_ij[2 * b] - 1, c = p.bond_ij[2 * b + 1] - 1;
                for (int e = 0; e < 2; ++e) {
                    const int me = e ? c : a, other = e ? a : c;
                    const int slot = fill[hs[s].off + me]++;
                    part[slot] = other;
                    pw[slot] = p.bond_p[b];
                    kk[slot] = p.bond_k[b];
                    eq[slot] = p.bond_eq[b];
                }
            }
        }
        bptr = dalloc<int>(ntot + 1);
        bpart = dalloc<int>(part.size());
        bpw = dalloc<int>(pw.size());
        bk = dalloc<double>(kk.size());
        beq = dalloc<double>(eq.size());
        up(bptr, deg.data(), (ntot + 1) * sizeof(int));
        up(bpart, part.data(), part.size() * sizeof(int));
        up(bpw, pw.data(), pw.size() * sizeof(int));
        up(bk, kk.data(), kk.size() * sizeof(double));
        up(beq, eq.data(), eq.size() * sizeof(double));
        // the bond table, in the initial internal order (MOLSIM order within each system),
        // when no particle has more than two bonds; list rebuilds rewrite it
        int maxdeg = 0;
        for (int i = 0; i < ntot; ++i) maxdeg = std::max(maxdeg, deg[i + 1] - deg[i]);
        if (deg[ntot] > 0 && maxdeg <= 2) {
            std::vector<int4> bt(ntot, make_int4(-1, 0, -1, 0));
            for (int s = 0; s < n; ++s)
                for (int i = 0; i < P[s].np; ++i) {
                    const int g = hs[s].off + i, b0 = deg[g], b1 = deg[g + 1];
                    if (b0 < b1) bt[g].x = hs[s].off + part[b0], bt[g].y = b0 | (i < part[b0] ? BT_COUNT : 0);
                    if (b0 + 1 < b1)
                        bt[g].z = hs[s].off + part[b0 + 1], bt[g].w = (b0 + 1) | (i < part[b0 + 1] ? BT_COUNT : 0);
                }
            btab = dalloc<int4>(ntot);
            up(btab, bt.data(), ntot * sizeof(int4));
        }
    }

    // --- work lists ---
    {
        std::vector<Tile> a128;
        std::vector<PairTask> pt16;
        std::vector<int4> ch;
        for (int s = 0; s < n; ++s) {
            const SysDev &S = hs[s];
            for (int i = 0; i < S.n; i += 128) a128.push_back(Tile{s, S.off + i, S.off + std::min(S.n, i + 128), 0});
            for (int i = 0; i < S.n; i += SK_CHUNK)
                ch.push_back(make_int4(s, S.off + i, S.off + std::min(S.n, i + SK_CHUNK), 0));
        }
        pt16 = make_pair_tasks(0);
        nptask = (int)pt16.size();
        set_pair_chunks(pt16, false);
        psched = dalloc<int>(n + 1);
        this->t128 = dalloc<Tile>(a128.size());
        ptask = dalloc<PairTask>(pt16.size());
        chunks = dalloc<int4>(ch.size());
        up(this->t128, a128.data(), a128.size() * sizeof(Tile));
        up(ptask, pt16.data(), pt16.size() * sizeof(PairTask));
        up(chunks, ch.data(), ch.size() * sizeof(int4));
    }

    // --- particles: MOLSIM order is the initial internal order ---
    for (int b = 0; b < 2; ++b) {
        pos[b] = dalloc<double4>(ntot);
        vel[b] = dalloc<double4>(ntot);
        acc[b] = dalloc<double4>(ntot);
        dsum[b] = dalloc<double4>(ntot);
        fo[b] = dalloc<double4>(ntot);
        typ[b] = dalloc<int>(ntot);
        orig[b] = dalloc<int>(ntot);
    }
    cellid = dalloc<int>(ntot);
    inv = dalloc<int>(ntot);
    sysid = dalloc<int>(ntot);
    fsr = dalloc<double4>(ntot);
    if (prec == MSG_PREC_MIXED) fpart = dalloc<unsigned long long>(3 * (size_t)ntot);
    ftot = dalloc<double4>(ntot);
    posfx = dalloc<int4>(ntot);
    {
        std::vector<double4> hp(ntot);
        std::vector<int> ht(ntot), ho(ntot), hsid(ntot);
        for (int s = 0; s < n; ++s) {
            const msg_params &p = P[s];
            for (int i = 0; i < p.np; ++i) {
                const int g = hs[s].off + i;
                if (p.iptpn[i] < 1 || p.iptpn[i] > p.npt) throw CudaError{MSG_ERR_ARG, "iptpn out of range"};
                hp[g] = make_double4(0.0, 0.0, 0.0, p.az[i]);
                ht[g] = p.iptpn[i] - 1;
                ho[g] = i;
                hsid[g] = s;
            }
        }
        up(pos[0], hp.data(), ntot * sizeof(double4));
        up(typ[0], ht.data(), ntot * sizeof(int));
        up(orig[0], ho.data(), ntot * sizeof(int));
        std::vector<int> idn(ntot);
        for (int i = 0; i < ntot; ++i) idn[i] = i;
        up(inv, idn.data(), ntot * sizeof(int));
        up(sysid, hsid.data(), ntot * sizeof(int));
        // until a system's first list build, its particles sit in its first cell
        std::vector<int> hc(ntot);
        for (int i = 0; i < ntot; ++i) hc[i] = hs[hsid[i]].cell_off;
        up(cellid, hc.data(), ntot * sizeof(int));
    }
    k0 = dalloc<uint32_t>(ntot);
    v0 = dalloc<uint32_t>(ntot);
    k1 = dalloc<uint32_t>(ntot);
    v1 = dalloc<uint32_t>(ntot);
    rhist = dalloc<uint32_t>((size_t)RS_BINS * ((ntot + RS_TILE - 1) / RS_TILE) + RS_BINS);
    cstart = dalloc<int>(ncell_tot);
    cend = dalloc<int>(ncell_tot);
    nbl = dalloc<int>(nbl_tot);
    nnb = dalloc<int>(ntot);
    nmaxrow = dalloc<int>(n);
    r2o = dalloc<double>(ntot);
    skinout = dalloc<double>(2 * (size_t)n);
    sc = dalloc<SkinChunk>(nchunk);
    flag = dalloc<int>(n);
    nrebuild = dalloc<long long>(n);
    istep2 = dalloc<unsigned>(n);
    if (any_llist) llinfo = dalloc<int4>(ntot);
    eacc = dalloc<long long>((size_t)n * EA_N);
    esys = dalloc<double>((size_t)n * ESZ);
    stepctr = dalloc<unsigned long long>(1);
    sstep = dalloc<unsigned long long>(n);
    rdone = dalloc<unsigned>(1);
    fdone = dalloc<unsigned>(n);
    errw = dalloc<ErrWord>(1);
    dsys = dalloc<SysDev>(n);
    up(dsys, hs.data(), n * sizeof(SysDev));
    if (!dry) {
        // persistent pair grid: as many blocks as fit the SMs at once
        int per = 0;
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
#define MSG_PAIR_CFG(PRC, NTV)                                                                           \
    do {                                                                                                \
        CK(cudaFuncSetAttribute(k_pair<PRC, NTV>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));      \
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pair<PRC, NTV>, PAIR_BLOCK, pair_smem)); \
    } while (0)
        if (prec == MSG_PREC_MIXED) {
            if (max_npt <= 2) MSG_PAIR_CFG(PrecM, 2); else MSG_PAIR_CFG(PrecM, 4);
            set_lean_grid(nsm);
        } else {
            if (max_npt <= 2) MSG_PAIR_CFG(PrecD, 2); else MSG_PAIR_CFG(PrecD, 4);
        }
#undef MSG_PAIR_CFG
        pair_blocks_max = nsm * std::max(1, per);
        if (prec != MSG_PREC_MIXED) pair_blocks_lean = pair_blocks_max;
        pair_grid = std::max(1, std::min(nptask, pair_blocks_max));
        if (conv_ntasks) {
            // convolution kernel: one block per SM (a block waiting for its system's
            // previous stage holds its SM's registers and shared memory, which the pair
            // kernel beside it needs), at most as many as the widest stage has tasks.  The shared-memory limit is
            // the kernel's largest (a process-wide attribute, shared by every handle).
            const int smax = (int)conv_smem_bytes(CONV_MAX_SMEM / (2 * (int)sizeof(double2)));
            const int smem = (int)conv_smem_bytes(conv_cap);
            if (prec == MSG_PREC_MIXED) {
                CK(cudaFuncSetAttribute(k_spme_conv<PrecM>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
                CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&conv_occ, k_spme_conv<PrecM>, CONV_THREADS, smem));
            } else {
                CK(cudaFuncSetAttribute(k_spme_conv<PrecD>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
                CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&conv_occ, k_spme_conv<PrecD>, CONV_THREADS, smem));
            }
            conv_occ = std::max(1, conv_occ);
            conv_widest = 0;   // tasks of the widest stage (one per plane or slab of every system)
            for (int s = 0; s < n; ++s)
                if (hs[s].lewald && !hs[s].recstd && hs[s].fft_rad) conv_widest += hs[s].s;
            set_conv_grid(0);
        }
    }
    if (!dry) CK(cudaStreamSynchronize(st));
}

// Grid of the convolution kernel: per_sm blocks on every SM (at most as many as
// fit), or with per_sm = 0 one per SM and at most one per task of the widest stage.
void msg_handle::set_conv_grid(int per_sm)
{
    if (!conv_ntasks) return;
    conv_grid = per_sm > 0 ? std::min(conv_ntasks, nsm * std::min(per_sm, conv_occ)) : std::min(conv_widest, nsm);
    conv_grid = std::max(1, conv_grid);
}

// Persistent grid of the lean pair kernel for its current unroll: as many
// blocks as fit the SMs at once.
void msg_handle::set_lean_grid(int nsm)
{
    int perm = 0;
#define MSG_LEAN_OCC(NTV, UV)                                                                                \
    do {                                                                                                     \
        int ph = 0;                                                                                          \
        CK(cudaFuncSetAttribute(k_pair_m<NTV, UV>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024)); \
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perm, k_pair_m<NTV, UV>, PAIR_BLOCK, pair_smem_m)); \
        CK(cudaFuncSetAttribute(k_pair_h<NTV, UV, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024)); \
        CK(cudaFuncSetAttribute(k_pair_h<NTV, UV, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024)); \
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ph, k_pair_h<NTV, UV, true>, PAIR_BLOCK, pair_smem_h)); \
        perm = std::min(perm, ph);                                                                           \
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ph, k_pair_h<NTV, UV, false>, PAIR_BLOCK, pair_smem_h)); \
        perm = std::min(perm, ph);                                                                           \
    } while (0)
    if (max_npt <= 2) {
        if (pair_unroll == 1) MSG_LEAN_OCC(2, 1); else if (pair_unroll == 2) MSG_LEAN_OCC(2, 2); else MSG_LEAN_OCC(2, 4);
    } else {
        if (pair_unroll == 1) MSG_LEAN_OCC(4, 1); else if (pair_unroll == 2) MSG_LEAN_OCC(4, 2); else MSG_LEAN_OCC(4, 4);
    }
#undef MSG_LEAN_OCC
    pair_blocks_lean = nsm * std::max(1, perm);
}

// Warp tasks of the pair kernel: 32/G consecutive particles of one system, G
// lanes per particle.  G follows the expected full-list row (about four row
// entries per lane), scaled by 2^shift (the pair-lane tuning knob), 2..32.
std::vector<PairTask> msg_handle::make_pair_tasks(int shift) const
{
    std::vector<PairTask> pt;
    for (int s = 0; s < nsys; ++s) {
        const SysDev &S = hs[s];
        const double rl = std::sqrt(S.rs2cut);
        const double nrow = S.n / S.vol * 4.0 / 3.0 * 3.1415926535897932 * rl * rl * rl * (list_half ? 0.5 : 1.0);
        int G = 4;
        while (G < 32 && 2 * G <= nrow / 4.0) G *= 2;
        for (int k = 0; k < shift && G < 32; ++k) G *= 2;
        for (int k = 0; k > shift && G > 2; --k) G /= 2;
        const int per = 32 / G;
        const size_t first = pt.size();
        for (int i = 0; i < S.n; i += per)
            pt.push_back(PairTask{s, S.off + i, S.off + std::min(S.n, i + per), G, 0, 0, 0, 0});
        for (size_t q = first; q < pt.size(); ++q) pt[q].send = (int)pt.size();
    }
    return pt;
}

// Each system's task range for the lean pair kernel's per-system counters.
void msg_handle::set_pair_chunks(const std::vector<PairTask> &pt, bool replace)
{
    std::vector<int2> r(nsys, make_int2(0, 0));
    std::vector<int> gs(nsys, 32);
    for (size_t a = 0; a < pt.size();) {
        const int end = pt[a].send;
        r[pt[a].sys] = make_int2((int)a, end);
        gs[pt[a].sys] = pt[a].g;
        a = (size_t)end;
    }
    if (replace) {
        dfree(psrange);
        dfree(pgsys);
    }
    psrange = dalloc<int2>(nsys);
    up(psrange, r.data(), r.size() * sizeof(int2));
    pgsys = dalloc<int>(nsys);
    up(pgsys, gs.data(), gs.size() * sizeof(int));
}

void msg_handle::set_pair_lanes(int shift, bool force)
{
    if (shift == pair_shift && !force) return;
    drop_graph();
    CK(cudaStreamSynchronize(st));
    std::vector<PairTask> pt = make_pair_tasks(shift);
    dfree(ptask);
    ptask = dalloc<PairTask>(pt.size());
    up(ptask, pt.data(), pt.size() * sizeof(PairTask));
    nptask = (int)pt.size();
    set_pair_chunks(pt, true);
    pair_grid = std::max(1, std::min(nptask, pair_blocks_max));
    pair_shift = shift;
    CK(cudaStreamSynchronize(st));
}

// Split each grid class into power-of-two sub-batches and take their plans
// from the cache; one work area (the largest any plan asks for) serves them
// all, since a handle runs its transforms one after another on its stream.
void msg_handle::plan_fft()
{
    const int f32 = prec == MSG_PREC_MIXED ? 1 : 0;
    size_t need = 0;
    for (auto &fc : fft) {
        if (fc.rad) continue;   // the convolution kernel's edge
        long long go = fc.grid_off, co = fc.cgrid_off;
        const long long rs = (long long)fc.s * fc.s * fc.s, cs = (long long)fc.s * fc.s * (fc.s / 2 + 1);
        for (int bit = 30; bit >= 0; --bit) {
            const int c = 1 << bit;
            if (!(fc.count & c)) continue;
            FftPart part;
            part.count = c;
            part.grid_off = go;
            part.cgrid_off = co;
            go += rs * c;
            co += cs * c;
            for (int dir = 1; dir >= 0; --dir) {
                // forward D2Z in both precisions; backward C2R (mixed) or Z2D (FP64)
                const PlanKey key{fc.s, c, dir ? 0 : f32, dir};
                cufftHandle hp = 0;
                size_t ws = 0;
                if (dry) {
                    // the estimate depends on the plan's shape only: asked once per shape
                    static std::mutex est_mu;
                    static std::map<PlanKey, size_t> est_cache;
                    std::lock_guard<std::mutex> lk(est_mu);
                    auto it = est_cache.find(key);
                    if (it != est_cache.end()) {
                        ws = it->second;
                    } else {
                        int dims[3] = {fc.s, fc.s, fc.s};
                        const cufftType t = dir ? CUFFT_D2Z : (f32 ? CUFFT_C2R : CUFFT_Z2D);
                        // without a device cuFFT cannot estimate: assume one complex grid per transform
                        if (cufftEstimateMany(3, dims, nullptr, 1, dir ? (int)rs : (int)cs, nullptr, 1,
                                              dir ? (int)cs : (int)rs, t, c, &ws) != CUFFT_SUCCESS)
                            ws = (size_t)c * (size_t)cs * (key.f32 ? sizeof(float2) : sizeof(double2));
                        est_cache[key] = ws;
                    }
                } else {
                    {
                        std::lock_guard<std::mutex> lk(g_plan_mu);
                        auto &v = g_plan_idle[key];
                        if (!v.empty()) {
                            hp = v.back().first;
                            ws = v.back().second;
                            v.pop_back();
                        }
                    }
                    if (!hp) CKF(make_plan(key, &hp, &ws));
                }
                (dir ? part.fwd : part.bwd) = hp;
                (dir ? part.ws_fwd : part.ws_bwd) = ws;
                need = std::max(need, ws);
            }
            fc.parts.push_back(part);
        }
    }
    fftwork = dalloc<unsigned char>(std::max<size_t>(need, 1));
    if (dry) return;
    for (auto &fc : fft)
        for (auto &pt : fc.parts)
            for (cufftHandle hp : {pt.fwd, pt.bwd}) {
                CKF(cufftSetWorkArea(hp, fftwork));
                CKF(cufftSetStream(hp, st));
            }
}

void msg_handle::release_fft()
{
    const int f32 = prec == MSG_PREC_MIXED ? 1 : 0;
    std::lock_guard<std::mutex> lk(g_plan_mu);
    for (auto &fc : fft)
        for (auto &pt : fc.parts) {
            if (pt.fwd) g_plan_idle[PlanKey{fc.s, pt.count, 0, 1}].push_back({pt.fwd, pt.ws_fwd});
            if (pt.bwd) g_plan_idle[PlanKey{fc.s, pt.count, f32, 0}].push_back({pt.bwd, pt.ws_bwd});
        }
    fft.clear();
}

// ---------------------------------------------------------------------------
// Kernel sequences.
// ---------------------------------------------------------------------------
void msg_handle::enqueue_rebuild()
{
    // cur stays 0: rebuilt systems are permuted into the [1] buffers and copied home
    tbeg(TM_REBUILD);
    k_rb_keys<<<nt128, 128, 0, st>>>(dsys, t128, flag, pos[0], orig[0], cellid, k0, v0, cstart, cend, ncell_tot);
    int nsort = 0;
    const bool in1 = radix_sort_pairs(k0, v0, k1, v1, rhist, ntot, cell_bits, st, &nsort);
    const uint32_t *sk = in1 ? k1 : k0, *sv = in1 ? v1 : v0;
    k_permute<<<nt128, 128, 0, st>>>(dsys, t128, flag, sk, sv, pos[0], pos[1], vel[0], vel[1], acc[0], acc[1],
                                      fo[0], fo[1], typ[0], typ[1], orig[0], orig[1], cellid, inv, cstart, cend,
                                      ntot);
    k_copyback<<<nt128, 128, 0, st>>>(dsys, t128, flag, pos[0], pos[1], vel[0], vel[1], acc[0], acc[1], fo[0],
                                       fo[1], typ[0], typ[1], orig[0], orig[1], dsum[0], posfx);
    if (btab) {
        k_bond_table<<<nt128, 128, 0, st>>>(dsys, t128, flag, orig[0], inv, bptr, bpart, btab);
        launches += 1;
    }
    if (any_llist) {
        k_llist_info<<<nt128, 128, 0, st>>>(dsys, t128, flag, pos[0], llinfo);
        launches += 1;
    }
    k_nlist<<<(ntot * 32 + 255) / 256, 256, 0, st>>>(dsys, sysid, flag, pos[0], typ[0], cellid, cstart, cend, nbl,
                                                     nnb, ntot, nmaxrow, errw, list_half, orig[0], llinfo);
    tend(TM_REBUILD);
    launches += 4 + nsort;
}

template <int P, class PR>
static void launch_spme(msg_handle *h)
{
    h->tbeg(TM_SPREAD);
    k_spread<P, PR><<<h->nt128 * (128 / SPREAD_PART), SPREAD_THREADS, 0, h->st>>>(h->dsys, h->t128, h->pos[0], h->rgrid, h->igrid,
                                                  h->eacc);
    h->launches += 1;
    bool cufft = false;
    for (auto &fc : h->fft) {
        if (fc.rad) continue;
        // cuFFT edges: the fixed-point grid to the FP64 input of the forward transform
        const long long ng = (long long)fc.count * fc.s * fc.s * fc.s;
        k_grid_to_f64<<<(unsigned)((ng + 255) / 256), 256, 0, h->st>>>(h->igrid + fc.grid_off, h->rgrid + fc.grid_off, ng);
        h->launches += 1;
        cufft = true;
    }
    h->tend(TM_SPREAD);
    if (h->conv_ntasks) {
        h->tbeg(TM_FFT);
        k_spme_conv<PR><<<h->conv_grid, CONV_THREADS, conv_smem_bytes(h->conv_cap), h->st>>>(
            h->dsys, h->conv_tasks, h->conv_ntasks, h->conv_cap, h->igrid, h->cgrid, h->cgrid32, h->rgrid,
            h->rgrid32, h->conv_tw, h->conv_tw32, h->mfac, h->emf, h->vmf, h->eacc, h->conv_ctr, h->conv_nctr,
            h->errw);
        h->launches += 1;
        h->tend(TM_FFT);
    }
    if (!cufft) return;
    h->tbeg(TM_FFT);
    for (auto &fc : h->fft)
        for (auto &f : fc.parts)
            CKF(cufftExecD2Z(f.fwd, h->rgrid + f.grid_off, reinterpret_cast<cufftDoubleComplex *>(h->cgrid + f.cgrid_off)));
    h->tend(TM_FFT);
    h->tbeg(TM_INFL);
    k_influence<PR><<<h->ninfl, INFL_THREADS, 0, h->st>>>(h->dsys, h->infl, h->cgrid, h->cgrid32, h->mfac, h->emf,
                                                          h->vmf, h->eacc);
    h->launches += 1;
    h->tend(TM_INFL);
    h->tbeg(TM_FFT);
    for (auto &fc : h->fft)
        for (auto &f : fc.parts) {
            if (PR::mixed)
                CKF(cufftExecC2R(f.bwd, reinterpret_cast<cufftComplex *>(h->cgrid32 + f.cgrid_off),
                                 h->rgrid32 + f.grid_off));
            else
                CKF(cufftExecZ2D(f.bwd, reinterpret_cast<cufftDoubleComplex *>(h->cgrid + f.cgrid_off),
                                 h->rgrid + f.grid_off));
        }
    h->tend(TM_FFT);
}

template <int P, class PR>
static void launch_finalize(msg_handle *h, int mode, bool record)
{
    FinOut fo;
    fo.esys = h->esys;
    fo.hist = record ? h->hist : nullptr;
    fo.hist_cap = h->hist_cap;
    fo.nsys = h->nsys;
    fo.stepctr = h->stepctr;
    fo.sstep = h->sstep;
    fo.fdone = h->fdone;
    fo.alldone = h->rdone;
    h->tbeg(TM_FINAL);
    h->launches += 1;
    k_finalize<P, PR><<<h->nt128 * FIN_SPLIT, FIN_THREADS, 0, h->st>>>(
        h->dsys, h->t128, h->pos[0], h->typ[0], h->rgrid, h->rgrid32, h->fsr, h->list_half ? h->fpart : nullptr,
        h->ntot, FinBonds{h->orig[0], h->inv, h->has_bonds ? h->bptr : nullptr, h->bpart, h->bpw, h->bk, h->beq,
                          h->has_bonds ? h->btab : nullptr},
        h->ew_fks, h->eacc, h->massip, h->massp,
        h->ftot, h->fo[0], h->vel[0], h->acc[0], mode, fo, h->errw);
    h->tend(TM_FINAL);
}

// Standard Ewald chain (tables; partial structure factors reduced by each k tile's
// last chunk, with the energy and virial; force slices); the finalize kernel adds
// the slices.
static void launch_ewald_std(msg_handle *h)
{
    h->tbeg(TM_EWSTD);
    k_ew_eik<<<h->nt128, 128, 0, h->st>>>(h->dsys, h->t128, h->pos[0], h->ew_eik, h->eacc);
    k_ew_sk<<<h->ew_nk, EWK_THREADS, h->ew_smem, h->st>>>(h->dsys, h->ew_kitems, h->ew_kv, h->ew_kfac, h->ew_eik,
                                                          h->ew_part, h->ew_sk, h->ew_tiledone, h->eacc);
    k_ew_force<<<h->ew_nf, EWF_THREADS, 0, h->st>>>(h->dsys, h->ew_fitems, h->pos[0], h->ew_kv, h->ew_kfac, h->ew_sk,
                                                    h->ew_fks);
    h->launches += 3;
    if (h->elc_nk) {
        k_elc_sum<<<h->elc_nk, ELC_THREADS, 0, h->st>>>(h->dsys, h->elc_kv, h->elc_kfac, h->pos[0], h->elc_st, h->eacc);
        k_elc_force<<<h->nt128, 128, 0, h->st>>>(h->dsys, h->t128, h->pos[0], h->elc_kv, h->elc_kfac, h->elc_st,
                                                 h->ew_fks);
        h->launches += 2;
    }
    h->tend(TM_EWSTD);
}

template <class PR>
static void launch_forces(msg_handle *h, int mode, bool record, bool skin)
{
    // The pair kernel and the SPME chain (spread, FFT, influence, FFT) read
    // different inputs and add into different accumulators: the pair kernel runs
    // on a second stream beside the chain and finalize waits for both.  (Per-kernel
    // timers need one stream, so timing serialises them.)
    const bool par = h->overlap && h->any_ewald && !h->timing;
    cudaStream_t ps = h->st;
    if (par) {
        CK(cudaEventRecord(h->ev_fork, h->st));
        CK(cudaStreamWaitEvent(h->st2, h->ev_fork, 0));
        ps = h->st2;
    }
    if (skin) {
        // the skin test's combine: needed only by the rebuild at the end of the step
        k_skin_combine<<<h->nsys, SK_THREADS, 0, ps>>>(h->dsys, h->r2o, h->sc, h->flag, h->nrebuild, h->skinout,
                                                       h->cond, h->use_cond, h->istep2);
        h->launches += 1;
    }
    h->tbeg(TM_PAIR);
    const typename PR::V4 *pp =
        reinterpret_cast<const typename PR::V4 *>(PR::mixed ? (const void *)h->posfx : (const void *)h->pos[0]);
    const typename PR::R *tzp = reinterpret_cast<const typename PR::R *>(PR::mixed ? (const void *)h->tz32 : (const void *)h->tz);
    const typename PR::R *tcp = reinterpret_cast<const typename PR::R *>(PR::mixed ? (const void *)h->tc32 : (const void *)h->tc);
    if (PR::mixed && h->pair_lean >= 2) {
        const int per_sm = h->pair_per_sm > 0 ? h->pair_per_sm : (par ? 2 : 0);
        const int cap = per_sm > 0 ? std::min(h->pair_blocks_lean, h->nsm * per_sm) : h->pair_blocks_lean;
        const int grid = std::max(1, std::min(h->nptask, cap));
#define MSG_HALF1(NTV, UV, HV)                                                                              \
    k_pair_h<NTV, UV, HV><<<grid, PAIR_BLOCK, h->pair_smem_h, ps>>>(h->dsys, h->pgsys, h->psrange, h->nsys,    \
                                                                    h->nptask, h->psched, h->posfx, h->typ[0], \
                                                                    h->nbl, h->nnb, h->ptmap, h->ptab, h->tch, \
                                                                    h->bkz, h->fsr, h->fpart, h->ntot, h->eacc, \
                                                                    h->errw)
#define MSG_HALF(NTV, UV)                          \
    do {                                           \
        if (h->list_half) MSG_HALF1(NTV, UV, true); \
        else MSG_HALF1(NTV, UV, false);            \
    } while (0)
        if (h->max_npt <= 2) {
            if (h->pair_unroll == 1) MSG_HALF(2, 1); else if (h->pair_unroll == 2) MSG_HALF(2, 2); else MSG_HALF(2, 4);
        } else {
            if (h->pair_unroll == 1) MSG_HALF(4, 1); else if (h->pair_unroll == 2) MSG_HALF(4, 2); else MSG_HALF(4, 4);
        }
#undef MSG_HALF
#undef MSG_HALF1
    } else if (PR::mixed && h->pair_lean) {
        // beside the SPME chain the pair kernel leaves room on each SM for the chain's blocks
        const int per_sm = h->pair_per_sm > 0 ? h->pair_per_sm : (par ? 2 : 0);
        const int cap = per_sm > 0 ? std::min(h->pair_blocks_lean, h->nsm * per_sm) : h->pair_blocks_lean;
        const int grid = std::max(1, std::min(h->nptask, cap));
#define MSG_LEAN(NTV, UV)                                                                                   \
    k_pair_m<NTV, UV><<<grid, PAIR_BLOCK, h->pair_smem_m, ps>>>(h->dsys, h->ptask, h->psrange, h->nsys,        \
                                                                h->nptask, h->psched, h->posfx,           \
                                                                   h->typ[0], h->nbl, h->nnb, h->ptmap,    \
                                                                   h->ptab, h->tc32, h->bkz, h->fsr,       \
                                                                   h->eacc, h->errw)
        if (h->max_npt <= 2) {
            if (h->pair_unroll == 1) MSG_LEAN(2, 1); else if (h->pair_unroll == 2) MSG_LEAN(2, 2); else MSG_LEAN(2, 4);
        } else {
            if (h->pair_unroll == 1) MSG_LEAN(4, 1); else if (h->pair_unroll == 2) MSG_LEAN(4, 2); else MSG_LEAN(4, 4);
        }
#undef MSG_LEAN
    } else if (h->max_npt <= 2)
        k_pair<PR, 2><<<h->pair_grid, PAIR_BLOCK, h->pair_smem, ps>>>(h->dsys, h->ptask, h->nptask, pp, h->typ[0], h->nbl,
                                                              h->nnb, h->ptmap, h->ptab, tzp, tcp, h->bst, h->fsr,
                                                              h->eacc, h->errw);
    else
        k_pair<PR, 4><<<h->pair_grid, PAIR_BLOCK, h->pair_smem, ps>>>(h->dsys, h->ptask, h->nptask, pp, h->typ[0], h->nbl,
                                                              h->nnb, h->ptmap, h->ptab, tzp, tcp, h->bst, h->fsr,
                                                              h->eacc, h->errw);
    h->tend(TM_PAIR);
    h->launches += 1;
    if (h->any_std) launch_ewald_std(h);
    if (h->any_spme) {
        switch (h->order) {
        case 4: launch_spme<4, PR>(h); break;
        case 5: launch_spme<5, PR>(h); break;
        default: launch_spme<6, PR>(h); break;
        }
    }
    if (par) {
        CK(cudaEventRecord(h->ev_join, h->st2));
        CK(cudaStreamWaitEvent(h->st, h->ev_join, 0));
    }
    switch (h->order) {
    case 4: launch_finalize<4, PR>(h, mode, record); break;
    case 5: launch_finalize<5, PR>(h, mode, record); break;
    default: launch_finalize<6, PR>(h, mode, record); break;
    }
}

void msg_handle::enqueue_forces(int mode, bool record, bool skin)
{
    if (prec == MSG_PREC_MIXED)
        launch_forces<PrecM>(this, mode, record, skin);
    else
        launch_forces<PrecD>(this, mode, record, skin);
}

void msg_handle::enqueue_md_step(bool record)
{
    tbeg(TM_POS);
    k_vv_skin<<<nchunk, SK_THREADS, 0, st>>>(dsys, chunks, inv, pos[0], vel[0], acc[0], dsum[0], posfx, r2o, sc);
    tend(TM_POS);
    launches += 1;
    if (io_ro) {
        // the new positions are final: send them to the host beside the force work
        CK(cudaEventRecord(ev_io0, st));
        CK(cudaStreamWaitEvent(st3, ev_io0, 0));
        const int nb = (hs[io_ro_sys].n + STATE_BLOCK - 1) / STATE_BLOCK;
        k_state_out<<<nb, STATE_BLOCK, 0, st3>>>(dsys, io_ro_sys, pos[0], vel[0], acc[0], io_ro, nullptr, nullptr, inv);
        launches += 1;
        CK(cudaEventRecord(ev_io1, st3));
    }
    enqueue_forces(1, record, true);
    if (!use_cond) enqueue_rebuild();
}

void msg_handle::enqueue_bd_step(uint64_t seed, const double *xin_step, double *xout_step, bool record)
{
    tbeg(TM_POS);
    k_bd_skin<<<nchunk, SK_THREADS, 0, st>>>(dsys, chunks, inv, pos[0], fo[0], dsum[0], typ[0], fac1, fac2, xin_step,
                                             xout_step, seed, sstep, posfx, r2o, sc);
    tend(TM_POS);
    launches += 1;
    enqueue_forces(0, record, true);
    if (!use_cond) enqueue_rebuild();
}

// Row capacity follows the longest row seen (x1.5 + 32).  When a system's rows
// outgrow it, every list is re-laid out and rebuilt.  Returns true on growth.
bool msg_handle::grow_lists(const int *mx_host)
{
    std::vector<int> mx(nsys);
    if (mx_host)
        std::memcpy(mx.data(), mx_host, nsys * sizeof(int));
    else
        down(mx.data(), nmaxrow, nsys * sizeof(int));
    bool grow = false;
    std::vector<int> cap(nsys);
    for (int s = 0; s < nsys; ++s) {
        int need = (int)std::ceil(1.5 * mx[s]) + 32;
        need = std::min(((need + 7) / 8) * 8, std::max(8, ((hs[s].n + 7) / 8) * 8));
        cap[s] = hs[s].cap;
        if (alloc_log && need > hs[s].cap)
            std::fprintf(stderr, "msg grow system %d: n %d longest row %d cap %d -> %d\n", s, hs[s].n, mx[s],
                         hs[s].cap, need);
        if (need > hs[s].cap) {
            cap[s] = need;
            grow = true;
        }
    }
    if (!grow) return false;
    drop_graph();
    long long acc = 0;
    for (int s = 0; s < nsys; ++s) {
        hs[s].cap = cap[s];
        hs[s].nbl_off = acc;
        acc += (long long)cap[s] * hs[s].n;
    }
    CK(cudaStreamSynchronize(st));
    dfree(nbl);
    nbl = dalloc<int>(acc);
    nbl_tot = acc;
    up(dsys, hs.data(), nsys * sizeof(SysDev));
    return true;
}

// Rebuild the flagged systems; on a capacity overflow grow the rows and rebuild all.
int msg_handle::rebuild_checked(const std::vector<int> &flags)
{
    h2d(flag, flags.data(), nsys, st);
    enqueue_rebuild();
    int rc = check();
    for (int attempt = 0; attempt < 3; ++attempt) {
        if (rc != MSG_OK && rc != MSG_ERR_CAPACITY) return rc;
        if (!grow_lists()) return rc;
        std::vector<int> all(placed.begin(), placed.end());
        h2d(flag, all.data(), nsys, st);
        enqueue_rebuild();
        rc = check();
    }
    return rc;
}

void msg_handle::drop_one(StepGraph &gr)
{
    if (gr.exec) cudaGraphExecDestroy(gr.exec);
    for (cudaEvent_t e : gr.ta) cudaEventDestroy(e);
    for (cudaEvent_t e : gr.tb) cudaEventDestroy(e);
    gr = StepGraph();
}

void msg_handle::drop_graph()
{
    drop_one(graph);
    drop_one(iograph);
}

void msg_handle::ensure_graph(int kind, bool record, uint64_t seed)
{
    if (graph.exec && graph.kind == kind && graph.record == record && graph.timing == timing &&
        (kind == 0 || graph.seed == seed) && graph.hist == (record ? hist : nullptr) &&
        graph.hist_cap == (record ? hist_cap : 0))
        return;
    drop_one(graph);
    double *none[3] = {nullptr, nullptr, nullptr};
    build_graph(graph, kind, record, seed, -1, none);
}

// One MD step with the host exchange of msg_velver_host on page-locked arrays:
// the conversion kernels read and write the caller's arrays in place, and the
// read-backs follow the rebuild node -- one launch, one wait.
void msg_handle::ensure_io_graph(bool record, int io_sys, double *const io[3])
{
    if (iograph.exec && iograph.record == record && iograph.io_sys == io_sys && iograph.io[0] == io[0] &&
        iograph.io[1] == io[1] && iograph.io[2] == io[2] && iograph.hist == (record ? hist : nullptr) &&
        iograph.hist_cap == (record ? hist_cap : 0) && !timing)
        return;
    drop_one(iograph);
    build_graph(iograph, 0, record, 0, io_sys, io);
}

void msg_handle::build_graph(StepGraph &gr, int kind, bool record, uint64_t seed, int io_sys, double *const io[3])
{
    CK(cudaStreamSynchronize(st));
    flush_timers();
    cudaGraph_t g;
    CK(cudaGraphCreate(&g, 0));
    CK(cudaGraphConditionalHandleCreate(&cond, g, 0u, cudaGraphCondAssignDefault));
    const long long l0 = launches;
    const size_t p0 = pend_k.size();
    CK(cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    capturing = true;
    use_cond = 1;
    if (io_sys >= 0) {
        // io[] are the mapped device addresses of the caller's page-locked arrays:
        // the conversion kernels read and write them directly, no staging copies
        const int nb = (hs[io_sys].n + STATE_BLOCK - 1) / STATE_BLOCK;
        k_state_in<<<nb, STATE_BLOCK, 0, st>>>(dsys, io_sys, io[0], io[1], io[2], pos[0], vel[0], acc[0], posfx, inv,
                                               record ? stepctr : nullptr);
        launches += 1;
        io_ro = io[0];
        io_ro_sys = io_sys;
    }
    if (kind == 0)
        enqueue_md_step(record);
    else
        enqueue_bd_step(seed, nullptr, nullptr, record);
    io_ro = nullptr;
    io_ro_sys = -1;
    if (io_sys >= 0) {
        if (io[1] || io[2]) {
            const int nb = (hs[io_sys].n + STATE_BLOCK - 1) / STATE_BLOCK;
            k_state_out<<<nb, STATE_BLOCK, 0, st>>>(dsys, io_sys, pos[0], vel[0], acc[0], nullptr, io[1], io[2], inv);
            launches += 1;
        }
        if (io[0] && kind == 0) CK(cudaStreamWaitEvent(st, ev_io1, 0));
    }
    use_cond = 0;
    // the rebuild: an IF node after everything captured so far
    tbeg(TM_REBUILD);
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    CK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &nd));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t cn;
    CK(cudaGraphAddNode(&cn, g, deps, nd, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CK(cudaStreamUpdateCaptureDependencies(st, &cn, 1, cudaStreamSetCaptureDependencies));
    if (io_sys >= 0) {
        // read-backs after the rebuild, straight into the mapped pinned block: the
        // longest rows (list growth), the energies, the error word
        k_readback<<<1, 256, 0, st>>>(nmaxrow, nsys, record ? hist : nullptr, record ? nsys * ESZ : 0, errw,
                                      map_host(pin_rows()), record ? map_host(pin_hist((size_t)nsys * ESZ)) : nullptr,
                                      map_host(pin_err()));
        launches += 1;
    }
    cudaEvent_t rb_begin = timing ? open_ev[TM_REBUILD] : nullptr;
    if (timing) {
        cudaEvent_t b = get_event();
        rec_event(b);
        pend_k.push_back(TM_REBUILD);
        pend_a.push_back(rb_begin);
        pend_b.push_back(b);
    }
    CK(cudaStreamEndCapture(st, &g));
    capturing = false;
    // capture the rebuild into the body graph (timers off inside: the IF node is timed as a whole)
    const bool tsave = timing;
    timing = false;
    CK(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    enqueue_rebuild();
    cudaGraph_t bdone;
    CK(cudaStreamEndCapture(st, &bdone));
    timing = tsave;
    CK(cudaGraphInstantiate(&gr.exec, g, 0));
    CK(cudaGraphDestroy(g));
    gr.kind = kind;
    gr.record = record;
    gr.timing = timing;
    gr.seed = seed;
    gr.hist = record ? hist : nullptr;
    gr.hist_cap = record ? hist_cap : 0;
    gr.launches = launches - l0;
    gr.io_sys = io_sys;
    for (int k = 0; k < 3; ++k) gr.io[k] = io[k];
    launches = l0;
    // events captured as graph nodes stay with the graph and are read after each launch
    for (size_t q = p0; q < pend_k.size(); ++q) {
        gr.tk.push_back(pend_k[q]);
        gr.ta.push_back(pend_a[q]);
        gr.tb.push_back(pend_b[q]);
    }
    pend_k.resize(p0);
    pend_a.resize(p0);
    pend_b.resize(p0);
}

void msg_handle::launch_graph() { launch_one(graph); }

void msg_handle::launch_one(StepGraph &gr)
{
    CK(cudaGraphLaunch(gr.exec, st));
    launches += gr.launches;
    if (gr.timing) {
        // the graph's event nodes are re-recorded by every launch: read them now
        CK(cudaStreamSynchronize(st));
        for (size_t q = 0; q < gr.tk.size(); ++q) {
            float ms = 0.0f;
            CK(cudaEventElapsedTime(&ms, gr.ta[q], gr.tb[q]));
            tm_ms[gr.tk[q]] += ms;
            tm_n[gr.tk[q]] += 1;
        }
    }
}

int msg_handle::check()
{
    ErrWord e;
    if (pin) {
        // the error word rides with whatever reads the caller queued: one wait
        CK(cudaMemcpyAsync(pin_err(), errw, sizeof(ErrWord), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        e = *pin_err();
    } else {
        CK(cudaStreamSynchronize(st));
        down(&e, errw, sizeof(e));
    }
    CK(cudaGetLastError());
    flush_timers();
    return check_word(e);
}

// Turns a device error word into a status and message, and clears what an aborted
// step may have left behind.
int msg_handle::check_word(const ErrWord &e)
{
    if (e.code) {
        static const char *names[] = {"ok", "r2 < r2umin (pair below the table minimum)", "table interval overrun",
                                      "neighbour-list capacity exceeded", "cuda", "device timeout", "argument",
                                      "non-finite force", "hard-core overlap"};
        char buf[256];
        std::snprintf(buf, sizeof(buf), "%s (system %d, particles %d, %d)",
                      (e.code >= 0 && e.code <= 8) ? names[e.code] : "error", e.sys, e.i, e.j);
        err = buf;
        const int code = e.code;
        CK(cudaMemsetAsync(errw, 0, sizeof(ErrWord), st));
        // an aborted step may leave partial sums and counters behind
        CK(cudaMemsetAsync(eacc, 0, sizeof(long long) * nsys * EA_N, st));
        CK(cudaMemsetAsync(fdone, 0, sizeof(unsigned) * nsys, st));
        CK(cudaMemsetAsync(rdone, 0, sizeof(unsigned), st));
        CK(cudaMemsetAsync(psched, 0, (nsys + 1) * sizeof(int), st));
        CK(cudaStreamSynchronize(st));
        return code;
    }
    return MSG_OK;
}

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
#define API_BEGIN try {
#define API_END                                       \
    }                                                 \
    catch (const CudaError &e) {                      \
        if (h) h->err = e.what;                       \
        return e.code;                                \
    }

// The device's default memory pool keeps freed blocks for reuse instead of
// returning them at every synchronisation (a process-local attribute).
static void keep_pool_blocks()
{
    static std::once_flag once;
    std::call_once(once, [] {
        int dev = 0;
        cudaMemPool_t pool;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t keep = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    });
}

static int create_impl(const msg_params *p, int32_t nsys, int32_t precision, msg_handle **out)
{
    if (!p || !out || nsys < 1 || (precision != MSG_PREC_FP64 && precision != MSG_PREC_MIXED)) return MSG_ERR_ARG;
    keep_pool_blocks();
    msg_handle *h = new msg_handle();
    if (const char *al = std::getenv("MSG_ALLOC_LOG")) h->alloc_log = (size_t)std::atoll(al);
    // MSG_NO_GRAPHS=1 launches every kernel directly instead of replaying a CUDA graph
    if (const char *ng = std::getenv("MSG_NO_GRAPHS")) h->use_graphs = !(ng[0] == '1');
    try {
        h->build(p, nsys, precision);
        // initial neighbour lists: every system is rebuilt from its set-up order
        std::vector<int> ones(nsys, 1);
        h->up(h->flag, ones.data(), nsys * sizeof(int));
    } catch (const CudaError &e) {
        std::fprintf(stderr, "msg_create: %s\n", e.what.c_str());
        delete h;
        *out = nullptr;
        return e.code;
    }
    *out = h;
    return MSG_OK;
}

extern "C" int msg_create(const msg_params *p, int32_t precision, msg_handle **out)
{
    return create_impl(p, 1, precision, out);
}

extern "C" int msg_create_batch(const msg_params *p, int32_t nsys, int32_t precision, msg_handle **out)
{
    return create_impl(p, nsys, precision, out);
}

extern "C" void msg_destroy(msg_handle *h) { delete h; }

extern "C" int msg_estimate_bytes(const msg_params *p, int32_t nsys, int32_t precision, int64_t *bytes)
{
    if (!p || !bytes || nsys < 1 || (precision != MSG_PREC_FP64 && precision != MSG_PREC_MIXED)) return MSG_ERR_ARG;
    msg_handle *h = new msg_handle();
    h->dry = true;
    if (const char *al = std::getenv("MSG_ALLOC_LOG")) h->alloc_log = (size_t)std::atoll(al);
    int rc = MSG_OK;
    try {
        h->build(p, nsys, precision);
        *bytes = h->bytes_live;
    } catch (const CudaError &e) {
        if (h->alloc_log) std::fprintf(stderr, "msg_estimate_bytes: %s\n", e.what.c_str());
        rc = e.code;
    }
    delete h;
    return rc;
}

extern "C" int64_t msg_device_bytes(const msg_handle *h) { return h ? h->bytes_live : -1; }

extern "C" int msg_trim_caches(void)
{
    {
        std::lock_guard<std::mutex> lk(g_plan_mu);
        for (auto &kv : g_plan_idle)
            for (auto &pw : kv.second) cufftDestroy(pw.first);
        g_plan_idle.clear();
    }
    int dev = 0;
    cudaMemPool_t pool;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess)
        return MSG_ERR_CUDA;
    return cudaMemPoolTrimTo(pool, 0) == cudaSuccess ? MSG_OK : MSG_ERR_CUDA;
}

extern "C" const char *msg_last_error(const msg_handle *h) { return h ? h->err.c_str() : "null handle"; }

extern "C" int32_t msg_nsys(const msg_handle *h) { return h ? h->nsys : 0; }

// Host state of system isys (MOLSIM layout, NULL arrays skipped) onto the
// device, stream-ordered: copies through one staging region per array, then one
// conversion kernel.
static void upload_state(msg_handle *h, int32_t isys, const double *ro, const double *rod, const double *rodd)
{
    const SysDev &S = h->hs[isys];
    // one staging region per array, so the copies and conversions do not wait on each other
    h->ensure_stage(9 * (size_t)S.n);
    const int c = h->cur, nb = (S.n + STATE_BLOCK - 1) / STATE_BLOCK;
    const double *src[3] = {ro, rod, rodd};
    const double *stg[3] = {nullptr, nullptr, nullptr};
    for (int k = 0; k < 3; ++k) {
        if (!src[k]) continue;
        double *p = h->stage + 3 * (size_t)S.n * k;
        h2d(p, src[k], 3 * (size_t)S.n, h->st);
        stg[k] = p;
    }
    if (ro || rod || rodd) {
        k_state_in<<<nb, STATE_BLOCK, 0, h->st>>>(h->dsys, isys, stg[0], stg[1], stg[2], h->pos[c], h->vel[c],
                                                  h->acc[c], h->posfx, h->inv, nullptr);
        h->launches += 1;
    }
    if (ro) h->placed[isys] = 1;
}

// The reverse, into host arrays; complete once the stream reaches it.
static void download_state(msg_handle *h, int32_t isys, double *ro, double *rod, double *rodd)
{
    const SysDev &S = h->hs[isys];
    h->ensure_stage(9 * (size_t)S.n);
    const int c = h->cur, nb = (S.n + STATE_BLOCK - 1) / STATE_BLOCK;
    double *dst[3] = {ro, rod, rodd};
    double *stg[3] = {nullptr, nullptr, nullptr};
    for (int k = 0; k < 3; ++k)
        if (dst[k]) stg[k] = h->stage + 3 * (size_t)S.n * k;
    if (ro || rod || rodd) {
        k_state_out<<<nb, STATE_BLOCK, 0, h->st>>>(h->dsys, isys, h->pos[c], h->vel[c], h->acc[c], stg[0], stg[1],
                                                   stg[2], h->inv);
        h->launches += 1;
    }
    for (int k = 0; k < 3; ++k)
        if (dst[k]) CK(cudaMemcpyAsync(dst[k], stg[k], 3 * sizeof(double) * S.n, cudaMemcpyDeviceToHost, h->st));
}

static int put_state(msg_handle *h, int32_t isys, const double *ro, const double *rod, const double *rodd,
                     bool keep_list)
{
    upload_state(h, isys, ro, rod, rodd);
    if (ro && !keep_list) {
        // new positions: rebuild this system's list now (the rebuild resets drosum)
        std::vector<int> f(h->nsys, 0);
        f[isys] = 1;
        return h->rebuild_checked(f);
    }
    return h->check();
}

extern "C" int msg_nlist_before_macrostep(msg_handle *h)
{
    if (!h) return MSG_ERR_ARG;
    API_BEGIN
    CK(cudaMemsetAsync(h->dsum[0], 0, sizeof(double4) * h->ntot, h->st));
    CK(cudaMemsetAsync(h->istep2, 0, sizeof(unsigned) * h->nsys, h->st));
    return h->check();
    API_END
}

extern "C" int msg_set_state(msg_handle *h, int32_t isys, const double *ro, const double *rod, const double *rodd)
{
    if (!h || isys < 0 || isys >= h->nsys) return MSG_ERR_ARG;
    API_BEGIN
    return put_state(h, isys, ro, rod, rodd, false);
    API_END
}

extern "C" int msg_set_state_all(msg_handle *h, const double *ro, const double *rod, const double *rodd)
{
    if (!h || !ro) return MSG_ERR_ARG;
    API_BEGIN
    // every system's copies and conversion on the stream, then one rebuild of every list
    size_t at = 0;
    for (int s = 0; s < h->nsys; ++s) {
        upload_state(h, s, ro + at, rod ? rod + at : nullptr, rodd ? rodd + at : nullptr);
        at += 3 * (size_t)h->hs[s].n;
    }
    std::vector<int> all(h->nsys, 1);
    return h->rebuild_checked(all);
    API_END
}

extern "C" int msg_put_state(msg_handle *h, int32_t isys, const double *ro, const double *rod, const double *rodd,
                             int32_t keep_list)
{
    if (!h || isys < 0 || isys >= h->nsys) return MSG_ERR_ARG;
    API_BEGIN
    return put_state(h, isys, ro, rod, rodd, keep_list != 0);
    API_END
}

extern "C" int msg_get_state(msg_handle *h, int32_t isys, double *ro, double *rod, double *rodd)
{
    if (!h || isys < 0 || isys >= h->nsys) return MSG_ERR_ARG;
    API_BEGIN
    download_state(h, isys, ro, rod, rodd);
    return h->check();
    API_END
}

extern "C" int msg_build_nlist(msg_handle *h, int32_t isys, int32_t *nneighpn, int32_t *jpnlist, int32_t maxnneigh,
                               int64_t *npair)
{
    if (!h || isys < 0 || isys >= h->nsys) return MSG_ERR_ARG;
    API_BEGIN
    std::vector<int> f(h->nsys, 0);
    f[isys] = 1;
    int rc = h->rebuild_checked(f);
    if (rc) return rc;
    const SysDev &S = h->hs[isys];
    if (npair) {
        std::vector<int> nn(S.n);
        h->down(nn.data(), h->nnb + S.off, S.n * sizeof(int));
        long long tot = 0;
        for (int v : nn) tot += v;
        *npair = h->list_half ? tot : tot / 2;
    }
    if (nneighpn && jpnlist) {
        if (maxnneigh < 1) return MSG_ERR_ARG;
        int *dn = h->dalloc<int>(S.n);
        long long *dj = h->dalloc<long long>((size_t)S.n * maxnneigh);
        int *ds = h->dalloc<int>((size_t)S.n * maxnneigh);
        const unsigned nb = (unsigned)(((long long)S.n * 32 + 255) / 256);
        k_export_scatter<<<nb, 256, 0, h->st>>>(h->dsys, isys, h->nbl, h->nnb, h->orig[h->cur], h->list_half,
                                                h->llinfo, dn, dj, maxnneigh, h->errw);
        k_export_sort<<<nb, 256, 0, h->st>>>(S.n, dn, dj, ds, maxnneigh);
        rc = h->check();
        if (!rc) {
            h->down(nneighpn, dn, S.n * sizeof(int));
            h->down(jpnlist, ds, (size_t)S.n * maxnneigh * sizeof(int));
        }
        h->dfree(dn);
        h->dfree(dj);
        h->dfree(ds);
        return rc;
    }
    return MSG_OK;
    API_END
}

static void fill_energy(const double *e, int natat, msg_energy *out)
{
    std::memset(out, 0, sizeof(*out));
    out->utot = e[0];
    out->utwob0 = e[1];
    for (int p = 0; p < natat && p < 10; ++p) out->utwob[p] = e[2 + p];
    out->urec = e[12];
    out->ubond = e[13];
    out->virial = e[14];
    out->ekin = e[15];
}

extern "C" int msg_utotal(msg_handle *h, int32_t isys, double *force, double *forceo, msg_energy *e)
{
    if (!h || isys < 0 || isys >= h->nsys) return MSG_ERR_ARG;
    API_BEGIN
    h->enqueue_forces(0, false);
    int rc = h->check();
    if (rc) return rc;
    const SysDev &S = h->hs[isys];
    h->ensure_stage(3 * (size_t)S.n);
    const int nb = (S.n + 255) / 256;
    if (force) {
        k_to_molsim<<<nb, 256, 0, h->st>>>(h->ftot, h->stage, h->inv, S.off, S.n, 1.0);
        CK(cudaMemcpyAsync(force, h->stage, 3 * sizeof(double) * S.n, cudaMemcpyDeviceToHost, h->st));
    }
    if (forceo) {
        k_to_molsim<<<nb, 256, 0, h->st>>>(h->fo[h->cur], h->stage, h->inv, S.off, S.n, 1.0);
        CK(cudaMemcpyAsync(forceo, h->stage, 3 * sizeof(double) * S.n, cudaMemcpyDeviceToHost, h->st));
    }
    if (e) {
        double he[ESZ];
        CK(cudaMemcpyAsync(he, h->esys + (size_t)isys * ESZ, sizeof(he), cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
        fill_energy(he, S.natat, e);
    }
    return h->check();
    API_END
}

extern "C" int msg_get_forces(msg_handle *h, int32_t isys, double *force, double *forceo)
{
    if (!h || isys < 0 || isys >= h->nsys) return MSG_ERR_ARG;
    API_BEGIN
    const SysDev &S = h->hs[isys];
    h->ensure_stage(3 * (size_t)S.n);
    const int nb = (S.n + 255) / 256;
    if (force) {
        k_to_molsim<<<nb, 256, 0, h->st>>>(h->ftot, h->stage, h->inv, S.off, S.n, 1.0);
        h->down(force, h->stage, 3 * sizeof(double) * S.n);
    }
    if (forceo) {
        k_to_molsim<<<nb, 256, 0, h->st>>>(h->fo[h->cur], h->stage, h->inv, S.off, S.n, 1.0);
        h->down(forceo, h->stage, 3 * sizeof(double) * S.n);
    }
    return h->check();
    API_END
}

extern "C" int msg_tune(msg_handle *h, int32_t key, int32_t value)
{
    if (!h) return MSG_ERR_ARG;
    API_BEGIN
    if (key == MSG_TUNE_PAIR_LANES) {
        if (value < -4 || value > 4) return MSG_ERR_ARG;
        h->set_pair_lanes(value);
        return MSG_OK;
    }
    if (key == MSG_TUNE_PAIR_UNROLL) {
        if (value != 1 && value != 2 && value != 4) return MSG_ERR_ARG;
        if (h->pair_unroll != value) {
            h->drop_graph();
            h->pair_unroll = value;
            if (h->prec == MSG_PREC_MIXED) h->set_lean_grid(h->nsm);
        }
        return MSG_OK;
    }
    if (key == MSG_TUNE_OVERLAP) {
        if (value != 0 && value != 1) return MSG_ERR_ARG;
        if (h->overlap != value) {
            h->drop_graph();
            h->overlap = value;
        }
        return MSG_OK;
    }
    if (key == MSG_TUNE_PAIR_BLOCKS) {
        if (value < 0 || value > 32) return MSG_ERR_ARG;
        if (h->pair_per_sm != value) {
            h->drop_graph();
            h->pair_per_sm = value;
        }
        return MSG_OK;
    }
    if (key == MSG_TUNE_CONV_BLOCKS) {
        if (value < 0 || value > 32) return MSG_ERR_ARG;
        h->drop_graph();
        h->set_conv_grid(value);
        return MSG_OK;
    }
    if (key == MSG_TUNE_PAIR_KERNEL) {
        if (value < 0 || value > 3 || (value >= 2 && h->prec != MSG_PREC_MIXED)) return MSG_ERR_ARG;
        if (h->pair_lean != value) {
            h->drop_graph();
            const int half = value == 2 ? 1 : 0;
            h->pair_lean = value;
            if (half != h->list_half) {
                // the other list layout: new task sizes and every placed system's list rebuilt
                h->list_half = half;
                h->set_pair_lanes(h->pair_shift, true);
                std::vector<int> all(h->placed.begin(), h->placed.end());
                const int rc = h->rebuild_checked(all);
                if (rc) return rc;
            }
        }
        return MSG_OK;
    }
    return MSG_ERR_ARG;
    API_END
}

extern "C" int msg_get_linacc(msg_handle *h)
{
    if (!h) return MSG_ERR_ARG;
    API_BEGIN
    const int c = h->cur;
    k_linacc<<<h->nt128, 128, 0, h->st>>>(h->dsys, h->t128, h->fo[c], h->typ[c], h->massip, h->acc[c]);
    return h->check();
    API_END
}

// Random's first-call state from iseed (Src/mollib.F90:2696-2701).
static int2 mc_seed_state(int32_t iseed)
{
    // abs(iseed) in two's complement (INT_MIN stays INT_MIN, as a 32-bit abs wraps)
    const int32_t a = iseed < 0 ? (int32_t)(0u - (uint32_t)iseed) : iseed;
    return make_int2(777755555 ^ a, (888889999 ^ a) | 1);
}

// Random's jump table: the xorshift (13, 17, 5) step as a 32x32 bit matrix and its
// squarings, and 16807^(2^b) mod (2^31 - 1).
static McJump make_jump_table()
{
    McJump J;
    for (int j = 0; j < 32; ++j) {
        unsigned v = 1u << j;
        v ^= v << 13;
        v ^= v >> 17;
        v ^= v << 5;
        J.xs[0][j] = v;
    }
    for (int b = 1; b < 32; ++b)
        for (int j = 0; j < 32; ++j) J.xs[b][j] = mc_xs_apply(J.xs[b - 1], J.xs[b - 1][j]);
    J.pm[0] = 16807ull;
    for (int b = 1; b < 32; ++b) J.pm[b] = (J.pm[b - 1] * J.pm[b - 1]) % 2147483647ull;
    return J;
}

static const McJump &jump_table()
{
    static const McJump J = make_jump_table();
    return J;
}

extern "C" int msg_random_jump(int32_t ix, int32_t iy, uint32_t k, int32_t out[2])
{
    if (!out || iy <= 0) return MSG_ERR_ARG;
    const int2 r = mc_jump(jump_table(), make_int2(ix, iy), k);
    out[0] = r.x;
    out[1] = r.y;
    return MSG_OK;
}

// Monte Carlo buffers, made on first use; an unseeded system starts from iseed = isys + 1.
void msg_handle::ensure_mc()
{
    if (mc_rng) return;                // mc_rng is made last: a set-up that failed part-way starts over
    {
        void **parts[] = {(void **)&mc_u, (void **)&mc_cnt, (void **)&mc_par, (void **)&mc_dtr, (void **)&ew_sktm,
                          (void **)&elc_sttm, (void **)&mc_ig, (void **)&mc_rg, (void **)&mc_F, (void **)&mc_jumpt,
                          (void **)&mca_psave, (void **)&mca_step, (void **)&mca_flag, (void **)&mca_esave,
                          (void **)&mca_beta, (void **)&mca_acc};
        for (void **pp : parts)
            if (*pp) {
                dfree(*pp);
                *pp = nullptr;
            }
        for (cufftHandle p : mc_plans) cufftDestroy(p);
        mc_plans.clear();
    }
    mc_u = dalloc<double>((size_t)nsys * ESZ);
    mc_cnt = dalloc<long long>(2 * (size_t)nsys);
    mc_par = dalloc<McPar>(nsys);
    mc_dtr = dalloc<double>(std::max(1, type_tot));
    if (any_std) ew_sktm = dalloc<double2>(4 * (size_t)ew_nkv_tot);
    if (elc_nk) elc_sttm = dalloc<double>(8 * (size_t)elc_nk);
    if (any_spme) {
        mc_ig = dalloc<unsigned long long>(grid_tot);
        CK(cudaMemsetAsync(mc_ig, 0, grid_tot * sizeof(unsigned long long), st));
        mc_rg = dalloc<double>(grid_tot);
        mc_F = dalloc<double2>(cgrid_tot);
        for (const FftClass &fc : fft) {
            cufftHandle p = 0;
            int dims[3] = {fc.s, fc.s, fc.s};
            const int rd = fc.s * fc.s * fc.s, cd = fc.s * fc.s * (fc.s / 2 + 1);
            CKF(cufftPlanMany(&p, 3, dims, nullptr, 1, rd, nullptr, 1, cd, CUFFT_D2Z, fc.count));
            mc_plans.push_back(p);
        }
    }
    mc_jumpt = dalloc<McJump>(1);
    up(mc_jumpt, &jump_table(), sizeof(McJump));
    mca_psave = dalloc<double4>(ntot);
    mca_step = dalloc<double4>(ntot);
    mca_flag = dalloc<int>(nsys);
    mca_esave = dalloc<double>((size_t)nsys * ESZ);
    mca_beta = dalloc<double>(nsys);
    mca_acc = dalloc<int>(nsys);
    std::vector<int2> st(nsys);
    for (int s = 0; s < nsys; ++s) st[s] = mc_seed_state(s + 1);
    int2 *rng = dalloc<int2>(nsys);
    up(rng, st.data(), nsys * sizeof(int2));
    mc_rng = rng;
}

extern "C" int msg_mc_seed(msg_handle *h, int32_t isys, int32_t iseed)
{
    if (!h || isys < 0 || isys >= h->nsys) return MSG_ERR_ARG;
    API_BEGIN
    h->ensure_mc();
    const int2 st = mc_seed_state(iseed);
    CK(cudaMemcpyAsync(h->mc_rng + isys, &st, sizeof(int2), cudaMemcpyHostToDevice, h->st));
    return h->check();
    API_END
}

extern "C" int msg_mc_pass(msg_handle *h, int32_t npass, const msg_mc_params *p, int64_t *accepted,
                           int64_t *hsreject, int32_t isys, msg_energy *e)
{
    if (!h || !p || npass < 0 || (e && (isys < 0 || isys >= h->nsys))) return MSG_ERR_ARG;
    API_BEGIN
    std::vector<McPar> par(h->nsys);
    std::vector<double> dtr(std::max(1, h->type_tot), 0.0);
    for (int s = 0; s < h->nsys; ++s) {
        const SysDev &S = h->hs[s];


        if (!p[s].dtran || (p[s].isamp != 0 && p[s].isamp != 1)) {
            h->err = "msg_mc_params needs dtran[npt] and isamp 0 or 1";
            return MSG_ERR_ARG;
        }
        par[s].beta = p[s].beta;
        par[s].isamp = p[s].isamp;
        par[s].pad = 0;
        for (int t = 0; t < S.npt; ++t) dtr[S.type_off + t] = p[s].dtran[t];
    }
    h->ensure_mc();
    h->up(h->mc_par, par.data(), h->nsys * sizeof(McPar));
    h->up(h->mc_dtr, dtr.data(), dtr.size() * sizeof(double));
    CK(cudaMemsetAsync(h->mc_cnt, 0, 2 * sizeof(long long) * h->nsys, h->st));
    // energies and structure factors of the current configuration (UTotal), carried
    // from here by the accepted moves' differences (MCUpdate)
    h->enqueue_forces(0, false);
    CK(cudaMemcpyAsync(h->mc_u, h->esys, sizeof(double) * ESZ * h->nsys, cudaMemcpyDeviceToDevice, h->st));
    if (npass > 0 && h->any_spme) {
        // the FP64 spectrum of every SPME system's charge mesh at the start of the pass
        k_mc_spread<<<h->nt128, 128, 0, h->st>>>(h->dsys, h->t128, h->pos[0], h->mc_ig);
        k_mc_mesh_f64<<<(unsigned)((h->grid_tot + 255) / 256), 256, 0, h->st>>>(h->grid_tot, h->mc_ig, h->mc_rg);
        for (size_t c = 0; c < h->fft.size(); ++c) {
            CKF(cufftSetStream(h->mc_plans[c], h->st));
            CKF(cufftExecD2Z(h->mc_plans[c], h->mc_rg + h->fft[c].grid_off,
                             reinterpret_cast<cufftDoubleComplex *>(h->mc_F + h->fft[c].cgrid_off)));
        }
        h->launches += 2;
    }
    if (npass > 0) {
        // a chain reads its system from shared memory when every system's share fits and
        // there are no more chains than SMs (each such block holds an SM on its own)
        const int wmax = h->any_std ? h->ew_maxw : 1;
        int smax = 0;
        for (int s = 0; s < h->nsys; ++s)
            if (h->hs[s].lewald && !h->hs[s].recstd) smax = std::max(smax, h->hs[s].s);
        const int etabn = std::max(6 * wmax, 7 * smax);
        const size_t etab = (size_t)etabn * sizeof(double2);
        size_t need = 0;
        for (int s = 0; s < h->nsys; ++s)
            need = std::max(need, mc_cache_bytes(h->hs[s].n, h->hs[s].tab_nk, h->hs[s].natat));
        const int cache = (h->nsys <= h->nsm && etab + need <= 200 * 1024) ? 1 : 0;
        const size_t smem = etab + (cache ? need : 0);
        const int feat = (h->any_spme ? 1 : 0) | (h->elc_nk ? 2 : 0);
        auto kern = feat == 3 ? k_mc_pass<3> : feat == 2 ? k_mc_pass<2> : feat == 1 ? k_mc_pass<1> : k_mc_pass<0>;
        if (smem > 48 * 1024)
            CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<h->nsys, MC_THREADS, smem, h->st>>>(
            h->dsys, h->pos[0], h->typ[0], h->inv, h->ptmap, h->ptab, h->tc, h->bst, h->ew_kv, h->ew_kfac, h->ew_sk,
            h->ew_sktm, h->has_bonds ? h->bptr : nullptr, h->bpart, h->bk, h->beq, h->bpw, h->mc_par, h->mc_dtr,
            h->mc_rng, h->mc_u, h->mc_cnt, npass, cache, wmax, h->elc_kv, h->elc_kfac, h->elc_st, h->elc_sttm,
            h->mc_F, h->emf, etabn);
        h->launches += 1;
    }
    std::vector<long long> cnt(2 * (size_t)h->nsys);
    CK(cudaMemcpyAsync(cnt.data(), h->mc_cnt, cnt.size() * sizeof(long long), cudaMemcpyDeviceToHost, h->st));
    double he[ESZ];
    if (e) CK(cudaMemcpyAsync(he, h->mc_u + (size_t)isys * ESZ, sizeof(he), cudaMemcpyDeviceToHost, h->st));
    int rc = h->check();
    if (rc) return rc;
    for (int s = 0; s < h->nsys; ++s) {
        if (accepted) accepted[s] = cnt[2 * (size_t)s];
        if (hsreject) hsreject[s] = cnt[2 * (size_t)s + 1];
    }
    if (e) fill_energy(he, h->hs[isys].natat, e);
    // the particles moved: every list is rebuilt (NList after the sweeps)
    if (npass > 0) {
        std::vector<int> all(h->placed.begin(), h->placed.end());
        return h->rebuild_checked(all);
    }
    return MSG_OK;
    API_END
}

static void prepare_hist(msg_handle *h, int nsteps)
{
    if (nsteps > h->hist_cap) {
        if (h->hist) h->dfree(h->hist);
        h->hist = h->dalloc<double>((size_t)nsteps * h->nsys * ESZ);
        h->hist_cap = nsteps;
    }
    CK(cudaMemsetAsync(h->stepctr, 0, sizeof(unsigned long long), h->st));
}

static void copy_hist(msg_handle *h, int nsteps, int isys, msg_energy *e)
{
    std::vector<double> buf((size_t)nsteps * h->nsys * ESZ);
    CK(cudaMemcpyAsync(buf.data(), h->hist, buf.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (int k = 0; k < nsteps; ++k) fill_energy(&buf[((size_t)k * h->nsys + isys) * ESZ], h->hs[isys].natat, &e[k]);
}

extern "C" int msg_velver(msg_handle *h, int32_t nsteps, int32_t isys, msg_energy *e)
{
    if (!h || nsteps < 0 || (e && (isys < 0 || isys >= h->nsys))) return MSG_ERR_ARG;
    API_BEGIN
    const bool rec = e != nullptr;
    if (rec) prepare_hist(h, nsteps);
    if (h->use_graphs && nsteps > 0) {
        h->ensure_graph(0, rec, 0);
        for (int k = 0; k < nsteps; ++k) h->launch_graph();
    } else {
        for (int k = 0; k < nsteps; ++k) h->enqueue_md_step(rec);
    }
    // the longest rows and the energy history come back with the error word: one wait
    int *prow = h->pin_rows();
    if (prow) CK(cudaMemcpyAsync(prow, h->nmaxrow, h->nsys * sizeof(int), cudaMemcpyDeviceToHost, h->st));
    const size_t nh = (size_t)nsteps * h->nsys * ESZ;
    double *ph = rec ? h->pin_hist(nh) : nullptr;
    if (ph) CK(cudaMemcpyAsync(ph, h->hist, nh * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    int rc = h->check();
    if (rc) return rc;
    if (rec) {
        if (ph)
            for (int k = 0; k < nsteps; ++k) fill_energy(&ph[((size_t)k * h->nsys + isys) * ESZ], h->hs[isys].natat, &e[k]);
        else
            copy_hist(h, nsteps, isys, e);
    }
    if (h->grow_lists(prow)) {
        std::vector<int> all(h->placed.begin(), h->placed.end());
        return h->rebuild_checked(all);
    }
    return MSG_OK;
    API_END
}

// The device address of a caller's host array of `bytes` bytes when the GPU may
// read and write it in place: page-locked, mapped at the same address, 8-byte
// aligned, and wholly inside one page-locked allocation (the driver's address-range
// attributes).  Null otherwise, and for a null array.
static double *mapped_span(double *p, size_t bytes)
{
    if (!p || (reinterpret_cast<uintptr_t>(p) & 7)) return nullptr;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a.type != cudaMemoryTypeHost || a.devicePointer != static_cast<void *>(p)) return nullptr;
    using RangeFn = CUresult (*)(void *, CUpointer_attribute, CUdeviceptr);
    static RangeFn get = [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuPointerGetAttribute", &fn, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            fn = nullptr;
        }
        return reinterpret_cast<RangeFn>(fn);
    }();
    if (!get) return nullptr;
    CUdeviceptr start = 0;
    size_t size = 0;
    const CUdeviceptr at = reinterpret_cast<CUdeviceptr>(p);
    if (get(&start, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, at) != CUDA_SUCCESS ||
        get(&size, CU_POINTER_ATTRIBUTE_RANGE_SIZE, at) != CUDA_SUCCESS)
        return nullptr;
    if (at < start || at - start + bytes > size) return nullptr;
    return p;
}

extern "C" int msg_velver_host(msg_handle *h, int32_t isys, int32_t nsteps, double *ro, double *rod, double *rodd,
                               msg_energy *e)
{
    if (!h || isys < 0 || isys >= h->nsys || nsteps < 0) return MSG_ERR_ARG;
    API_BEGIN
    const bool rec = e != nullptr;
    // one step on page-locked host arrays: the whole exchange is one graph launch and one wait
    const size_t nbytes = 3 * sizeof(double) * (size_t)h->hs[isys].n;
    double *io[3] = {mapped_span(ro, nbytes), mapped_span(rod, nbytes), mapped_span(rodd, nbytes)};
    if (h->use_graphs && !h->timing && nsteps == 1 && h->dpin && h->pin_rows() &&
        (!rec || h->pin_hist((size_t)h->nsys * ESZ)) && (ro || rod || rodd) && (!ro || io[0]) &&
        (!rod || io[1]) && (!rodd || io[2])) {
        if (rec && h->hist_cap < 1) prepare_hist(h, 1);
        h->ensure_io_graph(rec, isys, io);
        if (ro) h->placed[isys] = 1;
        h->launch_one(h->iograph);
        CK(cudaStreamSynchronize(h->st));
        CK(cudaGetLastError());
        const int rc = h->check_word(*h->pin_err());
        if (rc) return rc;
        if (rec) fill_energy(h->pin_hist((size_t)h->nsys * ESZ) + (size_t)isys * ESZ, h->hs[isys].natat, e);
        if (h->grow_lists(h->pin_rows())) {
            std::vector<int> all(h->placed.begin(), h->placed.end());
            return h->rebuild_checked(all);
        }
        return MSG_OK;
    }
    // the host arrays continue the device's trajectory: the list and drosum stay valid
    upload_state(h, isys, ro, rod, rodd);
    if (rec) prepare_hist(h, nsteps);
    if (h->use_graphs && nsteps > 0) {
        h->ensure_graph(0, rec, 0);
        for (int k = 0; k < nsteps; ++k) h->launch_graph();
    } else {
        for (int k = 0; k < nsteps; ++k) h->enqueue_md_step(rec);
    }
    download_state(h, isys, ro, rod, rodd);
    int *prow = h->pin_rows();
    if (prow) CK(cudaMemcpyAsync(prow, h->nmaxrow, h->nsys * sizeof(int), cudaMemcpyDeviceToHost, h->st));
    const size_t nh = (size_t)nsteps * h->nsys * ESZ;
    double *ph = rec ? h->pin_hist(nh) : nullptr;
    if (ph) CK(cudaMemcpyAsync(ph, h->hist, nh * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    int rc = h->check();
    if (rc) return rc;
    if (rec) {
        if (ph)
            for (int k = 0; k < nsteps; ++k) fill_energy(&ph[((size_t)k * h->nsys + isys) * ESZ], h->hs[isys].natat, &e[k]);
        else
            copy_hist(h, nsteps, isys, e);
    }
    if (h->grow_lists(prow)) {
        std::vector<int> all(h->placed.begin(), h->placed.end());
        return h->rebuild_checked(all);
    }
    return MSG_OK;
    API_END
}

extern "C" int msg_velver_async(msg_handle *h, int32_t nsteps)
{
    if (!h || nsteps < 0) return MSG_ERR_ARG;
    API_BEGIN
    if (h->timing) return MSG_ERR_ARG;   // timers need the synchronous call
    if (h->use_graphs && nsteps > 0) {
        h->ensure_graph(0, false, 0);
        for (int k = 0; k < nsteps; ++k) h->launch_graph();
    } else {
        for (int k = 0; k < nsteps; ++k) h->enqueue_md_step(false);
    }
    cudaEvent_t ev = h->get_event();
    CK(cudaEventRecord(ev, h->st));
    h->inflight.push_back(ev);
    CK(cudaGetLastError());
    return MSG_OK;
    API_END
}

extern "C" int msg_pending(msg_handle *h)
{
    if (!h) return -MSG_ERR_ARG;
    try {
        size_t done = 0;
        while (done < h->inflight.size()) {
            const cudaError_t q = cudaEventQuery(h->inflight[done]);
            if (q == cudaErrorNotReady) break;
            if (q != cudaSuccess) {
                h->err = std::string("msg_pending: ") + cudaGetErrorString(q);
                return -MSG_ERR_CUDA;
            }
            h->evpool.push_back(h->inflight[done]);
            ++done;
        }
        h->inflight.erase(h->inflight.begin(), h->inflight.begin() + done);
        if (!h->inflight.empty()) return (int)h->inflight.size();
        const int rc = h->check();
        return rc ? -rc : 0;
    } catch (const CudaError &e) {
        h->err = e.what;
        return -e.code;
    }
}

extern "C" int msg_get_energy(msg_handle *h, int32_t isys, msg_energy *e)
{
    if (!h || !e || isys < 0 || isys >= h->nsys) return MSG_ERR_ARG;
    API_BEGIN
    double he[ESZ];
    h->down(he, h->esys + (size_t)isys * ESZ, sizeof(he));
    fill_energy(he, h->hs[isys].natat, e);
    return h->check();
    API_END
}

extern "C" int msg_bd_step(msg_handle *h, int32_t nsteps, uint64_t seed, int32_t isys, const double *xi,
                           double *xi_out, msg_energy *e)
{
    if (!h || nsteps < 0 || ((xi || xi_out || e) && (isys < 0 || isys >= h->nsys))) return MSG_ERR_ARG;
    if (!h->has_bd) {
        h->err = "bd_fac1/bd_fac2 were not given at creation";
        return MSG_ERR_ARG;
    }
    API_BEGIN
    const bool rec = e != nullptr;
    if (rec) prepare_hist(h, nsteps);
    const size_t per = 3 * (size_t)h->ntot;
    if ((xi || xi_out) && per * std::max(1, nsteps) > h->xin_n) {
        if (h->xin) h->dfree(h->xin);
        h->xin_n = per * std::max(1, nsteps);
        h->xin = h->dalloc<double>(h->xin_n);
    }
    const SysDev &S = h->hs[std::max(0, isys)];
    if (xi) {
        for (int k = 0; k < nsteps; ++k)
            h2d(h->xin + k * per + 3 * (size_t)S.off, xi + (size_t)k * 3 * S.n, 3 * (size_t)S.n, h->st);
    }
    if (h->use_graphs && !xi && !xi_out && nsteps > 0) {
        h->ensure_graph(1, rec, seed);
        for (int k = 0; k < nsteps; ++k) h->launch_graph();
    } else {
        for (int k = 0; k < nsteps; ++k)
            h->enqueue_bd_step(seed, xi ? h->xin + k * per : nullptr, xi_out ? h->xin + k * per : nullptr, rec);
    }
    int rc = h->check();
    if (rc) return rc;
    if (xi_out) {
        std::vector<double> buf(per);
        for (int k = 0; k < nsteps; ++k) {
            h->down(buf.data(), h->xin + k * per, per * sizeof(double));
            std::memcpy(xi_out + (size_t)k * 3 * S.n, buf.data() + 3 * (size_t)S.off, 3 * sizeof(double) * S.n);
        }
    }
    if (rec) copy_hist(h, nsteps, isys, e);
    return MSG_OK;
    API_END
}

extern "C" int64_t msg_nrebuild(const msg_handle *h, int32_t isys)
{
    if (!h || isys < 0 || isys >= h->nsys) return -1;
    long long v = 0;
    if (cudaMemcpyAsync(&v, h->nrebuild + isys, sizeof(v), cudaMemcpyDeviceToHost, h->st) != cudaSuccess ||
        cudaStreamSynchronize(h->st) != cudaSuccess)
        return -1;
    return v;
}

extern "C" void *msg_stream(const msg_handle *h) { return h ? (void *)h->st : nullptr; }

extern "C" int64_t msg_launch_count(const msg_handle *h) { return h ? h->launches : -1; }

extern "C" int msg_set_timing(msg_handle *h, int32_t on)
{
    if (!h) return MSG_ERR_ARG;
    h->timing = on != 0;
    if (h->graph.exec && h->graph.timing != h->timing) h->drop_graph();
    for (int k = 0; k < TM_N; ++k) {
        h->tm_ms[k] = 0.0;
        h->tm_n[k] = 0;
    }
    return MSG_OK;
}

extern "C" int32_t msg_ntimers(void) { return TM_N; }

extern "C" int msg_kernel_time(const msg_handle *h, int32_t k, const char **name, double *total_ms, int64_t *launches)
{
    if (!h || k < 0 || k >= TM_N) return MSG_ERR_ARG;
    if (name) *name = kTimerNames[k];
    if (total_ms) *total_ms = h->tm_ms[k];
    if (launches) *launches = h->tm_n[k];
    return MSG_OK;
}

// MCAllPass (Src/mc.F90:4024-4178) for every system of the handle: npass trials, each
// displacing all particles at once (Random drawn on the device from each chain's place in
// the stream), rebuilding the lists, one UTotal of the trial, Metropolis on du%tot, and the
// saved configuration and energies back on rejection.
extern "C" int msg_mcall_pass(msg_handle *h, int32_t npass, const msg_mcall_params *p, int64_t *accepted,
                              int32_t isys, msg_energy *e)
{
    if (!h || !p || npass < 0 || (e && (isys < 0 || isys >= h->nsys))) return MSG_ERR_ARG;
    API_BEGIN
    std::vector<double> dtr(std::max(1, h->type_tot), 0.0), beta(h->nsys);
    for (int s = 0; s < h->nsys; ++s) {
        const SysDev &S = h->hs[s];
        if (!p[s].dtranall) {
            h->err = "msg_mcall_params needs dtranall[npt]";
            return MSG_ERR_ARG;
        }
        for (int t = 0; t < S.npt; ++t) dtr[S.type_off + t] = p[s].dtranall[t];
        beta[s] = p[s].beta;
    }
    h->ensure_mc();
    h->up(h->mc_dtr, dtr.data(), dtr.size() * sizeof(double));
    h->up(h->mca_beta, beta.data(), beta.size() * sizeof(double));
    CK(cudaMemsetAsync(h->mc_cnt, 0, 2 * sizeof(long long) * h->nsys, h->st));
    h->enqueue_forces(0, false);                       // the energies of the configuration
    int rc = h->check();
    if (rc) return rc;
    const long long n = h->ntot, nb = std::max<long long>(n, (long long)h->nsys * ESZ);
    int4 *fx = h->prec == MSG_PREC_MIXED ? h->posfx : nullptr;
    std::vector<int> flags(h->nsys);
    for (int pass = 0; pass < npass; ++pass) {
        k_mcall_save<<<(unsigned)((nb + 255) / 256), 256, 0, h->st>>>(n, h->pos[0], h->inv, h->mca_psave, h->nsys,
                                                                       h->esys, h->mca_esave);
        k_mcall_trial<<<(unsigned)((n + 255) / 256), 256, 0, h->st>>>(h->dsys, n, h->sysid, h->inv, h->typ[0],
                                                                       h->pos[0], h->mc_rng, h->mc_jumpt, h->mc_dtr,
                                                                       h->dsum[0], h->mca_step, fx);
        // NList: a system's lists are rebuilt only when its displacements since the last build
        // could have brought a pair from beyond rcut + drnlist inside rcut
        k_mcall_skin<<<h->nsys, 256, 0, h->st>>>(h->dsys, h->dsum[0], h->mca_flag);
        h->launches += 3;
        CK(cudaMemcpyAsync(flags.data(), h->mca_flag, h->nsys * sizeof(int), cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
        bool any = false;
        for (int s = 0; s < h->nsys; ++s) {
            flags[s] = flags[s] && h->placed[s];
            any = any || flags[s];
        }
        if (any) {
            rc = h->rebuild_checked(flags);
            if (rc) return rc;
        }
        h->enqueue_forces(0, false);
        k_mcall_decide<<<(h->nsys + 127) / 128, 128, 0, h->st>>>(h->dsys, h->nsys, h->mc_rng, h->mc_jumpt,
                                                                   h->mca_beta, h->esys, h->mca_esave, h->mca_acc,
                                                                   h->mc_cnt);
        k_mcall_restore<<<(unsigned)((n + 255) / 256), 256, 0, h->st>>>(h->dsys, n, h->sysid, h->inv, h->mca_acc,
                                                                         h->mca_psave, h->pos[0], h->dsum[0],
                                                                         h->mca_step, fx);
        h->launches += 2;
    }
    std::vector<long long> cnt(2 * (size_t)h->nsys);
    CK(cudaMemcpyAsync(cnt.data(), h->mc_cnt, cnt.size() * sizeof(long long), cudaMemcpyDeviceToHost, h->st));
    double he[ESZ];
    if (e) CK(cudaMemcpyAsync(he, h->esys + (size_t)isys * ESZ, sizeof(he), cudaMemcpyDeviceToHost, h->st));
    rc = h->check();
    if (rc) return rc;
    for (int s = 0; s < h->nsys && accepted; ++s) accepted[s] = cnt[2 * (size_t)s];
    if (e) fill_energy(he, h->hs[isys].natat, e);
    return MSG_OK;
    API_END
}

/*
 * molsim_gpu.h -- C-ABI of the B200 force/energy path for MOLSIM.
 *
 * The library is a drop-in for MOLSIM's per-step force/energy routines of a
 * monoatomic charged system.  The Fortran host keeps its own arrays and calls
 * these entry points through an ISO_C_BINDING interface (the same mechanism
 * MOLSIM already uses for FFTW, Src/energy.F90:100-110).  All arrays are
 * plain host pointers; Fortran (3,N) real(8) arrays are passed as C [N][3]
 * doubles.  Type indices, pair-table offsets and neighbour indices keep
 * MOLSIM's 1-based values.
 *
 * Entry points and the MOLSIM routine each one replaces:
 *   msg_create / msg_create_batch  -> set-up done by IOPotTwoBody+EwaldSetup
 *                                     (Src/potential.F90:294-446,
 *                                      Src/energy.F90:6601-7019) and IONList
 *                                     (Src/nlist.F90:184-281)
 *   msg_set_state / msg_get_state  -> the ro/rod/rodd globals (Src/mol.F90:1087-1098)
 *   msg_build_nlist                -> SetVList -> SetVListMD (Src/nlist.F90:686-759)
 *   msg_utotal                     -> UTotal (Src/energy.F90:280-434) with
 *                                     UTwoBodyA, UEwald (SPM or standard), UBond
 *   msg_get_linacc                 -> GetLinAcc (Src/md.F90:601-617)
 *   msg_velver                     -> MDDriver iSimulationStep: VelVer +
 *                                     GetKinEnergy (Src/md.F90:154-168, 252-410)
 *                                     followed by NList (Src/nlist.F90:597-621)
 *   msg_utwobody_p                 -> UTwoBodyP (Src/energy.F90:786-896), polyatomic particles
 *   msg_velver_p                   -> MDDriver with VelVer for rigid polyatomic particles
 *                                     (Src/md.F90:252-410, 628-663)
 *   msg_velver_p_ewald             -> the same steps with lewald: UTotal's UEwald over the sites
 *                                     (Src/energy.F90:335-352) in every step's forces and virial
 *   msg_uewald_sites               -> UEwald over the sites of polyatomic particles: UEwaldRecStd,
 *                                     UEwaldSelf with its molecular term, UEwaldSurf
 *                                     (Src/energy.F90:905-1104, 1301-1371)
 *   msg_uewald_sites_spm           -> the same with UEwaldRecSPM (Src/energy.F90:1207-1297)
 *   msg_mc_seed / msg_mc_pass      -> MCDriver iSimulationStep: MCPass with SPartMove
 *                                     (Src/mc.F90:1470-1755), DUTotal, Metropolis, MCUpdate
 *   msg_mcall_pass                 -> MCAllDriver iSimulationStep: MCAllPass (Src/mc.F90:4024-4178)
 *   msg_bd_step                    -> BDDriver iSimulationStep: BDStep + UTotal
 *                                     (Src/bd.F90:53-59, 120-155) followed by NList
 * Set-up helpers that restate MOLSIM's own set-up for callers without it:
 *   msg_rcut_to_alpha              -> RcutToAlpha (Src/energy.F90:7090-7105)
 *   msg_alpha_to_ncut              -> AlphaToNcut (Src/energy.F90:7066-7081)
 *   msg_pot_tab                    -> PotTwoBodyTab1/2/3 with Pot_1_6_12
 *                                     (Src/potential.F90:868-1258, 1349-1425)
 *
 * Status codes mirror MOLSIM's Stop() sites so the Fortran shim can stop with
 * the same message.
 */
#ifndef MOLSIM_GPU_H
#define MOLSIM_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MSG_OK               0
#define MSG_ERR_TABLE_MIN    1  /* r2 < r2umin           (Src/energy.F90:478-479) */
#define MSG_ERR_TABLE_RANGE  2  /* ibuf > nbuf           (Src/energy.F90:485)     */
#define MSG_ERR_CAPACITY     3  /* nneighpn > maxnneigh  (Src/nlist.F90:752)      */
#define MSG_ERR_CUDA         4  /* CUDA or cuFFT failure                          */
#define MSG_ERR_TIMEOUT      5  /* a bounded device wait gave up                  */
#define MSG_ERR_ARG          6  /* invalid argument                               */
#define MSG_ERR_NONFINITE    7  /* a force or energy became NaN/Inf               */
#define MSG_ERR_HARDCORE     8  /* r2 < r2atat (hard-core overlap, Src/energy.F90:476) */

#define MSG_PREC_FP64        0  /* FP64 everywhere: the plain drop-in path          */
#define MSG_PREC_MIXED       1  /* FP32 pair/grid forces, 64-bit fixed-point sums,
                                   FP64 positions, integrator, energies, b^2 moduli */

/* One system.  Mirrors the MolModule globals used on the path (Src/mol.F90). */
typedef struct msg_params {
    int32_t np;              /* particles (= atoms, monoatomic)                         */
    int32_t npt;             /* particle types                                          */
    double  boxlen[3];       /* periodic box, A (txbc='xyz')                            */
    double  rcut;            /* real-space cutoff, A                                    */
    double  drnlist;         /* Verlet skin, A                                          */
    const int32_t *iptpn;    /* [np] type of each particle, 1-based                     */
    const double  *az;       /* [np] charge, e                                          */
    const double  *masspt;   /* [npt] mass, g/mol                                       */
    const double  *ubuf;     /* pair table, 12 doubles per interval (Src/mol.F90:1120)  */
    int32_t        nbuf;     /* doubles in ubuf                                         */
    const int32_t *iubuflow; /* [natat] 1-based start of each type pair's table         */
    const double  *r2umin;   /* [natat] lower table limit, A^2                          */
    const double  *r2atat;   /* [natat] hard-core r^2 (0: none), A^2                    */
    int32_t lewald;          /* 0: none; 1: SPME (txewaldrec 'spm'); 2: standard Ewald
                              * ('std', UEwaldRecStd, Src/energy.F90:964-1104)          */
    int32_t order;           /* B-spline order                                          */
    int32_t nmesh;           /* SPME grid edge (even)                                   */
    int32_t lsurf;           /* 1: add the surface (dipole) term                        */
    double  ualpha;          /* Ewald alpha, 1/A                                        */
    double  epsi_four_pi;    /* Epsi0FourPi/relpermitt, kJ A / mol                      */
    int32_t nbond;           /* bonds                                                   */
    const int32_t *bond_ij;  /* [nbond][2] 1-based particle pairs                       */
    const double  *bond_k;   /* [nbond] force constant divided by the power             */
    const double  *bond_eq;  /* [nbond] equilibrium length, A                           */
    const int32_t *bond_p;   /* [nbond] power                                           */
    double  tstep;           /* time step, ps                                           */
    const double  *bd_fac1;  /* [npt] BD drift factor (Src/bd.F90:138), may be NULL    */
    const double  *bd_fac2;  /* [npt] BD noise factor (Src/bd.F90:139), may be NULL    */
    int32_t maxnneigh;       /* row capacity hint for the neighbour list (0: automatic) */
    int32_t ncut;            /* lewald 2: k = 2 pi n / L with 0 <= n_i <= ncut (1..100)  */
    int32_t ncutregion;      /* lewald 2: 0 'sphere' (|n|^2 <= ncut^2), 1 'cube'         */
    int32_t lewald2dlc;      /* 1: 2D layer correction (UEwaldRecStd2dlc, lewald 2) and    */
                             /*    UEwaldSurf's 2d-periodic form (Src/energy.F90:1106-1203, */
                             /*    1362-1369), in UTotal and in the Monte Carlo difference */
    int32_t inlist;          /* NList update interval (Src/nlist.F90:600-620): 0 the skin  */
                             /*    test; n > 0 a rebuild whenever mod(istep2, n) == 0,      */
                             /*    istep2 counting steps since msg_nlist_before_macrostep   */
    int32_t lvlistllist;     /* 1: the Verlet list is SetLList(rcut+drnlist) +             */
                             /*    SetVListMDLList's (Src/nlist.F90:698-702, 769-811,      */
                             /*    1168-1260): pair set and row order; at most 1000 cells  */
} msg_params;

typedef struct msg_handle msg_handle;

/* Energies of one system, MOLSIM's u%... fields (kJ/mol) and virial. */
typedef struct msg_energy {
    double utot;             /* u%tot                                   */
    double utwob0;           /* u%twob(0) = sum over type pairs          */
    double utwob[10];        /* u%twob(1..natat), natat <= 10 (npt <= 4) */
    double urec;             /* u%rec (reciprocal + self + surface)      */
    double ubond;            /* u%bond                                   */
    double virial;           /* virial                                   */
    double ekin;             /* kinetic energy after the step (MD)       */
} msg_energy;

/* Create a handle for one system on the current CUDA device. */
int  msg_create(const msg_params *p, int32_t precision, msg_handle **out);
/* Create a handle for nsys independent systems advanced together. */
int  msg_create_batch(const msg_params *p, int32_t nsys, int32_t precision, msg_handle **out);
void msg_destroy(msg_handle *h);
const char *msg_last_error(const msg_handle *h);
int32_t msg_nsys(const msg_handle *h);

/* NList(iBeforeMacrostep) (Src/nlist.F90:594-596) for every system of the handle:
 * drosum = 0, and the step count istep2 of the inlist > 0 rule restarts. */
int  msg_nlist_before_macrostep(msg_handle *h);

/* Positions ro, velocities rod, accelerations rodd of system isys, [np][3]; NULL skips. */
int  msg_set_state(msg_handle *h, int32_t isys, const double *ro, const double *rod, const double *rodd);
int  msg_get_state(msg_handle *h, int32_t isys, double *ro, double *rod, double *rodd);
/* msg_set_state for every system at once: ro, rod, rodd hold the systems' [np][3]
 * blocks one after another in handle order (rod, rodd may be NULL); every list is
 * rebuilt; one wait for the device. */
int  msg_set_state_all(msg_handle *h, const double *ro, const double *rod, const double *rodd);

/* Rebuild the Verlet list now (SetVListMD semantics: r2 < (rcut+drnlist)^2 with
 * MOLSIM's PBCr2).  Optionally export it in MOLSIM's layout: nneighpn[np] and
 * jpnlist[np][maxnneigh] with 1-based partners owned by the parity rule of
 * Src/nlist.F90:741-744, ascending within each row.  *npair = half-list pairs. */
int  msg_build_nlist(msg_handle *h, int32_t isys, int32_t *nneighpn, int32_t *jpnlist,
                     int32_t maxnneigh, int64_t *npair);

/* UTotal for every system; outputs for system isys: force (kJ/(mol A)),
 * forceo (internal units), energies.  NULL outputs are skipped. */
int  msg_utotal(msg_handle *h, int32_t isys, double *force, double *forceo, msg_energy *e);

/* The forces of system isys from the last force evaluation of the handle
 * (msg_utotal or a step), without recomputing them.  NULL outputs are skipped. */
int  msg_get_forces(msg_handle *h, int32_t isys, double *force, double *forceo);

/* Tuning knobs (no counterpart in the reference).  MSG_TUNE_PAIR_LANES: lanes
 * per particle in the pair kernel scaled by 2^value (-4..4) from the default
 * chosen by the expected row length.  FP64 results move by FP64 rounding only;
 * mixed results by FP32 rounding (a lane's partial sum is regrouped), and stay
 * deterministic for each setting. */
#define MSG_TUNE_PAIR_LANES 1
/* MSG_TUNE_PAIR_KERNEL (mixed path): 2 (default) the FP32 pair kernel with FP64
 * energy and virial sums over a half list (each pair once, partner forces as
 * 64-bit fixed-point atomics), 3 the same kernel over a full list (each pair from
 * both ends, no atomics), 1 the lean FP32 kernel with FP32 energy terms, 0 the
 * kernel shared with the FP64 path.  Switching between half and full lists
 * rebuilds the lists.  Forces agree within the mixed-precision tolerance. */
#define MSG_TUNE_PAIR_KERNEL 2
/* MSG_TUNE_PAIR_UNROLL (lean kernel): row entries each lane keeps in flight,
 * 1, 2 (default) or 4.  Results do not depend on it. */
#define MSG_TUNE_PAIR_UNROLL 3
/* MSG_TUNE_OVERLAP: 1 (default) runs the pair kernel on a second stream beside
 * the SPME chain, 0 runs them one after the other.  MSG_TUNE_PAIR_BLOCKS: pair
 * blocks per SM of the lean kernel (0, the default: as many as fit, or 2 when
 * the pair kernel runs beside the SPME chain).  Neither
 * changes results. */
#define MSG_TUNE_OVERLAP 4
#define MSG_TUNE_PAIR_BLOCKS 5
/* MSG_TUNE_CONV_BLOCKS: blocks per SM of the persistent SPME convolution kernel
 * of a handle created with MSG_SPME_CONV=1 in the environment (0, the default:
 * one per SM, at most one per plane of the handle's grids).  No effect on other
 * handles; results do not depend on it. */
#define MSG_TUNE_CONV_BLOCKS 6
int  msg_tune(msg_handle *h, int32_t key, int32_t value);

/* rodd = massip * forceo (GetLinAcc) from the last msg_utotal. */
int  msg_get_linacc(msg_handle *h);

/* Monte Carlo with single-particle translations (MCPass with SPartMove,
 * Src/mc.F90:1470-1755; DUTotal, Src/denergy.F90:110-230; Metropolis and MCUpdate,
 * Src/mc.F90:5135-5236).  Parameters of one system's sweeps: */
typedef struct msg_mc_params {
    double beta;             /* 1/kT in mol/kJ (MOLSIM's beta)                          */
    const double *dtran;     /* [npt] displacement per type: > 0 cube side, < 0 sphere   */
    int32_t isamp;           /* 0: particles in order; 1: a random particle per trial    */
    int32_t pad;
} msg_mc_params;

/* MCAll parameters of one system (MCAllPass, Src/mc.F90:4024-4178). */
typedef struct msg_mcall_params {
    double beta;                    /* MOLSIM's beta */
    const double *dtranall;         /* [npt] */
} msg_mcall_params;

/* npass MCAll trials for every system (p[nsys]): all particles displaced at once by
 * (Random - 1/2) dtranall(ipt) per coordinate, five draws per particle in MOLSIM order
 * (three displacements and GetRandomTrialOri's two), PBC, the lists rebuilt, one UTotal
 * of the trial and Metropolis on du%tot; a rejected trial restores the configuration and
 * its energies.  The chains use the msg_mc_seed streams; the draws are made in parallel
 * from each particle's place in the stream (the generator jumped ahead), equal to the
 * sequential ones.  accepted [nsys] (optional); e (optional): energies of system isys. */
int  msg_mcall_pass(msg_handle *h, int32_t npass, const msg_mcall_params *p, int64_t *accepted, int32_t isys,
                    msg_energy *e);

/* Random's SAVEd state (ix, iy) after k further draws (Src/mollib.F90:2689-2708), host
 * only: the xorshift part by powers of its GF(2) matrix, the Park-Miller part by powers of
 * 16807 mod 2^31 - 1.  MSG_ERR_ARG for iy <= 0. */
int  msg_random_jump(int32_t ix, int32_t iy, uint32_t k, int32_t out[2]);

/* Random's state of system isys from iseed (its first call, Src/mollib.F90:2689-2708).
 * A system never seeded starts from iseed = isys + 1. */
int  msg_mc_seed(msg_handle *h, int32_t isys, int32_t iseed);

/* npass sweeps of np trial moves for every system (p[nsys]), one Metropolis chain per
 * system, each drawing the reference's random numbers in the reference's order.
 * accepted / hsreject [nsys] (optional): moves accepted and moves rejected for a
 * hard-core or below-table overlap in this call.  e (optional): energies of system
 * isys after the sweeps, from a UTotal at the start plus the accepted moves'
 * differences (MCUpdate).  The lists are rebuilt afterwards.  Any reciprocal method:
 * standard Ewald (DUTwoBodyEwaldRecStd, with lewald2dlc its layer correction) or SPME
 * (DUTwoBodyEwaldRecSPM, Src/denergy.F90:1413-1495, from the spectrum of the mesh at the
 * call and the moved stencils' transforms). */
int  msg_mc_pass(msg_handle *h, int32_t npass, const msg_mc_params *p, int64_t *accepted,
                 int64_t *hsreject, int32_t isys, msg_energy *e);

/* nsteps velocity-Verlet steps of every system, entirely on the device.
 * e (optional): [nsteps] energies of system isys after each step. */
int  msg_velver(msg_handle *h, int32_t nsteps, int32_t isys, msg_energy *e);

/* The drop-in step with host-held state: ro, rod, rodd of system isys (the
 * host's arrays, [np][3], continuing the device's trajectory as with
 * msg_put_state(keep_list = 1)) go to the device, nsteps of MDDriver run, and
 * the new state comes back into the same arrays, with the energies of each
 * step in e (optional, [nsteps]).  Same result as msg_put_state + msg_velver +
 * msg_get_state, with one wait for the device instead of three.  NULL arrays
 * are neither sent nor returned.  With nsteps = 1 and page-locked arrays
 * (cudaHostAlloc / cudaMallocHost, or cudaHostRegister with
 * cudaHostRegisterMapped where the device uses the host address) the exchange
 * runs in place inside the step's CUDA graph, without copies. */
int  msg_velver_host(msg_handle *h, int32_t isys, int32_t nsteps, double *ro, double *rod, double *rodd,
                     msg_energy *e);

/* As msg_velver without energies, but returns once the steps are enqueued on
 * the handle's stream (msg_stream); device errors surface at the next
 * synchronous call. */
int  msg_velver_async(msg_handle *h, int32_t nsteps);

/* nsteps Brownian-dynamics steps.  xi == NULL: FP32 normal noise from a
 * Philox4x32-10 stream keyed by (seed, particle, step); otherwise xi holds
 * caller noise for system isys, [nsteps][np][3] (for the drop-in, MOLSIM's
 * GauRandom sequence).  xi_out (optional) receives the noise used. */
int  msg_bd_step(msg_handle *h, int32_t nsteps, uint64_t seed, int32_t isys,
                 const double *xi, double *xi_out, msg_energy *e);

/* Number of list rebuilds since creation, for system isys. */
int64_t msg_nrebuild(const msg_handle *h, int32_t isys);

/* Like msg_set_state; keep_list != 0 states that ro continues the trajectory the
 * device holds (e.g. it came back from msg_get_state), so the Verlet list and
 * the skin accumulator drosum stay valid and no rebuild is forced. */
int  msg_put_state(msg_handle *h, int32_t isys, const double *ro, const double *rod, const double *rodd,
                   int32_t keep_list);

/* --- Serving support (no counterpart in the reference, which runs one system
 * per process).  A serving loop keeps several handles resident, each on its
 * own stream, and advances them concurrently.  Handles allocate and free
 * device memory stream-ordered from the device's pool and take their cuFFT
 * plans from a process-wide cache, so creating or destroying one does not
 * wait for the others' work. */

/* Device bytes a handle for these systems would allocate (a dry set-up that
 * allocates nothing; cuFFT work areas by cufftEstimateMany). */
int  msg_estimate_bytes(const msg_params *p, int32_t nsys, int32_t precision, int64_t *bytes);
/* Device bytes the handle holds now (its buffers and cuFFT work area). */
int64_t msg_device_bytes(const msg_handle *h);
/* Number of msg_velver_async batches of this handle still running on the
 * device (0: idle and the device error word is clean).  A negative value is
 * minus a status code (a device error raised by the finished steps). */
int  msg_pending(msg_handle *h);
/* Energies of system isys after the last step enqueued (waits for the stream). */
int  msg_get_energy(msg_handle *h, int32_t isys, msg_energy *e);
/* Destroy idle cached cuFFT plans and return unused pool memory to the device
 * (may wait for the device). */
int  msg_trim_caches(void);

/* Instrumentation: the handle's CUDA stream (cudaStream_t), kernel launches
 * issued so far, and per-kernel CUDA-event timers (enabled by msg_set_timing). */
void   *msg_stream(const msg_handle *h);
int64_t msg_launch_count(const msg_handle *h);
int     msg_set_timing(msg_handle *h, int32_t on);
/* Timer k (0 <= k < msg_ntimers()): name, summed device milliseconds, launches. */
int32_t msg_ntimers(void);
int     msg_kernel_time(const msg_handle *h, int32_t k, const char **name, double *total_ms, int64_t *launches);

/* UTwoBodyA's pair force, energy and virial on the caller's own MOLSIM arrays,
 * allocating nothing.  No counterpart in the reference: it serves callers that
 * cannot call cudaMalloc (a host whose device memory all comes from its own
 * pool or a framework allocator, or a memory budget that forbids a library to
 * grow).  All arrays are device-accessible memory the caller owns: ro [np][3],
 * iptpn [np] (1-based), nneighpn [np] and jpnlist [np][maxnneigh] (1-based
 * partners), ubuf [nbuf]; force [np][3] is overwritten in kJ/(mol A) (MOLSIM
 * `force` before UTotal's unit scaling), utwob [natat+1] receives
 * u%twob(0..natat), virial [1] the pair virial.  lmc = 0: the list is MOLSIM's
 * MD half list (SetVList, every pair in one row); lmc = 1: a full list (every
 * pair in both rows, as Monte Carlo builds it), and pairs with jp < ip are
 * skipped as UTwoBodyA does under lmc (Src/energy.F90:466-468).  A row longer
 * than maxnneigh, or an index out of range, returns MSG_ERR_ARG.  boxlen,
 * iubuflow, r2umin and r2atat (may be NULL) are host arrays; stop_ipjp (may be
 * NULL) receives the 1-based ip and jp of the pair that raised a nonzero
 * status (StopUTwoBodyA's report), zeros otherwise.  Rectangular periodic box
 * only (PBCr2's lbcbox branch).  The only scratch is a fixed static device
 * array (about 88 KiB per GPU, held until exit), so np <= 262144; larger np
 * returns MSG_ERR_ARG.  The first call on a device looks up that array's
 * address: make it before any stream capture.  Calls share the array; calls
 * that overlap on the GPU race.  Every call waits for its work on `stream` (a
 * cudaStream_t, NULL for the default stream) before it returns. */
int  msg_utwobody_noalloc(int32_t np, int32_t npt, const double boxlen[3], double rcut, const double *ro,
                          const int32_t *iptpn, const int32_t *nneighpn, const int32_t *jpnlist,
                          int32_t maxnneigh, int32_t lmc, const double *ubuf, int32_t nbuf,
                          const int32_t *iubuflow, const double *r2umin, const double *r2atat, double *force,
                          double *utwob, double *virial, int32_t *stop_ipjp, void *stream);

/* UTwoBodyP (Src/energy.F90:786-896): site-site pair energy, forces and virial of
 * polyatomic particles over MOLSIM's particle list, as UTotal calls it for molecules.
 * Host arrays in MOLSIM's layout, 1-based indices: ro [np][3] particle positions,
 * r [na][3] atom positions, iptpn [np] particle type, ianpn [np] first atom of each
 * particle, napt [npt] atoms per particle type, iatan [na] atom type (nat types),
 * nneighpn [np] and jpnlist [np][maxnneigh] the particle list; ubuf/iubuflow/r2umin
 * the atom-type table (natat = nat(nat+1)/2 pairs).  A pair interacts when its centres
 * are within rcut after PBC2's box shift (box cell).  Out: force [na][3] (kJ/(mol A),
 * overwritten), utwob [npt(npt+1)/2 + 1] = u%twob(0:nptpt) by particle-type pair,
 * virial [1]; kernel_ms (optional): device time of the computation.
 * MSG_ERR_TABLE_MIN for an atom pair below r2umin (StopUTwoBodyP). */
int  msg_utwobody_p(int32_t np, int32_t na, int32_t npt, int32_t nat, const double boxlen[3], double rcut,
                    const double *ro, const double *r, const int32_t *iptpn, const int32_t *ianpn,
                    const int32_t *napt, const int32_t *iatan, const int32_t *nneighpn, const int32_t *jpnlist,
                    int32_t maxnneigh, const double *ubuf, int32_t nbuf, const int32_t *iubuflow,
                    const double *r2umin, double *force, double *utwob, double *virial, float *kernel_ms);

/* nsteps of MDDriver for rigid polyatomic particles (VelVer with lpolyatom,
 * Src/md.F90:252-410), the particle list held fixed: centre and quaternion update,
 * QuaNorm, QuaToOri, PBC of the centres, SetAtomPos, UTwoBodyP, forces, torques and
 * the molecular virial (UTotal, Src/energy.F90:403-426), GetLinAcc, and nvvite rounds of
 * QuaVelToAngVel + GetAngAcc for the quaternion velocities (tvvite: their trial step).
 * State (host arrays, MOLSIM layout) advanced in place: ro, rod, rodd [np][3], qua, quad,
 * quadd [np][4] (qua(0:3)), r [na][3]; ra [npt][maxsite][3] the sites in the principal
 * frame, masspt [npt], momp [npt][3] the principal moments; the rest as msg_utwobody_p.
 * utwob and virial of the last step; kernel_ms (optional): device time of the steps. */
int  msg_velver_p(int32_t nsteps, int32_t np, int32_t na, int32_t npt, int32_t nat, const double boxlen[3],
                  double rcut, double tstep, int32_t nvvite, double tvvite, double *ro, double *rod, double *rodd,
                  double *qua, double *quad, double *quadd, double *r, const int32_t *iptpn, const int32_t *ianpn,
                  const int32_t *napt, const int32_t *iatan, const double *ra, int32_t maxsite,
                  const double *masspt, const double *momp, const int32_t *nneighpn, const int32_t *jpnlist,
                  int32_t maxnneigh, const double *ubuf, int32_t nbuf, const int32_t *iubuflow,
                  const double *r2umin, double *utwob, double *virial, float *kernel_ms);

/* UEwald over the sites of polyatomic particles (Src/energy.F90:905-958) with the
 * standard reciprocal sum (UEwaldRecStd, :964-1104; k-vectors of EwaldSetup 'std' from
 * ncut and ncutregion 0 sphere / 1 cube), UEwaldSelf's atomic term and its molecular term
 * (the erf(alpha r)/r of every site pair inside a particle, :1301-1345) and, when lsurf,
 * UEwaldSurf (:1349-1371).  Sites r [na][3] with charges az [na]; the particles' sites
 * from iptpn, ianpn (1-based) and napt [npt].  force [na][3] is overwritten with the
 * Ewald forces; urec = u%rec and virrec its virial, both scaled by epsfp (EpsiFourPi)
 * as UEwald does.  The sums are deterministic (fixed point, fixed order).
 * MSG_ERR_ARG for ncut outside 1..100 or a particle whose sites leave 1..na. */
int  msg_uewald_sites(int32_t na, const double boxlen[3], double ualpha, int32_t ncut, int32_t ncutregion,
                      int32_t lsurf, double epsfp, const double *r, const double *az, int32_t np,
                      const int32_t *iptpn, const int32_t *ianpn, const int32_t *napt, int32_t npt,
                      double *force, double *urec, double *virrec, float *kernel_ms);

/* The site Ewald sum of msg_velver_p_ewald: MOLSIM's txewaldrec over the sites. */
typedef struct msg_site_ewald {
    int32_t lewald;                 /* 1: SPME ('spm'), 2: standard Ewald ('std') */
    int32_t order, nmesh;           /* SPME: spline order 4..8, mesh edge (even) */
    int32_t ncut, ncutregion;       /* standard Ewald: 1..100; 0 sphere, 1 cube */
    int32_t lsurf;                  /* UEwaldSurf */
    double ualpha, epsi_four_pi;
    const double *az;               /* [na] site charges, zat(iatan(ia)) */
} msg_site_ewald;

/* msg_uewald_sites with SPME over the sites (UEwaldRecSPM, Src/energy.F90:1207-1297, with
 * SPMFFTRec :6525-6587 and EwaldSetup's mesh factors :6980-7018): spline order 4..8, nmesh
 * even, 8..1024.  The charge mesh is spread in 64-bit fixed point, so the result repeats
 * bit for bit. */
int  msg_uewald_sites_spm(int32_t na, const double boxlen[3], double ualpha, int32_t order, int32_t nmesh,
                          int32_t lsurf, double epsfp, const double *r, const double *az, int32_t np,
                          const int32_t *iptpn, const int32_t *ianpn, const int32_t *napt, int32_t npt,
                          double *force, double *urec, double *virrec, float *kernel_ms);

/* msg_velver_p with lewald: every step adds the site Ewald sum (as msg_uewald_sites or
 * msg_uewald_sites_spm computes it) to the site forces before the forces, torques and
 * molecular virial (UTotal, Src/energy.F90:335-352, 403-426), and its reciprocal virial to
 * virial; urec = u%rec of the last step.  The table ubuf carries the erfc-screened site
 * pairs (lewald in PotTwoBodyTab).  MSG_ERR_ARG as the site Ewald calls. */
int  msg_velver_p_ewald(int32_t nsteps, int32_t np, int32_t na, int32_t npt, int32_t nat, const double boxlen[3],
                        double rcut, double tstep, int32_t nvvite, double tvvite, double *ro, double *rod,
                        double *rodd, double *qua, double *quad, double *quadd, double *r, const int32_t *iptpn,
                        const int32_t *ianpn, const int32_t *napt, const int32_t *iatan, const double *ra,
                        int32_t maxsite, const double *masspt, const double *momp, const int32_t *nneighpn,
                        const int32_t *jpnlist, int32_t maxnneigh, const double *ubuf, int32_t nbuf,
                        const int32_t *iubuflow, const double *r2umin, const msg_site_ewald *ew, double *utwob,
                        double *urec, double *virial, float *kernel_ms);

/* Set-up helpers (host only). */
double msg_rcut_to_alpha(double uewaldtol, double q2sum, double epsi_four_pi,
                         double boxlenshort, double rcut, int32_t *status);
/* ncut of the standard Ewald sum for alpha at uewaldtol (iewaldopt 3). */
int32_t msg_alpha_to_ncut(double uewaldtol, double q2sum, double epsi_four_pi,
                          double boxlenshort, double ualpha, int32_t *status);

typedef struct msg_tab_params {
    int32_t npt;
    const double *zat, *sigat, *epsat;   /* [npt] */
    double rcut, ualpha, epsi_four_pi;
    int32_t lewald, lljcut;
    double ljrcut, ljushift;
    double r2uminin, utoltab, ftoltab, umaxtab, fmaxtab, rumaxfac;
} msg_tab_params;

/* Build MOLSIM's pair table.  Returns MSG_OK or MSG_ERR_CAPACITY (nbuf too
 * small) or MSG_ERR_ARG (no convergence). */
int  msg_pot_tab(const msg_tab_params *p, double *ubuf, int32_t nbuf, int32_t *iubuflow,
                 int32_t *nugrid, double *r2umin, int32_t *nused);

#ifdef __cplusplus
}
#endif
#endif

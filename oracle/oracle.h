/*
 * oracle.h -- FP64 CPU restatement of MOLSIM's serial force/energy hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path is
 * compared against.  Only the tests, the smoke check and the CPU-baseline leg
 * of the benchmark may load it; the product library never links or calls it.
 *
 * Every routine names the MOLSIM (TomHoefken/molsim) source it restates,
 * as Src/<file>:<line>.  Arrays follow MOLSIM's layout: Fortran (3,N) is
 * C [N][3]; particle types, pair-table offsets and neighbour indices are
 * 1-based exactly as in MOLSIM's globals (Src/mol.F90:1087-1135).
 *
 * Parity status: PARITY UNPINNED against the reference itself.  The
 * reference is Fortran, ships no golden vectors for this path, and no Fortran
 * compiler is installed alongside this code, so no output of the compiled
 * reference is available.  These routines are checked instead against the
 * reference's own in-code self checks (CheckUBuffer tolerances, TestCellList
 * completeness, TestEwaldSPM-style SPME-vs-converged checks, standard Ewald)
 * and against analytic known answers (isolated ion pair, harmonic bond,
 * rock-salt Madelung constant, NumPy FFT conventions).
 */
#ifndef MOLSIM_ORACLE_H
#define MOLSIM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- physical constants and units, Src/mol.F90:60-80, Src/molsim.F90:786-805 ---- */
double or_epsi0_four_pi(void);          /* e^2/(4 pi eps0 A) N_A / 1e3  [kJ A / mol] */
double or_gas_constant(void);           /* J/(mol K) */

/* ---- scalar numerics ---- */
double or_erf2(double x);                                   /* Src/mollib.F90:215-274 */
void   or_ewald_ufac(double r1, double ualpha, double c[3]);/* Src/potential.F90:2938-2960 */
void   or_cardinal_bspline(int order, double pos, int32_t *kmax,
                           double *values, double *derivs);  /* Src/mollib.F90:1629-1683 */
double or_rcut_to_alpha(double uewaldtol, double q2sum, double epsi_four_pi,
                        double boxlenshort, double rcut, int32_t *status); /* Src/energy.F90:7090-7105 */
int32_t or_alpha_to_ncut(double uewaldtol, double q2sum, double epsi_four_pi,
                         double boxlenshort, double ualpha, int32_t *status); /* Src/energy.F90:7066-7081 */
double or_ewald_error_ureal(double q2sum, double l, double alpha, double rcut,
                            double unit);                   /* Src/potential.F90:2995-3018 */

/* ---- pair potential (1,6,12) and its table, Src/potential.F90:868-1258, 1349-1425 ---- */
typedef struct or_tab_params {
    int32_t npt;             /* particle (= atom) types */
    const double *zat;       /* [npt] charge, e */
    const double *sigat;     /* [npt] LJ sigma, A */
    const double *epsat;     /* [npt] LJ epsilon, kJ/mol */
    double rcut;             /* A */
    double ualpha;           /* Ewald alpha, 1/A */
    double epsi_four_pi;     /* Epsi0FourPi / relpermitt */
    int32_t lewald;          /* erfc-screened Coulomb */
    int32_t lljcut;          /* cut-and-shift LJ at ljrcut*sigma */
    double ljrcut;
    double ljushift;
    double r2uminin;
    double utoltab, ftoltab, umaxtab, fmaxtab;
    double rumaxfac;
} or_tab_params;

/* Potential value and r-derivatives u0, u1=du/dr, u2=d2u/dr2 (Pot_1_6_12 'calc'). */
void or_pot_1_6_12(const or_tab_params *p, int iat, int jat, double r1,
                   double *u0, double *u1, double *u2);

/* Build the full table (PotTwoBodyTab1/2/3 + SetUBuffer + CheckUBuffer).
 * ubuf capacity nbuf doubles; iubuflow/nugrid/r2umin/rumin/rumax sized natat.
 * Returns 0, or 2 when nbuf is too small, or 6 when dr/igrid did not converge. */
int or_pot_tab(const or_tab_params *p, double *ubuf, int32_t nbuf,
               int32_t *iubuflow, int32_t *nugrid, double *r2umin,
               double *rumin, double *rumax, int32_t *nused);

/* ---- SPME setup, Src/energy.F90:6855-7019 ---- */
void or_ewald_setup_spm(int s, int order, double ualpha, const double boxlen[3],
                        double *meshfac, double *energyfac, double *virfac);

/* ---- FFT with FFTW's unnormalised r2c (e^-i) / c2r (e^+i) conventions ----
 * real grid [s][s][s] (x fastest) <-> complex [s][s][s/2+1] interleaved re,im */
void or_fft3_r2c(int s, const double *in, double *out);
void or_fft3_c2r(int s, const double *in, double *out);

/* ---- the simulated system (mirrors the MolModule globals used on the path) ---- */
typedef struct or_params {
    int32_t np, npt;
    double boxlen[3];
    double rcut, drnlist;
    const int32_t *iptpn;    /* [np] 1-based type */
    const double *az;        /* [np] charge, e */
    const double *masspt;    /* [npt] mass, g/mol */
    const double *ubuf; int32_t nbuf;
    const int32_t *iubuflow; /* [natat] 1-based */
    const double *r2umin;    /* [natat] */
    const double *r2atat;    /* [natat] */
    int32_t lewald;          /* 0 none; 1 SPME (txewaldrec 'spm'); 2 standard Ewald ('std') */
    int32_t order, nmesh, lsurf;
    double ualpha, epsi_four_pi;
    int32_t nbond;
    const int32_t *bond_ij;  /* [nbond][2] 1-based, in chain order */
    const double *bond_k;    /* [nbond] force constant already divided by power */
    const double *bond_eq;   /* [nbond] */
    const int32_t *bond_p;   /* [nbond] power */
    double tstep;
    int32_t maxnneigh;       /* row capacity of jpnlist */
    int32_t lcellbuild;      /* 1: build the Verlet list through cells (same pair set) */
    int32_t ncut;            /* standard Ewald: largest |n| component of k = 2 pi n / L */
    int32_t ncutregion;      /* standard Ewald: 0 'sphere' (|n|^2 <= ncut^2), 1 'cube' */
    int32_t lewald2dlc;      /* 1: the 2D layer correction (UEwaldRecStd2dlc) and UEwaldSurf's 2D form */
    int32_t inlist;          /* NList: 0 skin test; n > 0 rebuild when mod(istep2, n) == 0 */
    int32_t lvlistllist;     /* 1: SetVList builds through linked lists (SetLList + SetVListMDLList) */
} or_params;

typedef struct or_sys or_sys;

or_sys *or_create(const or_params *p);
void    or_destroy(or_sys *s);
void    or_set_state(or_sys *s, const double *ro, const double *rod, const double *rodd);
void    or_get_state(const or_sys *s, double *ro, double *rod, double *rodd, double *drosum);
void    or_set_drosum(or_sys *s, const double *drosum);

/* SetVList for MD/BD, Src/nlist.F90:686-716: SetVListMD (:724-759), or with lvlistllist
 * SetLList(rcut+drnlist) + SetVListMDLList (:1168-1221, :769-811).  Returns 3 on a row
 * beyond maxnneigh; 6 when the linked-list grid has no cell or more than 1000 cells. */
int  or_set_vlist(or_sys *s);
/* NList(iBeforeMacrostep), Src/nlist.F90:594-596: drosum = 0; also restarts istep2. */
void or_nlist_before_macrostep(or_sys *s);
void or_get_vlist(const or_sys *s, int32_t *nneighpn, int32_t *jpnlist);
int64_t or_npair(const or_sys *s);

/* UTotal.  u = [tot, twob(0..nptpt), rec, bond]; virial scalar.
 * force is in kJ/(mol A) (MOLSIM `force`), forceo in internal units (`forceo`). */
int  or_utotal(or_sys *s, double *force, double *forceo, double *u, double *virial);

/* One velocity-Verlet step (VelVer linear part, GetKinEnergy, NList skin test).
 * Returns status; *rebuilt=1 when the list was rebuilt after the step. */
int  or_velver_step(or_sys *s, double *ekin, int32_t *rebuilt);

/* One Ermak-McCammon step (BDStep, UTotal, NList skin test) with caller noise
 * xi[np][3]; fac1/fac2 per type. */
int  or_bd_step(or_sys *s, const double *xi, const double *fac1, const double *fac2,
                int32_t *rebuilt);

/* MOLSIM's GauRandom with its SAVEd spare carried in (flag, save). */
double or_gau_random(int32_t *iseed, int32_t *flag, double *save);

/* The reference's own rebuild test (NList iSimulationStep branch) on a given
 * drostep; updates drosum, returns 1 when a rebuild is due. */
int  or_skin_test(or_sys *s, const double *drostep, double *max1, double *max2);

/* ---- Monte Carlo: single-particle translations ---- */
/* Random, Src/mollib.F90:2689-2708: state = {ix, iy}; or_random_init is its
 * first-call initialisation from iseed. */
void   or_random_init(int32_t iseed, int32_t state[2]);
double or_random_next(int32_t state[2]);
void   or_mc_seed(or_sys *s, int32_t iseed);
/* npass MCPass sweeps of single-particle translations (SPartMove, DUTotal,
 * Metropolis, MCUpdate).  dtran[npt] (>0 cube, <0 sphere), beta = 1/kT in the
 * energy unit; u = [tot, twob(0..natat), rec, bond] from the last or_utotal, advanced
 * by every accepted move.  Needs lewald 0 or 2 (standard Ewald); returns 6 otherwise. */
/* MCPass with single-particle and chain moves (CallMove's selection by the cumulative pspart,
 * pchain [npt]; ChainMove translates a whole chain by one displacement of dtranchain).
 * Chains are contiguous ranges chain_first (0-based) / chain_len. */
int    or_mc_pass_moves(or_sys *s, int npass, int isamp, const double *dtran, const double *pspart,
                        const double *pchain, const double *dtranchain, int nchain, const int32_t *chain_first,
                        const int32_t *chain_len, double beta, double *u, int64_t *accepted, int64_t *hsreject);
/* MCAllPass: all particles displaced at once (five draws each), UTotal, Metropolis. */
int    or_mcall_pass(or_sys *s, int npass, const double *dtranall, double beta, double *u, int64_t *accepted);
int    or_mc_pass(or_sys *s, int npass, int isamp, const double *dtran, double beta, double *u,
                  int64_t *accepted, int64_t *hsreject);

/* ---- polyatomic particles ---- */
/* UTwoBodyP (Src/energy.F90:786-896): site-site pair energy, forces and virial over the
 * particle list; 1-based MOLSIM arrays; force [na][3] overwritten, utwob [nptpt+1],
 * virial [1].  Returns 1 for an atom pair below r2umin, 2 for a table overrun. */
int    or_utwobody_p(int32_t np, int32_t na, int32_t npt, int32_t nat, const double boxlen[3], double rcut,
                     const double *ro, const double *r, const int32_t *iptpn, const int32_t *ianpn,
                     const int32_t *napt, const int32_t *iatan, const int32_t *nneighpn,
                     const int32_t *jpnlist, int32_t maxnneigh, const double *ubuf, int32_t nbuf,
                     const int32_t *iubuflow, const double *r2umin, double *force, double *utwob,
                     double *virial);

/* nsteps of VelVer for rigid polyatomic particles (Src/md.F90:252-410, lpolyatom), the
 * particle list held fixed; state arrays advanced in place (qua/quad/quadd [np][4]);
 * ra [npt][maxsite][3] sites in the principal frame, masspt [npt], momp [npt][3]. */
int    or_velver_p(int32_t nsteps, int32_t np, int32_t na, int32_t npt, int32_t nat, const double boxlen[3],
                   double rcut, double tstep, int32_t nvvite, double tvvite, double *ro, double *rod,
                   double *rodd, double *qua, double *quad, double *quadd, double *r, const int32_t *iptpn,
                   const int32_t *ianpn, const int32_t *napt, const int32_t *iatan, const double *ra,
                   int32_t maxsite, const double *masspt, const double *momp, const int32_t *nneighpn,
                   const int32_t *jpnlist, int32_t maxnneigh, const double *ubuf, int32_t nbuf,
                   const int32_t *iubuflow, const double *r2umin, double *utwob, double *virial);

/* or_velver_p with the site Ewald sum (or_uewald_sites) in every step's forces and virial;
 * *urec = u%rec of the last step. */
int    or_velver_p_ewald(int32_t nsteps, int32_t np, int32_t na, int32_t npt, int32_t nat, const double boxlen[3],
                         double rcut, double tstep, int32_t nvvite, double tvvite, double *ro, double *rod,
                         double *rodd, double *qua, double *quad, double *quadd, double *r, const int32_t *iptpn,
                         const int32_t *ianpn, const int32_t *napt, const int32_t *iatan, const double *ra,
                         int32_t maxsite, const double *masspt, const double *momp, const int32_t *nneighpn,
                         const int32_t *jpnlist, int32_t maxnneigh, const double *ubuf, int32_t nbuf,
                         const int32_t *iubuflow, const double *r2umin, const double *az, double ualpha,
                         int32_t lewald, int32_t ncut, int32_t ncutregion, int32_t order, int32_t nmesh,
                         int32_t lsurf, double epsfp, double *utwob, double *urec, double *virial);

/* UEwald over the sites of polyatomic particles: standard reciprocal sum, UEwaldSelf's
 * atomic and molecular (intramolecular erf) terms, surface term; force [na][3] overwritten. */
int    or_uewald_sites(int32_t na, const double boxlen[3], double ualpha, int32_t ncut, int32_t ncutregion,
                       int32_t lsurf, double epsfp, const double *r, const double *az, int32_t np,
                       const int32_t *iptpn, const int32_t *ianpn, const int32_t *napt, double *force,
                       double *urec, double *virrec);
/* The same with SPME over the sites (order, nmesh). */
int    or_uewald_sites_spm(int32_t na, const double boxlen[3], double ualpha, int32_t order, int32_t nmesh,
                           int32_t lsurf, double epsfp, const double *r, const double *az, int32_t np,
                           const int32_t *iptpn, const int32_t *ianpn, const int32_t *napt, double *force,
                           double *urec, double *virrec);

#ifdef __cplusplus
}
#endif
#endif

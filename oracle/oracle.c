/*
 * oracle.c -- FP64 CPU restatement of MOLSIM's serial force/energy hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Compiled with -O2
 * -ffp-contract=off so that every a*b+c rounds twice, as the reference's
 * gfortran/x86-64 build does.  Expressions keep the reference's evaluation
 * order (Fortran evaluates a*b*c as (a*b)*c; x**2 as x*x).
 */
#include "oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Src/mol.F90:60-80 */
static const double Pi = 3.1415926535897932;
static const double AvNo = 6.02214179e23;
static const double ECh = 1.602176487e-19;
static const double GasConstant = 8.314472;
static const double Epsi0 = 8.854187817e-12;

/* Default unit scales, Src/molsim.F90:786-795 */
static const double scllen = 1.0e-10, sclmas = 1.0e-03, scltim = 1.0e-12, sclene = 1.0e+03;

double or_gas_constant(void) { return GasConstant; }

/* Epsi0FourPi = ECh**2/(FourPi*Epsi0*scllen)*AvNo/sclene, Src/molsim.F90:805 */
double or_epsi0_four_pi(void)
{
    double FourPi = 4.0 * Pi;
    return ECh * ECh / (FourPi * Epsi0 * scllen) * AvNo / sclene;
}

static double sclfor(void)
{
    double sclvel = scllen / scltim;
    double sclacc = sclvel / scltim;
    return sclacc * sclmas;
}

/* ------------------------------------------------------------------ */
/* Erf2, Src/mollib.F90:215-274 (NAG Chebyshev form).                 */
/* The reference's second branch starts from c(18), runs j=16..2 and  */
/* finishes with c(j) where j==1 after the loop: c(17) is never used. */
/* ------------------------------------------------------------------ */
double or_erf2(double x)
{
    static const double c[19] = {0.0,
        1.9449071068178803, 4.20186582324414e-2, -1.86866103976769e-2,
        5.1281061839107e-3, -1.0683107461726e-3, 1.744737872522e-4,
        -2.15642065714e-5, 1.7282657974e-6, -2.00479241e-8,
        -1.64782105e-8, 2.0008475e-9, 2.57716e-11,
        -3.06343e-11, 1.9158e-12, 3.703e-13,
        -5.43e-14, -4.0e-15, 1.2e-15};
    static const double d[18] = {0.0,
        1.4831105640848036, -3.010710733865950e-1, 6.89948306898316e-2,
        -1.39162712647222e-2, 2.4207995224335e-3, -3.658639685849e-4,
        4.86209844323e-5, -5.7492565580e-6, 6.113243578e-7,
        -5.89910153e-8, 5.2070091e-9, -4.232976e-10,
        3.18811e-11, -2.2361e-12, 1.467e-13,
        -9.0e-15, 5.0e-16};
    const double sqrtpi = 1.7724538509055160, xup = 6.25;
    const int ncfc = 18, ncfd = 17;
    double xv = fabs(x), x2, bj = 0.0, bjp1, bjp2;
    int j;
    if (xv <= 2.0) {
        x2 = x * x - 2.0;
        bjp2 = 0.0;
        bjp1 = d[ncfd];
        for (j = ncfd - 1; j >= 2; --j) {
            bj = x2 * bjp1 - bjp2 + d[j];
            bjp2 = bjp1;
            bjp1 = bj;
        }
        bj = x2 * bjp1 - bjp2 + d[1];
        return 0.5 * (bj - bjp2) * x;
    } else if (xv < xup) {
        x2 = 2.0 - 20.0 / (xv + 3.0);
        bjp2 = 0.0;
        bjp1 = c[ncfc];
        for (j = ncfd - 1; j >= 2; --j) {
            bj = x2 * bjp1 - bjp2 + c[j];
            bjp2 = bjp1;
            bjp1 = bj;
        }
        /* Fortran loop variable after completion: j == 1 */
        bj = x2 * bjp1 - bjp2 + c[1];
        x2 = 0.5 * (bj - bjp2) / xv * exp(-x * x) / sqrtpi;
        return (1.0 - x2) * (x >= 0.0 ? 1.0 : -1.0);
    }
    /* xv > xup (xv == xup exactly is left undefined by the reference) */
    return x >= 0.0 ? 1.0 : -1.0;
}

/* CalcEwaldUfac, Src/potential.F90:2938-2960 */
void or_ewald_ufac(double r1, double ualpha, double c[3])
{
    const double fac = 1.12837916709;
    double ra = ualpha * r1;
    double er = or_erf2(ra);
    double ex = fac * exp(-(ra * ra));
    c[0] = 1.0 - (er);
    c[1] = 1.0 - (er - ra * ex);
    c[2] = 1.0 - (er - ra * (1.0 + ra * ra) * ex);
}

/* CardinalBSpline, Src/mollib.F90:1629-1683 (values + first derivatives) */
void or_cardinal_bspline(int order, double pos, int32_t *kmax, double *values, double *derivs)
{
    double lastvals[32];
    int v = (int)floor(pos), n, i;
    double x = pos - v, a;
    *kmax = v;
    for (i = 0; i < order; ++i) lastvals[i] = 0.0;
    values[0] = x;
    if (order > 1) {
        values[1] = 1.0 - x;
        for (n = 3; n <= order; ++n) {
            for (i = 0; i < order; ++i) lastvals[i] = values[i];
            values[0] = x * lastvals[0] / (n - 1);
            for (i = 1; i <= n - 2; ++i) {
                a = i + x;
                values[i] = (a * lastvals[i] + (n - a) * lastvals[i - 1]) / (n - 1);
            }
            values[n - 1] = (1 - x) * lastvals[n - 2] / (n - 1);
        }
        n = order;
        if (derivs) {
            derivs[0] = lastvals[0];
            for (i = 1; i <= n - 2; ++i) derivs[i] = lastvals[i] - lastvals[i - 1];
            derivs[n - 1] = -lastvals[n - 2];
        }
    }
}

/* RcutToAlpha, Src/energy.F90:7090-7105 (charged system, lq2sum == 0) */
double or_rcut_to_alpha(double uewaldtol, double q2sum, double epsi_four_pi,
                        double boxlenshort, double rcut, int32_t *status)
{
    double br = boxlenshort * rcut;
    double y = (uewaldtol / (q2sum * epsi_four_pi)) * sqrt(2.0 * (br * br * br));
    double xold = 1.0e-1, xnew = 0.0;
    int i;
    for (i = 1; i <= 40; ++i) {
        xnew = (1.0 / rcut) * sqrt(-log(y * (xold * xold)));
        if (fabs(xold - xnew) / xnew < 1.0e-6) break;
        xold = xnew;
    }
    if (status) *status = (i > 40) ? 6 : 0;
    return xnew;
}

/* AlphaToNcut, Src/energy.F90:7066-7081 (charged system, lq2sum == 0) */
int32_t or_alpha_to_ncut(double uewaldtol, double q2sum, double epsi_four_pi, double boxlenshort,
                         double ualpha, int32_t *status)
{
    double y = (uewaldtol / (q2sum * epsi_four_pi)) * (Pi * Pi / ((ualpha * ualpha) * boxlenshort));
    double xold = 1.0, xnew = 0.0;
    int i;
    for (i = 1; i <= 40; ++i) {
        xnew = (ualpha * boxlenshort / Pi) *
               sqrt(-log(y * xold / (1.0 + 1.0 / (ualpha * boxlenshort * sqrt(xold)))));
        if (fabs(xold - xnew) / xnew < 1.0e-6) break;
        xold = xnew;
    }
    if (status) *status = (i > 40) ? 6 : 0;
    return (int32_t)(xnew + 1.0);
}

/* EwaldErrorUReal, Src/potential.F90:2995-3018 (charges) */
double or_ewald_error_ureal(double q2sum, double l, double alpha, double rcut, double unit)
{
    double fac = (alpha * rcut) * (alpha * rcut);
    return unit * q2sum * sqrt(rcut / (2.0 * (l * l * l))) / fac * exp(-fac);
}

/* ------------------------------------------------------------------ */
/* Pair potential table                                                */
/* ------------------------------------------------------------------ */

/* iptpt / iatat enumeration, Src/particle.F90:1528-1562 (1-based) */
static int pair_index(int npt, int i, int j)
{
    int a = i < j ? i : j, b = i < j ? j : i, k = 0, ii, jj;
    for (ii = 1; ii <= npt; ++ii)
        for (jj = ii; jj <= npt; ++jj) {
            ++k;
            if (ii == a && jj == b) return k;
        }
    return 0;
}

/* x**6 as gfortran expands an integer power: (x*x*x)**2 */
static double pow6(double x) { double x3 = x * x * x; return x3 * x3; }

/* Pot_1_6_12 'calc', Src/potential.F90:1349-1425 (types are 1-based) */
void or_pot_1_6_12(const or_tab_params *p, int iat, int jat, double r1,
                   double *u0, double *u1, double *u2)
{
    double qq = p->zat[iat - 1] * p->zat[jat - 1] * p->epsi_four_pi;
    double sig = 0.5 * (p->sigat[iat - 1] + p->sigat[jat - 1]);
    double eps = sqrt(p->epsat[iat - 1] * p->epsat[jat - 1]);
    double r1i = 1.0 / r1;
    double fac = pow6(sig * r1i);
    double c[3] = {1.0, 1.0, 1.0};
    double us0, us1, us2;
    if (p->lewald) or_ewald_ufac(r1, p->ualpha, c);
    us0 = +4.0 * eps * (fac * fac - fac);
    us1 = -(24.0 * eps * (2.0 * (fac * fac) - fac) * r1i);
    us2 = +24.0 * eps * (26.0 * (fac * fac) - 7.0 * fac) * (r1i * r1i);
    if (p->lljcut) {
        if (r1 < p->ljrcut * sig) {
            us0 = us0 + p->ljushift * eps;
        } else {
            us0 = 0.0; us1 = 0.0; us2 = 0.0;
        }
    }
    *u0 = qq * c[0] * r1i + us0;
    *u1 = -(qq * c[1] * (r1i * r1i)) + us1;
    *u2 = 2.0 * qq * c[2] * (r1i * r1i * r1i) + us2;
}

/* SetUBuffer, Src/potential.F90:1139-1220 */
static void set_ubuffer(double zlow, double u0low, double u1low, double u2low,
                        double zupp, double u0upp, double u1upp, double u2upp, double *t)
{
    double dz1, dz2, dz3, rlow, rupp, w0low, w1low, w2low, w0upp, w1upp, w2upp, a, b, c;
    int k;
    if (u0low == 0.0 && u0upp == 0.0) {
        t[0] = zlow;
        for (k = 1; k < 12; ++k) t[k] = 0.0;
        return;
    }
    rlow = sqrt(zlow);
    rupp = sqrt(zupp);
    dz1 = zupp - zlow;
    dz2 = dz1 * dz1;
    dz3 = dz2 * dz1;
    w0low = u0low;
    w0upp = u0upp;
    w1low = 0.50 * u1low / rlow;
    w1upp = 0.50 * u1upp / rupp;
    w2low = 0.25 * (u2low - u1low / rlow) / zlow;
    w2upp = 0.25 * (u2upp - u1upp / rupp) / zupp;
    a = 6.0 * (w0upp - w0low - w1low * dz1 - 0.5 * w2low * dz2) / dz3;
    b = 2.0 * (w1upp - w1low - w2low * dz1) / dz2;
    c = (w2upp - w2low) / dz1;
    t[0] = zlow;
    t[1] = w0low;
    t[2] = w1low;
    t[3] = 0.5 * w2low;
    t[4] = (10.0 * a - 12.0 * b + 3.0 * c) / (6.0);
    t[5] = (-15.0 * a + 21.0 * b - 6.0 * c) / (6.0 * dz1);
    t[6] = (2.0 * a - 3.0 * b + c) / (2.0 * dz2);
    t[7] = -2.0 * t[2];
    t[8] = -4.0 * t[3];
    t[9] = -6.0 * t[4];
    t[10] = -8.0 * t[5];
    t[11] = -10.0 * t[6];
}

/* CheckUBuffer, Src/potential.F90:1224-1258 */
static void check_ubuffer(const or_tab_params *p, int iat, int jat, double rlow, double rupp,
                          const double *t, int *ok, int *repul)
{
    const int ncheck = 11;
    double dr = (rupp - rlow) / (ncheck - 1), r1, dz, usum, fsum, u0, u1, u2;
    int icheck;
    *ok = 0;
    *repul = 0;
    for (icheck = 1; icheck <= ncheck; ++icheck) {
        r1 = rlow + dr * (icheck - 1);
        or_pot_1_6_12(p, iat, jat, r1, &u0, &u1, &u2);
        dz = r1 * r1 - rlow * rlow;
        usum = t[1] + dz * (t[2] + dz * (t[3] + dz * (t[4] + dz * (t[5] + dz * t[6]))));
        fsum = t[7] + dz * (t[8] + dz * (t[9] + dz * (t[10] + dz * t[11])));
        fsum = r1 * fsum;
        if (fabs(usum - u0) > p->utoltab) return;
        if (fabs(fsum + u1) > p->ftoltab) return;
        if (fabs(usum) > p->umaxtab) *repul = 1;
        if (fabs(fsum) > p->fmaxtab) *repul = 1;
    }
    *ok = 1;
}

/* PotTwoBodyTab3, Src/potential.F90:1054-1135.  ibuf is a 1-based cursor. */
static int pot_tab3(const or_tab_params *p, int iat, int jat, int iatjat, int32_t *ibuf,
                    double *ubuf, int32_t nbuf, int32_t *iubuflow, int32_t *nugrid,
                    double *rumin, const double *rumax)
{
    const int mnugrid = 1200, ndr = 100;
    const double drfac = 0.9;
    double rlow = 0.0, rupp, zlow, zupp, dr, u0l, u1l, u2l, u0u, u1u, u2u, t[12];
    int igrid, idr, ok = 0, repul = 0, k;
    iubuflow[iatjat - 1] = *ibuf;
    rupp = rumax[iatjat - 1];
    dr = 0.5 * (rumax[iatjat - 1] - rumin[iatjat - 1]);
    for (igrid = 1; igrid <= mnugrid; ++igrid) {
        zupp = rupp * rupp;
        for (idr = 1; idr <= ndr; ++idr) {
            rlow = rupp - dr;
            rlow = fmax(rumin[iatjat - 1], rlow);
            zlow = rlow * rlow;
            or_pot_1_6_12(p, iat, jat, rlow, &u0l, &u1l, &u2l);
            or_pot_1_6_12(p, iat, jat, rupp, &u0u, &u1u, &u2u);
            set_ubuffer(zlow, u0l, u1l, u2l, zupp, u0u, u1u, u2u, t);
            check_ubuffer(p, iat, jat, rlow, rupp, t, &ok, &repul);
            if (ok) {
                rupp = rlow;
                if (p->lljcut) dr = 2.0 * dr;
                break;
            }
            dr = dr * drfac;
        }
        if (idr >= ndr + 1) return 6;
        if (*ibuf + 11 > nbuf) return 2;
        for (k = 0; k < 12; ++k) ubuf[*ibuf - 1 + k] = t[k];
        *ibuf += 12;
        if (repul) rumin[iatjat - 1] = rlow;
        if (rlow <= rumin[iatjat - 1]) break;
        if (repul) break;
    }
    if (igrid >= mnugrid + 1) return 6;
    nugrid[iatjat - 1] = igrid;
    return 0;
}

/* PotTwoBodyTab1 + PotTwoBodyTab2 + Pot_1_6_12 'init', Src/potential.F90:868-1050, 1370-1380 */
int or_pot_tab(const or_tab_params *p, double *ubuf, int32_t nbuf,
               int32_t *iubuflow, int32_t *nugrid, double *r2umin,
               double *rumin, double *rumax, int32_t *nused)
{
    int npt = p->npt, ipt, jpt, rc;
    int32_t ibuf = 1;
    memset(ubuf, 0, sizeof(double) * (size_t)nbuf);
    for (ipt = 1; ipt <= npt; ++ipt)
        for (jpt = ipt; jpt <= npt; ++jpt) {
            int ij = pair_index(npt, ipt, jpt);
            double r2umax = (p->rumaxfac * (p->rcut + 0.0 + 0.0));
            r2umax = r2umax * r2umax;
            r2umin[ij - 1] = p->r2uminin;
            rumax[ij - 1] = sqrt(r2umax);
            rumin[ij - 1] = sqrt(r2umin[ij - 1]);
            rc = pot_tab3(p, ipt, jpt, ij, &ibuf, ubuf, nbuf, iubuflow, nugrid, rumin, rumax);
            if (rc) return rc;
            r2umin[ij - 1] = rumin[ij - 1] * rumin[ij - 1];
        }
    if (nused) *nused = ibuf - 1;
    return 0;
}

/* ------------------------------------------------------------------ */
/* SPME setup, Src/energy.F90:6855-7019                                */
/* ------------------------------------------------------------------ */
void or_ewald_setup_spm(int s, int order, double ualpha, const double boxlen[3],
                        double *meshfac, double *energyfac, double *virfac)
{
    const double TwoPi = 2.0 * Pi, FourPi = 4.0 * Pi;
    double spl[32], b2[3][1024], vol, fac0, expfac, TwoPiBoxi[3];
    int32_t z;
    int i, m, k, nx, ny, nz, h = s / 2;
    or_cardinal_bspline(order, 0.0, &z, spl, NULL);
    for (i = 0; i < 3; ++i)
        for (m = 0; m < s; ++m) {
            double complex a = 0.0;
            if ((order % 2 == 1) && (2 * m == s)) {
                /* left unset by the reference; defined here as 0 (Nyquist plane dropped) */
                b2[i][m] = 0.0;
                continue;
            }
            for (k = 0; k <= order - 2; ++k) {
                /* cmplx(0, x) without KIND is default (single precision) complex */
                float ang = (float)(TwoPi * m * k / s);
                float complex e = cexpf(I * ang);
                a = a + spl[k + 1] * (double complex)e;
            }
            b2[i][m] = 1.0 / (creal(a) * creal(a) + cimag(a) * cimag(a));
        }
    vol = boxlen[0] * boxlen[1] * boxlen[2];
    for (i = 0; i < 3; ++i) TwoPiBoxi[i] = TwoPi * (1.0 / boxlen[i]);
    fac0 = FourPi / vol;
    expfac = -1.0 / (4.0 * (ualpha * ualpha));
    for (nz = 0; nz <= h; ++nz)
        for (ny = 0; ny <= h; ++ny)
            for (nx = 0; nx <= h; ++nx) {
                size_t idx = (size_t)nx + (size_t)(h + 1) * ((size_t)ny + (size_t)(h + 1) * nz);
                if (nx == 0 && ny == 0 && nz == 0) {
                    meshfac[idx] = 0.0;
                    energyfac[idx] = 0.0;
                    virfac[idx] = 0.0;
                } else {
                    double kx = nx * TwoPiBoxi[0], ky = ny * TwoPiBoxi[1], kz = nz * TwoPiBoxi[2];
                    double m2 = kx * kx + ky * ky + kz * kz;
                    double c = exp(m2 * expfac) / m2;
                    double mf = fac0 * c * b2[0][nx] * b2[1][ny] * b2[2][nz];
                    meshfac[idx] = mf;
                    if (nx == (s - nx) % s) mf = mf / 2;
                    if (ny == (s - ny) % s) mf = mf / 2;
                    if (nz == (s - nz) % s) mf = mf / 2;
                    energyfac[idx] = mf;
                    virfac[idx] = (1.0 + 2 * m2 * expfac) * mf;
                }
            }
}

/* ------------------------------------------------------------------ */
/* FFT: recursive mixed-radix complex DFT (FFTW 3.3.4 is the reference */
/* library; only its unnormalised conventions are restated here).     */
/* ------------------------------------------------------------------ */
/* x[k*stride], k<n; tw[e] = exp(sign*2*pi*i*e/N) for the top-level size N */
static void fft1(double complex *x, int n, int stride, const double complex *tw, int N,
                 double complex *tmp)
{
    int p, m, k, q, r;
    if (n == 1) return;
    for (p = 2; p <= n; ++p)
        if (n % p == 0) break;
    m = n / p;
    for (r = 0; r < p; ++r)
        for (k = 0; k < m; ++k) tmp[r * m + k] = x[(k * p + r) * stride];
    for (r = 0; r < p; ++r) fft1(tmp + r * m, m, 1, tw, N, tmp + n);
    for (k = 0; k < m; ++k)
        for (q = 0; q < p; ++q) {
            double complex acc = 0.0;
            int kk = k + q * m;
            for (r = 0; r < p; ++r) {
                long e = ((long)r * kk) % n;
                acc += tmp[r * m + k] * tw[e * (N / n)];
            }
            x[kk * stride] = acc;
        }
}

static void fft3_complex(int s, double complex *a, int sign)
{
    double complex *tmp = malloc(sizeof(double complex) * (size_t)s * 4);
    double complex *line = malloc(sizeof(double complex) * (size_t)s);
    double complex *tw = malloc(sizeof(double complex) * (size_t)s);
    int i, j, k;
    for (i = 0; i < s; ++i) {
        double ang = sign * 2.0 * Pi * (double)i / (double)s;
        tw[i] = cos(ang) + I * sin(ang);
    }
    for (k = 0; k < s; ++k)          /* x lines */
        for (j = 0; j < s; ++j) fft1(a + ((size_t)k * s + j) * s, s, 1, tw, s, tmp);
    for (k = 0; k < s; ++k)          /* y lines */
        for (i = 0; i < s; ++i) {
            for (j = 0; j < s; ++j) line[j] = a[((size_t)k * s + j) * s + i];
            fft1(line, s, 1, tw, s, tmp);
            for (j = 0; j < s; ++j) a[((size_t)k * s + j) * s + i] = line[j];
        }
    for (j = 0; j < s; ++j)          /* z lines */
        for (i = 0; i < s; ++i) {
            for (k = 0; k < s; ++k) line[k] = a[((size_t)k * s + j) * s + i];
            fft1(line, s, 1, tw, s, tmp);
            for (k = 0; k < s; ++k) a[((size_t)k * s + j) * s + i] = line[k];
        }
    free(tw);
    free(line);
    free(tmp);
}

void or_fft3_r2c(int s, const double *in, double *out)
{
    size_t n = (size_t)s * s * s, i;
    int h = s / 2 + 1, x, y, z;
    double complex *a = malloc(sizeof(double complex) * n);
    for (i = 0; i < n; ++i) a[i] = in[i];
    fft3_complex(s, a, -1);
    for (z = 0; z < s; ++z)
        for (y = 0; y < s; ++y)
            for (x = 0; x < h; ++x) {
                double complex v = a[((size_t)z * s + y) * s + x];
                size_t o = ((size_t)z * s + y) * h + x;
                out[2 * o] = creal(v);
                out[2 * o + 1] = cimag(v);
            }
    free(a);
}

void or_fft3_c2r(int s, const double *in, double *out)
{
    size_t n = (size_t)s * s * s, i;
    int h = s / 2 + 1, x, y, z;
    double complex *a = malloc(sizeof(double complex) * n);
    for (z = 0; z < s; ++z)
        for (y = 0; y < s; ++y)
            for (x = 0; x < s; ++x) {
                double complex v;
                if (x < h) {
                    size_t o = ((size_t)z * s + y) * h + x;
                    v = in[2 * o] + I * in[2 * o + 1];
                } else {
                    int xs = s - x, ys = (s - y) % s, zs = (s - z) % s;
                    size_t o = ((size_t)zs * s + ys) * h + xs;
                    v = in[2 * o] - I * in[2 * o + 1];
                }
                a[((size_t)z * s + y) * s + x] = v;
            }
    fft3_complex(s, a, +1);
    for (i = 0; i < n; ++i) out[i] = creal(a[i]);
    free(a);
}

/* ------------------------------------------------------------------ */
/* The system                                                          */
/* ------------------------------------------------------------------ */
struct or_sys {
    int np, npt, natat;
    double boxlen[3], boxlen2[3], boxleni[3], dpbc[3], vol;
    double rcut, rcut2, drnlist;
    int32_t *iptpn;
    double *az, *massp, *massip;
    double *ro, *rod, *rodd, *roddo, *drostep, *drosum, *force, *forceo;
    double *ubuf; int nbuf; int32_t *iubuflow; double *r2umin, *r2atat;
    int maxnneigh; int32_t *nneighpn, *jpnlist;
    int lewald, order, s, lsurf; double ualpha, epsfp;
    double *meshfac, *energyfac, *virfac, *qmesh, *fqmesh;
    /* standard Ewald (lewald == 2): k-space cut, kfac in the sums' order, work arrays */
    int ncut, ncut2, nkvec;
    double *kfac;
    double *eik[3];          /* [np][ncut+1] complex (re, im) */
    double *eyz, *eikr;      /* [np] 2 complex; [np] 4 complex */
    double *sumeikr;         /* [nkvec][4] complex: structure factors of the last UTotal / MC update */
    /* 2D layer correction (lewald2dlc): 2D k-vectors (nx, ny) with kfac2d, sin/cos tables */
    int elc, ncut2d2, nkvec2d;
    double *kfac2d;
    double *trig2d;          /* [np][4][ncut+1]: sin kx, cos kx, sin ky, cos ky */
    double *sumtrig;         /* [nkvec2d][8]: the sums of the last UTotal / MC update */
    /* Random's SAVEd state (Src/mollib.F90:2683-2687) */
    int32_t rix, riy;
    int nbond; int32_t *bond_ij; double *bond_k, *bond_eq; int32_t *bond_p;
    double tstep;
    int lcellbuild;
    int inlist, lvlistllist;
    int istep2;              /* steps since NList(iBeforeMacrostep): MOLSIM's istep2 */
};

static void *dup(const void *p, size_t n)
{
    void *q = malloc(n ? n : 1);
    if (p && n) memcpy(q, p, n);
    else memset(q, 0, n ? n : 1);
    return q;
}

/* EwaldSetup, txewaldrec = 'std': ncut2 from ncutregion and kfac over the
 * k-vectors in the order the sums visit them, Src/energy.F90:6752-6782 */
static void ewald_setup_std(or_sys *s, int ncut, int cube)
{
    int nx, ny, nz, n = 0, m;
    double tpbi[3], fac0 = 2.0 * Pi / s->vol;
    for (m = 0; m < 3; ++m) tpbi[m] = 2.0 * Pi * s->boxleni[m];
    s->ncut = ncut;
    s->ncut2 = cube ? 3 * ncut * ncut : ncut * ncut;
    s->kfac = malloc(sizeof(double) * ((size_t)ncut + 1) * (ncut + 1) * (ncut + 1));
    for (nz = 0; nz <= ncut; ++nz) {
        double facz = (nz == 0) ? 1.0 : 2.0;
        for (ny = 0; ny <= ncut; ++ny) {
            double facy = (ny == 0) ? 0.5 : 1.0;
            for (nx = 0; nx <= ncut; ++nx) {
                double facx, k2;
                if (nx * nx + ny * ny + nz * nz > s->ncut2) continue;
                if (nx == 0 && ny == 0 && nz == 0) continue;
                facx = (nx == 0) ? 0.5 : 1.0;
                k2 = (nx * tpbi[0]) * (nx * tpbi[0]) + (ny * tpbi[1]) * (ny * tpbi[1]) +
                     (nz * tpbi[2]) * (nz * tpbi[2]);
                s->kfac[n++] = fac0 * facz * facy * facx * exp(-k2 / (4.0 * (s->ualpha * s->ualpha))) / k2;
            }
        }
    }
    s->nkvec = n;
    s->sumeikr = calloc(8 * (size_t)(n > 0 ? n : 1), sizeof(double));
    for (m = 0; m < 3; ++m) s->eik[m] = malloc(sizeof(double) * 2 * (size_t)s->np * (ncut + 1));
    s->eyz = malloc(sizeof(double) * 4 * (size_t)s->np);
    s->eikr = malloc(sizeof(double) * 8 * (size_t)s->np);
}

/* EwaldSetup, lewald2dlc (Src/energy.F90:6785-6851): ncut2d = ncut; ncut2d2 = ncut2d^2
 * ('sphere') or 2 ncut2d^2 ('cube'); for each (nx, ny) != 0 with nx^2 + ny^2 <= ncut2d2, ny
 * outer, kfac2d = -2pi/(Lx Ly) fac / (kp (exp(kp Lz) - 1)), fac = 4 when both are nonzero. */
static void ewald_setup_2dlc(or_sys *s, int cube)
{
    const int nc = s->ncut;
    const double fac0 = 2.0 * Pi / (s->boxlen[0] * s->boxlen[1]);
    int nx, ny, n = 0;
    s->ncut2d2 = cube ? 2 * nc * nc : nc * nc;
    s->kfac2d = malloc(sizeof(double) * ((size_t)nc + 1) * (nc + 1));
    for (ny = 0; ny <= nc; ++ny)
        for (nx = 0; nx <= nc; ++nx) {
            double fac = 1.0, kp;
            if (nx * nx + ny * ny > s->ncut2d2) continue;
            if (nx == 0 && ny == 0) continue;
            if (nx != 0 && ny != 0) fac = 4.0 * fac;
            kp = sqrt((nx * (2.0 * Pi * s->boxleni[0])) * (nx * (2.0 * Pi * s->boxleni[0])) +
                      (ny * (2.0 * Pi * s->boxleni[1])) * (ny * (2.0 * Pi * s->boxleni[1])));
            s->kfac2d[n++] = -fac0 * fac / (kp * (exp(kp * s->boxlen[2]) - 1.0));
        }
    s->nkvec2d = n;
    s->trig2d = malloc(sizeof(double) * 4 * (size_t)s->np * ((size_t)nc + 1));
    s->sumtrig = calloc(8 * (size_t)(n > 0 ? n : 1), sizeof(double));
}

or_sys *or_create(const or_params *p)
{
    or_sys *s = calloc(1, sizeof(or_sys));
    int np = p->np, i, h;
    s->np = np;
    s->npt = p->npt;
    s->natat = p->npt * (p->npt + 1) / 2;
    /* SetBoxParam, Src/molaux.F90:325-336 (txbc='xyz') */
    for (i = 0; i < 3; ++i) {
        s->boxlen[i] = p->boxlen[i];
        s->boxlen2[i] = p->boxlen[i] / 2.0;
        s->boxleni[i] = 1.0 / p->boxlen[i];
        s->dpbc[i] = p->boxlen[i];
    }
    s->vol = p->boxlen[0] * p->boxlen[1] * p->boxlen[2];
    s->rcut = p->rcut;
    s->rcut2 = p->rcut * p->rcut;
    s->drnlist = p->drnlist;
    s->iptpn = dup(p->iptpn, sizeof(int32_t) * np);
    s->az = dup(p->az, sizeof(double) * np);
    s->massp = malloc(sizeof(double) * np);
    s->massip = malloc(sizeof(double) * np);
    for (i = 0; i < np; ++i) {
        double m = p->masspt[s->iptpn[i] - 1];
        s->massp[i] = m;
        s->massip[i] = m > 0.0 ? 1.0 / m : 0.0;
    }
    s->ro = calloc(3 * (size_t)np, sizeof(double));
    s->rod = calloc(3 * (size_t)np, sizeof(double));
    s->rodd = calloc(3 * (size_t)np, sizeof(double));
    s->roddo = calloc(3 * (size_t)np, sizeof(double));
    s->drostep = calloc(3 * (size_t)np, sizeof(double));
    s->drosum = calloc(3 * (size_t)np, sizeof(double));
    s->force = calloc(3 * (size_t)np, sizeof(double));
    s->forceo = calloc(3 * (size_t)np, sizeof(double));
    s->nbuf = p->nbuf;
    s->ubuf = dup(p->ubuf, sizeof(double) * p->nbuf);
    s->iubuflow = dup(p->iubuflow, sizeof(int32_t) * s->natat);
    s->r2umin = dup(p->r2umin, sizeof(double) * s->natat);
    s->r2atat = dup(p->r2atat, sizeof(double) * s->natat);
    s->maxnneigh = p->maxnneigh;
    s->nneighpn = calloc((size_t)np, sizeof(int32_t));
    s->jpnlist = calloc((size_t)np * (size_t)p->maxnneigh, sizeof(int32_t));
    s->lewald = p->lewald;
    s->order = p->order;
    s->s = p->nmesh;
    s->lsurf = p->lsurf;
    s->ualpha = p->ualpha;
    s->epsfp = p->epsi_four_pi;
    s->elc = p->lewald2dlc ? 1 : 0;
    if (s->lewald == 2) {
        ewald_setup_std(s, p->ncut, p->ncutregion);
        if (s->elc) ewald_setup_2dlc(s, p->ncutregion);
    } else if (s->lewald) {
        size_t n = (size_t)s->s * s->s * s->s;
        h = s->s / 2 + 1;
        s->meshfac = malloc(sizeof(double) * h * h * h);
        s->energyfac = malloc(sizeof(double) * h * h * h);
        s->virfac = malloc(sizeof(double) * h * h * h);
        or_ewald_setup_spm(s->s, s->order, s->ualpha, s->boxlen, s->meshfac, s->energyfac, s->virfac);
        s->qmesh = malloc(sizeof(double) * n);
        s->fqmesh = malloc(sizeof(double) * 2 * (size_t)h * s->s * s->s);
    }
    s->nbond = p->nbond;
    s->bond_ij = dup(p->bond_ij, sizeof(int32_t) * 2 * p->nbond);
    s->bond_k = dup(p->bond_k, sizeof(double) * p->nbond);
    s->bond_eq = dup(p->bond_eq, sizeof(double) * p->nbond);
    s->bond_p = dup(p->bond_p, sizeof(int32_t) * p->nbond);
    s->tstep = p->tstep;
    s->lcellbuild = p->lcellbuild;
    s->inlist = p->inlist;
    s->lvlistllist = p->lvlistllist;
    s->istep2 = 0;
    return s;
}

void or_destroy(or_sys *s)
{
    if (!s) return;
    free(s->iptpn); free(s->az); free(s->massp); free(s->massip);
    free(s->ro); free(s->rod); free(s->rodd); free(s->roddo); free(s->drostep); free(s->drosum);
    free(s->force); free(s->forceo);
    free(s->ubuf); free(s->iubuflow); free(s->r2umin); free(s->r2atat);
    free(s->nneighpn); free(s->jpnlist);
    free(s->meshfac); free(s->energyfac); free(s->virfac); free(s->qmesh); free(s->fqmesh);
    free(s->kfac2d); free(s->trig2d); free(s->sumtrig);
    free(s->kfac); free(s->eik[0]); free(s->eik[1]); free(s->eik[2]); free(s->eyz); free(s->eikr);
    free(s->sumeikr);
    free(s->bond_ij); free(s->bond_k); free(s->bond_eq); free(s->bond_p);
    free(s);
}

void or_set_state(or_sys *s, const double *ro, const double *rod, const double *rodd)
{
    size_t n = 3 * (size_t)s->np * sizeof(double);
    if (ro) memcpy(s->ro, ro, n);
    if (rod) memcpy(s->rod, rod, n);
    if (rodd) memcpy(s->rodd, rodd, n);
}

void or_get_state(const or_sys *s, double *ro, double *rod, double *rodd, double *drosum)
{
    size_t n = 3 * (size_t)s->np * sizeof(double);
    if (ro) memcpy(ro, s->ro, n);
    if (rod) memcpy(rod, s->rod, n);
    if (rodd) memcpy(rodd, s->rodd, n);
    if (drosum) memcpy(drosum, s->drosum, n);
}

void or_set_drosum(or_sys *s, const double *drosum)
{
    memcpy(s->drosum, drosum, 3 * (size_t)s->np * sizeof(double));
}

/* PBC (box), Src/molaux.F90:104-118: anint-wrap of one coordinate */
static double pbc1(double d, double half, double len, double leni)
{
    if (fabs(d) > half) d = d - len * round(d * leni);
    return d;
}

/* PBCr2 (box), Src/molaux.F90:149-161: single sign(dpbc,d) shift */
static double pbcr2(const or_sys *s, double *dx, double *dy, double *dz)
{
    if (fabs(*dx) > s->boxlen2[0]) *dx = *dx - copysign(s->dpbc[0], *dx);
    if (fabs(*dy) > s->boxlen2[1]) *dy = *dy - copysign(s->dpbc[1], *dy);
    if (fabs(*dz) > s->boxlen2[2]) *dz = *dz - copysign(s->dpbc[2], *dz);
    return *dx * *dx + *dy * *dy + *dz * *dz;
}

/* parity rule of SetVListMD, Src/nlist.F90:741-744 (1-based ip, jp) */
static int owns(int ip, int jp)
{
    int itemp = (ip + jp) % 2;
    if (ip < jp && itemp == 0) return 0;
    if (ip > jp && itemp != 0) return 0;
    return ip != jp;
}

/* SetVListMD, Src/nlist.F90:724-759 */
static int set_vlist_md(or_sys *s)
{
    double rs2cut = (s->rcut + s->drnlist) * (s->rcut + s->drnlist);
    int ip, jp, np = s->np;
    for (ip = 1; ip <= np; ++ip) {
        int32_t *row = s->jpnlist + (size_t)(ip - 1) * s->maxnneigh;
        int nn = 0;
        for (jp = 1; jp <= np; ++jp) {
            double dx, dy, dz, r2;
            if (!owns(ip, jp)) continue;
            dx = s->ro[3 * (ip - 1)] - s->ro[3 * (jp - 1)];
            dy = s->ro[3 * (ip - 1) + 1] - s->ro[3 * (jp - 1) + 1];
            dz = s->ro[3 * (ip - 1) + 2] - s->ro[3 * (jp - 1) + 2];
            r2 = pbcr2(s, &dx, &dy, &dz);
            if (r2 < rs2cut) {
                if (nn >= s->maxnneigh) return 3;
                row[nn++] = jp;
            }
        }
        s->nneighpn[ip - 1] = nn;
    }
    return 0;
}

static int cmp_i32(const void *a, const void *b)
{
    int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

/* Same pair set and row order as SetVListMD, found through a cell grid
 * (cell side >= rcut+drnlist) so that large N stays tractable; rows are
 * sorted by jp, which is the order SetVListMD's jp loop produces. */
static int set_vlist_cells(or_sys *s)
{
    double rl = s->rcut + s->drnlist, rs2cut = rl * rl;
    int nc[3], d, np = s->np, ip, i;
    for (d = 0; d < 3; ++d) {
        nc[d] = (int)floor(s->boxlen[d] / rl);
        if (nc[d] < 1) nc[d] = 1;
    }
    {
        size_t ncell = (size_t)nc[0] * nc[1] * nc[2];
        int32_t *head = malloc(sizeof(int32_t) * ncell), *next = malloc(sizeof(int32_t) * np);
        int32_t *cell = malloc(sizeof(int32_t) * np);
        for (i = 0; i < (int)ncell; ++i) head[i] = -1;
        for (ip = np - 1; ip >= 0; --ip) {
            int c[3];
            for (d = 0; d < 3; ++d) {
                int k = (int)floor((s->ro[3 * ip + d] + s->boxlen2[d]) * nc[d] / s->boxlen[d]);
                if (k < 0) k = 0;
                if (k >= nc[d]) k = nc[d] - 1;
                c[d] = k;
            }
            cell[ip] = c[0] + nc[0] * (c[1] + nc[1] * c[2]);
            next[ip] = head[cell[ip]];
            head[cell[ip]] = ip;
        }
        for (ip = 0; ip < np; ++ip) {
            int32_t *row = s->jpnlist + (size_t)ip * s->maxnneigh;
            int nn = 0, cx = cell[ip] % nc[0], cy = (cell[ip] / nc[0]) % nc[1], cz = cell[ip] / (nc[0] * nc[1]);
            int off[3][3], no[3], a, b, e;
            for (d = 0; d < 3; ++d) {
                int cc = d == 0 ? cx : (d == 1 ? cy : cz);
                if (nc[d] >= 3) { no[d] = 3; off[d][0] = (cc + nc[d] - 1) % nc[d]; off[d][1] = cc; off[d][2] = (cc + 1) % nc[d]; }
                else { no[d] = nc[d]; for (a = 0; a < nc[d]; ++a) off[d][a] = a; }
            }
            for (a = 0; a < no[2]; ++a)
                for (b = 0; b < no[1]; ++b)
                    for (e = 0; e < no[0]; ++e) {
                        int32_t jp = head[off[0][e] + nc[0] * (off[1][b] + nc[1] * off[2][a])];
                        for (; jp >= 0; jp = next[jp]) {
                            double dx, dy, dz, r2;
                            if (!owns(ip + 1, jp + 1)) continue;
                            dx = s->ro[3 * ip] - s->ro[3 * jp];
                            dy = s->ro[3 * ip + 1] - s->ro[3 * jp + 1];
                            dz = s->ro[3 * ip + 2] - s->ro[3 * jp + 2];
                            r2 = pbcr2(s, &dx, &dy, &dz);
                            if (r2 < rs2cut) {
                                if (nn >= s->maxnneigh) { free(head); free(next); free(cell); return 3; }
                                row[nn++] = jp + 1;
                            }
                        }
                    }
            qsort(row, nn, sizeof(int32_t), cmp_i32);
            s->nneighpn[ip] = nn;
        }
        free(head); free(next); free(cell);
    }
    return 0;
}

/* Row rule of SetVListMDLList, Src/nlist.F90:790-792: the pair is skipped when
 * (ip > jp, ip+jp even) or (ip < jp, ip+jp odd), the opposite rows from SetVListMD's. */
static int owns_llist(int ip, int jp)
{
    int itemp = (ip + jp) % 2;
    if (ip > jp && itemp == 0) return 0;
    if (ip < jp && itemp != 0) return 0;
    return ip != jp;
}

/* SetLList(distance), Src/nlist.F90:1168-1221: ndivllist = int(boxlen/distance), celli =
 * real(ndivllist)*boxleni (real() is default real; exact for these integers), cells
 * numbered 1 + ix + iy nx + iz nx ny from aint((ro+boxlen2)*celli); each cell's chain runs
 * from its smallest ip upwards (particles inserted np..1).  The reference caps the cell
 * arrays at 1000 and does not guard larger grids; this restatement refuses them (6). */
static int llist_cell(const or_sys *s, const int nd[3], const double celli[3], const double *r)
{
    int c[3], d;
    for (d = 0; d < 3; ++d) {
        c[d] = (int)((r[d] + s->boxlen2[d]) * celli[d]);
        if (c[d] >= nd[d]) c[d] = nd[d] - 1;     /* r = +boxlen2 exactly: outside the reference's grid */
        if (c[d] < 0) c[d] = 0;
    }
    return c[0] + c[1] * nd[0] + c[2] * nd[0] * nd[1];
}

/* SetVListMDLList, Src/nlist.F90:769-811, over SetLList(rcut+drnlist) and, per particle,
 * SetNCell(ro(ip), rcut) (:1231-1260): the cells of the 27 points ro(ip) + (i, j, k) rcut,
 * i, j, k in {-1, 0, 1}, each put in the box by PBC, are scanned in ascending cell number,
 * each cell's chain in ascending ip. */
static int set_vlist_md_llist(or_sys *s)
{
    double dist = s->rcut + s->drnlist, rs2cut = dist * dist, celli[3];
    int nd[3], d, np = s->np, ip, ncell;
    for (d = 0; d < 3; ++d) {
        nd[d] = (int)(s->boxlen[d] / dist);
        celli[d] = (double)(float)nd[d] * s->boxleni[d];
    }
    ncell = nd[0] * nd[1] * nd[2];
    if (ncell < 1 || ncell > 1000) return 6;
    {
        int32_t *head = malloc(sizeof(int32_t) * ncell), *next = malloc(sizeof(int32_t) * np);
        unsigned char *mark = malloc((size_t)ncell);
        int c;
        for (c = 0; c < ncell; ++c) head[c] = -1;
        for (ip = np - 1; ip >= 0; --ip) {
            c = llist_cell(s, nd, celli, s->ro + 3 * ip);
            next[ip] = head[c];
            head[c] = ip;
        }
        for (ip = 0; ip < np; ++ip) {
            int32_t *row = s->jpnlist + (size_t)ip * s->maxnneigh;
            int nn = 0, a, b, e;
            memset(mark, 0, (size_t)ncell);
            for (a = -1; a <= 1; ++a)
                for (b = -1; b <= 1; ++b)
                    for (e = -1; e <= 1; ++e) {
                        double q[3];
                        q[0] = s->ro[3 * ip] + a * s->rcut;
                        q[1] = s->ro[3 * ip + 1] + b * s->rcut;
                        q[2] = s->ro[3 * ip + 2] + e * s->rcut;
                        for (d = 0; d < 3; ++d) q[d] = pbc1(q[d], s->boxlen2[d], s->dpbc[d], s->boxleni[d]);
                        mark[llist_cell(s, nd, celli, q)] = 1;
                    }
            for (c = 0; c < ncell; ++c) {
                int32_t jp;
                if (!mark[c]) continue;
                for (jp = head[c]; jp >= 0; jp = next[jp]) {
                    double dx, dy, dz, r2;
                    if (!owns_llist(ip + 1, jp + 1)) continue;
                    dx = s->ro[3 * ip] - s->ro[3 * jp];
                    dy = s->ro[3 * ip + 1] - s->ro[3 * jp + 1];
                    dz = s->ro[3 * ip + 2] - s->ro[3 * jp + 2];
                    r2 = pbcr2(s, &dx, &dy, &dz);
                    if (r2 < rs2cut) {
                        if (nn >= s->maxnneigh) { free(head); free(next); free(mark); return 3; }
                        row[nn++] = jp + 1;
                    }
                }
            }
            s->nneighpn[ip] = nn;
        }
        free(head); free(next); free(mark);
    }
    return 0;
}

int or_set_vlist(or_sys *s)
{
    if (s->lvlistllist) return set_vlist_md_llist(s);
    return s->lcellbuild ? set_vlist_cells(s) : set_vlist_md(s);
}

void or_nlist_before_macrostep(or_sys *s)
{
    memset(s->drosum, 0, sizeof(double) * 3 * s->np);
    s->istep2 = 0;
}

/* NList(iSimulationStep), Src/nlist.F90:597-621: the skin test when inlist == 0; with
 * inlist > 0 a rebuild whenever mod(istep2, inlist) == 0, drosum untouched. */
static int nlist_step(or_sys *s, int32_t *rebuilt)
{
    int due;
    s->istep2 += 1;
    if (s->inlist > 0)
        due = (s->istep2 % s->inlist) == 0;
    else
        due = or_skin_test(s, s->drostep, NULL, NULL);
    if (rebuilt) *rebuilt = due;
    return due ? or_set_vlist(s) : 0;
}

void or_get_vlist(const or_sys *s, int32_t *nneighpn, int32_t *jpnlist)
{
    if (nneighpn) memcpy(nneighpn, s->nneighpn, sizeof(int32_t) * s->np);
    if (jpnlist) memcpy(jpnlist, s->jpnlist, sizeof(int32_t) * (size_t)s->np * s->maxnneigh);
}

int64_t or_npair(const or_sys *s)
{
    int64_t n = 0;
    int i;
    for (i = 0; i < s->np; ++i) n += s->nneighpn[i];
    return n;
}

/* UTwoBodyA, Src/energy.F90:445-544 (serial: iploc == ip) */
static int utwobody_a(or_sys *s, double *utwob, double *virtwob)
{
    int ip, k, npt = s->npt;
    double vir = 0.0;
    for (k = 0; k <= s->natat; ++k) utwob[k] = 0.0;
    for (ip = 1; ip <= s->np; ++ip) {
        int ipt = s->iptpn[ip - 1];
        const int32_t *row = s->jpnlist + (size_t)(ip - 1) * s->maxnneigh;
        for (k = 0; k < s->nneighpn[ip - 1]; ++k) {
            int jp = row[k], jpt = s->iptpn[jp - 1], iptjpt = pair_index(npt, ipt, jpt);
            double dx = s->ro[3 * (ip - 1)] - s->ro[3 * (jp - 1)];
            double dy = s->ro[3 * (ip - 1) + 1] - s->ro[3 * (jp - 1) + 1];
            double dz = s->ro[3 * (ip - 1) + 2] - s->ro[3 * (jp - 1) + 2];
            double r2 = pbcr2(s, &dx, &dy, &dz), usum, fsum = 0.0;
            if (r2 > s->rcut2) continue;
            if (r2 < s->r2atat[iptjpt - 1]) {
                usum = 1e10;   /* hard-core overlap; the reference leaves fsum stale here */
            } else if (r2 < s->r2umin[iptjpt - 1]) {
                return 1;
            } else {
                int ibuf = s->iubuflow[iptjpt - 1];
                const double *u;
                for (;;) {
                    if (r2 >= s->ubuf[ibuf - 1]) break;
                    ibuf += 12;
                    if (ibuf > s->nbuf) return 2;
                }
                u = s->ubuf + ibuf - 1;
                {
                    double d = r2 - u[0];
                    usum = u[1] + d * (u[2] + d * (u[3] + d * (u[4] + d * (u[5] + d * u[6]))));
                    fsum = u[7] + d * (u[8] + d * (u[9] + d * (u[10] + d * u[11])));
                }
            }
            utwob[iptjpt] = utwob[iptjpt] + usum;
            s->force[3 * (ip - 1)] += (fsum * dx);
            s->force[3 * (ip - 1) + 1] += (fsum * dy);
            s->force[3 * (ip - 1) + 2] += (fsum * dz);
            s->force[3 * (jp - 1)] -= (fsum * dx);
            s->force[3 * (jp - 1) + 1] -= (fsum * dy);
            s->force[3 * (jp - 1) + 2] -= (fsum * dz);
            vir = vir - (fsum * r2);
        }
    }
    utwob[0] = 0.0;
    for (k = 1; k <= s->natat; ++k) utwob[0] += utwob[k];
    *virtwob = vir;
    return 0;
}

/* UEwaldRecSPM + SPMFFTRec, Src/energy.F90:1207-1297, 6525-6587 */
static void uewald_rec_spm(or_sys *s, double *urec, double *virrec)
{
    int S = s->s, order = s->order, h = S / 2, hp = S / 2 + 1, ia, m, ix, iy, iz;
    size_t n = (size_t)S * S * S;
    double dkdr[3], spline[3][32], deriv[3][32];
    int32_t meshmax[3];
    double uloc = 0.0, virloc = *virrec;
    for (m = 0; m < 3; ++m) dkdr[m] = S / s->boxlen[m];
    memset(s->qmesh, 0, sizeof(double) * n);
    for (ia = 0; ia < s->np; ++ia) {
        for (m = 0; m < 3; ++m) {
            or_cardinal_bspline(order, dkdr[m] * s->ro[3 * ia + m], &meshmax[m], spline[m], deriv[m]);
            meshmax[m] = (meshmax[m] + S) % S;
        }
        for (iz = 0; iz < order; ++iz) {
            int nz = (S + meshmax[2] - iz) % S;
            double qz = s->az[ia] * spline[2][iz];
            for (iy = 0; iy < order; ++iy) {
                int ny = (S + meshmax[1] - iy) % S;
                double qyz = qz * spline[1][iy];
                for (ix = 0; ix < order; ++ix) {
                    int nx = (S + meshmax[0] - ix) % S;
                    double q = qyz * spline[0][ix];
                    s->qmesh[(size_t)nx + S * ((size_t)ny + (size_t)S * nz)] += q;
                }
            }
        }
    }
    or_fft3_r2c(S, s->qmesh, s->fqmesh);
    {
        int nx, ny, nz;
        for (nz = 0; nz <= h; ++nz) {
            int nza = (S - nz) % S;
            for (ny = 0; ny <= h; ++ny) {
                int nya = (S - ny) % S;
                for (nx = 0; nx <= h; ++nx) {
                    size_t f = (size_t)nx + (size_t)hp * ((size_t)ny + (size_t)hp * nz);
                    size_t i1 = (size_t)nx + (size_t)hp * ((size_t)ny + (size_t)S * nz);
                    size_t i2 = (size_t)nx + (size_t)hp * ((size_t)ny + (size_t)S * nza);
                    size_t i3 = (size_t)nx + (size_t)hp * ((size_t)nya + (size_t)S * nz);
                    size_t i4 = (size_t)nx + (size_t)hp * ((size_t)nya + (size_t)S * nza);
                    double *F = s->fqmesh;
                    double v1r = F[2 * i1], v1i = F[2 * i1 + 1], v2r = F[2 * i2], v2i = F[2 * i2 + 1];
                    double v3r = F[2 * i3], v3i = F[2 * i3 + 1], v4r = F[2 * i4], v4i = F[2 * i4 + 1];
                    double Qsum = v1r * v1r + v1i * v1i + v2r * v2r + v2i * v2i
                                + v3r * v3r + v3i * v3i + v4r * v4r + v4i * v4i;
                    double mf = s->meshfac[f];
                    uloc = uloc + Qsum * s->energyfac[f];
                    virloc = virloc - Qsum * s->virfac[f];
                    F[2 * i1] = v1r * mf; F[2 * i1 + 1] = v1i * mf;
                    F[2 * i2] = v2r * mf; F[2 * i2 + 1] = v2i * mf;
                    F[2 * i3] = v3r * mf; F[2 * i3 + 1] = v3i * mf;
                    F[2 * i4] = v4r * mf; F[2 * i4 + 1] = v4i * mf;
                }
            }
        }
    }
    or_fft3_c2r(S, s->fqmesh, s->qmesh);
    for (ia = 0; ia < s->np; ++ia) {
        double esum[3] = {0.0, 0.0, 0.0};
        for (m = 0; m < 3; ++m) {
            or_cardinal_bspline(order, dkdr[m] * s->ro[3 * ia + m], &meshmax[m], spline[m], deriv[m]);
            meshmax[m] = (meshmax[m] + S) % S;
        }
        for (iz = 0; iz < order; ++iz) {
            int nz = (S + meshmax[2] - iz) % S;
            double splz = spline[2][iz], dsdz = deriv[2][iz];
            for (iy = 0; iy < order; ++iy) {
                int ny = (S + meshmax[1] - iy) % S;
                double sply = spline[1][iy], dsdy = deriv[1][iy];
                for (ix = 0; ix < order; ++ix) {
                    int nx = (S + meshmax[0] - ix) % S;
                    double splx = spline[0][ix], dsdx = deriv[0][ix];
                    double Qval = s->qmesh[(size_t)nx + S * ((size_t)ny + (size_t)S * nz)];
                    esum[0] = esum[0] + dsdx * sply * splz * Qval;
                    esum[1] = esum[1] + splx * dsdy * splz * Qval;
                    esum[2] = esum[2] + splx * sply * dsdz * Qval;
                }
            }
        }
        for (m = 0; m < 3; ++m)
            s->force[3 * ia + m] = s->force[3 * ia + m] - s->az[ia] * esum[m] * dkdr[m] * s->epsfp;
    }
    *urec = uloc;
    *virrec = virloc;
}

/* Complex arithmetic on (re, im) pairs, as Fortran complex(8) evaluates it. */
typedef struct { double r, i; } cx;
static cx cmul(cx a, cx b)
{
    cx c;
    c.r = a.r * b.r - a.i * b.i;
    c.i = a.r * b.i + a.i * b.r;
    return c;
}

/* UEwaldRecStd (serial branch) with EwaldSetArray, Src/energy.F90:1045-1100, 1401-1426.
 * Returns the reciprocal energy and virial before the EpsiFourPi scale of UEwald and
 * adds the reciprocal forces (already scaled by EpsiFourPi) into s->force. */
static void uewald_rec_std(or_sys *s, double *urec, double *virrec)
{
    const int np = s->np, nc = s->ncut, ncut2 = s->ncut2;
    const size_t w = (size_t)nc + 1;
    cx *ex = (cx *)s->eik[0], *ey = (cx *)s->eik[1], *ez = (cx *)s->eik[2];
    cx *eyz = (cx *)s->eyz, *eikr = (cx *)s->eikr;
    double tpbi[3], uloc = 0.0, virloc = *virrec;
    int ia, nx, ny, nz, m, kn = 0, icut;
    cx *e[3];
    e[0] = ex; e[1] = ey; e[2] = ez;
    for (m = 0; m < 3; ++m) tpbi[m] = 2.0 * Pi * s->boxleni[m];
    /* EwaldSetArray: e(0) = 1, e(1) = exp(i 2pi/L r), e(n) = e(n-1) e(1) */
    for (ia = 0; ia < np; ++ia)
        for (m = 0; m < 3; ++m) {
            cx *t = e[m] + (size_t)ia * w;
            t[0].r = 1.0; t[0].i = 0.0;
            t[1].r = cos(tpbi[m] * s->ro[3 * ia + m]);
            t[1].i = sin(tpbi[m] * s->ro[3 * ia + m]);
        }
    for (icut = 2; icut <= nc; ++icut)
        for (ia = 0; ia < np; ++ia)
            for (m = 0; m < 3; ++m) {
                cx *t = e[m] + (size_t)ia * w;
                t[icut] = cmul(t[icut - 1], t[1]);
            }
    for (nz = 0; nz <= nc; ++nz) {
        for (ny = 0; ny <= nc; ++ny) {
            if (ny * ny + nz * nz > ncut2) continue;
            for (ia = 0; ia < np; ++ia) {
                cx yc = ey[(size_t)ia * w + ny], zz = ez[(size_t)ia * w + nz];
                cx yconj;
                yconj.r = yc.r; yconj.i = -yc.i;
                eyz[2 * ia] = cmul(yconj, zz);      /* eikyzm */
                eyz[2 * ia + 1] = cmul(yc, zz);     /* eikyzp */
            }
            for (nx = 0; nx <= nc; ++nx) {
                cx sum[4];
                double term, kfac2, kx, ky, kz, k2;
                int c;
                if (nx * nx + ny * ny + nz * nz > ncut2) continue;
                if (nx == 0 && ny == 0 && nz == 0) continue;
                for (c = 0; c < 4; ++c) sum[c].r = sum[c].i = 0.0;
                for (ia = 0; ia < np; ++ia) {
                    cx x = ex[(size_t)ia * w + nx], qxc, qx;
                    const double q = s->az[ia];
                    qxc.r = q * x.r; qxc.i = q * (-x.i);    /* az * conjg(eikx) */
                    qx.r = q * x.r; qx.i = q * x.i;         /* az * eikx */
                    eikr[4 * ia] = cmul(qxc, eyz[2 * ia]);
                    eikr[4 * ia + 1] = cmul(qxc, eyz[2 * ia + 1]);
                    eikr[4 * ia + 2] = cmul(qx, eyz[2 * ia]);
                    eikr[4 * ia + 3] = cmul(qx, eyz[2 * ia + 1]);
                    for (c = 0; c < 4; ++c) {
                        sum[c].r = sum[c].r + eikr[4 * ia + c].r;
                        sum[c].i = sum[c].i + eikr[4 * ia + c].i;
                    }
                }
                term = 0.0;
                for (c = 0; c < 4; ++c) term = term + (sum[c].r * sum[c].r + sum[c].i * sum[c].i);
                for (c = 0; c < 4; ++c) ((cx *)s->sumeikr)[4 * (size_t)kn + c] = sum[c];
                term = s->kfac[kn] * term;
                uloc = uloc + term;
                kfac2 = s->epsfp * 2.0 * s->kfac[kn];
                kx = kfac2 * nx * tpbi[0];
                ky = kfac2 * ny * tpbi[1];
                kz = kfac2 * nz * tpbi[2];
                for (ia = 0; ia < np; ++ia) {
                    const cx *r = eikr + 4 * (size_t)ia;
                    double fmm = -r[0].r * sum[0].i + r[0].i * sum[0].r;
                    double fmp = -r[1].r * sum[1].i + r[1].i * sum[1].r;
                    double fpm = -r[2].r * sum[2].i + r[2].i * sum[2].r;
                    double fpp = -r[3].r * sum[3].i + r[3].i * sum[3].r;
                    s->force[3 * ia] = s->force[3 * ia] + kx * (-fmm - fmp + fpm + fpp);
                    s->force[3 * ia + 1] = s->force[3 * ia + 1] + ky * (-fmm + fmp - fpm + fpp);
                    s->force[3 * ia + 2] = s->force[3 * ia + 2] + kz * (fmm + fmp + fpm + fpp);
                }
                k2 = (nx * tpbi[0]) * (nx * tpbi[0]) + (ny * tpbi[1]) * (ny * tpbi[1]) +
                     (nz * tpbi[2]) * (nz * tpbi[2]);
                virloc = virloc - (1.0 - k2 / (2.0 * (s->ualpha * s->ualpha))) * term;
                ++kn;
            }
        }
    }
    *urec = uloc;
    *virrec = virloc;
}

/* UEwaldRecStd2dlc with EwaldSetArray2d, Src/energy.F90:1106-1203, 1435-1463: the layer
 * correction of Arnold et al. over the 2D k-vectors.  The tables keep the reference's
 * sin(0) = cos(0) = 1 at n = 0.  Adds to *urec (before the EpsiFourPi scale) and the
 * forces (scaled); the virial is untouched, as in the reference. */
static void uewald_rec_std2dlc(or_sys *s, double *urec)
{
    const int np = s->np, nc = s->ncut;
    const size_t w = (size_t)nc + 1;
    double tpbi[2], uloc = *urec;
    int ia, nx, ny, icut, kn = 0, c;
    tpbi[0] = 2.0 * Pi * s->boxleni[0];
    tpbi[1] = 2.0 * Pi * s->boxleni[1];
    for (ia = 0; ia < np; ++ia) {
        double *t = s->trig2d + (size_t)ia * 4 * w;       /* sx, cx, sy, cy rows */
        t[0] = 1.0; t[w] = 1.0; t[2 * w] = 1.0; t[3 * w] = 1.0;
        if (nc >= 1) {
            t[1] = sin(tpbi[0] * s->ro[3 * ia]);
            t[w + 1] = cos(tpbi[0] * s->ro[3 * ia]);
            t[2 * w + 1] = sin(tpbi[1] * s->ro[3 * ia + 1]);
            t[3 * w + 1] = cos(tpbi[1] * s->ro[3 * ia + 1]);
        }
        for (icut = 2; icut <= nc; ++icut) {
            t[icut] = t[icut - 1] * t[w + 1] + t[w + icut - 1] * t[1];
            t[w + icut] = t[w + icut - 1] * t[w + 1] - t[icut - 1] * t[1];
            t[2 * w + icut] = t[2 * w + icut - 1] * t[3 * w + 1] + t[3 * w + icut - 1] * t[2 * w + 1];
            t[3 * w + icut] = t[3 * w + icut - 1] * t[3 * w + 1] - t[2 * w + icut - 1] * t[2 * w + 1];
        }
    }
    for (ny = 0; ny <= nc; ++ny) {
        const double ky = ny * tpbi[1];
        for (nx = 0; nx <= nc; ++nx) {
            const double kx = nx * tpbi[0];
            double kp, st[8], term, kfac2, kxx, kyy, kpp;
            if (nx * nx + ny * ny > s->ncut2d2) continue;
            if (nx == 0 && ny == 0) continue;
            kp = sqrt(kx * kx + ky * ky);
            for (c = 0; c < 8; ++c) st[c] = 0.0;
            for (ia = 0; ia < np; ++ia) {
                const double *t = s->trig2d + (size_t)ia * 4 * w;
                const double sx = t[nx], cx = t[w + nx], sy = t[2 * w + ny], cy = t[3 * w + ny];
                const double e = exp(kp * s->ro[3 * ia + 2]), ei = 1.0 / e;
                const double sh = 0.5 * (e - ei), ch = 0.5 * (e + ei), q = s->az[ia];
                st[0] = st[0] + q * sx * sy * sh;
                st[1] = st[1] + q * cx * sy * sh;
                st[2] = st[2] + q * sx * cy * sh;
                st[3] = st[3] + q * cx * cy * sh;
                st[4] = st[4] + q * sx * sy * ch;
                st[5] = st[5] + q * cx * sy * ch;
                st[6] = st[6] + q * sx * cy * ch;
                st[7] = st[7] + q * cx * cy * ch;
            }
            term = s->kfac2d[kn] * (-st[0] * st[0] - st[1] * st[1] - st[2] * st[2] - st[3] * st[3] +
                                    st[4] * st[4] + st[5] * st[5] + st[6] * st[6] + st[7] * st[7]);
            uloc = uloc + term;
            for (c = 0; c < 8; ++c) s->sumtrig[8 * (size_t)kn + c] = st[c];
            kfac2 = s->epsfp * 2.0 * s->kfac2d[kn];
            kxx = kfac2 * kx;
            kyy = kfac2 * ky;
            kpp = kfac2 * kp;
            for (ia = 0; ia < np; ++ia) {
                const double *t = s->trig2d + (size_t)ia * 4 * w;
                const double sx = t[nx], cx = t[w + nx], sy = t[2 * w + ny], cy = t[3 * w + ny];
                const double e = exp(kp * s->ro[3 * ia + 2]), ei = 1.0 / e;
                const double sh = 0.5 * (e - ei), ch = 0.5 * (e + ei), q = s->az[ia];
                s->force[3 * ia] = s->force[3 * ia] -
                    kxx * q * (-(cx) * (sy) * sh * st[0] - (-sx) * (sy) * sh * st[1] - (cx) * (cy) * sh * st[2] -
                               (-sx) * (cy) * sh * st[3] + (cx) * (sy) * ch * st[4] + (-sx) * (sy) * ch * st[5] +
                               (cx) * (cy) * ch * st[6] + (-sx) * (cy) * ch * st[7]);
                s->force[3 * ia + 1] = s->force[3 * ia + 1] -
                    kyy * q * (-(sx) * (cy) * sh * st[0] - (cx) * (cy) * sh * st[1] - (sx) * (-sy) * sh * st[2] -
                               (cx) * (-sy) * sh * st[3] + (sx) * (cy) * ch * st[4] + (cx) * (cy) * ch * st[5] +
                               (sx) * (-sy) * ch * st[6] + (cx) * (-sy) * ch * st[7]);
                s->force[3 * ia + 2] = s->force[3 * ia + 2] -
                    kpp * q * (-(sx) * (sy) * ch * st[0] - (cx) * (sy) * ch * st[1] - (sx) * (cy) * ch * st[2] -
                               (cx) * (cy) * ch * st[3] + (sx) * (sy) * sh * st[4] + (cx) * (sy) * sh * st[5] +
                               (sx) * (cy) * sh * st[6] + (cx) * (cy) * sh * st[7]);
            }
            ++kn;
        }
    }
    *urec = uloc;
}

/* UEwald + UEwaldSelf + UEwaldSurf, Src/energy.F90:905-958, 1301-1371 (monoatomic) */
static void uewald(or_sys *s, double *urec_out, double *utot, double *virial)
{
    double urec = 0.0, virrec = 0.0, q2 = 0.0;
    int ia;
    if (s->lewald == 2) {
        uewald_rec_std(s, &urec, &virrec);
        if (s->elc) uewald_rec_std2dlc(s, &urec);
    } else {
        uewald_rec_spm(s, &urec, &virrec);
    }
    for (ia = 0; ia < s->np; ++ia) q2 += s->az[ia] * s->az[ia];
    urec = urec - s->ualpha / sqrt(Pi) * q2;
    if (s->lsurf && s->elc) {                  /* 2d-periodic system (Src/energy.F90:1362-1369) */
        double fac = 2.0 * Pi / s->vol, sz = 0.0, term;
        for (ia = 0; ia < s->np; ++ia) sz += s->az[ia] * s->ro[3 * ia + 2];
        term = fac * (sz * sz);
        urec = urec + term;
        for (ia = 0; ia < s->np; ++ia)
            s->force[3 * ia + 2] = s->force[3 * ia + 2] - s->epsfp * (2.0 * fac) * s->az[ia] * sz;
        virrec = virrec - term;
    } else if (s->lsurf) {
        double fac = 2.0 * Pi / (3.0 * s->vol), sx = 0.0, sy = 0.0, sz = 0.0, term;
        for (ia = 0; ia < s->np; ++ia) {
            sx += s->az[ia] * s->ro[3 * ia];
            sy += s->az[ia] * s->ro[3 * ia + 1];
            sz += s->az[ia] * s->ro[3 * ia + 2];
        }
        term = fac * (sx * sx + sy * sy + sz * sz);
        urec = urec + term;
        for (ia = 0; ia < s->np; ++ia) {
            s->force[3 * ia] = s->force[3 * ia] - s->epsfp * (2.0 * fac) * s->az[ia] * sx;
            s->force[3 * ia + 1] = s->force[3 * ia + 1] - s->epsfp * (2.0 * fac) * s->az[ia] * sy;
            s->force[3 * ia + 2] = s->force[3 * ia + 2] - s->epsfp * (2.0 * fac) * s->az[ia] * sz;
        }
        virrec = virrec - term;
    }
    urec = s->epsfp * urec;
    *utot = *utot + urec;
    *virial = *virial + s->epsfp * virrec;
    *urec_out = urec;
}

/* UBond, Src/energy.F90:5335-5387 */
static void ubond(or_sys *s, double *ub, double *utot, double *virial)
{
    double u = 0.0, vir = 0.0;
    int b, k;
    for (b = 0; b < s->nbond; ++b) {
        int ip = s->bond_ij[2 * b] - 1, jp = s->bond_ij[2 * b + 1] - 1, pw = s->bond_p[b];
        double dx = s->ro[3 * ip] - s->ro[3 * jp];
        double dy = s->ro[3 * ip + 1] - s->ro[3 * jp + 1];
        double dz = s->ro[3 * ip + 2] - s->ro[3 * jp + 2];
        double r2 = pbcr2(s, &dx, &dy, &dz), r1 = sqrt(r2), term = r1 - s->bond_eq[b];
        double tp = 1.0, fac;
        for (k = 0; k < pw - 1; ++k) tp = tp * term;
        fac = s->bond_k[b] * tp;
        u = u + fac * term;
        fac = -(pw * fac / r1);
        s->force[3 * ip] += (fac * dx);
        s->force[3 * ip + 1] += (fac * dy);
        s->force[3 * ip + 2] += (fac * dz);
        s->force[3 * jp] -= (fac * dx);
        s->force[3 * jp + 1] -= (fac * dy);
        s->force[3 * jp + 2] -= (fac * dz);
        vir = vir - (fac * r2);
    }
    *ub = u;
    *utot = *utot + u;
    *virial = *virial + vir;
}

/* UTotal, Src/energy.F90:280-434 (monoatomic, charged, vlist) */
int or_utotal(or_sys *s, double *force, double *forceo, double *u, double *virial)
{
    double utot = 0.0, vir = 0.0, virtwob = 0.0, urec = 0.0, ub = 0.0, fac;
    double *utwob = malloc(sizeof(double) * (s->natat + 1));
    int rc, i, k, n3 = 3 * s->np;
    for (i = 0; i < n3; ++i) s->force[i] = 0.0;
    rc = utwobody_a(s, utwob, &virtwob);
    if (rc) { free(utwob); return rc; }
    utot = utot + utwob[0];
    vir = vir + virtwob;
    if (s->lewald) uewald(s, &urec, &utot, &vir);
    if (s->nbond > 0) ubond(s, &ub, &utot, &vir);
    /* force -> internal units, forceo; virmolecule == 0 for monoatomic */
    fac = (sclene / scllen) / sclfor();
    if (force) memcpy(force, s->force, sizeof(double) * n3);
    for (i = 0; i < n3; ++i) {
        s->force[i] = s->force[i] * fac;
        s->forceo[i] = 0.0 + s->force[i];
    }
    if (forceo) memcpy(forceo, s->forceo, sizeof(double) * n3);
    if (u) {
        u[0] = utot;
        for (k = 0; k <= s->natat; ++k) u[1 + k] = utwob[k];
        u[2 + s->natat] = urec;
        u[3 + s->natat] = ub;
    }
    if (virial) *virial = vir;
    free(utwob);
    return 0;
}

/* NList iSimulationStep with inlist == 0, Src/nlist.F90:597-613 */
int or_skin_test(or_sys *s, const double *drostep, double *max1, double *max2)
{
    double r2max1 = 0.0, r2max2 = 0.0;
    int ip, m;
    for (ip = 0; ip < s->np; ++ip) {
        double r2;
        for (m = 0; m < 3; ++m) s->drosum[3 * ip + m] = s->drosum[3 * ip + m] + drostep[3 * ip + m];
        r2 = s->drosum[3 * ip] * s->drosum[3 * ip] + s->drosum[3 * ip + 1] * s->drosum[3 * ip + 1]
           + s->drosum[3 * ip + 2] * s->drosum[3 * ip + 2];
        if (r2 > r2max1) r2max1 = r2;
        else if (r2 > r2max2) r2max2 = r2;
    }
    if (max1) *max1 = r2max1;
    if (max2) *max2 = r2max2;
    if (sqrt(r2max1) + sqrt(r2max2) > s->drnlist) {
        memset(s->drosum, 0, sizeof(double) * 3 * s->np);
        return 1;
    }
    return 0;
}

/* VelVer (linear) + GetLinAcc + GetKinEnergy + NList, Src/md.F90:252-410, 601-617, 1089-1112 */
int or_velver_step(or_sys *s, double *ekin, int32_t *rebuilt)
{
    double dt = s->tstep, fac = 0.5 * (dt * dt), ek = 0.0;
    int ip, m, rc, n3 = 3 * s->np;
    for (ip = 0; ip < s->np; ++ip) {
        for (m = 0; m < 3; ++m) {
            int i = 3 * ip + m;
            s->drostep[i] = dt * s->rod[i] + fac * s->rodd[i];
            s->ro[i] = s->ro[i] + s->drostep[i];
        }
        for (m = 0; m < 3; ++m)
            s->ro[3 * ip + m] = pbc1(s->ro[3 * ip + m], s->boxlen2[m], s->dpbc[m], s->boxleni[m]);
    }
    rc = or_utotal(s, NULL, NULL, NULL, NULL);
    if (rc) return rc;
    for (m = 0; m < n3; ++m) s->roddo[m] = s->rodd[m];
    for (ip = 0; ip < s->np; ++ip)
        for (m = 0; m < 3; ++m) s->rodd[3 * ip + m] = s->massip[ip] * s->forceo[3 * ip + m];
    for (m = 0; m < n3; ++m) s->rod[m] = s->rod[m] + 0.5 * dt * (s->rodd[m] + s->roddo[m]);
    for (ip = 0; ip < s->np; ++ip) {
        const double *v = s->rod + 3 * ip;
        ek = ek + 0.5 * s->massp[ip] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    }
    {
        double sclvel = scllen / scltim;
        ek = ek * sclmas * (sclvel * sclvel) / sclene;
    }
    if (ekin) *ekin = ek;
    return nlist_step(s, rebuilt);
}

/* BDDriver iSimulationStep: BDStep then UTotal, then NList; Src/bd.F90:53-59, 120-155 */
int or_bd_step(or_sys *s, const double *xi, const double *fac1, const double *fac2, int32_t *rebuilt)
{
    int ip, m, rc;
    for (ip = 0; ip < s->np; ++ip) {
        int ipt = s->iptpn[ip] - 1;
        for (m = 0; m < 3; ++m) {
            int i = 3 * ip + m;
            s->drostep[i] = fac1[ipt] * s->forceo[i] + fac2[ipt] * xi[i];
            s->ro[i] = s->ro[i] + s->drostep[i];
        }
        for (m = 0; m < 3; ++m)
            s->ro[3 * ip + m] = pbc1(s->ro[3 * ip + m], s->boxlen2[m], s->dpbc[m], s->boxleni[m]);
    }
    rc = or_utotal(s, NULL, NULL, NULL, NULL);
    if (rc) return rc;
    return nlist_step(s, rebuilt);
}

/* GauRandom, Src/mollib.F90:2739-2766 (polar Box-Muller over a 31-bit LCG) */
double or_gau_random(int32_t *iseed, int32_t *flag, double *save)
{
    const int32_t k = 16087;
    const double f = 1.0 / 2147483648.0;
    double rx, ry, r, fac;
    if (*flag) {
        for (;;) {
            *iseed = (int32_t)(((uint32_t)*iseed * (uint32_t)k) & 0x7fffffffu);
            rx = 2.0 * (f * *iseed - 0.5);
            *iseed = (int32_t)(((uint32_t)*iseed * (uint32_t)k) & 0x7fffffffu);
            ry = 2.0 * (f * *iseed - 0.5);
            r = rx * rx + ry * ry;
            if (r < 1.0) break;
        }
        fac = sqrt(-2.0 * log(r) / r);
        *save = ry * fac;
        *flag = 0;
        return rx * fac;
    }
    *flag = 1;
    return *save;
}

/* ------------------------------------------------------------------ */
/* Monte Carlo: single-particle translations                          */
/* ------------------------------------------------------------------ */

/* Random, Src/mollib.F90:2689-2708: Marsaglia xorshift (period 2^32-1) combined with
 * Park-Miller by Schrage's method (period 2^31-2), masked to a nonzero 31-bit
 * integer and scaled by am = nearest(1.0,-1.0)/im, a default-real (single
 * precision) quotient: (1 - 2^-24) 2^-31 exactly. */
static const double or_am = (1.0 - 5.9604644775390625e-08) * 4.656612873077392578125e-10;

void or_random_init(int32_t iseed, int32_t state[2])
{
    int32_t a = iseed < 0 ? (int32_t)(0u - (uint32_t)iseed) : iseed;   /* abs, wrapping at INT_MIN */
    state[1] = (888889999 ^ a) | 1;          /* iy */
    state[0] = 777755555 ^ a;                /* ix */
}

double or_random_next(int32_t state[2])
{
    uint32_t x = (uint32_t)state[0];
    int32_t iy = state[1], k;
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    state[0] = (int32_t)x;
    k = iy / 127773;
    iy = 16807 * (iy - k * 127773) - 2836 * k;
    if (iy < 0) iy += 2147483647;
    state[1] = iy;
    return or_am * (double)((2147483647 & (state[0] ^ state[1])) | 1);
}

void or_mc_seed(or_sys *s, int32_t iseed)
{
    int32_t st[2];
    or_random_init(iseed, st);
    s->rix = st[0];
    s->riy = st[1];
}

static double mc_random(or_sys *s)
{
    int32_t st[2];
    double r;
    st[0] = s->rix;
    st[1] = s->riy;
    r = or_random_next(st);
    s->rix = st[0];
    s->riy = st[1];
    return r;
}

/* u(r2) of one type pair by the table walk of UTwoBodyANewCellList,
 * Src/energy.F90:779-785 pattern (0-based iptjpt). */
static double tab_u(const or_sys *s, int iptjpt, double r2)
{
    int ibuf = s->iubuflow[iptjpt] - 1;
    double d;
    while (r2 < s->ubuf[ibuf]) ibuf += 12;
    d = r2 - s->ubuf[ibuf];
    return s->ubuf[ibuf + 1] + d * (s->ubuf[ibuf + 2] + d * (s->ubuf[ibuf + 3] + d * (s->ubuf[ibuf + 4] +
           d * (s->ubuf[ibuf + 5] + d * s->ubuf[ibuf + 6]))));
}

/* npass MCPass sweeps of SPartMove (Src/mc.F90:1470-1583, 1583-1755) with one
 * particle per trial: GetRandomTrialPos (:4527-4580), CheckPartBCTM with txbc 'xyz'
 * (PBC, :4810-4858), DUTotal (Src/denergy.F90:110-230) = DUTwoBody with the cell-list
 * routines' pair set (every partner inside rcut, :728-912: a hard-core or below-table
 * partner rejects the move) + DUTwoBodyEwald (:1240-1335 'std' and :1504-1536 surface)
 * + DUBond (:2893-2957), Metropolis (Src/mc.F90:5135-5175, weight 1) and MCUpdate
 * (:5203-5236, EwaldUpdateArray Src/denergy.F90:1776-1792).  u = [tot, twob(0..natat),
 * rec, bond] from the last UTotal, advanced by every accepted move.  Counts: accepted,
 * hard-core rejects. */
/* The SPME reciprocal energy of a charge mesh (before the EpsiFourPi scale): r2c transform
 * and the energyfac sum of UEwaldRecSPM / DUTwoBodyEwaldRecSPM (Src/denergy.F90:1480-1495). */
static double spm_mesh_energy(const or_sys *s, const double *Q, double *F)
{
    const int S = s->s, h = S / 2, hp = S / 2 + 1;
    double u = 0.0;
    int nx, ny, nz;
    or_fft3_r2c(S, Q, F);
    for (nz = 0; nz <= h; ++nz) {
        const int nza = (S - nz) % S;
        for (ny = 0; ny <= h; ++ny) {
            const int nya = (S - ny) % S;
            for (nx = 0; nx <= h; ++nx) {
                const size_t f = (size_t)nx + (size_t)hp * ((size_t)ny + (size_t)hp * nz);
                const size_t i1 = (size_t)nx + (size_t)hp * ((size_t)ny + (size_t)S * nz);
                const size_t i2 = (size_t)nx + (size_t)hp * ((size_t)ny + (size_t)S * nza);
                const size_t i3 = (size_t)nx + (size_t)hp * ((size_t)nya + (size_t)S * nz);
                const size_t i4 = (size_t)nx + (size_t)hp * ((size_t)nya + (size_t)S * nza);
                const double Qsum = F[2 * i1] * F[2 * i1] + F[2 * i1 + 1] * F[2 * i1 + 1] +
                                    F[2 * i2] * F[2 * i2] + F[2 * i2 + 1] * F[2 * i2 + 1] +
                                    F[2 * i3] * F[2 * i3] + F[2 * i3 + 1] * F[2 * i3 + 1] +
                                    F[2 * i4] * F[2 * i4] + F[2 * i4 + 1] * F[2 * i4 + 1];
                u = u + Qsum * s->energyfac[f];
            }
        }
    }
    return u;
}

/* q M M M of one particle at r added (sign +1) or removed (-1) on the charge mesh Q
 * (Src/denergy.F90:1441-1470). */
static void spm_stencil(const or_sys *s, double *Q, const double r[3], double q, double sign)
{
    const int S = s->s, order = s->order;
    double spline[3][32], deriv[3][32];
    int32_t km[3];
    int m, ix, iy, iz;
    for (m = 0; m < 3; ++m) {
        or_cardinal_bspline(order, (S / s->boxlen[m]) * r[m], &km[m], spline[m], deriv[m]);
        km[m] = (km[m] + S) % S;
    }
    for (iz = 0; iz < order; ++iz) {
        const int nz = (S + km[2] - iz) % S;
        const double qz = q * spline[2][iz];
        for (iy = 0; iy < order; ++iy) {
            const int ny = (S + km[1] - iy) % S;
            const double qyz = qz * spline[1][iy];
            for (ix = 0; ix < order; ++ix) {
                const int nx = (S + km[0] - ix) % S;
                Q[(size_t)nx + S * ((size_t)ny + (size_t)S * nz)] += sign * (qyz * spline[0][ix]);
            }
        }
    }
}

int or_mc_pass(or_sys *s, int npass, int isamp, const double *dtran, double beta, double *u,
               int64_t *accepted, int64_t *hsreject)
{
    const int np = s->np, natat = s->natat;
    int pass, ipass, k;
    double *dtwob = malloc(sizeof(double) * (natat + 1)), *unew = malloc(sizeof(double) * (natat + 1));
    double *uold = malloc(sizeof(double) * (natat + 1));
    cx *tm[3] = {NULL, NULL, NULL}, *stm = NULL, *yzt = NULL;
    double *trigtm = NULL, *sttm = NULL;     /* layer correction: trial tables and sums */
    double *qm = NULL, *qmtm = NULL, *fq = NULL, urecold = 0.0, urecnew = 0.0;   /* SPME */
    const size_t w = (size_t)s->ncut + 1;
    if (s->lewald == 1) {
        /* DUTwoBodyEwaldRecSPM: the charge mesh of the configuration and its energy */
        const size_t n = (size_t)s->s * s->s * s->s;
        int ia;
        qm = calloc(n, sizeof(double));
        qmtm = malloc(sizeof(double) * n);
        fq = malloc(sizeof(double) * 2 * (size_t)(s->s / 2 + 1) * s->s * s->s);
        for (ia = 0; ia < np; ++ia) spm_stencil(s, qm, s->ro + 3 * ia, s->az[ia], 1.0);
        urecold = spm_mesh_energy(s, qm, fq);
    }
    if (s->lewald == 2) {
        for (k = 0; k < 3; ++k) tm[k] = malloc(sizeof(cx) * w);
        stm = malloc(sizeof(cx) * 4 * (size_t)(s->nkvec > 0 ? s->nkvec : 1));
        yzt = malloc(sizeof(cx) * 2);
    }
    if (s->elc && s->lewald == 2) {
        trigtm = malloc(sizeof(double) * 4 * w);
        sttm = malloc(sizeof(double) * 8 * (size_t)(s->nkvec2d > 0 ? s->nkvec2d : 1));
    }
    for (pass = 0; pass < npass; ++pass) {
        for (ipass = 0; ipass < np; ++ipass) {
            int ip, ipt, jp, m, overlap = 0;
            double dtr, d[3], rtm[3], dutot = 0.0, durec = 0.0, dubond = 0.0, dured;
            /* select a particle */
            if (isamp == 0) {
                ip = ipass + 1;
            } else {
                ip = 1 + (int)(np * mc_random(s));
            }
            ip = ip < 1 ? 1 : (ip > np ? np : ip);
            ip -= 1;
            ipt = s->iptpn[ip] - 1;
            dtr = dtran[ipt];
            /* GetRandomTrialPos */
            if (dtr >= 0.0) {
                d[0] = (mc_random(s) - 0.5) * dtr;
                d[1] = (mc_random(s) - 0.5) * dtr;
                d[2] = (mc_random(s) - 0.5) * dtr;
            } else {
                for (;;) {
                    d[0] = mc_random(s) - 0.5;
                    d[1] = mc_random(s) - 0.5;
                    d[2] = mc_random(s) - 0.5;
                    if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < 0.5 * 0.5) break;
                }
                for (m = 0; m < 3; ++m) d[m] = d[m] * fabs(dtr);
            }
            for (m = 0; m < 3; ++m) rtm[m] = s->ro[3 * ip + m] + d[m];
            /* CheckPartBCTM, txbc 'xyz': PBC */
            for (m = 0; m < 3; ++m) rtm[m] = pbc1(rtm[m], s->boxlen2[m], s->boxlen[m], s->boxleni[m]);
            /* DUTwoBody: new configuration, with the overlap checks */
            for (k = 0; k <= natat; ++k) unew[k] = uold[k] = 0.0;
            for (jp = 0; jp < np && !overlap; ++jp) {
                double dx, dy, dz, r2;
                int ij;
                if (jp == ip) continue;
                dx = rtm[0] - s->ro[3 * jp];
                dy = rtm[1] - s->ro[3 * jp + 1];
                dz = rtm[2] - s->ro[3 * jp + 2];
                r2 = pbcr2(s, &dx, &dy, &dz);
                if (!(r2 < s->rcut2)) continue;
                ij = pair_index(s->npt, ipt + 1, s->iptpn[jp]);        /* 1-based iptjpt */
                if (r2 < s->r2atat[ij - 1] || r2 < s->r2umin[ij - 1]) { overlap = 1; break; }
                unew[ij] += tab_u(s, ij - 1, r2);
            }
            if (overlap) {
                if (hsreject) ++*hsreject;
                continue;                            /* Metropolis: imchsreject, no random number */
            }
            for (jp = 0; jp < np; ++jp) {
                double dx, dy, dz, r2;
                int ij;
                if (jp == ip) continue;
                dx = s->ro[3 * ip] - s->ro[3 * jp];
                dy = s->ro[3 * ip + 1] - s->ro[3 * jp + 1];
                dz = s->ro[3 * ip + 2] - s->ro[3 * jp + 2];
                r2 = pbcr2(s, &dx, &dy, &dz);
                if (!(r2 < s->rcut2)) continue;
                ij = pair_index(s->npt, ipt + 1, s->iptpn[jp]);
                uold[ij] += tab_u(s, ij - 1, r2);
            }
            for (k = 1; k <= natat; ++k) { unew[0] += unew[k]; uold[0] += uold[k]; }
            for (k = 0; k <= natat; ++k) dtwob[k] = unew[k] - uold[k];
            dutot = dutot + dtwob[0];
            /* DUTwoBodyEwald: SPME reciprocal difference (the whole mesh re-transformed) */
            if (s->lewald == 1) {
                const double q = s->az[ip];
                memcpy(qmtm, qm, sizeof(double) * (size_t)s->s * s->s * s->s);
                spm_stencil(s, qmtm, s->ro + 3 * ip, q, -1.0);
                spm_stencil(s, qmtm, rtm, q, 1.0);
                urecnew = spm_mesh_energy(s, qmtm, fq);
                durec = urecnew - urecold;
                if (s->lsurf) {
                    const double fac = 2.0 * Pi / (3.0 * s->vol);
                    double sx = 0.0, sy = 0.0, sz = 0.0, tx, ty, tz;
                    int ia;
                    for (ia = 0; ia < np; ++ia) {
                        sx += s->az[ia] * s->ro[3 * ia];
                        sy += s->az[ia] * s->ro[3 * ia + 1];
                        sz += s->az[ia] * s->ro[3 * ia + 2];
                    }
                    if (s->elc) {
                        tz = sz + q * (rtm[2] - s->ro[3 * ip + 2]);
                        durec = durec + (2.0 * Pi / s->vol) * (tz * tz - sz * sz);
                    } else {
                        tx = sx + q * (rtm[0] - s->ro[3 * ip]);
                        ty = sy + q * (rtm[1] - s->ro[3 * ip + 1]);
                        tz = sz + q * (rtm[2] - s->ro[3 * ip + 2]);
                        durec = durec + fac * ((tx * tx + ty * ty + tz * tz) - (sx * sx + sy * sy + sz * sz));
                    }
                }
                durec = s->epsfp * durec;
                dutot = dutot + durec;
            }
            /* DUTwoBodyEwald: 'std' reciprocal sum and the surface term */
            if (s->lewald == 2) {
                const int nc = s->ncut, ncut2 = s->ncut2;
                const double q = s->az[ip];
                const cx *ex = (const cx *)s->eik[0] + (size_t)ip * w;
                const cx *ey = (const cx *)s->eik[1] + (size_t)ip * w;
                const cx *ez = (const cx *)s->eik[2] + (size_t)ip * w;
                const cx *S4 = (const cx *)s->sumeikr;
                double tpbi[3];
                int nx, ny, nz, kn = 0, icut;
                for (m = 0; m < 3; ++m) tpbi[m] = 2.0 * Pi * s->boxleni[m];
                /* EwaldSetArrayTM (Src/energy.F90:1440-1466 pattern): tables of the trial position */
                for (m = 0; m < 3; ++m) {
                    tm[m][0].r = 1.0; tm[m][0].i = 0.0;
                    tm[m][1].r = cos(tpbi[m] * rtm[m]);
                    tm[m][1].i = sin(tpbi[m] * rtm[m]);
                    for (icut = 2; icut <= nc; ++icut) tm[m][icut] = cmul(tm[m][icut - 1], tm[m][1]);
                }
                for (nz = 0; nz <= nc; ++nz) {
                    for (ny = 0; ny <= nc; ++ny) {
                        cx yc, yct, yzm, yzp, yzmt, yzpt;
                        if (ny * ny + nz * nz > ncut2) continue;
                        yc.r = ey[ny].r; yc.i = -ey[ny].i;
                        yzm = cmul(yc, ez[nz]);
                        yzp = cmul(ey[ny], ez[nz]);
                        yct.r = tm[1][ny].r; yct.i = -tm[1][ny].i;
                        yzmt = cmul(yct, tm[2][nz]);
                        yzpt = cmul(tm[1][ny], tm[2][nz]);
                        for (nx = 0; nx <= nc; ++nx) {
                            cx xo = ex[nx], xt = tm[0][nx], xoc, xtc, a, b, *st;
                            double termnew, termold;
                            if (nx * nx + ny * ny + nz * nz > ncut2) continue;
                            if (nx == 0 && ny == 0 && nz == 0) continue;
                            xoc.r = xo.r; xoc.i = -xo.i;
                            xtc.r = xt.r; xtc.i = -xt.i;
                            st = stm + 4 * (size_t)kn;
                            for (k = 0; k < 4; ++k) st[k] = S4[4 * (size_t)kn + k];
                            /* sumeikrtm = sumeikr + az*(new - old), per sign pattern */
                            a = cmul(xtc, yzmt); b = cmul(xoc, yzm);
                            st[0].r = st[0].r + q * (a.r - b.r); st[0].i = st[0].i + q * (a.i - b.i);
                            a = cmul(xtc, yzpt); b = cmul(xoc, yzp);
                            st[1].r = st[1].r + q * (a.r - b.r); st[1].i = st[1].i + q * (a.i - b.i);
                            a = cmul(xt, yzmt); b = cmul(xo, yzm);
                            st[2].r = st[2].r + q * (a.r - b.r); st[2].i = st[2].i + q * (a.i - b.i);
                            a = cmul(xt, yzpt); b = cmul(xo, yzp);
                            st[3].r = st[3].r + q * (a.r - b.r); st[3].i = st[3].i + q * (a.i - b.i);
                            termnew = st[0].r * st[0].r + st[0].i * st[0].i + st[1].r * st[1].r + st[1].i * st[1].i +
                                      st[2].r * st[2].r + st[2].i * st[2].i + st[3].r * st[3].r + st[3].i * st[3].i;
                            {
                                const cx *so = S4 + 4 * (size_t)kn;
                                termold = so[0].r * so[0].r + so[0].i * so[0].i + so[1].r * so[1].r +
                                          so[1].i * so[1].i + so[2].r * so[2].r + so[2].i * so[2].i +
                                          so[3].r * so[3].r + so[3].i * so[3].i;
                            }
                            durec = durec + s->kfac[kn] * (termnew - termold);
                            ++kn;
                        }
                    }
                }
                if (s->elc) {
                    /* DUTwoBodyEwaldRec2dlc (Src/denergy.F90:1339-1409) with EwaldSetArray2dTM */
                    const double *to = s->trig2d + (size_t)ip * 4 * w;
                    for (m = 0; m < 4; ++m) trigtm[m * w] = 1.0;
                    if (nc >= 1) {
                        trigtm[1] = sin(tpbi[0] * rtm[0]);
                        trigtm[w + 1] = cos(tpbi[0] * rtm[0]);
                        trigtm[2 * w + 1] = sin(tpbi[1] * rtm[1]);
                        trigtm[3 * w + 1] = cos(tpbi[1] * rtm[1]);
                    }
                    for (icut = 2; icut <= nc; ++icut) {
                        trigtm[icut] = trigtm[icut - 1] * trigtm[w + 1] + trigtm[w + icut - 1] * trigtm[1];
                        trigtm[w + icut] = trigtm[w + icut - 1] * trigtm[w + 1] - trigtm[icut - 1] * trigtm[1];
                        trigtm[2 * w + icut] = trigtm[2 * w + icut - 1] * trigtm[3 * w + 1] +
                                               trigtm[3 * w + icut - 1] * trigtm[2 * w + 1];
                        trigtm[3 * w + icut] = trigtm[3 * w + icut - 1] * trigtm[3 * w + 1] -
                                               trigtm[2 * w + icut - 1] * trigtm[2 * w + 1];
                    }
                    kn = 0;
                    for (ny = 0; ny <= nc; ++ny) {
                        const double ky = ny * tpbi[1];
                        for (nx = 0; nx <= nc; ++nx) {
                            const double kx = nx * tpbi[0];
                            double kp, e, ei, sht, cht, sho, cho, tn, to_, *st = sttm + 8 * (size_t)kn;
                            const double *so = s->sumtrig + 8 * (size_t)kn;
                            const double sxt = trigtm[nx], cxt = trigtm[w + nx], syt = trigtm[2 * w + ny],
                                         cyt = trigtm[3 * w + ny];
                            const double sxo = to[nx], cxo = to[w + nx], syo = to[2 * w + ny], cyo = to[3 * w + ny];
                            if (nx * nx + ny * ny > s->ncut2d2) continue;
                            if (nx == 0 && ny == 0) continue;
                            kp = sqrt(kx * kx + ky * ky);
                            e = exp(kp * rtm[2]); ei = 1.0 / e;
                            sht = 0.5 * (e - ei); cht = 0.5 * (e + ei);
                            e = exp(kp * s->ro[3 * ip + 2]); ei = 1.0 / e;
                            sho = 0.5 * (e - ei); cho = 0.5 * (e + ei);
                            st[0] = so[0] + q * (sxt * syt * sht - sxo * syo * sho);
                            st[1] = so[1] + q * (cxt * syt * sht - cxo * syo * sho);
                            st[2] = so[2] + q * (sxt * cyt * sht - sxo * cyo * sho);
                            st[3] = so[3] + q * (cxt * cyt * sht - cxo * cyo * sho);
                            st[4] = so[4] + q * (sxt * syt * cht - sxo * syo * cho);
                            st[5] = so[5] + q * (cxt * syt * cht - cxo * syo * cho);
                            st[6] = so[6] + q * (sxt * cyt * cht - sxo * cyo * cho);
                            st[7] = so[7] + q * (cxt * cyt * cht - cxo * cyo * cho);
                            tn = -st[0] * st[0] - st[1] * st[1] - st[2] * st[2] - st[3] * st[3] +
                                 st[4] * st[4] + st[5] * st[5] + st[6] * st[6] + st[7] * st[7];
                            to_ = -so[0] * so[0] - so[1] * so[1] - so[2] * so[2] - so[3] * so[3] +
                                  so[4] * so[4] + so[5] * so[5] + so[6] * so[6] + so[7] * so[7];
                            durec = durec + s->kfac2d[kn] * (tn - to_);
                            ++kn;
                        }
                    }
                }
                if (s->lsurf && s->elc) {
                    /* DUTwoBodyEwaldSurf, 2d-periodic form: the z dipole */
                    const double fac = 2.0 * Pi / s->vol;
                    double sz = 0.0, tz;
                    int ia;
                    for (ia = 0; ia < np; ++ia) sz += s->az[ia] * s->ro[3 * ia + 2];
                    tz = sz + q * (rtm[2] - s->ro[3 * ip + 2]);
                    durec = durec + fac * (tz * tz - sz * sz);
                } else if (s->lsurf) {
                    const double fac = 2.0 * Pi / (3.0 * s->vol);
                    double sx = 0.0, sy = 0.0, sz = 0.0, tx, ty, tz;
                    int ia;
                    for (ia = 0; ia < np; ++ia) {
                        sx += s->az[ia] * s->ro[3 * ia];
                        sy += s->az[ia] * s->ro[3 * ia + 1];
                        sz += s->az[ia] * s->ro[3 * ia + 2];
                    }
                    tx = sx + q * (rtm[0] - s->ro[3 * ip]);
                    ty = sy + q * (rtm[1] - s->ro[3 * ip + 1]);
                    tz = sz + q * (rtm[2] - s->ro[3 * ip + 2]);
                    durec = durec + fac * ((tx * tx + ty * ty + tz * tz) - (sx * sx + sy * sy + sz * sz));
                }
                durec = s->epsfp * durec;
                dutot = dutot + durec;
            }
            /* DUBond: every bond of the moved particle, lower neighbour first */
            if (s->nbond > 0) {
                int b;
                for (b = 0; b < s->nbond; ++b) {
                    int a1 = s->bond_ij[2 * b] - 1, a2 = s->bond_ij[2 * b + 1] - 1, other, pw, e;
                    double dx, dy, dz, r2n, r2o, xn, xo, pn = 1.0, po = 1.0;
                    if (a1 != ip && a2 != ip) continue;
                    other = (a1 == ip) ? a2 : a1;
                    dx = rtm[0] - s->ro[3 * other];
                    dy = rtm[1] - s->ro[3 * other + 1];
                    dz = rtm[2] - s->ro[3 * other + 2];
                    r2n = pbcr2(s, &dx, &dy, &dz);
                    dx = s->ro[3 * ip] - s->ro[3 * other];
                    dy = s->ro[3 * ip + 1] - s->ro[3 * other + 1];
                    dz = s->ro[3 * ip + 2] - s->ro[3 * other + 2];
                    r2o = pbcr2(s, &dx, &dy, &dz);
                    xn = sqrt(r2n) - s->bond_eq[b];
                    xo = sqrt(r2o) - s->bond_eq[b];
                    pw = s->bond_p[b];
                    for (e = 0; e < pw; ++e) { pn *= xn; po *= xo; }
                    dubond = dubond + s->bond_k[b] * (pn - po);
                }
                dutot = dutot + dubond;
            }
            /* Metropolis, weight 1, expmax = 87 (Src/mol.F90:62) */
            dured = dutot * beta;
            {
                int accept;
                if (dured > 87.0) {
                    accept = 0;
                } else if (dured < -87.0) {
                    accept = 1;
                } else {
                    double fac = exp(-dured);
                    accept = (fac > 1.0) ? 1 : (fac > mc_random(s));
                }
                if (!accept) continue;
            }
            /* MCUpdate */
            if (accepted) ++*accepted;
            u[0] = u[0] + dutot;
            for (k = 0; k <= natat; ++k) u[1 + k] = u[1 + k] + dtwob[k];
            if (s->lewald) u[2 + natat] = u[2 + natat] + durec;
            if (s->nbond > 0) u[3 + natat] = u[3 + natat] + dubond;
            if (s->lewald == 2) {
                for (m = 0; m < 3; ++m) memcpy((cx *)s->eik[m] + (size_t)ip * w, tm[m], sizeof(cx) * w);
                memcpy(s->sumeikr, stm, sizeof(cx) * 4 * (size_t)s->nkvec);
            }
            if (s->elc && s->lewald == 2) {
                memcpy(s->trig2d + (size_t)ip * 4 * w, trigtm, sizeof(double) * 4 * w);
                memcpy(s->sumtrig, sttm, sizeof(double) * 8 * (size_t)s->nkvec2d);
            }
            if (s->lewald == 1) {
                double *t_ = qm;
                qm = qmtm;
                qmtm = t_;
                urecold = urecnew;
            }
            for (m = 0; m < 3; ++m) {
                s->ro[3 * ip + m] = rtm[m];
                s->drostep[3 * ip + m] += d[m];
            }
        }
    }
    free(dtwob); free(unew); free(uold);
    for (k = 0; k < 3; ++k) free(tm[k]);
    free(stm); free(yzt); free(trigtm); free(sttm); free(qm); free(qmtm); free(fq);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Polyatomic particles: UTwoBodyP                                     */
/* ------------------------------------------------------------------ */

/* UTwoBodyP, Src/energy.F90:786-896 (box cell), with PBC2 (Src/molaux.F90:193-210):
 * the particle list decides the pairs (particle centres within rcut), every site
 * pair of the two particles interacts through the atom-type table with the centres'
 * periodic shift.  1-based MOLSIM arrays; force [na][3] is overwritten (kJ/(mol A)),
 * utwob [nptpt+1] = u%twob(0:nptpt) by particle-type pair, *virial the pair virial.
 * Returns 1 when an atom pair lies below r2umin (StopUTwoBodyP), 2 on a table overrun. */
int or_utwobody_p(int32_t np, int32_t na, int32_t npt, int32_t nat, const double boxlen[3], double rcut,
                  const double *ro, const double *r, const int32_t *iptpn, const int32_t *ianpn,
                  const int32_t *napt, const int32_t *iatan, const int32_t *nneighpn, const int32_t *jpnlist,
                  int32_t maxnneigh, const double *ubuf, int32_t nbuf, const int32_t *iubuflow,
                  const double *r2umin, double *force, double *utwob, double *virial)
{
    const double rcut2 = rcut * rcut;
    const int nptpt = npt * (npt + 1) / 2;
    double half[3], vir = 0.0;
    int ip, m, k;
    for (m = 0; m < 3; ++m) half[m] = boxlen[m] / 2.0;
    for (k = 0; k < 3 * na; ++k) force[k] = 0.0;
    for (k = 0; k <= nptpt; ++k) utwob[k] = 0.0;
    for (ip = 0; ip < np; ++ip) {
        const int ipt = iptpn[ip], ialow = ianpn[ip] - 1, iaupp = ialow + napt[ipt - 1] - 1;
        int jploc;
        for (jploc = 0; jploc < nneighpn[ip]; ++jploc) {
            const int jp = jpnlist[(size_t)ip * maxnneigh + jploc] - 1;
            const int jpt = iptpn[jp], iptjpt = pair_index(npt, ipt, jpt);
            const int jalow = ianpn[jp] - 1, jaupp = jalow + napt[jpt - 1] - 1;
            double d[3], sh[3], r2, usum = 0.0;
            int ia, ja;
            for (m = 0; m < 3; ++m) {
                d[m] = ro[3 * ip + m] - ro[3 * jp + m];
                sh[m] = fabs(d[m]) > half[m] ? copysign(boxlen[m], d[m]) : 0.0;   /* PBC2 */
                d[m] = d[m] - sh[m];
            }
            r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (r2 > rcut2) continue;
            for (ia = ialow; ia <= iaupp; ++ia) {
                const int iat = iatan[ia];
                for (ja = jalow; ja <= jaupp; ++ja) {
                    const int jat = iatan[ja], iatjat = pair_index(nat, iat, jat);
                    double dx = r[3 * ia] - r[3 * ja] - sh[0];
                    double dy = r[3 * ia + 1] - r[3 * ja + 1] - sh[1];
                    double dz = r[3 * ia + 2] - r[3 * ja + 2] - sh[2];
                    double a2 = dx * dx + dy * dy + dz * dz, dd, fsum;
                    int ibuf;
                    if (a2 < r2umin[iatjat - 1]) return 1;
                    ibuf = iubuflow[iatjat - 1] - 1;
                    while (a2 < ubuf[ibuf]) {
                        ibuf += 12;
                        if (ibuf + 12 > nbuf) return 2;
                    }
                    dd = a2 - ubuf[ibuf];
                    usum = usum + ubuf[ibuf + 1] + dd * (ubuf[ibuf + 2] + dd * (ubuf[ibuf + 3] +
                           dd * (ubuf[ibuf + 4] + dd * (ubuf[ibuf + 5] + dd * ubuf[ibuf + 6]))));
                    fsum = ubuf[ibuf + 7] + dd * (ubuf[ibuf + 8] + dd * (ubuf[ibuf + 9] +
                           dd * (ubuf[ibuf + 10] + dd * ubuf[ibuf + 11])));
                    force[3 * ia] += fsum * dx;
                    force[3 * ia + 1] += fsum * dy;
                    force[3 * ia + 2] += fsum * dz;
                    force[3 * ja] -= fsum * dx;
                    force[3 * ja + 1] -= fsum * dy;
                    force[3 * ja + 2] -= fsum * dz;
                    vir = vir - fsum * a2;
                }
            }
            utwob[iptjpt] = utwob[iptjpt] + usum;
        }
    }
    for (k = 1; k <= nptpt; ++k) utwob[0] += utwob[k];
    *virial = vir;
    return 0;
}

/* ------------------------------------------------------------------ */
/* Rigid polyatomic particles: VelVer with lpolyatom                   */
/* ------------------------------------------------------------------ */

/* QuaToOri, Src/mollib.F90:2221-2255: ori[3][3] (row i, column j) of one quaternion */
static void qua_to_ori(const double *q, double *o)
{
    const double q00 = q[0] * q[0], q11 = q[1] * q[1], q22 = q[2] * q[2], q33 = q[3] * q[3];
    const double q01 = q[0] * q[1], q02 = q[0] * q[2], q03 = q[0] * q[3];
    const double q12 = q[1] * q[2], q13 = q[1] * q[3], q23 = q[2] * q[3];
    o[0] = -q22 + q11 - q33 + q00;          /* ori(1,1) */
    o[3] = 2.0 * (q03 - q12);               /* ori(2,1) */
    o[6] = 2.0 * (q13 + q02);               /* ori(3,1) */
    o[1] = -2.0 * (q12 + q03);              /* ori(1,2) */
    o[4] = q22 - q11 - q33 + q00;           /* ori(2,2) */
    o[7] = 2.0 * (q01 - q23);               /* ori(3,2) */
    o[2] = 2.0 * (q13 - q02);               /* ori(1,3) */
    o[5] = -2.0 * (q23 + q01);              /* ori(2,3) */
    o[8] = -q22 - q11 + q33 + q00;          /* ori(3,3) */
}

/* QuaNorm, Src/mollib.F90:2594-2612 */
static void qua_norm(double *q)
{
    const double norm = 1.0 / sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    int k;
    for (k = 0; k < 4; ++k) q[k] = q[k] * norm;
}

/* QuaVelToAngVel, Src/mollib.F90:2651-2669 */
static void qua_vel_to_ang_vel(const double *q, const double *qd, double *w)
{
    w[0] = 2.0 * (-q[3] * qd[2] + q[0] * qd[1] + q[2] * qd[3] - q[1] * qd[0]);
    w[1] = 2.0 * (-q[0] * qd[2] - q[3] * qd[1] + q[1] * qd[3] + q[2] * qd[0]);
    w[2] = 2.0 * (+q[1] * qd[2] - q[2] * qd[1] + q[0] * qd[3] - q[3] * qd[0]);
}

/* GetAngAcc, Src/md.F90:628-663: quaternion acceleration from the lab-frame torque */
static void get_ang_acc(const double *tor, const double *o, const double *w, const double *momp,
                        const double *q, const double *qd, double *qdd)
{
    const double t1 = tor[0] * o[0] + tor[1] * o[3] + tor[2] * o[6];
    const double t2 = tor[0] * o[1] + tor[1] * o[4] + tor[2] * o[7];
    const double t3 = tor[0] * o[2] + tor[1] * o[5] + tor[2] * o[8];
    const double a1 = (t1 + w[1] * w[2] * (momp[1] - momp[2])) * (1.0 / momp[0]);
    const double a2 = (t2 + w[2] * w[0] * (momp[2] - momp[0])) * (1.0 / momp[1]);
    const double a3 = (t3 + w[0] * w[1] * (momp[0] - momp[1])) * (1.0 / momp[2]);
    const double fac = -2.0 * (qd[2] * qd[2] + qd[1] * qd[1] + qd[3] * qd[3] + qd[0] * qd[0]);
    qdd[0] = 0.5 * (-q[1] * a1 + q[2] * a2 - q[3] * a3 + q[0] * fac);
    qdd[1] = 0.5 * (+q[0] * a1 - q[3] * a2 - q[2] * a3 + q[1] * fac);
    qdd[2] = 0.5 * (-q[3] * a1 - q[0] * a2 + q[1] * a3 + q[2] * fac);
    qdd[3] = 0.5 * (+q[2] * a1 + q[1] * a2 + q[0] * a3 + q[3] * fac);
}

/* SetAtomPos (ra), Src/molaux.F90:526-545: r = ro + ori ra for the sites of every particle */
static void set_atom_pos(int32_t np, const double *ro, const double *ori, const int32_t *iptpn,
                         const int32_t *ianpn, const int32_t *napt, const double *ra, int32_t maxsite, double *r)
{
    int ip, a, m;
    for (ip = 0; ip < np; ++ip) {
        const int ipt = iptpn[ip] - 1, ia0 = ianpn[ip] - 1;
        const double *o = ori + 9 * (size_t)ip;
        for (a = 0; a < napt[ipt]; ++a) {
            const double *x = ra + 3 * ((size_t)ipt * maxsite + a);
            for (m = 0; m < 3; ++m)
                r[3 * (size_t)(ia0 + a) + m] = ro[3 * ip + m] + o[3 * m] * x[0] + o[3 * m + 1] * x[1] + o[3 * m + 2] * x[2];
        }
    }
}

/* Forces, torques and the molecular virial of UTotal, Src/energy.F90:403-426 (no site
 * torques): force (kJ/(mol A)) is converted in place; forceo/torqueo per particle. */
static double rigid_forces(int32_t np, const double *ro, const double *r, const int32_t *iptpn, const int32_t *ianpn,
                           const int32_t *napt, double *force, double *forceo, double *torqueo)
{
    const double fac = (sclene / scllen) / sclfor();
    double virmol = 0.0;
    int ip, a;
    for (ip = 0; ip < np; ++ip) {
        const int ia0 = ianpn[ip] - 1, nat_ = napt[iptpn[ip] - 1];
        double *fo = forceo + 3 * (size_t)ip, *to = torqueo + 3 * (size_t)ip;
        fo[0] = fo[1] = fo[2] = to[0] = to[1] = to[2] = 0.0;
        for (a = 0; a < nat_; ++a) {
            double *f = force + 3 * (size_t)(ia0 + a);
            const double dx = r[3 * (size_t)(ia0 + a)] - ro[3 * ip];
            const double dy = r[3 * (size_t)(ia0 + a) + 1] - ro[3 * ip + 1];
            const double dz = r[3 * (size_t)(ia0 + a) + 2] - ro[3 * ip + 2];
            virmol = virmol + dx * f[0] + dy * f[1] + dz * f[2];
            f[0] = f[0] * fac;
            f[1] = f[1] * fac;
            f[2] = f[2] * fac;
            fo[0] = fo[0] + f[0];
            fo[1] = fo[1] + f[1];
            fo[2] = fo[2] + f[2];
            to[0] = to[0] + dy * f[2] - dz * f[1];
            to[1] = to[1] + dz * f[0] - dx * f[2];
            to[2] = to[2] + dx * f[1] - dy * f[0];
        }
    }
    return virmol;
}

/* nsteps of VelVer for rigid polyatomic particles, Src/md.F90:252-410 (lpolyatom, the
 * particle list held fixed): linear and quaternion position update, QuaNorm, QuaToOri,
 * PBC of the centres, SetAtomPos, UTotal's pair part (UTwoBodyP) with forces, torques
 * and the molecular virial, GetLinAcc and the linear half-kick, then the quaternion
 * velocities by nvvite iterations of QuaVelToAngVel + GetAngAcc (tvvite's trial step).
 * State arrays (MOLSIM layout) are advanced in place; ra [npt][maxsite][3] are the
 * sites in the principal frame, masspt [npt] and momp [npt][3] the particle masses and
 * principal moments.  Energies and virial of the last step.  Returns UTwoBodyP's status. */
/* Site Ewald parameters of the rigid-body step (or_velver_p_ewald). */
typedef struct {
    const double *az;
    double ualpha, epsfp;
    int32_t lewald, ncut, ncutregion, order, nmesh, lsurf;
} site_ew;

static int uewald_sites_impl(int32_t lewald, int32_t na, const double boxlen[3], double ualpha, int32_t ncut,
                             int32_t ncutregion, int32_t order, int32_t nmesh, int32_t lsurf, double epsfp,
                             const double *r, const double *az, int32_t np, const int32_t *iptpn,
                             const int32_t *ianpn, const int32_t *napt, double *force, double *urec, double *virrec);

static int velver_p_impl(const site_ew *ew, double *urec, int32_t nsteps, int32_t np, int32_t na, int32_t npt,
                         int32_t nat, const double boxlen[3], double rcut, double tstep, int32_t nvvite, double tvvite,
                         double *ro, double *rod, double *rodd, double *qua, double *quad, double *quadd, double *r,
                         const int32_t *iptpn, const int32_t *ianpn, const int32_t *napt, const int32_t *iatan,
                         const double *ra, int32_t maxsite, const double *masspt, const double *momp,
                         const int32_t *nneighpn, const int32_t *jpnlist, int32_t maxnneigh, const double *ubuf,
                         int32_t nbuf, const int32_t *iubuflow, const double *r2umin, double *utwob, double *virial)
{
    const double fac = 0.5 * tstep * tstep;
    double *ori = malloc(sizeof(double) * 9 * (size_t)np), *force = malloc(sizeof(double) * 3 * (size_t)na);
    double *forceo = malloc(sizeof(double) * 3 * (size_t)np), *torqueo = malloc(sizeof(double) * 3 * (size_t)np);
    double half[3];
    int step, ip, m, k, it, rc = 0;
    for (m = 0; m < 3; ++m) half[m] = boxlen[m] / 2.0;
    for (step = 0; step < nsteps && !rc; ++step) {
        double vpair = 0.0;
        for (ip = 0; ip < np; ++ip) {
            for (m = 0; m < 3; ++m) {
                const double d = tstep * rod[3 * ip + m] + fac * rodd[3 * ip + m];
                ro[3 * ip + m] = pbc1(ro[3 * ip + m] + d, half[m], boxlen[m], 1.0 / boxlen[m]);
            }
            for (k = 0; k < 4; ++k) qua[4 * ip + k] = qua[4 * ip + k] + tstep * quad[4 * ip + k] + fac * quadd[4 * ip + k];
            qua_norm(qua + 4 * ip);
            qua_to_ori(qua + 4 * ip, ori + 9 * (size_t)ip);
        }
        set_atom_pos(np, ro, ori, iptpn, ianpn, napt, ra, maxsite, r);
        rc = or_utwobody_p(np, na, npt, nat, boxlen, rcut, ro, r, iptpn, ianpn, napt, iatan, nneighpn, jpnlist,
                           maxnneigh, ubuf, nbuf, iubuflow, r2umin, force, utwob, &vpair);
        if (rc) break;
        if (ew) {                                  /* UTotal's UEwald over the sites (Src/energy.F90:335-352) */
            double *fe = malloc(sizeof(double) * 3 * (size_t)na), vr = 0.0;
            uewald_sites_impl(ew->lewald, na, boxlen, ew->ualpha, ew->ncut, ew->ncutregion, ew->order, ew->nmesh,
                              ew->lsurf, ew->epsfp, r, ew->az, np, iptpn, ianpn, napt, fe, urec, &vr);
            for (m = 0; m < 3 * na; ++m) force[m] = force[m] + fe[m];
            vpair = vpair + vr;
            free(fe);
        }
        *virial = vpair + rigid_forces(np, ro, r, iptpn, ianpn, napt, force, forceo, torqueo);
        for (ip = 0; ip < np; ++ip) {
            const int ipt = iptpn[ip] - 1;
            const double mi = 1.0 / masspt[ipt];
            double qdo[4], qddo[4], w[3];
            for (m = 0; m < 3; ++m) {                         /* GetLinAcc and the half-kick */
                const double ao = rodd[3 * ip + m];
                rodd[3 * ip + m] = forceo[3 * ip + m] * mi;
                rod[3 * ip + m] = rod[3 * ip + m] + 0.5 * tstep * (rodd[3 * ip + m] + ao);
            }
            for (k = 0; k < 4; ++k) {
                qddo[k] = quadd[4 * ip + k];
                qdo[k] = quad[4 * ip + k];
                quad[4 * ip + k] = qdo[k] + (tvvite * tstep) * qddo[k];
            }
            for (it = 0; it < nvvite; ++it) {
                qua_vel_to_ang_vel(qua + 4 * ip, quad + 4 * ip, w);
                get_ang_acc(torqueo + 3 * ip, ori + 9 * (size_t)ip, w, momp + 3 * ipt, qua + 4 * ip, quad + 4 * ip,
                            quadd + 4 * ip);
                for (k = 0; k < 4; ++k) quad[4 * ip + k] = qdo[k] + (0.5 * tstep) * (quadd[4 * ip + k] + qddo[k]);
            }
        }
    }
    free(ori); free(force); free(forceo); free(torqueo);
    return rc;
}

int or_velver_p(int32_t nsteps, int32_t np, int32_t na, int32_t npt, int32_t nat, const double boxlen[3],
                double rcut, double tstep, int32_t nvvite, double tvvite, double *ro, double *rod, double *rodd,
                double *qua, double *quad, double *quadd, double *r, const int32_t *iptpn, const int32_t *ianpn,
                const int32_t *napt, const int32_t *iatan, const double *ra, int32_t maxsite, const double *masspt,
                const double *momp, const int32_t *nneighpn, const int32_t *jpnlist, int32_t maxnneigh,
                const double *ubuf, int32_t nbuf, const int32_t *iubuflow, const double *r2umin, double *utwob,
                double *virial)
{
    return velver_p_impl(NULL, NULL, nsteps, np, na, npt, nat, boxlen, rcut, tstep, nvvite, tvvite, ro, rod, rodd, qua,
                         quad, quadd, r, iptpn, ianpn, napt, iatan, ra, maxsite, masspt, momp, nneighpn, jpnlist,
                         maxnneigh, ubuf, nbuf, iubuflow, r2umin, utwob, virial);
}

/* The rigid-body step with the site Ewald sum in UTotal (lewald with polyatomic particles;
 * lewald 1: SPME with order, nmesh; 2: standard Ewald with ncut, ncutregion): the Ewald site forces join the pair forces before the forces, torques and molecular virial;
 * the reciprocal virial joins the virial; *urec = u%rec of the last step. */
int or_velver_p_ewald(int32_t nsteps, int32_t np, int32_t na, int32_t npt, int32_t nat, const double boxlen[3],
                      double rcut, double tstep, int32_t nvvite, double tvvite, double *ro, double *rod, double *rodd,
                      double *qua, double *quad, double *quadd, double *r, const int32_t *iptpn,
                      const int32_t *ianpn, const int32_t *napt, const int32_t *iatan, const double *ra,
                      int32_t maxsite, const double *masspt, const double *momp, const int32_t *nneighpn,
                      const int32_t *jpnlist, int32_t maxnneigh, const double *ubuf, int32_t nbuf,
                      const int32_t *iubuflow, const double *r2umin, const double *az, double ualpha,
                      int32_t lewald, int32_t ncut, int32_t ncutregion, int32_t order, int32_t nmesh, int32_t lsurf,
                      double epsfp, double *utwob, double *urec, double *virial)
{
    site_ew ew;
    ew.az = az;
    ew.ualpha = ualpha;
    ew.epsfp = epsfp;
    ew.lewald = lewald;
    ew.ncut = ncut;
    ew.ncutregion = ncutregion;
    ew.order = order;
    ew.nmesh = nmesh;
    ew.lsurf = lsurf;
    return velver_p_impl(&ew, urec, nsteps, np, na, npt, nat, boxlen, rcut, tstep, nvvite, tvvite, ro, rod, rodd, qua,
                         quad, quadd, r, iptpn, ianpn, napt, iatan, ra, maxsite, masspt, momp, nneighpn, jpnlist,
                         maxnneigh, ubuf, nbuf, iubuflow, r2umin, utwob, virial);
}

/* UEwald over the sites of polyatomic particles (Src/energy.F90:905-958): the standard
 * reciprocal sum over sites (UEwaldRecStd), UEwaldSelf's atomic and molecular parts
 * (Src/energy.F90:1301-1345: the intramolecular site pairs' erf(alpha r)/r, with
 * ErfLocal = Erf2) and the surface term when lsurf.  Sites r [na][3], charges az [na];
 * particles give the molecules (iptpn, ianpn, napt, 1-based).  force [na][3] is
 * overwritten with the Ewald forces (kJ/(mol A)); *urec = u%rec, *virrec its virial
 * (both scaled by EpsiFourPi as UEwald does). */
static int uewald_sites_impl(int32_t lewald, int32_t na, const double boxlen[3], double ualpha, int32_t ncut,
                             int32_t ncutregion, int32_t order, int32_t nmesh, int32_t lsurf, double epsfp,
                             const double *r, const double *az, int32_t np, const int32_t *iptpn,
                             const int32_t *ianpn, const int32_t *napt, double *force, double *urec, double *virrec)
{
    static const int32_t one = 1;
    static const double dummy_buf[12] = {0.0};
    or_params p;
    or_sys *s;
    int32_t *types = malloc(sizeof(int32_t) * (size_t)na);
    double mass = 1.0, r2u = 0.0, ua = 0.0, utot = 0.0, vir = 0.0;
    int ia, ip;
    for (ia = 0; ia < na; ++ia) types[ia] = 1;
    memset(&p, 0, sizeof(p));
    p.np = na;
    p.npt = 1;
    memcpy(p.boxlen, boxlen, sizeof(double) * 3);
    p.rcut = 1.0;
    p.iptpn = types;
    p.az = az;
    p.masspt = &mass;
    p.ubuf = dummy_buf;
    p.nbuf = 12;
    p.iubuflow = &one;
    p.r2umin = &r2u;
    p.r2atat = &r2u;
    p.lewald = lewald;
    p.lsurf = lsurf;
    p.ualpha = ualpha;
    p.epsi_four_pi = epsfp;
    p.maxnneigh = 1;
    p.ncut = ncut;
    p.ncutregion = ncutregion;
    p.order = order;
    p.nmesh = nmesh;
    s = or_create(&p);
    or_set_state(s, r, NULL, NULL);
    for (ia = 0; ia < 3 * na; ++ia) s->force[ia] = 0.0;
    uewald(s, &ua, &utot, &vir);          /* reciprocal sum, atomic self term, surface */
    /* UEwaldSelf, molecular contribution: every site pair inside a particle */
    {
        const double ewaldfac1 = (1.0 / (sqrt(Pi) * ualpha)) * 2.0 * (ualpha * ualpha);
        double umol = 0.0;
        for (ip = 0; ip < np; ++ip) {
            const int ialow = ianpn[ip] - 1, iaupp = ialow + napt[iptpn[ip] - 1] - 1;
            int i, j;
            for (i = ialow; i <= iaupp; ++i)
                for (j = i + 1; j <= iaupp; ++j) {
                    const double dx = r[3 * i] - r[3 * j], dy = r[3 * i + 1] - r[3 * j + 1],
                                 dz = r[3 * i + 2] - r[3 * j + 2];
                    const double r2 = dx * dx + dy * dy + dz * dz, r1 = sqrt(r2);
                    double r1i = 1.0 / r1, r2i = r1i * r1i, ex = exp(-(ualpha * ualpha) * r2), r3i, fac;
                    r1i = r1i * or_erf2(ualpha * r1);
                    r3i = r2i * (r1i - ewaldfac1 * ex);
                    umol = umol - (az[i] * az[j] * r1i);
                    fac = epsfp * az[i] * az[j] * r3i;
                    s->force[3 * i] -= fac * dx;
                    s->force[3 * i + 1] -= fac * dy;
                    s->force[3 * i + 2] -= fac * dz;
                    s->force[3 * j] += fac * dx;
                    s->force[3 * j + 1] += fac * dy;
                    s->force[3 * j + 2] += fac * dz;
                }
        }
        ua = ua + epsfp * umol;
    }
    memcpy(force, s->force, sizeof(double) * 3 * (size_t)na);
    *urec = ua;
    *virrec = vir;
    or_destroy(s);
    free(types);
    return 0;
}

int or_uewald_sites(int32_t na, const double boxlen[3], double ualpha, int32_t ncut, int32_t ncutregion,
                    int32_t lsurf, double epsfp, const double *r, const double *az, int32_t np,
                    const int32_t *iptpn, const int32_t *ianpn, const int32_t *napt, double *force, double *urec,
                    double *virrec)
{
    return uewald_sites_impl(2, na, boxlen, ualpha, ncut, ncutregion, 0, 0, lsurf, epsfp, r, az, np, iptpn, ianpn,
                             napt, force, urec, virrec);
}

/* The same with SPME over the sites (UEwaldRecSPM, Src/energy.F90:1207-1297: order, nmesh). */
int or_uewald_sites_spm(int32_t na, const double boxlen[3], double ualpha, int32_t order, int32_t nmesh,
                        int32_t lsurf, double epsfp, const double *r, const double *az, int32_t np,
                        const int32_t *iptpn, const int32_t *ianpn, const int32_t *napt, double *force,
                        double *urec, double *virrec)
{
    return uewald_sites_impl(1, na, boxlen, ualpha, 0, 0, order, nmesh, lsurf, epsfp, r, az, np, iptpn, ianpn, napt,
                             force, urec, virrec);
}

/* MCAllPass (Src/mc.F90:4024-4178), monoatomic, txbc 'xyz': per trial every particle in order
 * draws (Random - 1/2) dtranall(ipt) for x, y, z and the two numbers of GetRandomTrialOri
 * (Src/mc.F90:4583-4622, the orientation itself unused for points), is wrapped by PBC; the
 * list is rebuilt and UTotal evaluated; Metropolis on du%tot; rejection restores the
 * configuration.  u = [tot, twob(0..natat), rec, bond] of the current configuration. */
int or_mcall_pass(or_sys *s, int npass, const double *dtranall, double beta, double *u, int64_t *accepted)
{
    const int np = s->np, nu = s->natat + 4;
    double *save = malloc(sizeof(double) * 3 * (size_t)np), *unew = malloc(sizeof(double) * (size_t)nu);
    double *f = malloc(sizeof(double) * 3 * (size_t)np), *fo = malloc(sizeof(double) * 3 * (size_t)np), vir;
    int pass, ip, m, k, rc = 0;
    for (pass = 0; pass < npass && !rc; ++pass) {
        double dured;
        int accept;
        memcpy(save, s->ro, sizeof(double) * 3 * (size_t)np);
        for (ip = 0; ip < np; ++ip) {
            const double dt = dtranall[s->iptpn[ip] - 1];
            double d[3];
            for (m = 0; m < 3; ++m) d[m] = (mc_random(s) - 0.5) * dt;
            (void)mc_random(s);                  /* GetRandomTrialOri: iaxis */
            (void)mc_random(s);                  /* and drottemp */
            for (m = 0; m < 3; ++m)
                s->ro[3 * ip + m] = pbc1(s->ro[3 * ip + m] + d[m], s->boxlen2[m], s->boxlen[m], s->boxleni[m]);
        }
        rc = or_set_vlist(s);
        if (!rc) rc = or_utotal(s, f, fo, unew, &vir);
        if (rc) break;
        dured = (unew[0] - u[0]) * beta;
        if (dured > 87.0) {
            accept = 0;
        } else if (dured < -87.0) {
            accept = 1;
        } else {
            const double fac = exp(-dured);
            accept = (fac > 1.0) ? 1 : (fac > mc_random(s));
        }
        if (accept) {
            if (accepted) ++*accepted;
            for (k = 0; k < nu; ++k) u[k] = unew[k];
        } else {
            memcpy(s->ro, save, sizeof(double) * 3 * (size_t)np);
            rc = or_set_vlist(s);
        }
    }
    free(save); free(unew); free(f); free(fo);
    return rc;
}

/* MCPass with single-particle and chain moves: CallMove's selection (Src/mc.F90:669-708;
 * MCPass :1470-1582), SPartMove and ChainMove (:2541-2636), GetRandomTrialPos (:4527-4580):
 * a type with pspart >= 1 - 1e-15 makes single-particle moves only; otherwise Random picks
 * a single-particle move below pspart and a chain move below pchain (MOLSIM's cumulative
 * probabilities, [npt]).  A chain move translates the whole chain of the chosen particle by
 * one displacement of dtranchain(ipt).  Chains: nchain contiguous ranges (chain_first
 * 0-based, chain_len).  DUTotal over the moved set: pair differences between moved and fixed
 * particles (pairs inside the set are unchanged, Src/denergy.F90:728-800), the reciprocal
 * difference (standard Ewald with the layer correction, or SPME re-transformed), the surface
 * term, and every bond with a moved end.  u as in or_mc_pass.  Returns 6 for a move type
 * outside these two or a chain move of a particle in no chain. */
int or_mc_pass_moves(or_sys *s, int npass, int isamp, const double *dtran, const double *pspart,
                     const double *pchain, const double *dtranchain, int nchain, const int32_t *chain_first,
                     const int32_t *chain_len, double beta, double *u, int64_t *accepted, int64_t *hsreject)
{
    const int np = s->np, natat = s->natat, nc = s->ncut;
    const size_t w = (size_t)nc + 1;
    int *moved = calloc((size_t)np, sizeof(int)), *mv = malloc(sizeof(int) * (size_t)np);
    double *rtm = malloc(sizeof(double) * 3 * (size_t)np);
    double *dtwob = malloc(sizeof(double) * (natat + 1)), *unew = malloc(sizeof(double) * (natat + 1));
    double *uold = malloc(sizeof(double) * (natat + 1));
    cx *tm = NULL, *stm = NULL;                      /* standard Ewald: [nmv][3][w], trial sums */
    double *trigtm = NULL, *sttm = NULL;             /* layer correction */
    double *qm = NULL, *qmtm = NULL, *fq = NULL, urecold = 0.0, urecnew = 0.0;   /* SPME */
    int pass, ipass, k, m, rc = 0;
    if (s->lewald == 2) {
        tm = malloc(sizeof(cx) * 3 * w * (size_t)np);
        stm = malloc(sizeof(cx) * 4 * (size_t)(s->nkvec > 0 ? s->nkvec : 1));
        if (s->elc) {
            trigtm = malloc(sizeof(double) * 4 * w * (size_t)np);
            sttm = malloc(sizeof(double) * 8 * (size_t)(s->nkvec2d > 0 ? s->nkvec2d : 1));
        }
    } else if (s->lewald == 1) {
        const size_t n = (size_t)s->s * s->s * s->s;
        int ia;
        qm = calloc(n, sizeof(double));
        qmtm = malloc(sizeof(double) * n);
        fq = malloc(sizeof(double) * 2 * (size_t)(s->s / 2 + 1) * s->s * s->s);
        for (ia = 0; ia < np; ++ia) spm_stencil(s, qm, s->ro + 3 * ia, s->az[ia], 1.0);
        urecold = spm_mesh_energy(s, qm, fq);
    }
    for (pass = 0; pass < npass && !rc; ++pass) {
        for (ipass = 0; ipass < np && !rc; ++ipass) {
            int ip, ipt, nmv = 0, chain = 0, overlap = 0, a;
            double dtr, d[3], dutot = 0.0, durec = 0.0, dubond = 0.0, dured;
            ip = (isamp == 0) ? ipass + 1 : 1 + (int)(np * mc_random(s));
            ip = (ip < 1 ? 1 : (ip > np ? np : ip)) - 1;
            ipt = s->iptpn[ip] - 1;
            if (!(pspart[ipt] > 1.0 - 1e-15)) {
                const double pr = mc_random(s);
                if (pr < pspart[ipt]) chain = 0;
                else if (pr < pchain[ipt]) chain = 1;
                else { rc = 6; break; }
            }
            if (chain) {
                int c, found = -1;
                for (c = 0; c < nchain; ++c)
                    if (ip >= chain_first[c] && ip < chain_first[c] + chain_len[c]) found = c;
                if (found < 0) { rc = 6; break; }
                for (a = 0; a < chain_len[found]; ++a) mv[nmv++] = chain_first[found] + a;
                dtr = dtranchain[ipt];
            } else {
                mv[nmv++] = ip;
                dtr = dtran[ipt];
            }
            /* GetRandomTrialPos: one displacement for the moved set */
            if (dtr >= 0.0) {
                for (m = 0; m < 3; ++m) d[m] = (mc_random(s) - 0.5) * dtr;
            } else {
                for (;;) {
                    for (m = 0; m < 3; ++m) d[m] = mc_random(s) - 0.5;
                    if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < 0.25) break;
                }
                for (m = 0; m < 3; ++m) d[m] = d[m] * fabs(dtr);
            }
            for (a = 0; a < nmv; ++a) {
                const int i = mv[a];
                moved[i] = 1;
                for (m = 0; m < 3; ++m)
                    rtm[3 * a + m] = pbc1(s->ro[3 * i + m] + d[m], s->boxlen2[m], s->boxlen[m], s->boxleni[m]);
            }
            /* DUTwoBody: moved against fixed particles; the new configuration first, with its checks */
            for (k = 0; k <= natat; ++k) unew[k] = uold[k] = 0.0;
            for (a = 0; a < nmv && !overlap; ++a) {
                const int i = mv[a], it = s->iptpn[i];
                int jp;
                for (jp = 0; jp < np; ++jp) {
                    double dx, dy, dz, r2;
                    int ij;
                    if (moved[jp]) continue;
                    dx = rtm[3 * a] - s->ro[3 * jp];
                    dy = rtm[3 * a + 1] - s->ro[3 * jp + 1];
                    dz = rtm[3 * a + 2] - s->ro[3 * jp + 2];
                    r2 = pbcr2(s, &dx, &dy, &dz);
                    if (!(r2 < s->rcut2)) continue;
                    ij = pair_index(s->npt, it, s->iptpn[jp]);
                    if (r2 < s->r2atat[ij - 1] || r2 < s->r2umin[ij - 1]) { overlap = 1; break; }
                    unew[ij] += tab_u(s, ij - 1, r2);
                }
            }
            if (overlap) {
                if (hsreject) ++*hsreject;
                for (a = 0; a < nmv; ++a) moved[mv[a]] = 0;
                continue;                            /* Metropolis: imchsreject, no random number */
            }
            for (a = 0; a < nmv; ++a) {
                const int i = mv[a], it = s->iptpn[i];
                int jp;
                for (jp = 0; jp < np; ++jp) {
                    double dx, dy, dz, r2;
                    int ij;
                    if (moved[jp]) continue;
                    dx = s->ro[3 * i] - s->ro[3 * jp];
                    dy = s->ro[3 * i + 1] - s->ro[3 * jp + 1];
                    dz = s->ro[3 * i + 2] - s->ro[3 * jp + 2];
                    r2 = pbcr2(s, &dx, &dy, &dz);
                    if (!(r2 < s->rcut2)) continue;
                    ij = pair_index(s->npt, it, s->iptpn[jp]);
                    uold[ij] += tab_u(s, ij - 1, r2);
                }
            }
            for (k = 1; k <= natat; ++k) { unew[0] += unew[k]; uold[0] += uold[k]; }
            for (k = 0; k <= natat; ++k) dtwob[k] = unew[k] - uold[k];
            dutot = dtwob[0];
            /* DUTwoBodyEwald */
            if (s->lewald == 2) {
                const int ncut2 = s->ncut2;
                const cx *S4 = (const cx *)s->sumeikr;
                double tpbi[3];
                int nx, ny, nz, kn = 0, icut;
                for (m = 0; m < 3; ++m) tpbi[m] = 2.0 * Pi * s->boxleni[m];
                for (a = 0; a < nmv; ++a)                /* EwaldSetArrayTM per moved particle */
                    for (m = 0; m < 3; ++m) {
                        cx *t = tm + ((size_t)a * 3 + m) * w;
                        t[0].r = 1.0; t[0].i = 0.0;
                        if (nc >= 1) {
                            t[1].r = cos(tpbi[m] * rtm[3 * a + m]);
                            t[1].i = sin(tpbi[m] * rtm[3 * a + m]);
                        }
                        for (icut = 2; icut <= nc; ++icut) t[icut] = cmul(t[icut - 1], t[1]);
                    }
                for (nz = 0; nz <= nc; ++nz)
                    for (ny = 0; ny <= nc; ++ny) {
                        if (ny * ny + nz * nz > ncut2) continue;
                        for (nx = 0; nx <= nc; ++nx) {
                            cx *st = stm + 4 * (size_t)kn;
                            const cx *so = S4 + 4 * (size_t)kn;
                            double termnew, termold;
                            if (nx * nx + ny * ny + nz * nz > ncut2) continue;
                            if (nx == 0 && ny == 0 && nz == 0) continue;
                            for (k = 0; k < 4; ++k) st[k] = so[k];
                            for (a = 0; a < nmv; ++a) {
                                const int i = mv[a];
                                const double q = s->az[i];
                                const cx *ex = (const cx *)s->eik[0] + (size_t)i * w;
                                const cx *ey = (const cx *)s->eik[1] + (size_t)i * w;
                                const cx *ez = (const cx *)s->eik[2] + (size_t)i * w;
                                const cx *tx = tm + ((size_t)a * 3) * w, *ty = tx + w, *tz = tx + 2 * w;
                                cx yc, yct, yzm, yzp, yzmt, yzpt, xo = ex[nx], xt = tx[nx], xoc, xtc, p, o;
                                yc.r = ey[ny].r; yc.i = -ey[ny].i;
                                yzm = cmul(yc, ez[nz]);
                                yzp = cmul(ey[ny], ez[nz]);
                                yct.r = ty[ny].r; yct.i = -ty[ny].i;
                                yzmt = cmul(yct, tz[nz]);
                                yzpt = cmul(ty[ny], tz[nz]);
                                xoc.r = xo.r; xoc.i = -xo.i;
                                xtc.r = xt.r; xtc.i = -xt.i;
                                p = cmul(xtc, yzmt); o = cmul(xoc, yzm);
                                st[0].r += q * (p.r - o.r); st[0].i += q * (p.i - o.i);
                                p = cmul(xtc, yzpt); o = cmul(xoc, yzp);
                                st[1].r += q * (p.r - o.r); st[1].i += q * (p.i - o.i);
                                p = cmul(xt, yzmt); o = cmul(xo, yzm);
                                st[2].r += q * (p.r - o.r); st[2].i += q * (p.i - o.i);
                                p = cmul(xt, yzpt); o = cmul(xo, yzp);
                                st[3].r += q * (p.r - o.r); st[3].i += q * (p.i - o.i);
                            }
                            termnew = termold = 0.0;
                            for (k = 0; k < 4; ++k) {
                                termnew += st[k].r * st[k].r + st[k].i * st[k].i;
                                termold += so[k].r * so[k].r + so[k].i * so[k].i;
                            }
                            durec += s->kfac[kn] * (termnew - termold);
                            ++kn;
                        }
                    }
                if (s->elc) {                            /* DUTwoBodyEwaldRec2dlc over the moved set */
                    for (a = 0; a < nmv; ++a) {
                        double *t = trigtm + (size_t)a * 4 * w;
                        for (m = 0; m < 4; ++m) t[m * w] = 1.0;
                        if (nc >= 1) {
                            t[1] = sin(tpbi[0] * rtm[3 * a]);
                            t[w + 1] = cos(tpbi[0] * rtm[3 * a]);
                            t[2 * w + 1] = sin(tpbi[1] * rtm[3 * a + 1]);
                            t[3 * w + 1] = cos(tpbi[1] * rtm[3 * a + 1]);
                        }
                        for (icut = 2; icut <= nc; ++icut) {
                            t[icut] = t[icut - 1] * t[w + 1] + t[w + icut - 1] * t[1];
                            t[w + icut] = t[w + icut - 1] * t[w + 1] - t[icut - 1] * t[1];
                            t[2 * w + icut] = t[2 * w + icut - 1] * t[3 * w + 1] + t[3 * w + icut - 1] * t[2 * w + 1];
                            t[3 * w + icut] = t[3 * w + icut - 1] * t[3 * w + 1] - t[2 * w + icut - 1] * t[2 * w + 1];
                        }
                    }
                    kn = 0;
                    for (ny = 0; ny <= nc; ++ny)
                        for (nx = 0; nx <= nc; ++nx) {
                            const double kx = nx * tpbi[0], ky = ny * tpbi[1];
                            double kp, tn, to_, *st = sttm + 8 * (size_t)kn;
                            const double *so = s->sumtrig + 8 * (size_t)kn;
                            if (nx * nx + ny * ny > s->ncut2d2) continue;
                            if (nx == 0 && ny == 0) continue;
                            kp = sqrt(kx * kx + ky * ky);
                            for (k = 0; k < 8; ++k) st[k] = so[k];
                            for (a = 0; a < nmv; ++a) {
                                const int i = mv[a];
                                const double q = s->az[i], *tt = trigtm + (size_t)a * 4 * w;
                                const double *to = s->trig2d + (size_t)i * 4 * w;
                                double e = exp(kp * rtm[3 * a + 2]), ei = 1.0 / e;
                                const double sht = 0.5 * (e - ei), cht = 0.5 * (e + ei);
                                double sho, cho;
                                e = exp(kp * s->ro[3 * i + 2]); ei = 1.0 / e;
                                sho = 0.5 * (e - ei); cho = 0.5 * (e + ei);
                                st[0] += q * (tt[nx] * tt[2 * w + ny] * sht - to[nx] * to[2 * w + ny] * sho);
                                st[1] += q * (tt[w + nx] * tt[2 * w + ny] * sht - to[w + nx] * to[2 * w + ny] * sho);
                                st[2] += q * (tt[nx] * tt[3 * w + ny] * sht - to[nx] * to[3 * w + ny] * sho);
                                st[3] += q * (tt[w + nx] * tt[3 * w + ny] * sht - to[w + nx] * to[3 * w + ny] * sho);
                                st[4] += q * (tt[nx] * tt[2 * w + ny] * cht - to[nx] * to[2 * w + ny] * cho);
                                st[5] += q * (tt[w + nx] * tt[2 * w + ny] * cht - to[w + nx] * to[2 * w + ny] * cho);
                                st[6] += q * (tt[nx] * tt[3 * w + ny] * cht - to[nx] * to[3 * w + ny] * cho);
                                st[7] += q * (tt[w + nx] * tt[3 * w + ny] * cht - to[w + nx] * to[3 * w + ny] * cho);
                            }
                            tn = -st[0] * st[0] - st[1] * st[1] - st[2] * st[2] - st[3] * st[3] +
                                 st[4] * st[4] + st[5] * st[5] + st[6] * st[6] + st[7] * st[7];
                            to_ = -so[0] * so[0] - so[1] * so[1] - so[2] * so[2] - so[3] * so[3] +
                                  so[4] * so[4] + so[5] * so[5] + so[6] * so[6] + so[7] * so[7];
                            durec += s->kfac2d[kn] * (tn - to_);
                            ++kn;
                        }
                }
            } else if (s->lewald == 1) {
                memcpy(qmtm, qm, sizeof(double) * (size_t)s->s * s->s * s->s);
                for (a = 0; a < nmv; ++a) {
                    spm_stencil(s, qmtm, s->ro + 3 * mv[a], s->az[mv[a]], -1.0);
                    spm_stencil(s, qmtm, rtm + 3 * a, s->az[mv[a]], 1.0);
                }
                urecnew = spm_mesh_energy(s, qmtm, fq);
                durec = urecnew - urecold;
            }
            if (s->lewald) {
                if (s->lsurf) {                          /* DUTwoBodyEwaldSurf */
                    double M[3] = {0.0, 0.0, 0.0}, T[3];
                    int ia;
                    for (ia = 0; ia < np; ++ia)
                        for (m = 0; m < 3; ++m) M[m] += s->az[ia] * s->ro[3 * ia + m];
                    for (m = 0; m < 3; ++m) {
                        T[m] = M[m];
                        for (a = 0; a < nmv; ++a) T[m] += s->az[mv[a]] * (rtm[3 * a + m] - s->ro[3 * mv[a] + m]);
                    }
                    if (s->elc)
                        durec += (2.0 * Pi / s->vol) * (T[2] * T[2] - M[2] * M[2]);
                    else
                        durec += 2.0 * Pi / (3.0 * s->vol) *
                                 ((T[0] * T[0] + T[1] * T[1] + T[2] * T[2]) - (M[0] * M[0] + M[1] * M[1] + M[2] * M[2]));
                }
                durec = s->epsfp * durec;
                dutot += durec;
            }
            /* DUBond: every bond with a moved end, once */
            if (s->nbond > 0) {
                int b;
                for (b = 0; b < s->nbond; ++b) {
                    const int a1 = s->bond_ij[2 * b] - 1, a2 = s->bond_ij[2 * b + 1] - 1;
                    double r1[3], r2v[3], dx, dy, dz, r2n, r2o, xn, xo, pn = 1.0, po = 1.0;
                    int e, la;
                    if (!moved[a1] && !moved[a2]) continue;
                    for (m = 0; m < 3; ++m) { r1[m] = s->ro[3 * a1 + m]; r2v[m] = s->ro[3 * a2 + m]; }
                    for (la = 0; la < nmv; ++la) {
                        if (mv[la] == a1) for (m = 0; m < 3; ++m) r1[m] = rtm[3 * la + m];
                        if (mv[la] == a2) for (m = 0; m < 3; ++m) r2v[m] = rtm[3 * la + m];
                    }
                    dx = r1[0] - r2v[0]; dy = r1[1] - r2v[1]; dz = r1[2] - r2v[2];
                    r2n = pbcr2(s, &dx, &dy, &dz);
                    dx = s->ro[3 * a1] - s->ro[3 * a2]; dy = s->ro[3 * a1 + 1] - s->ro[3 * a2 + 1];
                    dz = s->ro[3 * a1 + 2] - s->ro[3 * a2 + 2];
                    r2o = pbcr2(s, &dx, &dy, &dz);
                    xn = sqrt(r2n) - s->bond_eq[b];
                    xo = sqrt(r2o) - s->bond_eq[b];
                    for (e = 0; e < s->bond_p[b]; ++e) { pn *= xn; po *= xo; }
                    dubond += s->bond_k[b] * (pn - po);
                }
                dutot += dubond;
            }
            /* Metropolis, then MCUpdate */
            dured = dutot * beta;
            {
                int accept;
                if (dured > 87.0) accept = 0;
                else if (dured < -87.0) accept = 1;
                else {
                    const double fac = exp(-dured);
                    accept = (fac > 1.0) ? 1 : (fac > mc_random(s));
                }
                if (accept) {
                    if (accepted) ++*accepted;
                    u[0] += dutot;
                    for (k = 0; k <= natat; ++k) u[1 + k] += dtwob[k];
                    if (s->lewald) u[2 + natat] += durec;
                    if (s->nbond > 0) u[3 + natat] += dubond;
                    for (a = 0; a < nmv; ++a) {
                        const int i = mv[a];
                        if (s->lewald == 2) {
                            for (m = 0; m < 3; ++m)
                                memcpy((cx *)s->eik[m] + (size_t)i * w, tm + ((size_t)a * 3 + m) * w, sizeof(cx) * w);
                            if (s->elc) memcpy(s->trig2d + (size_t)i * 4 * w, trigtm + (size_t)a * 4 * w, sizeof(double) * 4 * w);
                        }
                        for (m = 0; m < 3; ++m) {
                            s->drostep[3 * i + m] += d[m];
                            s->ro[3 * i + m] = rtm[3 * a + m];
                        }
                    }
                    if (s->lewald == 2) {
                        memcpy(s->sumeikr, stm, sizeof(cx) * 4 * (size_t)s->nkvec);
                        if (s->elc) memcpy(s->sumtrig, sttm, sizeof(double) * 8 * (size_t)s->nkvec2d);
                    } else if (s->lewald == 1) {
                        double *t_ = qm;
                        qm = qmtm;
                        qmtm = t_;
                        urecold = urecnew;
                    }
                }
            }
            for (a = 0; a < nmv; ++a) moved[mv[a]] = 0;
        }
    }
    free(moved); free(mv); free(rtm); free(dtwob); free(unew); free(uold);
    free(tm); free(stm); free(trigtm); free(sttm); free(qm); free(qmtm); free(fq);
    return rc;
}

// setup.cpp -- host set-up of the B200 path: MOLSIM's pair table, Ewald alpha
// and SPME influence factors, in FP64.  These run once per system, before any
// kernel; the table format and the adaptive interval search are a contract
// with MOLSIM (a Fortran caller hands its own `ubuf` to msg_create), so they
// follow the reference's steps.
#include "setup.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

namespace msg {

static const double kPi = 3.1415926535897932;   // Src/mol.F90:63

// MOLSIM's Erf2 (Src/mollib.F90:215-274), a Chebyshev expansion (NAG Mark 4).
// Its second branch starts from c(18), runs j = 16..2 and ends with c(1):
// c(17) does not enter the sum.
double erf_molsim(double x)
{
    static const double c[19] = {0.0,
        1.9449071068178803, 4.20186582324414e-2, -1.86866103976769e-2, 5.1281061839107e-3,
        -1.0683107461726e-3, 1.744737872522e-4, -2.15642065714e-5, 1.7282657974e-6,
        -2.00479241e-8, -1.64782105e-8, 2.0008475e-9, 2.57716e-11, -3.06343e-11, 1.9158e-12,
        3.703e-13, -5.43e-14, -4.0e-15, 1.2e-15};
    static const double d[18] = {0.0,
        1.4831105640848036, -3.010710733865950e-1, 6.89948306898316e-2, -1.39162712647222e-2,
        2.4207995224335e-3, -3.658639685849e-4, 4.86209844323e-5, -5.7492565580e-6,
        6.113243578e-7, -5.89910153e-8, 5.2070091e-9, -4.232976e-10, 3.18811e-11,
        -2.2361e-12, 1.467e-13, -9.0e-15, 5.0e-16};
    const double av = std::fabs(x);
    if (av <= 2.0) {
        const double t = x * x - 2.0;
        double b2 = 0.0, b1 = d[17], b0 = 0.0;
        for (int j = 16; j >= 2; --j) {
            b0 = t * b1 - b2 + d[j];
            b2 = b1;
            b1 = b0;
        }
        b0 = t * b1 - b2 + d[1];
        return 0.5 * (b0 - b2) * x;
    }
    if (av < 6.25) {
        const double t = 2.0 - 20.0 / (av + 3.0);
        double b2 = 0.0, b1 = c[18], b0 = 0.0;
        for (int j = 16; j >= 2; --j) {
            b0 = t * b1 - b2 + c[j];
            b2 = b1;
            b1 = b0;
        }
        b0 = t * b1 - b2 + c[1];
        const double tail = 0.5 * (b0 - b2) / av * std::exp(-x * x) / 1.7724538509055160;
        return (1.0 - tail) * (x >= 0.0 ? 1.0 : -1.0);
    }
    return x >= 0.0 ? 1.0 : -1.0;
}

// u(r), u'(r), u''(r) of the (1,6,12) potential with erfc-screened Coulomb and
// optional cut-and-shift LJ (Pot_1_6_12 + CalcEwaldUfac, Src/potential.F90:1384-1419,
// 2938-2960).  Types are 0-based here.
static void pot_1_6_12(const msg_tab_params &p, int it, int jt, double r1, double &u0, double &u1,
                       double &u2)
{
    const double qq = p.zat[it] * p.zat[jt] * p.epsi_four_pi;
    const double sig = 0.5 * (p.sigat[it] + p.sigat[jt]);
    const double eps = std::sqrt(p.epsat[it] * p.epsat[jt]);
    const double r1i = 1.0 / r1;
    const double sr = sig * r1i, sr3 = sr * sr * sr, fac = sr3 * sr3;
    double c0 = 1.0, c1 = 1.0, c2 = 1.0;
    if (p.lewald) {
        const double ra = p.ualpha * r1, er = erf_molsim(ra);
        const double ex = 1.12837916709 * std::exp(-(ra * ra));
        c0 = 1.0 - er;
        c1 = 1.0 - (er - ra * ex);
        c2 = 1.0 - (er - ra * (1.0 + ra * ra) * ex);
    }
    double s0 = 4.0 * eps * (fac * fac - fac);
    double s1 = -(24.0 * eps * (2.0 * (fac * fac) - fac) * r1i);
    double s2 = 24.0 * eps * (26.0 * (fac * fac) - 7.0 * fac) * (r1i * r1i);
    if (p.lljcut) {
        if (r1 < p.ljrcut * sig) {
            s0 = s0 + p.ljushift * eps;
        } else {
            s0 = s1 = s2 = 0.0;
        }
    }
    u0 = qq * c0 * r1i + s0;
    u1 = -(qq * c1 * (r1i * r1i)) + s1;
    u2 = 2.0 * qq * c2 * (r1i * r1i * r1i) + s2;
}

// Quintic in z = r^2 matching w, w', w'' at both ends (SetUBuffer,
// Src/potential.F90:1139-1220; Andrea, Swope, Andersen, JCP 79, 4576 (1983)).
static void quintic(double zl, double u0l, double u1l, double u2l, double zu, double u0u, double u1u,
                    double u2u, double *t)
{
    if (u0l == 0.0 && u0u == 0.0) {
        t[0] = zl;
        for (int k = 1; k < 12; ++k) t[k] = 0.0;
        return;
    }
    const double rl = std::sqrt(zl), ru = std::sqrt(zu);
    const double dz1 = zu - zl, dz2 = dz1 * dz1, dz3 = dz2 * dz1;
    const double w1l = 0.50 * u1l / rl, w1u = 0.50 * u1u / ru;
    const double w2l = 0.25 * (u2l - u1l / rl) / zl, w2u = 0.25 * (u2u - u1u / ru) / zu;
    const double a = 6.0 * (u0u - u0l - w1l * dz1 - 0.5 * w2l * dz2) / dz3;
    const double b = 2.0 * (w1u - w1l - w2l * dz1) / dz2;
    const double c = (w2u - w2l) / dz1;
    t[0] = zl;
    t[1] = u0l;
    t[2] = w1l;
    t[3] = 0.5 * w2l;
    t[4] = (10.0 * a - 12.0 * b + 3.0 * c) / (6.0);
    t[5] = (-15.0 * a + 21.0 * b - 6.0 * c) / (6.0 * dz1);
    t[6] = (2.0 * a - 3.0 * b + c) / (2.0 * dz2);
    t[7] = -2.0 * t[2];
    t[8] = -4.0 * t[3];
    t[9] = -6.0 * t[4];
    t[10] = -8.0 * t[5];
    t[11] = -10.0 * t[6];
}

// Accuracy of one interval at 11 points (CheckUBuffer, Src/potential.F90:1224-1258).
static void check_interval(const msg_tab_params &p, int it, int jt, double rl, double ru, const double *t,
                           bool &ok, bool &repul)
{
    ok = false;
    repul = false;
    const double dr = (ru - rl) / 10;
    for (int k = 1; k <= 11; ++k) {
        const double r1 = rl + dr * (k - 1);
        double u0, u1, u2;
        pot_1_6_12(p, it, jt, r1, u0, u1, u2);
        const double dz = r1 * r1 - rl * rl;
        const double us = t[1] + dz * (t[2] + dz * (t[3] + dz * (t[4] + dz * (t[5] + dz * t[6]))));
        double fs = t[7] + dz * (t[8] + dz * (t[9] + dz * (t[10] + dz * t[11])));
        fs = r1 * fs;
        if (std::fabs(us - u0) > p.utoltab) return;
        if (std::fabs(fs + u1) > p.ftoltab) return;
        if (std::fabs(us) > p.umaxtab) repul = true;
        if (std::fabs(fs) > p.fmaxtab) repul = true;
    }
    ok = true;
}

}  // namespace msg

extern "C" double msg_rcut_to_alpha(double uewaldtol, double q2sum, double epsi_four_pi,
                                    double boxlenshort, double rcut, int32_t *status)
{
    // RcutToAlpha (Src/energy.F90:7090-7105), Kolafa-Perram fixed point.
    const double br = boxlenshort * rcut;
    const double y = (uewaldtol / (q2sum * epsi_four_pi)) * std::sqrt(2.0 * (br * br * br));
    double xold = 1.0e-1, xnew = 0.0;
    int i;
    for (i = 1; i <= 40; ++i) {
        xnew = (1.0 / rcut) * std::sqrt(-std::log(y * (xold * xold)));
        if (std::fabs(xold - xnew) / xnew < 1.0e-6) break;
        xold = xnew;
    }
    if (status) *status = (i > 40) ? MSG_ERR_ARG : MSG_OK;
    return xnew;
}

extern "C" int32_t msg_alpha_to_ncut(double uewaldtol, double q2sum, double epsi_four_pi, double boxlenshort,
                                     double ualpha, int32_t *status)
{
    // AlphaToNcut (Src/energy.F90:7066-7081): the k-space cut of the standard Ewald
    // sum from the Kolafa-Perram estimate of its error at uewaldtol.
    const double y = (uewaldtol / (q2sum * epsi_four_pi)) * (msg::kPi * msg::kPi / ((ualpha * ualpha) * boxlenshort));
    double xold = 1.0, xnew = 0.0;
    int i;
    for (i = 1; i <= 40; ++i) {
        xnew = (ualpha * boxlenshort / msg::kPi) *
               std::sqrt(-std::log(y * xold / (1.0 + 1.0 / (ualpha * boxlenshort * std::sqrt(xold)))));
        if (std::fabs(xold - xnew) / xnew < 1.0e-6) break;
        xold = xnew;
    }
    if (status) *status = (i > 40) ? MSG_ERR_ARG : MSG_OK;
    return (int32_t)(xnew + 1.0);
}

extern "C" int msg_pot_tab(const msg_tab_params *p, double *ubuf, int32_t nbuf, int32_t *iubuflow,
                           int32_t *nugrid, double *r2umin, int32_t *nused)
{
    // PotTwoBodyTab1/2/3 (Src/potential.F90:868-1135): tables from rumax down to
    // rumin, widening dr after each accepted interval and shrinking it by 0.9
    // until the interval passes the 11-point check.
    if (!p || !ubuf || p->npt < 1 || p->npt > 4) return MSG_ERR_ARG;
    std::memset(ubuf, 0, sizeof(double) * (size_t)nbuf);
    int ibuf = 1, pidx = 0;
    for (int it = 0; it < p->npt; ++it)
        for (int jt = it; jt < p->npt; ++jt, ++pidx) {
            double r2umax = p->rumaxfac * (p->rcut + 0.0 + 0.0);
            r2umax = r2umax * r2umax;
            const double rumax = std::sqrt(r2umax);
            double rumin = std::sqrt(p->r2uminin);
            iubuflow[pidx] = ibuf;
            double rupp = rumax, dr = 0.5 * (rumax - rumin), rlow = 0.0;
            int igrid;
            for (igrid = 1; igrid <= 1200; ++igrid) {
                const double zupp = rupp * rupp;
                double t[12];
                bool ok = false, repul = false;
                int idr;
                for (idr = 1; idr <= 100; ++idr) {
                    rlow = std::fmax(rumin, rupp - dr);
                    const double zlow = rlow * rlow;
                    double a0, a1, a2, b0, b1, b2;
                    msg::pot_1_6_12(*p, it, jt, rlow, a0, a1, a2);
                    msg::pot_1_6_12(*p, it, jt, rupp, b0, b1, b2);
                    msg::quintic(zlow, a0, a1, a2, zupp, b0, b1, b2, t);
                    msg::check_interval(*p, it, jt, rlow, rupp, t, ok, repul);
                    if (ok) {
                        rupp = rlow;
                        if (p->lljcut) dr = 2.0 * dr;
                        break;
                    }
                    dr = dr * 0.9;
                }
                if (idr > 100) return MSG_ERR_ARG;
                if (ibuf + 11 > nbuf) return MSG_ERR_CAPACITY;
                for (int k = 0; k < 12; ++k) ubuf[ibuf - 1 + k] = t[k];
                ibuf += 12;
                if (repul) rumin = rlow;
                if (rlow <= rumin) break;
                if (repul) break;
            }
            if (igrid > 1200) return MSG_ERR_ARG;
            if (nugrid) nugrid[pidx] = igrid;
            r2umin[pidx] = rumin * rumin;
        }
    if (nused) *nused = ibuf - 1;
    return MSG_OK;
}

namespace msg {

// SPME influence factors (EwaldSetup SPM branch, Src/energy.F90:6980-7018) on
// the folded half grid (s/2+1)^3, x fastest:
//   mfac = 4 pi/V exp(-k^2/4a^2)/k^2 * b2x b2y b2z       (meshfac)
//   emf  = mfac * (1/2 at kx = 0, s/2)                    (energy weight per r2c entry)
//   vmf  = (1 - 2 k^2/4a^2) * emf                          (virial weight per r2c entry)
// The reference halves energyfac also for ky, kz in {0, s/2} and visits those
// entries twice through its mirror loop; per distinct entry the weight is the
// unhalved value, which is what emf/vmf hold.  b^2 uses a single-precision
// phase, as the reference's cmplx() without a kind does; for odd orders the
// Nyquist modulus (where the sum vanishes and the reference leaves b2 unset)
// is defined as zero.
void spme_factors(int s, int order, double alpha, const double box[3], double *mfac, double *emf, double *vmf)
{
    std::vector<double> spl(order), b2(3 * (size_t)s);
    {
        // CardinalBSpline(order, 0): values(k) = M_order(k)
        std::vector<double> v(order, 0.0), last(order, 0.0);
        v[0] = 0.0;
        if (order > 1) v[1] = 1.0;
        for (int n = 3; n <= order; ++n) {
            last = v;
            v[0] = 0.0 * last[0] / (n - 1);
            for (int i = 1; i <= n - 2; ++i) {
                const double a = i + 0.0;
                v[i] = (a * last[i] + (n - a) * last[i - 1]) / (n - 1);
            }
            v[n - 1] = (1 - 0.0) * last[n - 2] / (n - 1);
        }
        spl = v;
    }
    const double TwoPi = 2.0 * kPi;
    for (int d = 0; d < 3; ++d)
        for (int m = 0; m < s; ++m) {
            if ((order % 2 == 1) && (2 * m == s)) {
                b2[d * s + m] = 0.0;
                continue;
            }
            std::complex<double> a(0.0, 0.0);
            for (int k = 0; k <= order - 2; ++k) {
                const float ang = (float)(TwoPi * m * k / s);
                const std::complex<float> e = std::exp(std::complex<float>(0.0f, ang));
                a = a + spl[k + 1] * std::complex<double>(e.real(), e.imag());
            }
            b2[d * s + m] = 1.0 / (a.real() * a.real() + a.imag() * a.imag());
        }
    const double vol = box[0] * box[1] * box[2];
    const double tpb[3] = {TwoPi * (1.0 / box[0]), TwoPi * (1.0 / box[1]), TwoPi * (1.0 / box[2])};
    const double fac0 = 4.0 * kPi / vol, expf = -1.0 / (4.0 * (alpha * alpha));
    const int h = s / 2 + 1;
    for (int nz = 0; nz < h; ++nz)
        for (int ny = 0; ny < h; ++ny)
            for (int nx = 0; nx < h; ++nx) {
                const size_t idx = nx + (size_t)h * (ny + (size_t)h * nz);
                if (nx == 0 && ny == 0 && nz == 0) {
                    mfac[idx] = emf[idx] = vmf[idx] = 0.0;
                    continue;
                }
                const double kx = nx * tpb[0], ky = ny * tpb[1], kz = nz * tpb[2];
                const double m2 = kx * kx + ky * ky + kz * kz;
                const double c = std::exp(m2 * expf) / m2;
                const double mf = fac0 * c * b2[nx] * b2[s + ny] * b2[2 * s + nz];
                mfac[idx] = mf;
                const double e = (nx == 0 || 2 * nx == s) ? mf / 2 : mf;
                emf[idx] = e;
                vmf[idx] = (1.0 + 2 * m2 * expf) * e;
            }
}

}  // namespace msg

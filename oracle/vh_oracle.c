/*
 * vh_oracle.c -- TEST INFRASTRUCTURE ONLY: CPU restatement of the cpu-vh hot
 * path (Kurganov-Tadmor RK2 step, inference, regulation, ghost cells) used as
 * the parity checker for the CUDA implementation and as the "port" CPU
 * baseline.  It is never linked into, or called by, the product.
 *
 * Every function restates one reference function in plain C, in the same
 * floating-point operation order (built with -ffp-contract=off so that no
 * multiply-add is fused), calling the same libm functions.  Citations are
 * file:line in derekeverett/cpu-vh.  Parity of this file against the
 * reference's own sources (oracle/_ref) is checked bit for bit by
 * tests/test_oracle_vs_reference.py.
 *
 * Lattice layout: padded SoA arrays of ncx*ncy*ncz doubles, index
 * i + ncx*(j + ncy*k) (DynamicalVariables.cpp:35-41), two ghost cells a side.
 *
 * The per-cell loops run under OpenMP (each cell writes only itself, so the
 * results do not depend on the thread count); error flags are reduced.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAXQ 15
#define HBARC 0.197326938

typedef struct {
    int nx, ny, nz, nq, bulk;          /* nq = 14 (shear) or 15 (shear + bulk) */
    int ncx, ncy, ncz;
    double dx, dy, dz, dt, t0, etabar, theta;
    int eos_table;                      /* 0 conformal, 1 tabulated */
    double eos_a;                       /* conformal e = a T^4 */
    double T_reg_GeV, T_fo_GeV;
    int fofac;
    /* tabulated EoS in fm units, as EquationOfState.cpp:292-327 stores it */
    int e_length;
    double e_min, e_max, e_spacing;
    double *p_tb, *T_tb;
    int zeta_law;                       /* 0: SourceTerms.cpp:40-48, 1: Gaussian in T[GeV] */
    double zeta_norm, zeta_T0, zeta_w;
    /* state */
    double *q[MAXQ], *Q[MAXQ], *qS[MAXQ];
    double *e, *p;
    double *u[4], *up[4], *uS[4];
    int n;                              /* completed steps */
    double t;
    double e_reg;
    int nan_flag;
    /* freezeout slabs: 2 x [11][N] (e, ux, uy, un, e, pixx, pixy, pixn, piyy, piyn, Pi) */
    double *slab[2];
    int fo_prev;
    /* thermal vorticity (allocated by the first vho_vorticity): wtx wty wtn wxy wxn wyn, beta t x y n */
    double *w[6], *beta[4];
    /* dynamical sources (vho_set_sources): t, x, y, eta components, padded; NULL when none */
    double *src[4];
    /* regulation factors of the last stage (regFacShear, regFacBulk), allocated by the first step */
    double *regfac[2];
} vho_t;

/* ------------------------------------------------------------------ EoS */
/* EquationOfState.cpp:329-360 */
static double interp1d(const vho_t *h, double ed, const double *table)
{
    double local_ed = ed;
    const double e0 = h->e_min;
    const double delta_e = h->e_spacing;
    const int N_e = h->e_length;
    int idx_e = (int)((local_ed - e0) / delta_e);
    if (idx_e > N_e - 2) idx_e = N_e - 2;
    if (idx_e < 0) idx_e = 0;
    const double frac_e = (local_ed - (idx_e * delta_e + e0)) / delta_e;
    double temp1 = table[idx_e];
    double temp2 = table[idx_e + 1];
    return temp1 * (1. - frac_e) + temp2 * frac_e;
}
static double dmax(double a, double b) { return (a < b) ? b : a; }  /* std::max */
static double dmin(double a, double b) { return (b < a) ? b : a; }  /* std::min */

/* EquationOfState.cpp:44-107 */
static double eos_p(const vho_t *h, double ed)
{
    if (h->eos_table) { double f = interp1d(h, ed, h->p_tb); return dmax(1.e-15, f); }
    return ed / 3.;
}
/* EquationOfState.cpp:109-160 */
static double eos_cs2(const vho_t *h, double ed)
{
    if (h->eos_table) {
        double v_min = 0.01, v_max = 1. / 3.;
        double delta_e = h->e_spacing;
        double pp = eos_p(h, ed);
        double p_r = eos_p(h, ed + delta_e);
        double delta_p = p_r - pp;
        double dpde = delta_e / delta_p;
        double v_sound = dpde;
        v_sound = dmax(v_min, dmin(v_max, v_sound));
        return v_sound;
    }
    return 1. / 3.;
}
/* EquationOfState.cpp:162-199 */
static double eos_T(const vho_t *h, double ed)
{
    if (h->eos_table) { double f = interp1d(h, ed, h->T_tb); return dmax(1.e-15, f); }
    return powf((float)(ed / h->eos_a), 0.25f);
}
/* EquationOfState.cpp:201-290 */
static double eos_e_of_T(const vho_t *h, double T)
{
    if (h->eos_table) {
        double T_goal = T, eps_lower = 1e-15, eps_upper = h->e_max;
        double eps_mid = (eps_upper + eps_lower) / 2.;
        double T_lower = eos_T(h, eps_lower);
        int ntol = 1000, iter = 0;
        double rel_accuracy = 1e-8, abs_accuracy = 1e-15, T_mid;
        (void)eos_T(h, eps_upper);
        if (T_goal < T_lower) return eps_lower;
        while (((eps_upper - eps_lower) / eps_mid > rel_accuracy && (eps_upper - eps_lower) > abs_accuracy) && iter < ntol) {
            T_mid = eos_T(h, eps_mid);
            if (T_goal < T_mid) eps_upper = eps_mid; else eps_lower = eps_mid;
            eps_mid = (eps_upper + eps_lower) / 2.;
            iter++;
        }
        return eps_mid;
    }
    return h->eos_a * (double)powf((float)T, 4.0f);
}

/* ------------------------------------------------------- limiter / flux */
/* FluxLimiter.cpp:14-32 */
static int sgn(double x) { return (x < 0) ? -1 : 1; }
static double minmod(double x, double y) { return (sgn(x) + sgn(y)) * fmin(fabs(x), fabs(y)) / 2.0; }
static double approx_deriv(double th, double x, double y, double z)
{
    double l = th * (y - x);
    double c = (z - x) / 2.0;
    double r = th * (z - y);
    return minmod(l, minmod(c, r));
}

/* EnergyMomentumTensor.cpp:22-115 */
static double e_from_conserved(const vho_t *h, double ePrev, double M0, double M, double Pi, int *bad)
{
    if (!h->eos_table)
        return fabsf(sqrtf(fabsf(4 * M0 * M0 - 3 * M)) - M0);
    double e0 = ePrev;
    for (int j = 0; j < 10000; ++j) {
        double pp = eos_p(h, e0);
        double cs2 = eos_cs2(h, e0);
        double cst2 = pp / e0;
        double A = M0 * (1.0 - cst2) + Pi;
        double B = M0 * (M0 + Pi) - M;
        double H = sqrtf(fabsf(A * A + 4 * cst2 * B));
        double D = (A - H) / (2 * cst2);
        double f = e0 + D;
        double fp = 1.0 - ((cs2 - cst2) * (B + D * H - ((cs2 - cst2) * cst2 * D * M0) / e0)) / (cst2 * e0 * H);
        if (isnan(f / fp)) { *bad = 1; return NAN; }
        double ee = e0 - f / fp;
        if (fabsf(ee - e0) <= 1.0e-3 * fabsf(ee)) return ee;
        e0 = ee;
    }
    /* bisection fallback, EnergyMomentumTensor.cpp:48-111 */
    {
        double e_lo = 0.0, e_mid = ePrev, e_hi = 2.0 * (ePrev + 1.0);
        for (int j = 0; j < 1000000; ++j) {
            double p_lo = eos_p(h, e_lo), p_mid = eos_p(h, e_mid), p_hi = eos_p(h, e_hi);
            double cst2_lo = p_lo / e_lo, cst2_mid = p_mid / e_mid, cst2_hi = p_hi / e_hi;
            double A_lo = M0 * (1.0 - cst2_lo) + Pi, A_mid = M0 * (1.0 - cst2_mid) + Pi, A_hi = M0 * (1.0 - cst2_hi) + Pi;
            double B = M0 * (M0 + Pi) - M;
            double H_lo = sqrtf(fabsf(A_lo * A_lo + 4 * cst2_lo * B));
            double H_mid = sqrtf(fabsf(A_mid * A_mid + 4 * cst2_mid * B));
            double H_hi = sqrtf(fabsf(A_hi * A_hi + 4 * cst2_hi * B));
            double D_lo = (A_lo - H_lo) / (2 * cst2_lo), D_mid = (A_mid - H_mid) / (2 * cst2_mid), D_hi = (A_hi - H_hi) / (2 * cst2_hi);
            double f_lo = e_lo + D_lo, f_mid = e_mid + D_mid, f_hi = e_hi + D_hi;
            if ((e_hi - e_lo) < (1.0e-3 * e_hi) / 2.0) return e_mid;
            if (f_lo * f_mid < 0.0) { e_hi = e_mid; e_mid = (e_lo + e_hi) / 2.0; }
            else if (f_mid * f_hi < 0.0) { e_lo = e_mid; e_mid = (e_lo + e_hi) / 2.0; }
        }
        return ePrev;
    }
}

/* EnergyMomentumTensor.cpp:117-233 */
static void inferred(const vho_t *h, double t, const double *qv, double ePrev,
                     double *e_, double *p_, double *ut, double *ux, double *uy, double *un, int *bad)
{
    double ttt = qv[0], ttx = qv[1], tty = qv[2], ttn = qv[3];
    double pitt = qv[4], pitx = qv[5], pity = qv[6], pitn = qv[7];
    double Pi = h->bulk ? qv[14] : 0;
    double M0 = ttt - pitt;
    double M1 = ttx - pitx;
    double M2 = tty - pity;
    double M3 = ttn - pitn;
    double M = M1 * M1 + M2 * M2 + t * t * M3 * M3;
    if (ePrev <= 0.1) *e_ = M0 - M / M0;
    else *e_ = e_from_conserved(h, ePrev, M0, M, Pi, bad);
    if (isnan(*e_)) *bad = 1;
    *p_ = eos_p(h, *e_);
    if (*e_ < 1.e-7) { *e_ = 1.e-7; *p_ = 1.e-7; }
    double P = *p_ + Pi;
    double E = 1.0 / (*e_ + P);
    *ut = sqrtf(fabsf((M0 + P) * E));
    double E2 = E / (*ut);
    *ux = M1 * E2;
    *uy = M2 * E2;
    *un = M3 * E2;
    if (*ut > 1.0e3) { *ut = 1.0; *ux = 0.0; *uy = 0.0; *un = 0.0; }
}

/* SemiDiscreteKurganovTadmorScheme.cpp:14-62 with HalfSiteExtrapolation.cpp,
 * LocalPropagationSpeed.cpp, SpectralRadius.cpp and FluxFunctions.cpp.
 * data: 5 stencil values per component; fwd=1 is the i+1/2 face, 0 the i-1/2
 * face; dir 1/2/3 selects x/y/eta. */
static void flux(const vho_t *h, const double *data, double *result, int fwd, int dir, double t, double ePrev, int *bad)
{
    double qR[MAXQ], qL[MAXQ];
    const double th = h->theta;
    for (int n = 0; n < h->nq; ++n) {
        const double *d = data + 5 * n;
        double qmm = d[0], qm = d[1], qq = d[2], qp = d[3], qpp = d[4];
        if (fwd) {
            qR[n] = qp - approx_deriv(th, qq, qp, qpp) / 2;
            qL[n] = qq + approx_deriv(th, qm, qq, qp) / 2;
        } else {
            qR[n] = qq - approx_deriv(th, qm, qq, qp) / 2;
            qL[n] = qm + approx_deriv(th, qmm, qm, qq) / 2;
        }
    }
    double eR, pR, utR, uxR, uyR, unR, eL, pL, utL, uxL, uyL, unL;
    inferred(h, t, qR, ePrev, &eR, &pR, &utR, &uxR, &uyR, &unR, bad);
    inferred(h, t, qL, ePrev, &eL, &pL, &utL, &uxL, &uyL, &unL, bad);
    double vR = (dir == 1) ? uxR : (dir == 2) ? uyR : unR;
    double vL = (dir == 1) ? uxL : (dir == 2) ? uyL : unL;
    double rhoL = fabs(vL / utL);
    double rhoR = fabs(vR / utR);
    double a = fmax(rhoL, rhoR);
    for (int n = 0; n < h->nq; ++n) {
        double FqR = vR * qR[n] / utR;
        double FqL = vL * qL[n] / utL;
        double res = FqR + FqL - a * (qR[n] - qL[n]);
        res /= 2;
        result[n] = res;
    }
}

/* ------------------------------------------------------------- sources */
/* SourceTerms.cpp:40-48 (reference law, T in fm^-1) or the Gaussian law */
static double zeta_over_s(const vho_t *h, double T)
{
    if (h->zeta_law == 1) {
        double TG = T * HBARC;
        double z = (TG - h->zeta_T0) / h->zeta_w;
        return h->zeta_norm * exp(-(z * z));
    }
    double x = T / 1.01355;
    if (x > 1.05) return 0.9 * exp(-(x - 1) / 0.025) + 0.25 * exp(-(x - 1) / 0.13) + 0.001;
    else if (x < 0.995) return 0.9 * exp((x - 1) / 0.0025) + 0.22 * exp((x - 1) / 0.022) + 0.03;
    else return -13.77 * x * x + 27.55 * x - 13.45;
}

/* SourceTerms.cpp:55-313 */
static void pimunu_sources(const vho_t *h, double *rhs, double t, double e, double p,
    double ut, double ux, double uy, double un, double utp, double uxp, double uyp, double unp,
    double pitt, double pitx, double pity, double pitn, double pixx, double pixy, double pixn, double piyy,
    double piyn, double pinn, double Pi,
    double dxut, double dyut, double dnut, double dxux, double dyux, double dnux,
    double dxuy, double dyuy, double dnuy, double dxun, double dyun, double dnun, double dkvk,
    double d_etabar, double d_dt)
{
    const double delta_pipi = 1.33333, tau_pipi = 1.42857, delta_PiPi = 0.666667, lambda_piPi = 1.2;
    double T = eos_T(h, e);
    double taupiInv = T / 5 / d_etabar;
    double beta_pi = (e + p) / 5;
    double cs2 = eos_cs2(h, e);
    double a = 1.0 / 3.0 - cs2;
    double a2 = a * a;
    double beta_Pi = 15 * a2 * (e + p);
    double lambda_Pipi = 8 * a / 5;
    double zetabar = zeta_over_s(h, T);
    double tauPiInv = 15 * a2 * T / zetabar;
    double ut2 = ut * ut, un2 = un * un, t2 = t * t, t3 = t * t2;
    double dtut = (ut - utp) / d_dt, dtux = (ux - uxp) / d_dt, dtuy = (uy - uyp) / d_dt, dtun = (un - unp) / d_dt;
    double Dut = ut * dtut + ux * dxut + uy * dyut + un * dnut + t * un * un;
    double DuxUpper = ut * dtux + ux * dxux + uy * dyux + un * dnux;
    double Dux = -DuxUpper;
    double DuyUpper = ut * dtuy + ux * dxuy + uy * dyuy + un * dnuy;
    double Duy = -DuyUpper;
    double DunUpper = ut * dtun + ux * dxun + uy * dyun + un * dnun + 2 * ut * un / t;
    double Dun = -t2 * DunUpper;
    double dut = Dut - t * un * un;
    double dux = ut * dtux + ux * dxux + uy * dyux + un * dnux;
    double duy = ut * dtuy + ux * dxuy + uy * dyuy + un * dnuy;
    double dun = ut * dtun + ux * dxun + uy * dyun + un * dnun;
    double theta = ut / t + dtut + dxux + dyuy + dnun;
    double stt = -t * ut * un2 + (dtut - ut * dut) + (ut2 - 1) * theta / 3.0;
    double stx = -(t * un2 * ux) / 2.0 + (dtux - dxut) / 2.0 - (ux * dut + ut * dux) / 2.0 + ut * ux * theta / 3.0;
    double sty = -(t * un2 * uy) / 2.0 + (dtuy - dyut) / 2.0 - (uy * dut + ut * duy) / 2.0 + ut * uy * theta / 3.0;
    double stn = -un * (2.0 * ut2 + t2 * un2) / (2.0 * t) + (dtun - dnut / t2) / 2.0 - (un * dut + ut * dun) / 2.0 + ut * un * theta / 3.0;
    double sxx = -(dxux + ux * dux) + (1.0 + ux * ux) * theta / 3.0;
    double sxy = -(dxuy + dyux) / 2.0 - (uy * dux + ux * duy) / 2.0 + ux * uy * theta / 3.0;
    double sxn = -ut * ux * un / t - (dxun + dnux / t2) / 2.0 - (un * dux + ux * dun) / 2.0 + ux * un * theta / 3.0;
    double syy = -(dyuy + uy * duy) + (1.0 + uy * uy) * theta / 3.0;
    double syn = -ut * uy * un / t - (dyun + dnuy / t2) / 2.0 - (un * duy + uy * dun) / 2.0 + uy * un * theta / 3.0;
    double snn = -ut * (1.0 + 2.0 * t2 * un2) / t3 - dnun / t2 - un * dun + (1.0 / t2 + un2) * theta / 3.0;
    double wtx = (-dtux - dxut + ut * dux - ux * dut - t * un2 * ux) / 2.0;
    double wty = (-dtuy - dyut + ut * duy - uy * dut - t * un2 * uy) / 2.0;
    double wtn = (-t2 * dtun - 2.0 * t * un - dnut - ut * Dun - t2 * un * dut - t3 * un * un2) / 2.0;
    double wxy = (dxuy - dyux + ux * duy - uy * dux) / 2.0;
    double wxn = (t2 * dxun - dnux - ux * Dun - t2 * un * dux) / 2.0;
    double wyn = (t2 * dyun - dnuy - uy * Dun - t2 * un * duy) / 2.0;
    double wxt = wtx, wyt = wty, wnt = wtn / t2, wyx = -wxy, wnx = -wxn / t2, wny = -wyn / t2;
    double I1tt = 2.0 * ut * (pitt * Dut + pitx * Dux + pity * Duy + pitn * Dun);
    double I1tx = (pitt * ux + pitx * ut) * Dut + (pitx * ux + pixx * ut) * Dux + (pity * ux + pixy * ut) * Duy + (pitn * ux + pixn * ut) * Dun;
    double I1ty = (pitt * uy + pity * ut) * Dut + (pitx * uy + pixy * ut) * Dux + (pity * uy + piyy * ut) * Duy + (pitn * uy + piyn * ut) * Dun;
    double I1tn = (pitt * un + pitn * ut) * Dut + (pitx * un + pixn * ut) * Dux + (pity * un + piyn * ut) * Duy + (pitn * un + pinn * ut) * Dun;
    double I1xx = 2.0 * ux * (pitx * Dut + pixx * Dux + pixy * Duy + pixn * Dun);
    double I1xy = (pitx * uy + pity * ux) * Dut + (pixx * uy + pixy * ux) * Dux + (pixy * uy + piyy * ux) * Duy + (pixn * uy + piyn * ux) * Dun;
    double I1xn = (pitx * un + pitn * ux) * Dut + (pixx * un + pixn * ux) * Dux + (pixy * un + piyn * ux) * Duy + (pixn * un + pinn * ux) * Dun;
    double I1yy = 2.0 * uy * (pity * Dut + pixy * Dux + piyy * Duy + piyn * Dun);
    double I1yn = (pity * un + pitn * uy) * Dut + (pixy * un + pixn * uy) * Dux + (piyy * un + piyn * uy) * Duy + (piyn * un + pinn * uy) * Dun;
    double I1nn = 2.0 * un * (pitn * Dut + pixn * Dux + piyn * Duy + pinn * Dun);
    double I2tt = theta * pitt, I2tx = theta * pitx, I2ty = theta * pity, I2tn = theta * pitn, I2xx = theta * pixx;
    double I2xy = theta * pixy, I2xn = theta * pixn, I2yy = theta * piyy, I2yn = theta * piyn, I2nn = theta * pinn;
    double I3tt = 2.0 * (pitx * wtx + pity * wty + pitn * wtn);
    double I3tx = pitt * wxt + pity * wxy + pitn * wxn + pixx * wtx + pixy * wty + pixn * wtn;
    double I3ty = pitt * wyt + pitx * wyx + pitn * wyn + pixy * wtx + piyy * wty + piyn * wtn;
    double I3tn = pitt * wnt + pitx * wnx + pity * wny + pixn * wtx + piyn * wty + pinn * wtn;
    double I3xx = 2.0 * (pitx * wxt + pixy * wxy + pixn * wxn);
    double I3xy = pitx * wyt + pity * wxt + pixx * wyx + piyy * wxy + pixn * wyn + piyn * wxn;
    double I3xn = pitx * wnt + pitn * wxt + pixx * wnx + pixy * wny + piyn * wxy + pinn * wxn;
    double I3yy = 2.0 * (pity * wyt + pixy * wyx + piyn * wyn);
    double I3yn = pity * wnt + pitn * wyt + pixy * wnx + pixn * wyx + piyy * wny + pinn * wyn;
    double I3nn = 2.0 * (pitn * wnt + pixn * wnx + piyn * wny);
    double ux2 = ux * ux, uy2 = uy * uy;
    double ps = pitt * stt - 2.0 * pitx * stx - 2.0 * pity * sty + pixx * sxx + 2.0 * pixy * sxy + piyy * syy - 2.0 * pitn * stn * t2 + 2.0 * pixn * sxn * t2 + 2.0 * piyn * syn * t2 + pinn * snn * t2 * t2;
    double I4tt = (pitt * stt - pitx * stx - pity * sty - t2 * pitn * stn) - (1.0 - ut2) * ps / 3.0;
    double I4tx = (pitt * stx + pitx * stt) / 2.0 - (pitx * sxx + pixx * stx) / 2.0 - (pity * sxy + pixy * sty) / 2.0 - t2 * (pitn * sxn + pixn * stn) / 2.0 + (ut * ux) * ps / 3.0;
    double I4ty = (pitt * sty + pity * stt) / 2.0 - (pitx * sxy + pixy * stx) / 2.0 - (pity * syy + piyy * sty) / 2.0 - t2 * (pitn * syn + piyn * stn) / 2.0 + (ut * uy) * ps / 3.0;
    double I4tn = (pitt * stn + pitn * stt) / 2.0 - (pitx * sxn + pixn * stx) / 2.0 - (pity * syn + piyn * sty) / 2.0 - t2 * (pitn * snn + pinn * stn) / 2.0 + (ut * un) * ps / 3.0;
    double I4xx = (pitx * stx - pixx * sxx - pixy * sxy - t2 * pixn * sxn) + (1.0 + ux2) * ps / 3.0;
    double I4xy = (pitx * sty + pity * stx) / 2.0 - (pixx * sxy + pixy * sxx) / 2.0 - (pixy * syy + piyy * sxy) / 2.0 - t2 * (pixn * syn + piyn * sxn) / 2.0 + (ux * uy) * ps / 3.0;
    double I4xn = (pitx * stn + pitn * stx) / 2.0 - (pixx * sxn + pixn * sxx) / 2.0 - (pixy * syn + piyn * sxy) / 2.0 - t2 * (pixn * snn + pinn * sxn) / 2.0 + (ux * un) * ps / 3.0;
    double I4yy = (pity * sty - pixy * sxy - piyy * syy - t2 * piyn * syn) + (1.0 + uy2) * ps / 3.0;
    double I4yn = (pity * stn + pitn * sty) / 2.0 - (pixy * sxn + pixn * sxy) / 2.0 - (piyy * syn + piyn * syy) / 2.0 - t2 * (piyn * snn + pinn * syn) / 2.0 + (uy * un) * ps / 3.0;
    double I4nn = (pitn * stn - pixn * sxn - piyn * syn - t2 * pinn * snn) + (1.0 / t2 + un2) * ps / 3.0;
    double Itt = I1tt + delta_pipi * I2tt - I3tt + tau_pipi * I4tt - lambda_piPi * Pi * stt;
    double Itx = I1tx + delta_pipi * I2tx - I3tx + tau_pipi * I4tx - lambda_piPi * Pi * stx;
    double Ity = I1ty + delta_pipi * I2ty - I3ty + tau_pipi * I4ty - lambda_piPi * Pi * sty;
    double Itn = I1tn + delta_pipi * I2tn - I3tn + tau_pipi * I4tn - lambda_piPi * Pi * stn;
    double Ixx = I1xx + delta_pipi * I2xx - I3xx + tau_pipi * I4xx - lambda_piPi * Pi * sxx;
    double Ixy = I1xy + delta_pipi * I2xy - I3xy + tau_pipi * I4xy - lambda_piPi * Pi * sxy;
    double Ixn = I1xn + delta_pipi * I2xn - I3xn + tau_pipi * I4xn - lambda_piPi * Pi * sxn;
    double Iyy = I1yy + delta_pipi * I2yy - I3yy + tau_pipi * I4yy - lambda_piPi * Pi * syy;
    double Iyn = I1yn + delta_pipi * I2yn - I3yn + tau_pipi * I4yn - lambda_piPi * Pi * syn;
    double Inn = I1nn + delta_pipi * I2nn - I3nn + tau_pipi * I4nn - lambda_piPi * Pi * snn;
    double dpitt = 2.0 * beta_pi * stt - pitt * taupiInv - Itt - 2.0 * un * t * pitn;
    double dpitx = 2.0 * beta_pi * stx - pitx * taupiInv - Itx - un * t * pixn;
    double dpity = 2.0 * beta_pi * sty - pity * taupiInv - Ity - un * t * piyn;
    double dpitn = 2.0 * beta_pi * stn - pitn * taupiInv - Itn - un * t * pinn - (ut * pitn + un * pitt) / t;
    double dpixx = 2.0 * beta_pi * sxx - pixx * taupiInv - Ixx;
    double dpixy = 2.0 * beta_pi * sxy - pixy * taupiInv - Ixy;
    double dpixn = 2.0 * beta_pi * sxn - pixn * taupiInv - Ixn - (ut * pixn + un * pitx) / t;
    double dpiyy = 2.0 * beta_pi * syy - piyy * taupiInv - Iyy;
    double dpiyn = 2.0 * beta_pi * syn - piyn * taupiInv - Iyn - (ut * piyn + un * pity) / t;
    double dpinn = 2.0 * beta_pi * snn - pinn * taupiInv - Inn - 2 * (ut * pinn + un * pitn) / t;
    double dPi = -beta_Pi * theta - Pi * tauPiInv - delta_PiPi * Pi * theta + lambda_Pipi * ps;
    rhs[0] = dpitt / ut + pitt * dkvk;
    rhs[1] = dpitx / ut + pitx * dkvk;
    rhs[2] = dpity / ut + pity * dkvk;
    rhs[3] = dpitn / ut + pitn * dkvk;
    rhs[4] = dpixx / ut + pixx * dkvk;
    rhs[5] = dpixy / ut + pixy * dkvk;
    rhs[6] = dpixn / ut + pixn * dkvk;
    rhs[7] = dpiyy / ut + piyy * dkvk;
    rhs[8] = dpiyn / ut + piyn * dkvk;
    rhs[9] = dpinn / ut + pinn * dkvk;
    if (h->bulk) rhs[10] = dPi / ut + Pi * dkvk;
}

/* SourceTerms.cpp:421-612 (USE_APPROX_DERIVATIVE branch, no Cartesian override;
 * the dynamical source arrays are zero unless vho_set_sources gave them). */
static void sources2(const vho_t *h, const double *Qv, double *S, double **uu,
                     double utp, double uxp, double uyp, double unp, double t, double e, const double *pvec, int s)
{
    double ttt = Qv[0], ttx = Qv[1], tty = Qv[2], ttn = Qv[3];
    double pitt = Qv[4], pitx = Qv[5], pity = Qv[6], pitn = Qv[7], pixx = Qv[8], pixy = Qv[9];
    double pixn = Qv[10], piyy = Qv[11], piyn = Qv[12], pinn = Qv[13];
    double Pi = h->bulk ? Qv[14] : 0;
    const double *utv = uu[0], *uxv = uu[1], *uyv = uu[2], *unv = uu[3];
    double p = pvec[s], ut = utv[s], ux = uxv[s], uy = uyv[s], un = unv[s];
    int sx = 1, sy = h->ncx, sz = h->ncx * h->ncy;
    const double th = h->theta;
    double dxut = approx_deriv(th, utv[s - sx], ut, utv[s + sx]) / h->dx;
    double dxux = approx_deriv(th, uxv[s - sx], ux, uxv[s + sx]) / h->dx;
    double dxuy = approx_deriv(th, uyv[s - sx], uy, uyv[s + sx]) / h->dx;
    double dxun = approx_deriv(th, unv[s - sx], un, unv[s + sx]) / h->dx;
    double dyut = approx_deriv(th, utv[s - sy], ut, utv[s + sy]) / h->dy;
    double dyux = approx_deriv(th, uxv[s - sy], ux, uxv[s + sy]) / h->dy;
    double dyuy = approx_deriv(th, uyv[s - sy], uy, uyv[s + sy]) / h->dy;
    double dyun = approx_deriv(th, unv[s - sy], un, unv[s + sy]) / h->dy;
    double dnut = approx_deriv(th, utv[s - sz], ut, utv[s + sz]) / h->dz;
    double dnux = approx_deriv(th, uxv[s - sz], ux, uxv[s + sz]) / h->dz;
    double dnuy = approx_deriv(th, uyv[s - sz], uy, uyv[s + sz]) / h->dz;
    double dnun = approx_deriv(th, unv[s - sz], un, unv[s + sz]) / h->dz;
    double dxp = approx_deriv(th, pvec[s - sx], p, pvec[s + sx]) / h->dx;
    double dyp = approx_deriv(th, pvec[s - sy], p, pvec[s + sy]) / h->dy;
    double dnp = approx_deriv(th, pvec[s - sz], p, pvec[s + sz]) / h->dz;
    /* Tnn(e, p+Pi, un, pinn, t), EnergyMomentumTensor.cpp:328-330 */
    double pP = p + Pi;
    double tnn = (e + pP) * un * un + pP / t / t + pinn;
    double vx = ux / ut, vy = uy / ut, vn = un / ut;
    double dxvx = (dxux - vx * dxut) / ut;
    double dyvy = (dyuy - vy * dyut) / ut;
    double dnvn = (dnun - vn * dnut) / ut;
    double dkvk = dxvx + dyvy + dnvn;
    double t2pow = pow(t, 2);
    const double s0 = h->src[0] ? h->src[0][s] : 0.0, s1 = h->src[0] ? h->src[1][s] : 0.0;
    const double s2 = h->src[0] ? h->src[2][s] : 0.0, s3 = h->src[0] ? h->src[3][s] : 0.0;
    S[0] = s0 - (ttt / t + t * tnn) + dkvk * (pitt - p - Pi) - vx * dxp - vy * dyp - vn * dnp;
    S[1] = s1 - ttx / t - dxp + dkvk * pitx;
    S[2] = s2 - tty / t - dyp + dkvk * pity;
    S[3] = s3 - 3 * ttn / t - dnp / t2pow + dkvk * pitn;
    double rhs[11];
    pimunu_sources(h, rhs, t, e, p, ut, ux, uy, un, utp, uxp, uyp, unp,
                   pitt, pitx, pity, pitn, pixx, pixy, pixn, piyy, piyn, pinn, Pi,
                   dxut, dyut, dnut, dxux, dyux, dnux, dxuy, dyuy, dnuy, dxun, dyun, dnun, dkvk, h->etabar, h->dt);
    for (int n = 0; n < h->nq - 4; ++n) S[n + 4] = rhs[n];
}

/* SourceTerms.cpp:316-419: the d(pi)/dx^i sources of the T^{tau mu} rows */
static void sources_dir(const vho_t *h, const double *I, double *S, double **uu, int s, double t, double d, int dir)
{
    double fac = 1 / d / 2;
    const double *v = (dir == 1) ? uu[1] : (dir == 2) ? uu[2] : uu[3];
    double ut = uu[0][s];
    double vv = v[s] / ut;
#define DER(n) ((I[5 * (n) + 3] - I[5 * (n) + 1]) * fac)
    if (dir == 1) {
        double dpitt = DER(4), dpitx = DER(5), dpity = DER(6), dpitn = DER(7), dpixx = DER(8), dpixy = DER(9), dpixn = DER(10);
        if (!h->bulk) { S[0] = dpitt * vv - dpitx; S[1] = dpitx * vv - dpixx; }
        else { double dPi = DER(14); S[0] = dpitt * vv - dpitx - vv * dPi; S[1] = dpitx * vv - dpixx - dPi; }
        S[2] = dpity * vv - dpixy;
        S[3] = dpitn * vv - dpixn;
    } else if (dir == 2) {
        double dpitt = DER(4), dpitx = DER(5), dpity = DER(6), dpitn = DER(7), dpixy = DER(9), dpiyy = DER(11), dpiyn = DER(12);
        if (!h->bulk) { S[0] = dpitt * vv - dpity; S[2] = dpity * vv - dpiyy; }
        else { double dPi = DER(14); S[0] = dpitt * vv - dpity - vv * dPi; S[2] = dpity * vv - dpiyy - dPi; }
        S[1] = dpitx * vv - dpixy;
        S[3] = dpitn * vv - dpiyn;
    } else {
        double dpitt = DER(4), dpitx = DER(5), dpity = DER(6), dpitn = DER(7), dpixn = DER(10), dpiyn = DER(12), dpinn = DER(13);
        if (!h->bulk) { S[0] = dpitt * vv - dpitn; S[3] = dpitn * vv - dpinn; }
        else { double dPi = DER(14); S[0] = dpitt * vv - dpitn - vv * dPi; S[3] = dpitn * vv - dpinn - dPi / pow(t, 2); }
        S[1] = dpitx * vv - dpixn;
        S[2] = dpity * vv - dpiyn;
    }
#undef DER
}

/* ------------------------------------------------------------- kernels */
static int IDX(const vho_t *h, int i, int j, int k) { return i + h->ncx * (j + h->ncy * k); }

/* FullyDiscreteKurganovTadmorScheme.cpp:155-298 */
static void euler_source(vho_t *h, double t, double **cur, double **upd, double **uu, double **upv)
{
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 2; k < h->ncz - 2; ++k)
        for (int j = 2; j < h->ncy - 2; ++j)
            for (int i = 2; i < h->ncx - 2; ++i) {
                int s = IDX(h, i, j, k);
                double Qv[MAXQ], S[MAXQ];
                for (int n = 0; n < h->nq; ++n) Qv[n] = cur[n][s];
                sources2(h, Qv, S, uu, upv[0][s], upv[1][s], upv[2][s], upv[3][s], t, h->e[s], h->p, s);
                for (int n = 0; n < h->nq; ++n) upd[n][s] = Qv[n] + h->dt * S[n];
            }
}

/* FullyDiscreteKurganovTadmorScheme.cpp:300-634 (dir 1, 2, 3) */
static void euler_dir(vho_t *h, double t, double **cur, double **upd, double **uu, int dir)
{
    int stride = (dir == 1) ? 1 : (dir == 2) ? h->ncx : h->ncx * h->ncy;
    double d = (dir == 1) ? h->dx : (dir == 2) ? h->dy : h->dz;
    int bad = 0;
#pragma omp parallel for collapse(2) schedule(static) reduction(| : bad)
    for (int k = 2; k < h->ncz - 2; ++k)
        for (int j = 2; j < h->ncy - 2; ++j)
            for (int i = 2; i < h->ncx - 2; ++i) {
                int s = IDX(h, i, j, k);
                double I[5 * MAXQ], H[MAXQ], result[MAXQ];
                for (int n = 0; n < h->nq; ++n) {
                    I[5 * n + 0] = cur[n][s - 2 * stride];
                    I[5 * n + 1] = cur[n][s - stride];
                    I[5 * n + 2] = cur[n][s];
                    I[5 * n + 3] = cur[n][s + stride];
                    I[5 * n + 4] = cur[n][s + 2 * stride];
                }
                flux(h, I, H, 1, dir, t, h->e[s], &bad);
                for (int n = 0; n < h->nq; ++n) result[n] = -H[n];
                flux(h, I, H, 0, dir, t, h->e[s], &bad);
                for (int n = 0; n < h->nq; ++n) { result[n] += H[n]; result[n] /= d; }
                sources_dir(h, I, H, uu, s, t, d, dir);
                for (int n = 0; n < 4; ++n) { result[n] += H[n]; result[n] *= h->dt; }
                for (int n = 4; n < h->nq; ++n) result[n] *= h->dt;
                for (int n = 0; n < h->nq; ++n) upd[n][s] += result[n];
            }
    if (bad) h->nan_flag = 1;
}

/* FullyDiscreteKurganovTadmorScheme.cpp:638-686 */
static void convex(vho_t *h, double **qq, double **QQ)
{
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 2; k < h->ncz - 2; ++k)
        for (int j = 2; j < h->ncy - 2; ++j)
            for (int i = 2; i < h->ncx - 2; ++i) {
                int s = IDX(h, i, j, k);
                for (int n = 0; n < h->nq; ++n) { QQ[n][s] += qq[n][s]; QQ[n][s] /= 2; }
            }
}

/* EnergyMomentumTensor.cpp:235-287 */
static void set_inferred(vho_t *h, double **qq, double **uu, double t)
{
    int bad = 0;
#pragma omp parallel for collapse(2) schedule(static) reduction(| : bad)
    for (int k = 2; k < h->ncz - 2; ++k)
        for (int j = 2; j < h->ncy - 2; ++j)
            for (int i = 2; i < h->ncx - 2; ++i) {
                int s = IDX(h, i, j, k);
                double qs[MAXQ], e_, p_, ut, ux, uy, un;
                for (int n = 0; n < h->nq; ++n) qs[n] = qq[n][s];
                inferred(h, t, qs, h->e[s], &e_, &p_, &ut, &ux, &uy, &un, &bad);
                h->e[s] = e_; h->p[s] = p_;
                uu[0][s] = ut; uu[1][s] = ux; uu[2][s] = uy; uu[3][s] = un;
            }
    if (bad) h->nan_flag = 1;
}

/* FullyDiscreteKurganovTadmorScheme.cpp:690-859 (REG_SCHEME_1) */
static void regulate(vho_t *h, double t, double **qq, double **uu)
{
    if (!h->regfac[0]) {
        size_t len = (size_t)h->ncx * h->ncy * h->ncz;
        h->regfac[0] = (double *)calloc(len, 8);
        h->regfac[1] = (double *)calloc(len, 8);
    }
    int bad = 0;
#pragma omp parallel for collapse(2) schedule(static) reduction(| : bad)
    for (int k = 2; k < h->ncz - 2; ++k)
        for (int j = 2; j < h->ncy - 2; ++j)
            for (int i = 2; i < h->ncx - 2; ++i) {
                int s = IDX(h, i, j, k);
                double pitt = qq[4][s], pitx = qq[5][s], pity = qq[6][s], pitn = qq[7][s], pixx = qq[8][s];
                double pixy = qq[9][s], pixn = qq[10][s], piyy = qq[11][s], piyn = qq[12][s], pinn = qq[13][s];
                double Pi = h->bulk ? qq[14][s] : 0;
                double ut = uu[0][s], ux = uu[1][s], uy = uu[2][s], un = uu[3][s];
                double t2 = t * t;
                double facShear, facBulk;
                double xi0 = 0.1, rhomax = 1.0;
                double pipi = pitt * pitt - 2 * pitx * pitx - 2 * pity * pity + pixx * pixx + 2 * pixy * pixy + piyy * piyy - 2 * pitn * pitn * t2 + 2 * pixn * pixn * t2 + 2 * piyn * piyn * t2 + pinn * pinn * t2 * t2;
                double spipi = sqrt(fabs(pipi));
                double pimumu = pitt - pixx - piyy - pinn * t * t;
                double piu0 = -(pitn * t2 * un) + pitt * ut - pitx * ux - pity * uy;
                double piu1 = -(pixn * t2 * un) + pitx * ut - pixx * ux - pixy * uy;
                double piu2 = -(piyn * t2 * un) + pity * ut - pixy * ux - piyy * uy;
                double piu3 = -(pinn * t2 * un) + pitn * ut - pixn * ux - piyn * uy;
                double a1 = spipi / rhomax / sqrtf(h->e[s] * h->e[s] + 3 * h->p[s] * h->p[s]);
                double a2 = pimumu / xi0 / rhomax / spipi;
                double a3 = piu0 / xi0 / rhomax / spipi;
                double a4 = piu1 / xi0 / rhomax / spipi;
                double a5 = piu2 / xi0 / rhomax / spipi;
                double a6 = piu3 / xi0 / rhomax / spipi;
                double a12 = fmax(a1, a2), a34 = fmax(a3, a4), a56 = fmax(a5, a6), a3456 = fmax(a34, a56);
                double rho = fmax(a12, a3456);
                facShear = tanh(rho) / rho;
                if (fabs(rho) < 1.e-7) facShear = 1.0;
                double rhoBulk = fabs(Pi) / h->p[s];
                facBulk = tanh(rhoBulk) / rhoBulk;
                if (fabs(rhoBulk) < 1.e-7) facBulk = 1.0;
                if (h->e[s] > h->e_reg) { facShear = 1.0; facBulk = 1.0; }
                for (int n = 4; n < 14; ++n) qq[n][s] *= facShear;
                h->regfac[0][s] = facShear;
                if (isnan(facShear)) bad = 1;
                if (h->bulk) { qq[14][s] *= facBulk; h->regfac[1][s] = facBulk; if (isnan(facBulk)) bad = 1; }
            }
    if (bad) h->nan_flag = 1;
}

/* DynamicalVariables.cpp:220-378, the face ghosts only: corner and edge ghost
 * cells are never read by the axis-aligned stencils. */
static void ghost_copy(vho_t *h, double **qq, double **uu, int s, int sBC)
{
    h->e[s] = h->e[sBC]; h->p[s] = h->p[sBC];
    for (int c = 0; c < 4; ++c) uu[c][s] = uu[c][sBC];
    for (int n = 0; n < h->nq; ++n) qq[n][s] = qq[n][sBC];
}
static void ghosts(vho_t *h, double **qq, double **uu)
{
    int nx = h->nx, ny = h->ny, nz = h->nz;
    for (int j = 2; j < ny + 2; ++j) for (int k = 2; k < nz + 2; ++k) {
        for (int i = 0; i <= 1; ++i) ghost_copy(h, qq, uu, IDX(h, i, j, k), IDX(h, 2, j, k));
        for (int i = nx + 2; i <= nx + 3; ++i) ghost_copy(h, qq, uu, IDX(h, i, j, k), IDX(h, nx + 1, j, k));
    }
    for (int i = 2; i < nx + 2; ++i) for (int k = 2; k < nz + 2; ++k) {
        for (int j = 0; j <= 1; ++j) ghost_copy(h, qq, uu, IDX(h, i, j, k), IDX(h, i, 2, k));
        for (int j = ny + 2; j <= ny + 3; ++j) ghost_copy(h, qq, uu, IDX(h, i, j, k), IDX(h, i, ny + 1, k));
    }
    for (int i = 2; i < nx + 2; ++i) for (int j = 2; j < ny + 2; ++j) {
        for (int k = 0; k <= 1; ++k) ghost_copy(h, qq, uu, IDX(h, i, j, k), IDX(h, i, j, 2));
        for (int k = nz + 2; k <= nz + 3; ++k) ghost_copy(h, qq, uu, IDX(h, i, j, k), IDX(h, i, j, nz + 1));
    }
}

/* FullyDiscreteKurganovTadmorScheme.cpp:867-924 */
static void rk2(vho_t *h, double t)
{
    double dt = h->dt;
    euler_source(h, t, h->q, h->qS, h->u, h->up);
    euler_dir(h, t, h->q, h->qS, h->u, 1);
    euler_dir(h, t, h->q, h->qS, h->u, 2);
    euler_dir(h, t, h->q, h->qS, h->u, 3);
    t += dt;
    set_inferred(h, h->qS, h->uS, t);
    regulate(h, t, h->qS, h->uS);
    ghosts(h, h->qS, h->uS);
    euler_source(h, t, h->qS, h->Q, h->uS, h->u);
    euler_dir(h, t, h->qS, h->Q, h->uS, 1);
    euler_dir(h, t, h->qS, h->Q, h->uS, 2);
    euler_dir(h, t, h->qS, h->Q, h->uS, 3);
    convex(h, h->q, h->Q);
    for (int c = 0; c < 4; ++c) { double *tmp = h->up[c]; h->up[c] = h->u[c]; h->u[c] = tmp; }
    set_inferred(h, h->Q, h->u, t);
    regulate(h, t, h->Q, h->u);
    ghosts(h, h->Q, h->u);
}

/* ------------------------------------------------------------- C API */
vho_t *vho_create(int nx, int ny, int nz, double dx, double dy, double dz, double dt, double t0,
                  double etabar, double theta, int bulk, double T_reg_GeV, double T_fo_GeV, int fofac)
{
    vho_t *h = (vho_t *)calloc(1, sizeof(vho_t));
    h->nx = nx; h->ny = ny; h->nz = nz; h->ncx = nx + 4; h->ncy = ny + 4; h->ncz = nz + 4;
    h->dx = dx; h->dy = dy; h->dz = dz; h->dt = dt; h->t0 = t0; h->etabar = etabar; h->theta = theta;
    h->bulk = bulk; h->nq = bulk ? 15 : 14;
    h->eos_a = 13.8997; h->T_reg_GeV = T_reg_GeV; h->T_fo_GeV = T_fo_GeV; h->fofac = fofac;
    size_t len = (size_t)h->ncx * h->ncy * h->ncz;
    for (int n = 0; n < h->nq; ++n) {
        h->q[n] = (double *)calloc(len, 8); h->Q[n] = (double *)calloc(len, 8); h->qS[n] = (double *)calloc(len, 8);
    }
    h->e = (double *)calloc(len, 8); h->p = (double *)calloc(len, 8);
    for (int c = 0; c < 4; ++c) {
        h->u[c] = (double *)calloc(len, 8); h->up[c] = (double *)calloc(len, 8); h->uS[c] = (double *)calloc(len, 8);
    }
    size_t N = (size_t)nx * ny * nz;
    for (int s = 0; s < 2; ++s) h->slab[s] = (double *)calloc(11 * N, 8);
    return h;
}

void vho_set_conformal(vho_t *h, double a) { h->eos_table = 0; h->eos_a = a; }
void vho_set_zeta(vho_t *h, int law, double norm, double T0GeV, double wGeV)
{
    h->zeta_law = law; h->zeta_norm = norm; h->zeta_T0 = T0GeV; h->zeta_w = wGeV;
}

/* rows: e[GeV/fm^3], P[GeV/fm^3], s, T[GeV] (EquationOfState.cpp:308-324) */
int vho_set_table(vho_t *h, const double *rows, int nrows)
{
    if (nrows < 2) return -1;
    h->eos_table = 1;
    h->e_length = nrows;
    free(h->p_tb); free(h->T_tb);
    h->p_tb = (double *)malloc(8 * (size_t)nrows); h->T_tb = (double *)malloc(8 * (size_t)nrows);
    for (int ii = 0; ii < nrows; ++ii) {
        double temp = rows[4 * ii] / HBARC;
        if (ii == 0) h->e_min = temp;
        if (ii == 1) h->e_spacing = temp - h->e_min;
        if (ii == nrows - 1) h->e_max = temp;
        h->p_tb[ii] = rows[4 * ii + 1] / HBARC;
        h->T_tb[ii] = rows[4 * ii + 3] / HBARC;
    }
    return 0;
}

double vho_eos_p(vho_t *h, double ed) { return eos_p(h, ed); }
double vho_eos_T(vho_t *h, double ed) { return eos_T(h, ed); }
double vho_eos_cs2(vho_t *h, double ed) { return eos_cs2(h, ed); }
double vho_eos_e(vho_t *h, double T) { return eos_e_of_T(h, T); }

/* interior arrays: e, p, u(4 x N: ut ux uy un), pi(10 x N: pitt..pinn), Pi(N) */
void vho_set_ic(vho_t *h, const double *e, const double *p, const double *u, const double *pi, const double *Pi)
{
    int nx = h->nx, ny = h->ny, nz = h->nz;
    size_t N = (size_t)nx * ny * nz;
    for (int k = 0; k < nz; ++k) for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) {
        int s = IDX(h, i + 2, j + 2, k + 2);
        size_t m = i + (size_t)nx * (j + (size_t)ny * k);
        h->e[s] = e[m]; h->p[s] = p[m];
        for (int c = 0; c < 4; ++c) { h->u[c][s] = u[c * N + m]; h->up[c][s] = u[c * N + m]; }
        for (int c = 0; c < 10; ++c) h->q[4 + c][s] = pi ? pi[c * N + m] : 0.0;
        if (h->bulk) h->q[14][s] = Pi ? Pi[m] : 0.0;
        /* DynamicalVariables.cpp:169-218 with EnergyMomentumTensor.cpp:292-306 */
        double ut = h->u[0][s], ux = h->u[1][s], uy = h->u[2][s], un = h->u[3][s];
        double P = h->p[s] + (h->bulk ? h->q[14][s] : 0.);
        double ee = h->e[s];
        h->q[0][s] = (ee + P) * ut * ut - P + h->q[4][s];
        h->q[1][s] = (ee + P) * ut * ux + h->q[5][s];
        h->q[2][s] = (ee + P) * ut * uy + h->q[6][s];
        h->q[3][s] = (ee + P) * ut * un + h->q[7][s];
    }
    ghosts(h, h->q, h->u);
    h->n = 0; h->t = h->t0;
    h->e_reg = eos_e_of_T(h, h->T_reg_GeV / HBARC);
    h->fo_prev = 0;
    for (int s = 0; s < 2; ++s) memset(h->slab[s], 0, 8 * 11 * N);
}

/* HydroPlugin.cpp:292-307 */
int vho_step(vho_t *h, int nsteps)
{
    for (int s = 0; s < nsteps; ++s) {
        rk2(h, h->t);
        for (int n = 0; n < h->nq; ++n) { double *tmp = h->q[n]; h->q[n] = h->Q[n]; h->Q[n] = tmp; }
        h->n += 1;
        h->t = h->t0 + h->n * h->dt;
    }
    return h->nan_flag;
}

/* Dynamical sources (the Source arrays of SourceTerms.cpp:584-587): interior
 * arrays t, x, y, eta of nx*ny*nz values each; st == NULL removes them. */
void vho_set_sources(vho_t *h, const double *st, const double *sx, const double *sy, const double *sn)
{
    size_t len = (size_t)h->ncx * h->ncy * h->ncz;
    if (!st) {
        for (int c = 0; c < 4; ++c) { free(h->src[c]); h->src[c] = NULL; }
        return;
    }
    const double *in[4] = {st, sx, sy, sn};
    for (int c = 0; c < 4; ++c) {
        if (!h->src[c]) h->src[c] = (double *)calloc(len, 8);
        for (int k = 0; k < h->nz; ++k)
            for (int j = 0; j < h->ny; ++j)
                for (int i = 0; i < h->nx; ++i)
                    h->src[c][IDX(h, i + 2, j + 2, k + 2)] = in[c][i + (size_t)h->nx * (j + (size_t)h->ny * k)];
    }
}

/* Vorticity.cpp:6-171: thermal velocity beta_mu = u_mu / T and the thermal
 * vorticity w_{mu nu} = -(d_mu beta_nu - d_nu beta_mu) / 2 with a backward
 * time difference (u against the previous step's up, both divided by the
 * cell's T) and central spatial differences (neighbours' u over the cell's
 * T), on the interior; u_mu = (u^t, -u^x, -u^y, -u^eta). */
void vho_vorticity(vho_t *h)
{
    size_t len = (size_t)h->ncx * h->ncy * h->ncz;
    if (!h->w[0]) {
        for (int c = 0; c < 6; ++c) h->w[c] = (double *)calloc(len, 8);
        for (int c = 0; c < 4; ++c) h->beta[c] = (double *)calloc(len, 8);
    }
    const double dt = h->dt, dx = h->dx, dy = h->dy, dz = h->dz;
    for (int k = 2; k < h->ncz - 2; ++k)
        for (int j = 2; j < h->ncy - 2; ++j)
            for (int i = 2; i < h->ncx - 2; ++i) {
                const int s = IDX(h, i, j, k);
                const int nb[6] = {IDX(h, i - 1, j, k), IDX(h, i + 1, j, k), IDX(h, i, j - 1, k),
                                   IDX(h, i, j + 1, k), IDX(h, i, j, k - 1), IDX(h, i, j, k + 1)};
                const double T = eos_T(h, h->e[s]);
                double b[4], bp[4], bn[6][4];
                for (int c = 0; c < 4; ++c) {
                    const double sg = (c == 0) ? 1.0 : -1.0;
                    b[c] = (c == 0 ? h->u[c][s] : h->u[c][s] * sg) / T;
                    bp[c] = (c == 0 ? h->up[c][s] : h->up[c][s] * sg) / T;
                    for (int m = 0; m < 6; ++m) bn[m][c] = (c == 0 ? h->u[c][nb[m]] : h->u[c][nb[m]] * sg) / T;
                }
                for (int c = 0; c < 4; ++c) h->beta[c][s] = b[c];
                double ddt[4], ddx[4], ddy[4], ddn[4];
                for (int c = 0; c < 4; ++c) {
                    ddt[c] = (b[c] - bp[c]) / dt;
                    ddx[c] = (bn[1][c] - bn[0][c]) / (2.0 * dx);
                    ddy[c] = (bn[3][c] - bn[2][c]) / (2.0 * dy);
                    ddn[c] = (bn[5][c] - bn[4][c]) / (2.0 * dz);
                }
                h->w[0][s] = (-1.0 / 2.0) * (ddt[1] - ddx[0]);
                h->w[1][s] = (-1.0 / 2.0) * (ddt[2] - ddy[0]);
                h->w[2][s] = (-1.0 / 2.0) * (ddt[3] - ddn[0]);
                h->w[3][s] = (-1.0 / 2.0) * (ddx[2] - ddy[1]);
                h->w[4][s] = (-1.0 / 2.0) * (ddx[3] - ddn[1]);
                h->w[5][s] = (-1.0 / 2.0) * (ddy[3] - ddn[2]);
            }
}

/* which: 0..nq-1 -> q; 100+c -> u; 110+c -> up; 200 -> e; 201 -> p;
 * 300+c -> w (tx ty tn xy xn yn); 310+c -> beta (t x y n) (padded arrays) */
int vho_get(vho_t *h, int which, double *out)
{
    size_t len = (size_t)h->ncx * h->ncy * h->ncz;
    const double *src = NULL;
    if (which >= 0 && which < h->nq) src = h->q[which];
    else if (which >= 100 && which < 104) src = h->u[which - 100];
    else if (which >= 110 && which < 114) src = h->up[which - 110];
    else if (which == 200) src = h->e;
    else if (which == 201) src = h->p;
    else if (which >= 300 && which < 306) src = h->w[which - 300];
    else if (which >= 310 && which < 314) src = h->beta[which - 310];
    else if (which == 400 || which == 401) {
        if (!h->regfac[0]) { memset(out, 0, 8 * len); return 0; }   /* before the first step */
        src = h->regfac[which - 400];
    }
    if (!src) return -1;
    memcpy(out, src, 8 * len);
    return 0;
}
int vho_steps_done(vho_t *h) { return h->n; }
double vho_time(vho_t *h) { return h->t; }

void vho_destroy(vho_t *h)
{
    if (!h) return;
    for (int n = 0; n < h->nq; ++n) { free(h->q[n]); free(h->Q[n]); free(h->qS[n]); }
    free(h->e); free(h->p);
    for (int c = 0; c < 4; ++c) { free(h->u[c]); free(h->up[c]); free(h->uS[c]); }
    for (int s = 0; s < 2; ++s) free(h->slab[s]);
    for (int c = 0; c < 6; ++c) free(h->w[c]);
    for (int c = 0; c < 4; ++c) free(h->src[c]);
    free(h->regfac[0]); free(h->regfac[1]);
    for (int c = 0; c < 4; ++c) free(h->beta[c]);
    free(h->p_tb); free(h->T_tb);
    free(h);
}

/* freezeout (vho_freezeout) lives in cornelius_oracle.c */
double vho_fo_eF(vho_t *h) { return eos_e_of_T(h, h->T_fo_GeV / HBARC); }
double vho_T_of_e(vho_t *h, double ed) { return eos_T(h, ed); }
double vho_p_of_e(vho_t *h, double ed) { return eos_p(h, ed); }

/* state view for the freezeout driver in cornelius_oracle.c */
int vho_fo_view(vho_t *h, int *dims, double *spacing, double *t0dt_t, int *n_next, double **e, double **u,
                double **q, int *nq, double **slabs_prev, double **slabs_cur, double *eF)
{
    dims[0] = h->nx; dims[1] = h->ny; dims[2] = h->nz;
    spacing[0] = h->dt * h->fofac; spacing[1] = h->dx; spacing[2] = h->dy; spacing[3] = h->dz;
    t0dt_t[0] = h->t0; t0dt_t[1] = h->dt; t0dt_t[2] = h->t;
    *n_next = h->n + 1;
    *e = h->e;
    /* u and q planes are separate allocations; expose them through a packed copy */
    size_t L = (size_t)h->ncx * h->ncy * h->ncz;
    static __thread double *pack = NULL;
    static __thread size_t packlen = 0;
    size_t need = (4 + (size_t)h->nq) * L;
    if (packlen < need) { free(pack); pack = (double *)malloc(8 * need); packlen = need; }
    for (int c = 0; c < 4; ++c) memcpy(pack + c * L, h->u[c], 8 * L);
    for (int n = 0; n < h->nq; ++n) memcpy(pack + (4 + n) * L, h->q[n], 8 * L);
    *u = pack;
    *q = pack + 4 * L;
    *nq = h->nq;
    *slabs_prev = h->slab[h->fo_prev];
    *slabs_cur = h->slab[1 - h->fo_prev];
    *eF = eos_e_of_T(h, h->T_fo_GeV / HBARC);
    return 0;
}
void vho_fo_flip(vho_t *h) { h->fo_prev = 1 - h->fo_prev; }

/*
 * workload_gen.c -- TEST INFRASTRUCTURE ONLY: the seeded synthetic workloads
 * (crossover EoS table, optical-Glauber, hotspot and Gubser initial
 * conditions) restated in plain C for the CPU side of the benchmark and the
 * tests, so that the reference's own code (oracle/_ref, which links this
 * file) can be given its inputs without loading the CUDA library.
 *
 * Each function restates, operation for operation and with the same libm
 * calls, the library's host generator of the same name in
 * cpu-vh_b200/host/vh_host.cpp (vh_eos_synthetic_table, vh_ic_glauber,
 * vh_ic_hotspots, vh_ic_gubser); tests/test_host_cpu.py checks that both
 * produce the same bits.  The pressure of a tabulated-EoS initial state is
 * left to the caller's EoS (the generators here return e and u, plus pi for
 * Gubser, whose conformal p = e/3 is returned too).  The longitudinal
 * profile follows InitialConditions.cpp:1046-1063 and the Woods-Saxon
 * thickness GlauberModel.cpp:26-108 (n0 = 0.17 fm^-3).
 *
 * Compiles as C11 (liboracle_vh.so) and as C++ (the oracle/_ref libraries).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VHG_HBARC 0.197326938

/* ------------------------------------------------------ synthetic table */
/* cs^2(T) = 1/3 - dip exp(-((T-Tc)/w)^2), integrated from a conformal gas of
 * factor a at T_lo with RK4 steps of 1e-5 GeV in (ln s, p); rows (e [GeV/fm^3],
 * P [GeV/fm^3], s [fm^-3], T [GeV]) uniform in e up to e_max. */
static double vhg_cs2(double T, double dip, double Tc, double w)
{
    double z = (T - Tc) / w;
    return 1. / 3. - dip * exp(-z * z);
}

int vhg_eos_synthetic_table(int nrows, double T_lo, double e_max_GeV, double a_conf, double dip, double Tc, double w,
                            double *rows)
{
    if (nrows < 2 || !rows || T_lo <= 0) return 1;
    const double hc3 = VHG_HBARC * VHG_HBARC * VHG_HBARC;
    size_t cap = 1 << 16, n = 0;
    double *TT = (double *)malloc(cap * sizeof(double)), *ee = (double *)malloc(cap * sizeof(double));
    double *pp = (double *)malloc(cap * sizeof(double)), *ss = (double *)malloc(cap * sizeof(double));
    double T = T_lo, s = 4. / 3. * a_conf * T_lo * T_lo * T_lo, p = a_conf * T_lo * T_lo * T_lo * T_lo / 3.;
    const double hT = 1e-5;
    double ecur = T * s - p;
    for (;;) {
        if (n == cap) {
            cap *= 2;
            TT = (double *)realloc(TT, cap * sizeof(double));
            ee = (double *)realloc(ee, cap * sizeof(double));
            pp = (double *)realloc(pp, cap * sizeof(double));
            ss = (double *)realloc(ss, cap * sizeof(double));
        }
        TT[n] = T; ss[n] = s; pp[n] = p; ee[n] = ecur; ++n;
        if (ecur / hc3 > e_max_GeV * 1.0001) break;
        double ls = log(s);
        double k1 = 1. / (T * vhg_cs2(T, dip, Tc, w));
        double k2 = 1. / ((T + hT / 2) * vhg_cs2(T + hT / 2, dip, Tc, w));
        double k4 = 1. / ((T + hT) * vhg_cs2(T + hT, dip, Tc, w));
        double ls_new = ls + hT * (k1 + 4 * k2 + k4) / 6.;
        double s_mid = exp(ls + hT * (k1 + k2) / 4.);
        double s_new = exp(ls_new);
        p += hT * (s + 4 * s_mid + s_new) / 6.;
        s = s_new;
        T += hT;
        ecur = T * s - p;
        if (T > 10.0) break;
    }
    const double e_lo = ee[0] / hc3;
    const double de = (e_max_GeV - e_lo) / (nrows - 1);
    size_t m = 0;
    for (int r = 0; r < nrows; ++r) {
        double eg = e_lo + r * de;
        double en = eg * hc3;
        while (m + 2 < n && ee[m + 1] < en) ++m;
        double f = (en - ee[m]) / (ee[m + 1] - ee[m]);
        rows[4 * r + 0] = eg;
        rows[4 * r + 1] = (pp[m] + f * (pp[m + 1] - pp[m])) / hc3;
        rows[4 * r + 2] = (ss[m] + f * (ss[m + 1] - ss[m])) / hc3;
        rows[4 * r + 3] = TT[m] + f * (TT[m + 1] - TT[m]);
    }
    free(TT); free(ee); free(pp); free(ss);
    return 0;
}

/* ------------------------------------------------------------ Glauber */
static double vhg_ws_thickness(double r2, double R, double a)
{
    const double n0 = 0.17;
    const double zmax = R + 15. * a;
    const int nzq = 600;
    const double hz = 2. * zmax / nzq;
    double sum = 0.;
    for (int k = 0; k <= nzq; ++k) {
        double z = -zmax + k * hz;
        double rr = sqrt(r2 + z * z);
        double f = n0 / (1. + exp((rr - R) / a));
        double wgt = (k == 0 || k == nzq) ? 1. : (k % 2 ? 4. : 2.);
        sum += wgt * f;
    }
    return sum * hz / 3.;
}

/* e (fm^-4) of the optical-Glauber event on nx x ny x nz cells, u at rest */
int vhg_ic_glauber(int nx, int ny, int nz, double dx, double dy, double dz, double R, double a, double sigma_nn,
                   double b, double e0_GeV, double eta_flat, double eta_sigma, double *e, double *u)
{
    if (!e || !u || nx < 1 || ny < 1 || nz < 1) return 1;
    const size_t N = (size_t)nx * ny * nz;
    double *npart = (double *)malloc((size_t)nx * ny * sizeof(double));
    double mx = 0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            double x = (i - (nx - 1) / 2.) * dx, y = (j - (ny - 1) / 2.) * dy;
            double TA = vhg_ws_thickness((x + b / 2) * (x + b / 2) + y * y, R, a);
            double TB = vhg_ws_thickness((x - b / 2) * (x - b / 2) + y * y, R, a);
            double np = TA * (1. - exp(-sigma_nn * TB)) + TB * (1. - exp(-sigma_nn * TA));
            npart[i + (size_t)nx * j] = np;
            mx = (mx < np) ? np : mx;
        }
    const double e0 = e0_GeV / VHG_HBARC;
    const double var = eta_sigma * eta_sigma;
    for (int k = 0; k < nz; ++k) {
        double eta = (k - (nz - 1) / 2) * dz;
        double sc = fabs(eta) - eta_flat / 2;
        double L = sc > 0 ? exp(-sc * sc / var / 2) : 1.0;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                size_t m = i + (size_t)nx * (j + (size_t)ny * k);
                e[m] = e0 * (npart[i + (size_t)nx * j] / mx) * L + 1.e-3;
                u[m] = 1.0; u[N + m] = 0.0; u[2 * N + m] = 0.0; u[3 * N + m] = 0.0;
            }
    }
    free(npart);
    return 0;
}

/* ------------------------------------------------------------ hotspots */
/* SplitMix64 keyed by (seed, counter) */
typedef struct { uint64_t key, ctr; } vhg_rng;

static uint64_t vhg_next(vhg_rng *r)
{
    uint64_t z = r->key + 0x9E3779B97F4A7C15ULL * (++r->ctr);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static double vhg_uniform(vhg_rng *r) { return ((vhg_next(r) >> 11) + 0.5) * 0x1p-53; }
static double vhg_normal(vhg_rng *r)
{
    double u1 = vhg_uniform(r), u2 = vhg_uniform(r);
    return sqrt(-2. * log(u1)) * cos(6.283185307179586 * u2);
}
static int vhg_poisson(vhg_rng *r, double mean)
{
    double L = exp(-mean), pk = L, cum = L, x = vhg_uniform(r);
    int k = 0;
    while (x > cum && k < 100000) { ++k; pk *= mean / k; cum += pk; }
    return k;
}
static double vhg_gamma(vhg_rng *r, double k)
{
    double d = k - 1. / 3., c = 1. / sqrt(9. * d);
    for (;;) {
        double xx, v;
        do { xx = vhg_normal(r); v = 1. + c * xx; } while (v <= 0);
        v = v * v * v;
        double uu = vhg_uniform(r);
        if (uu < 1. - 0.0331 * xx * xx * xx * xx) return d * v;
        if (log(uu) < 0.5 * xx * xx + d * (1. - v + log(v))) return d * v;
    }
}

/* e (fm^-4) of the 2+1D hotspot event `seed` on nx x ny cells, u at rest */
int vhg_ic_hotspots(int nx, int ny, double dx, double dy, uint64_t seed, double mean_spots, double w, double k_gamma,
                    double amp_mean_GeV, double R, double a, double *e, double *u)
{
    if (!e || !u || nx < 1 || ny < 1 || k_gamma < 1.0) return 1;
    vhg_rng rng = {seed * 0x9E3779B97F4A7C15ULL + 0x632BE59BD9B4E019ULL, 0};
    const double sigma_nn = 4.2;
    const double box = R + 3. * a;
    const double TA0 = vhg_ws_thickness(0.0, R, a);
    const double wmax = 2. * TA0 * (1. - exp(-sigma_nn * TA0));
    const int nspots = vhg_poisson(&rng, mean_spots);
    double *cx = (double *)calloc((size_t)nspots + 1, sizeof(double));
    double *cy = (double *)calloc((size_t)nspots + 1, sizeof(double));
    double *amp = (double *)calloc((size_t)nspots + 1, sizeof(double));
    for (int s = 0; s < nspots; ++s) {
        for (int tries = 0; tries < 100000; ++tries) {
            double x = (2. * vhg_uniform(&rng) - 1.) * box, y = (2. * vhg_uniform(&rng) - 1.) * box;
            double TA = vhg_ws_thickness(x * x + y * y, R, a);
            double wgt = 2. * TA * (1. - exp(-sigma_nn * TA));
            if (vhg_uniform(&rng) * wmax <= wgt) { cx[s] = x; cy[s] = y; break; }
        }
        amp[s] = amp_mean_GeV / VHG_HBARC * vhg_gamma(&rng, k_gamma) / k_gamma;
    }
    const size_t N = (size_t)nx * ny;
    const double inv2w2 = 1. / (2. * w * w);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            size_t m = i + (size_t)nx * j;
            double x = (i - (nx - 1) / 2.) * dx, y = (j - (ny - 1) / 2.) * dy;
            double ed = 1.e-3;
            for (int s = 0; s < nspots; ++s) {
                double ddx = x - cx[s], ddy = y - cy[s];
                double r2 = ddx * ddx + ddy * ddy;
                if (r2 < 50. * w * w) ed += amp[s] * exp(-r2 * inv2w2);
            }
            e[m] = ed;
            u[m] = 1.0; u[N + m] = 0.0; u[2 * N + m] = 0.0; u[3 * N + m] = 0.0;
        }
    free(cx); free(cy); free(amp);
    return 0;
}

/* -------------------------------------------------------------- Gubser */
static void vhg_gubser_u(double tau, double x, double y, double q, double *ut, double *ux, double *uy)
{
    double r2 = x * x + y * y;
    double den = 1. + q * q * tau * tau + q * q * r2;
    double kap = 2. * q * q * tau / den;
    double vr2 = kap * kap * r2;
    double g = 1. / sqrt(1. - vr2);
    *ut = g; *ux = g * kap * x; *uy = g * kap * y;
}

static double vhg_gubser_shape(double r2, double q, double t)
{
    double sh = (1. - q * q * t * t + q * q * r2) / (2. * q * t);
    return 1. / (t * cbrt(1. + sh * sh));
}

/* ideal Gubser profile at t0 with T(0) = T0 (conformal e = a T^4, p = e/3)
 * and the Navier-Stokes shear stress 2 etabar (e+p)/T sigma^{mu nu} (pi may
 * be null) */
int vhg_ic_gubser(int nx, int ny, double dx, double dy, double t0, double eos_a, double etabar, double q,
                  double T0_GeV, double *e, double *p, double *u, double *pi)
{
    if (!e || !p || !u || nx < 1 || ny < 1) return 1;
    const size_t N = (size_t)nx * ny;
    const double t = t0, a = eos_a;
    const double T0 = T0_GeV / VHG_HBARC;
    const double norm = T0 / vhg_gubser_shape(0.0, q, t);
    const double h = 1e-4;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            size_t m = i + (size_t)nx * j;
            double x = (i - (nx - 1) / 2.) * dx, y = (j - (ny - 1) / 2.) * dy;
            double T = norm * vhg_gubser_shape(x * x + y * y, q, t);
            double ed = a * T * T * T * T;
            double pr = ed / 3.;
            e[m] = ed; p[m] = pr;
            double ut, ux, uy;
            vhg_gubser_u(t, x, y, q, &ut, &ux, &uy);
            u[0 * N + m] = ut; u[1 * N + m] = ux; u[2 * N + m] = uy; u[3 * N + m] = 0.0;
            if (!pi) continue;
            double c[3][3];
            for (int d = 0; d < 3; ++d) {
                double v[4][3];
                const double off[4] = {-2 * h, -h, h, 2 * h};
                for (int o = 0; o < 4; ++o) {
                    double tt = t + (d == 0 ? off[o] : 0), xx = x + (d == 1 ? off[o] : 0), yy = y + (d == 2 ? off[o] : 0);
                    vhg_gubser_u(tt, xx, yy, q, &v[o][0], &v[o][1], &v[o][2]);
                }
                for (int cc = 0; cc < 3; ++cc) c[d][cc] = (v[0][cc] - 8 * v[1][cc] + 8 * v[2][cc] - v[3][cc]) / (12 * h);
            }
            double dtut = c[0][0], dtux = c[0][1], dtuy = c[0][2];
            double dxut = c[1][0], dxux = c[1][1], dxuy = c[1][2];
            double dyut = c[2][0], dyux = c[2][1], dyuy = c[2][2];
            double theta = ut / t + dtut + dxux + dyuy;
            double dut = ut * dtut + ux * dxut + uy * dyut;
            double dux = ut * dtux + ux * dxux + uy * dyux;
            double duy = ut * dtuy + ux * dxuy + uy * dyuy;
            double stt = (dtut - ut * dut) + (ut * ut - 1) * theta / 3.0;
            double stx = (dtux - dxut) / 2.0 - (ux * dut + ut * dux) / 2.0 + ut * ux * theta / 3.0;
            double sty = (dtuy - dyut) / 2.0 - (uy * dut + ut * duy) / 2.0 + ut * uy * theta / 3.0;
            double sxx = -(dxux + ux * dux) + (1.0 + ux * ux) * theta / 3.0;
            double sxy = -(dxuy + dyux) / 2.0 - (uy * dux + ux * duy) / 2.0 + ux * uy * theta / 3.0;
            double syy = -(dyuy + uy * duy) + (1.0 + uy * uy) * theta / 3.0;
            double snn = -ut / (t * t * t) + (1.0 / (t * t)) * theta / 3.0;
            double eta2 = 2. * etabar * (ed + pr) / T;
            double comp[10] = {stt, stx, sty, 0.0, sxx, sxy, 0.0, syy, 0.0, snn};
            for (int cc = 0; cc < 10; ++cc) pi[cc * N + m] = eta2 * comp[cc];
        }
    return 0;
}

#ifdef __cplusplus
}
#endif

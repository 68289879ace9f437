/*
 * vh_host.cpp -- host-side pieces of the C ABI that need no GPU:
 * configuration defaults, the host copy of the reference EoS (for e_F, e_reg
 * and initial pressures), the synthetic crossover EoS table and the seeded
 * initial-condition generators shared by the CUDA path, the oracle tests and
 * the benchmark.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

#include "vh_b200.h"
#include "vh_internal.h"

namespace vh {

/* ------------------------------------------------------------------ EoS */
void HostEos::init(const vh_config &cfg, const double *rows, int nrows)
{
    kind = cfg.eos_kind;
    a = cfg.eos_factor;
    if (kind == VH_EOS_TABLE) {
        /* EquationOfState.cpp:292-327, the loader's unit conversion */
        e_length = nrows;
        p_tb.resize(nrows);
        T_tb.resize(nrows);
        for (int ii = 0; ii < nrows; ++ii) {
            double temp = rows[4 * ii] / kHbarc;
            if (ii == 0) e_min = temp;
            if (ii == 1) e_spacing = temp - e_min;
            if (ii == nrows - 1) e_max = temp;
            p_tb[ii] = rows[4 * ii + 1] / kHbarc;
            T_tb[ii] = rows[4 * ii + 3] / kHbarc;
        }
        cs2_third_hi = cs2_third_bound();
    }
}

/* The table sound speed of the reference, e_spacing / (p(e + e_spacing) -
 * p(e)) clamped to [0.01, 1/3] (EquationOfState.cpp:109-160), is exactly the
 * clamp's 1/3 wherever the computed pressure step dp = p(e + de) - p(e) lies
 * in [0, 3 de): the quotient is then above 1/3 or +inf.  If the pressure
 * column rises with every segment slope in (0, 2.9], the exact step of the
 * interpolation (the last segment extrapolated above the table, the first
 * one below it, both floored at 1e-15, which is monotone) lies in
 * [0, 2.9 de], and the computed one differs from it by the rounding of the
 * interpolation, which grows with e.  This returns the largest e (four table
 * lengths, or the table's end) at which that rounding stays below 1 % of the
 * smallest exact step, or -inf when the table lacks these properties; up to
 * that e the device takes 1/3 without evaluating the expression, with
 * identical results, and evaluates it beyond. */
double HostEos::cs2_third_bound() const
{
    const int N = e_length;
    if (N < 2 || !(e_spacing > 0) || !(p_tb[0] >= 0)) return -INFINITY;
    double smin = INFINITY, smax = -INFINITY, pmax = 0;
    for (int i = 0; i + 1 < N; ++i) {
        const double sl = (p_tb[i + 1] - p_tb[i]) / e_spacing;
        smin = std::min(smin, sl);
        smax = std::max(smax, sl);
    }
    for (int i = 0; i < N; ++i) pmax = std::max(pmax, std::fabs(p_tb[i]));
    if (!(smin > 0) || !(smax <= 2.9) || !std::isfinite(pmax)) return -INFINITY;
    auto ulp = [](double x) { x = std::fabs(x); return std::nextafter(x, INFINITY) - x; };
    for (double lengths : {4.0, 1.0}) {
        const double hi = e_min + lengths * (N - 1) * e_spacing;
        /* |frac| + 1 bounds the interpolation weights for e in [e_min, hi + de];
         * below e_min the pressure is floored long before the weights grow */
        const double w = (hi + e_spacing - e_min) / e_spacing + 2;
        const double M = pmax * 2 * w;                        /* largest product and sum */
        const double err = 2 * (4 * ulp(M) + smax * 2 * ulp(hi + e_spacing)) + ulp(smax * e_spacing);
        if (err <= 0.01 * smin * e_spacing) return hi;
    }
    return -INFINITY;
}

/* EquationOfState.cpp:329-360 */
double HostEos::interp(double ed, const std::vector<double> &tb) const
{
    int idx = (int)((ed - e_min) / e_spacing);
    idx = std::min(e_length - 2, idx);
    idx = std::max(0, idx);
    const double frac = (ed - (idx * e_spacing + e_min)) / e_spacing;
    return tb[idx] * (1. - frac) + tb[idx + 1] * frac;
}

double HostEos::pressure(double ed) const
{
    if (kind == VH_EOS_TABLE) return std::max(1.e-15, interp(ed, p_tb));
    return ed / 3.;
}

double HostEos::cs2(double ed) const
{
    if (kind == VH_EOS_TABLE) {
        double pp = pressure(ed), pr = pressure(ed + e_spacing);
        double v = e_spacing / (pr - pp);
        return std::max(0.01, std::min(1. / 3., v));
    }
    return 1. / 3.;
}

double HostEos::temperature(double ed) const
{
    if (kind == VH_EOS_TABLE) return std::max(1.e-15, interp(ed, T_tb));
    return powf((float)(ed / a), 0.25f);
}

/* EquationOfState.cpp:201-290 */
double HostEos::energy_of_T(double T) const
{
    if (kind == VH_EOS_TABLE) {
        double lo = 1e-15, hi = e_max, mid = (hi + lo) / 2.;
        if (T < temperature(lo)) return lo;
        int iter = 0;
        while (((hi - lo) / mid > 1e-8 && (hi - lo) > 1e-15) && iter < 1000) {
            if (T < temperature(mid)) hi = mid; else lo = mid;
            mid = (hi + lo) / 2.;
            ++iter;
        }
        return mid;
    }
    return a * (double)powf((float)T, 4.0f);
}

} // namespace vh

using vh::kHbarc;

extern "C" {

int vh_config_default(vh_config *cfg)
{
    if (!cfg) return VH_ERR_ARG;
    std::memset(cfg, 0, sizeof(*cfg));
    /* rhic-conf/lattice.properties and hydro.properties as shipped */
    cfg->nx = 101; cfg->ny = 101; cfg->nz = 1;
    cfg->dx = 0.2; cfg->dy = 0.2; cfg->dz = 0.1; cfg->dt = 0.05;
    cfg->t0 = 0.5; cfg->etabar = 0.2; cfg->T_freezeout_GeV = 0.155; cfg->T_reg_GeV = 0.1;
    cfg->fo_factor = 2;
    /* compile-time macros: FluxLimiter.h:13, EquationOfState.h:13,19, DynamicalVariables.h:13-14 */
    cfg->theta = 1.1;
    cfg->eos_kind = VH_EOS_CONFORMAL; cfg->eos_factor = 13.8997;
    cfg->bulk = 0;
    cfg->zeta_law = VH_ZETA_REFERENCE;
    cfg->precision = VH_PREC_FP64;
    return VH_OK;
}

int vh_config_nq(const vh_config *cfg) { return cfg && cfg->bulk ? 15 : 14; }

double vh_eos_eval(const vh_config *cfg, const double *rows, int nrows, int what, double x)
{
    vh::HostEos eos;
    eos.init(*cfg, rows, nrows);
    switch (what) {
    case 0: return eos.pressure(x);
    case 1: return eos.cs2(x);
    case 2: return eos.temperature(x);
    case 4: return eos.kind == VH_EOS_TABLE ? eos.cs2_third_hi : -INFINITY;
    default: return eos.energy_of_T(x);
    }
}

int vh_eos_synthetic_table(int nrows, double T_lo, double e_max_GeV, double a_conf,
                           double dip, double Tc, double w, double *rows)
{
    if (nrows < 2 || !rows || T_lo <= 0) return VH_ERR_ARG;
    const double hc3 = kHbarc * kHbarc * kHbarc;
    /* integrate d ln s / dT = 1/(T cs^2) from a conformal gas of factor a at T_lo
     * (natural units: T [GeV], s [GeV^3], p and e [GeV^4]) */
    auto cs2 = [&](double T) { double z = (T - Tc) / w; return 1. / 3. - dip * std::exp(-z * z); };
    std::vector<double> TT, ee, pp, ss;
    double T = T_lo, s = 4. / 3. * a_conf * T_lo * T_lo * T_lo, p = a_conf * T_lo * T_lo * T_lo * T_lo / 3.;
    const double hT = 1e-5;
    double ecur = T * s - p;
    while (true) {
        TT.push_back(T); ss.push_back(s); pp.push_back(p); ee.push_back(ecur);
        if (ecur / hc3 > e_max_GeV * 1.0001) break;
        /* RK4 on (ln s, p) */
        auto f = [&](double Tv) { return 1. / (Tv * cs2(Tv)); };
        double ls = std::log(s);
        double k1 = f(T), k2 = f(T + hT / 2), k4 = f(T + hT);
        double ls_new = ls + hT * (k1 + 4 * k2 + k4) / 6.;
        double s_mid = std::exp(ls + hT * (k1 + k2) / 4.);  /* approximate midpoint value */
        double s_new = std::exp(ls_new);
        p += hT * (s + 4 * s_mid + s_new) / 6.;
        s = s_new;
        T += hT;
        ecur = T * s - p;
        if (T > 10.0) break;
    }
    const double e_lo = ee.front() / hc3;
    const double de = (e_max_GeV - e_lo) / (nrows - 1);
    size_t m = 0;
    for (int r = 0; r < nrows; ++r) {
        double eg = e_lo + r * de;          /* GeV/fm^3 */
        double en = eg * hc3;               /* GeV^4 */
        while (m + 2 < ee.size() && ee[m + 1] < en) ++m;
        double f = (en - ee[m]) / (ee[m + 1] - ee[m]);
        double Tr = TT[m] + f * (TT[m + 1] - TT[m]);
        double pr = pp[m] + f * (pp[m + 1] - pp[m]);
        double sr = ss[m] + f * (ss[m + 1] - ss[m]);
        rows[4 * r + 0] = eg;
        rows[4 * r + 1] = pr / hc3;
        rows[4 * r + 2] = sr / hc3;
        rows[4 * r + 3] = Tr;
    }
    return VH_OK;
}

/* ----------------------------------------------------------- Gubser IC */
/* Ideal Gubser profile (the shape InitialConditions.cpp:1146-1194 uses, there
 * for t0 = q = 1) at proper time t0 with T(0) = T0, and the Navier-Stokes shear
 * stress 2 eta sigma^{mu nu} with eta = etabar (e+p)/T.  sigma^{mu nu} is
 * assembled with the same component formulas as the reference's relaxation
 * equation (SourceTerms.cpp:98-128) from the analytic velocity field, whose
 * derivatives are taken by fourth-order central differences. */
static void gubser_u(double tau, double x, double y, double q, double *ut, double *ux, double *uy)
{
    double r2 = x * x + y * y;
    double den = 1. + q * q * tau * tau + q * q * r2;
    double kap = 2. * q * q * tau / den;   /* v_r / r */
    double vr2 = kap * kap * r2;
    double g = 1. / std::sqrt(1. - vr2);
    *ut = g; *ux = g * kap * x; *uy = g * kap * y;
}

int vh_ic_gubser(const vh_config *cfg, double q, double T0_GeV, double *e, double *p, double *u, double *pi)
{
    if (!cfg || !e || !p || !u || cfg->nz != 1) return VH_ERR_ARG;
    const int nx = cfg->nx, ny = cfg->ny;
    const size_t N = (size_t)nx * ny;
    const double t = cfg->t0, a = cfg->eos_factor;
    const double T0 = T0_GeV / kHbarc;
    auto shape = [&](double r2) {
        double sh = (1. - q * q * t * t + q * q * r2) / (2. * q * t);
        return 1. / (t * std::cbrt(1. + sh * sh));
    };
    const double norm = T0 / shape(0.0);
    const double h = 1e-4;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            size_t m = i + (size_t)nx * j;
            double x = (i - (nx - 1) / 2.) * cfg->dx, y = (j - (ny - 1) / 2.) * cfg->dy;
            double T = norm * shape(x * x + y * y);
            double ed = a * T * T * T * T;
            double pr = ed / 3.;
            e[m] = ed; p[m] = pr;
            double ut, ux, uy;
            gubser_u(t, x, y, q, &ut, &ux, &uy);
            u[0 * N + m] = ut; u[1 * N + m] = ux; u[2 * N + m] = uy; u[3 * N + m] = 0.0;
            if (!pi) continue;
            /* 4th-order central differences of the analytic field */
            double c[3][3];  /* [derivative dir t,x,y][component ut,ux,uy] */
            for (int d = 0; d < 3; ++d) {
                double v[4][3];
                const double off[4] = {-2 * h, -h, h, 2 * h};
                for (int o = 0; o < 4; ++o) {
                    double tt = t + (d == 0 ? off[o] : 0), xx = x + (d == 1 ? off[o] : 0), yy = y + (d == 2 ? off[o] : 0);
                    gubser_u(tt, xx, yy, q, &v[o][0], &v[o][1], &v[o][2]);
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
            double eta2 = 2. * cfg->etabar * (ed + pr) / T;
            double comp[10] = {stt, stx, sty, 0.0, sxx, sxy, 0.0, syy, 0.0, snn};
            for (int cc = 0; cc < 10; ++cc) pi[cc * N + m] = eta2 * comp[cc];
        }
    return VH_OK;
}

/* ---------------------------------------------------------- Glauber IC */
static double ws_thickness(double r2, double R, double a)
{
    const double n0 = 0.17;
    const double zmax = R + 15. * a;
    const int nzq = 600;   /* Simpson, even number of intervals */
    const double hz = 2. * zmax / nzq;
    double sum = 0.;
    for (int k = 0; k <= nzq; ++k) {
        double z = -zmax + k * hz;
        double rr = std::sqrt(r2 + z * z);
        double f = n0 / (1. + std::exp((rr - R) / a));
        double wgt = (k == 0 || k == nzq) ? 1. : (k % 2 ? 4. : 2.);
        sum += wgt * f;
    }
    return sum * hz / 3.;
}

int vh_ic_glauber(const vh_config *cfg, const double *rows, int nrows,
                  double R, double a, double sigma_nn, double b, double e0_GeV,
                  double eta_flat, double eta_sigma, double *e, double *p, double *u)
{
    if (!cfg || !e || !p || !u) return VH_ERR_ARG;
    vh::HostEos eos;
    eos.init(*cfg, rows, nrows);
    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz;
    const size_t N = (size_t)nx * ny * nz;
    std::vector<double> npart((size_t)nx * ny);
    double mx = 0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            double x = (i - (nx - 1) / 2.) * cfg->dx, y = (j - (ny - 1) / 2.) * cfg->dy;
            double TA = ws_thickness((x + b / 2) * (x + b / 2) + y * y, R, a);
            double TB = ws_thickness((x - b / 2) * (x - b / 2) + y * y, R, a);
            double np = TA * (1. - std::exp(-sigma_nn * TB)) + TB * (1. - std::exp(-sigma_nn * TA));
            npart[i + (size_t)nx * j] = np;
            mx = std::max(mx, np);
        }
    const double e0 = e0_GeV / kHbarc;
    const double var = eta_sigma * eta_sigma;
    for (int k = 0; k < nz; ++k) {
        /* InitialConditions.cpp:1046-1063 (integer (nz-1)/2 as there) */
        double eta = (k - (nz - 1) / 2) * cfg->dz;
        double sc = std::fabs(eta) - eta_flat / 2;
        double L = sc > 0 ? std::exp(-sc * sc / var / 2) : 1.0;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                size_t m = i + (size_t)nx * (j + (size_t)ny * k);
                double ed = e0 * (npart[i + (size_t)nx * j] / mx) * L + 1.e-3;
                e[m] = ed;
                p[m] = eos.pressure(ed);
                u[m] = 1.0; u[N + m] = 0.0; u[2 * N + m] = 0.0; u[3 * N + m] = 0.0;
            }
    }
    return VH_OK;
}

/* --------------------------------------------------------- hotspot IC */
/* SplitMix64 keyed by (seed, counter): a counter-based stream, so event `seed`
 * draws the same numbers whatever else runs. */
struct CounterRng {
    uint64_t key, ctr = 0;
    explicit CounterRng(uint64_t s) : key(s * 0x9E3779B97F4A7C15ULL + 0x632BE59BD9B4E019ULL) {}
    uint64_t next()
    {
        uint64_t z = key + 0x9E3779B97F4A7C15ULL * (++ctr);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    double uniform() { return ((next() >> 11) + 0.5) * 0x1p-53; }
    double normal() { double u1 = uniform(), u2 = uniform(); return std::sqrt(-2. * std::log(u1)) * std::cos(6.283185307179586 * u2); }
    int poisson(double mean)
    {   /* inversion by sequential search */
        double L = std::exp(-mean), pk = L, cum = L, x = uniform();
        int k = 0;
        while (x > cum && k < 100000) { ++k; pk *= mean / k; cum += pk; }
        return k;
    }
    double gamma(double k)
    {   /* Marsaglia-Tsang; k >= 1 */
        double d = k - 1. / 3., c = 1. / std::sqrt(9. * d);
        for (;;) {
            double xx, v;
            do { xx = normal(); v = 1. + c * xx; } while (v <= 0);
            v = v * v * v;
            double uu = uniform();
            if (uu < 1. - 0.0331 * xx * xx * xx * xx) return d * v;
            if (std::log(uu) < 0.5 * xx * xx + d * (1. - v + std::log(v))) return d * v;
        }
    }
};

} /* extern "C" */

/* The random part of the hotspot initial condition: Poisson(mean_spots)
 * centres accepted with the b = 0 Woods-Saxon participant density, Gamma(k)
 * amplitudes scaled to a mean of amp_mean_GeV; shared by the host generator
 * and the device one (vh_event_init_hotspots). */
void vh::draw_hotspots(uint64_t seed, double mean_spots, double k_gamma, double amp_mean_GeV, double R, double a,
                       std::vector<double> &cx, std::vector<double> &cy, std::vector<double> &amp)
{
    CounterRng rng(seed);
    const double sigma_nn = 4.2;
    const double box = R + 3. * a;
    const double TA0 = ws_thickness(0.0, R, a);
    const double wmax = 2. * TA0 * (1. - std::exp(-sigma_nn * TA0));
    int nspots = rng.poisson(mean_spots);
    cx.assign(nspots, 0.0);
    cy.assign(nspots, 0.0);
    amp.assign(nspots, 0.0);
    for (int s = 0; s < nspots; ++s) {
        for (int tries = 0; tries < 100000; ++tries) {
            double x = (2. * rng.uniform() - 1.) * box, y = (2. * rng.uniform() - 1.) * box;
            double TA = ws_thickness(x * x + y * y, R, a);
            double wgt = 2. * TA * (1. - std::exp(-sigma_nn * TA));
            if (rng.uniform() * wmax <= wgt) { cx[s] = x; cy[s] = y; break; }
        }
        amp[s] = amp_mean_GeV / kHbarc * rng.gamma(k_gamma) / k_gamma;
    }
}

extern "C" {

int vh_ic_hotspots(const vh_config *cfg, const double *rows, int nrows, uint64_t seed, double mean_spots,
                   double w, double k_gamma, double amp_mean_GeV, double R, double a,
                   double *e, double *p, double *u)
{
    if (!cfg || !e || !p || !u || cfg->nz != 1 || k_gamma < 1.0) return VH_ERR_ARG;
    vh::HostEos eos;
    eos.init(*cfg, rows, nrows);
    std::vector<double> cx, cy, amp;
    vh::draw_hotspots(seed, mean_spots, k_gamma, amp_mean_GeV, R, a, cx, cy, amp);
    const int nspots = (int)cx.size();
    const int nx = cfg->nx, ny = cfg->ny;
    const size_t N = (size_t)nx * ny;
    const double inv2w2 = 1. / (2. * w * w);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            size_t m = i + (size_t)nx * j;
            double x = (i - (nx - 1) / 2.) * cfg->dx, y = (j - (ny - 1) / 2.) * cfg->dy;
            double ed = 1.e-3;
            for (int s = 0; s < nspots; ++s) {
                double dx = x - cx[s], dy = y - cy[s];
                double r2 = dx * dx + dy * dy;
                if (r2 < 50. * w * w) ed += amp[s] * std::exp(-r2 * inv2w2);
            }
            e[m] = ed;
            p[m] = eos.pressure(ed);
            u[m] = 1.0; u[N + m] = 0.0; u[2 * N + m] = 0.0; u[3 * N + m] = 0.0;
        }
    return VH_OK;
}

} /* extern "C" */

/*
 * vh_physics.cuh -- per-cell device physics of the KT RK2 step, in FP64 and in
 * the reference's floating-point operation order (the library is compiled
 * with --fmad=false, so nothing below is fused unless written as fma()).
 *
 * Each function names the reference code it reproduces (file:line in
 * derekeverett/cpu-vh).  The state lives in padded SoA arrays (stride L
 * doubles between components) indexed i + ncx*(j + ncy*k).
 */
#ifndef VH_PHYSICS_CUH
#define VH_PHYSICS_CUH

#include "vh_math.cuh"

namespace vh {

/* error codes raised on the device (match VH_ERR_* in vh_b200.h) */
constexpr int kErrNan = 4;

struct DevEos {
    int kind;                 /* 0 conformal, 1 table */
    double a;                 /* conformal e = a T^4 */
    const double *p_tb;       /* tabulated P(e) [fm^-4] */
    const double *T_tb;       /* tabulated T(e) [fm^-1] */
    int e_length;
    double e_min, e_spacing;
    double inv_spacing;       /* RN(1/e_spacing), for div_rcp */
    double cs2_third_hi;      /* eos_cs2 is exactly 1/3 for e <= this (HostEos::cs2_third_bound) */
    PowfTab pq;               /* host-exact powf(x, 0.25) */
    const int *stop;          /* the event's device error code (or null): see e_bisect_table */
};

struct DevErr {
    int *code;                /* first error code, 0 if none */
    long long *cell;          /* padded index of the first failing cell */
    int *step;                /* step counter at the time */
};

__device__ __forceinline__ void raise_error(const DevErr &E, int code, long long cell, int step)
{
    if (atomicCAS(E.code, 0, code) == 0) { *E.cell = cell; *E.step = step; }
}

/* ---------------------------------------------- division, shared divisor */
/* IEEE a/b, kept out of line: the fallback of div_rcp */
static __device__ __noinline__ double div_ieee(double a, double b) { return a / b; }

/* The correctly rounded quotient a/b given y = RN(1/b), by Markstein's
 * theorem (P. Markstein, IBM J. Res. Dev. 34(1), 1990; Muller et al.,
 * Handbook of Floating-Point Arithmetic, ch. 4): q0 = RN(a*y) is within one
 * ulp of a/b, r = a - q0*b is exact with an FMA, and RN(q0 + r*y) = RN(a/b).
 * One reciprocal then serves every division by the same b at the cost of a
 * multiply and two FMAs each -- bit-identical to `a / b`.  The range test
 * (|a|, |y| >= 2^-960 and 2^-960 <= |q0| < 2^1000) reads the high words
 * with integer operations.  A zero numerator over a finite b gives q0 = a * y =
 * +-0 with the sign of a XOR the sign of b, which is a / b exactly (zero
 * numerators are common: velocity and viscous components that are still
 * exactly 0).  Non-finite, huge or near-subnormal operands, where the
 * exactness argument needs more care, take the IEEE division. */
__device__ __forceinline__ double div_rcp(double a, double b, double y)
{
    constexpr unsigned kLo = 0x03f00000u;      /* high word of 2^-960 */
    constexpr unsigned kHi = 0x7e700000u;      /* high word of 2^1000 */
    const double q0 = a * y;
    const unsigned ha = (unsigned)__double2hiint(a) & 0x7fffffffu;
    const unsigned hq = (unsigned)__double2hiint(q0) & 0x7fffffffu;
    const unsigned hy = (unsigned)__double2hiint(y) & 0x7fffffffu;
    if (ha >= kLo && hq >= kLo && hq < kHi && hy >= kLo) {
        const double r = fma(-q0, b, a);
        return fma(r, y, q0);
    }
    if ((ha | (unsigned)__double2loint(a)) == 0u && hq < 0x7ff00000u) return q0;
    return div_ieee(a, b);
}

/* ------------------------------------------------------------------ EoS */
/* EquationOfState.cpp:329-360 */
__device__ __forceinline__ double eos_interp(const DevEos &E, double ed, const double *tb)
{
    int idx = (int)div_rcp(ed - E.e_min, E.e_spacing, E.inv_spacing);
    idx = (E.e_length - 2 < idx) ? E.e_length - 2 : idx;   /* std::min(N_e - 2, idx) */
    idx = (idx < 0) ? 0 : idx;                              /* std::max(0, idx)       */
    const double frac = div_rcp(ed - (idx * E.e_spacing + E.e_min), E.e_spacing, E.inv_spacing);
    return __ldg(tb + idx) * (1. - frac) + __ldg(tb + idx + 1) * frac;
}
/* std::max(1.e-15, f): (1e-15 < f) ? f : 1e-15 */
__device__ __forceinline__ double floor15(double f) { return (1.e-15 < f) ? f : 1.e-15; }

template <int EOS>
__device__ __forceinline__ double eos_p(const DevEos &E, double ed)          /* EquationOfState.cpp:44-107 */
{
    if (EOS == 1) return floor15(eos_interp(E, ed, E.p_tb));
    return ed / 3.;
}
template <int EOS>
__device__ __forceinline__ double eos_cs2(const DevEos &E, double ed)        /* EquationOfState.cpp:109-160 */
{
    if (EOS == 1) {
        const double v_min = 0.01, v_max = 1. / 3.;
        if (ed <= E.cs2_third_hi) return v_max;    /* the clamp's value, proven for this table */
        double pp = eos_p<1>(E, ed);
        double p_r = eos_p<1>(E, ed + E.e_spacing);
        double v = E.e_spacing / (p_r - pp);
        v = (v < v_max) ? v : v_max;            /* std::min(v_max, v) */
        return (v_min < v) ? v : v_min;         /* std::max(v_min, v) */
    }
    return 1. / 3.;
}
template <int EOS>
__device__ __forceinline__ double eos_T(const DevEos &E, double ed)          /* EquationOfState.cpp:162-199 */
{
    if (EOS == 1) return floor15(eos_interp(E, ed, E.T_tb));
    return (double)powf_quarter(__double2float_rn(ed / E.a), E.pq);
}

/* --------------------------------------------------------- limiter */
/* FluxLimiter.cpp:14-32, generalised minmod with sign(0) = +1:
 * (sign(x) + sign(y)) * min(|x|, |y|) / 2, evaluated without the integer
 * sum and its conversion.  The factor is +-2 or 0, and 2m / 2 = m exactly
 * for m = min(|x|, |y|) below 2^1023 (no overflow in 2m), so the result is
 * +-m when the signs agree and 0 * m (+0, or NaN for m = inf) when they
 * differ -- the same value, sign of zero and NaN cases included. */
__device__ __forceinline__ double minmod(double x, double y)
{
    const bool nx = x < 0, ny = y < 0;
    const double m = fmin(fabs(x), fabs(y));
    return (nx == ny) ? (nx ? -m : m) : 0.0 * m;
}
__device__ __forceinline__ double approx_deriv(double th, double x, double y, double z)
{
    double l = th * (y - x);
    double c = (z - x) / 2.0;
    double r = th * (z - y);
    return minmod(l, minmod(c, r));
}

/* -------------------------------------------------------- inversion */
/* EnergyMomentumTensor.cpp:48-111: the bisection the tabulated-EoS root solve
 * falls back to when Newton has not converged in 10^4 iterations.  Out of
 * line: no valid state here reaches it, and every caller shares one copy.
 * Once the event's device has flagged an error, the bisection gives up after
 * 64 iterations: the state is then invalid (the reference exits at its first
 * NaN), and the cells of a garbage state would each spend its 10^6
 * iterations before the host reads the error.  The flag is read through L2
 * (another block may have just set it). */
static __device__ __noinline__ double e_bisect_table(const DevEos &E, double ePrev, double M0, double M, double Pi)
{
    double e_lo = 0.0, e_mid = ePrev, e_hi = 2.0 * (ePrev + 1.0);
    for (int j = 0; j < 1000000; ++j) {                            /* MAX_ITERS_BI */
        if ((j & 63) == 63 && E.stop && *(const volatile int *)E.stop != 0) return ePrev;
        double p_lo = eos_p<1>(E, e_lo), p_mid = eos_p<1>(E, e_mid), p_hi = eos_p<1>(E, e_hi);
        double c_lo = p_lo / e_lo, c_mid = p_mid / e_mid, c_hi = p_hi / e_hi;
        double A_lo = M0 * (1.0 - c_lo) + Pi, A_mid = M0 * (1.0 - c_mid) + Pi, A_hi = M0 * (1.0 - c_hi) + Pi;
        double B = M0 * (M0 + Pi) - M;
        double H_lo = (double)sqrtf(fabsf(__double2float_rn(A_lo * A_lo + 4 * c_lo * B)));
        double H_mid = (double)sqrtf(fabsf(__double2float_rn(A_mid * A_mid + 4 * c_mid * B)));
        double H_hi = (double)sqrtf(fabsf(__double2float_rn(A_hi * A_hi + 4 * c_hi * B)));
        double f_lo = e_lo + (A_lo - H_lo) / (2 * c_lo);
        double f_mid = e_mid + (A_mid - H_mid) / (2 * c_mid);
        double f_hi = e_hi + (A_hi - H_hi) / (2 * c_hi);
        if ((e_hi - e_lo) < (1.0e-3 * e_hi) / 2.0) return e_mid;
        if (f_lo * f_mid < 0.0) { e_hi = e_mid; e_mid = (e_lo + e_hi) / 2.0; }
        else if (f_mid * f_hi < 0.0) { e_lo = e_mid; e_mid = (e_lo + e_hi) / 2.0; }
    }
    return ePrev;
}

/* One Newton iteration of EnergyMomentumTensor.cpp:22-44 from e0: the next
 * iterate, whether f/f' is NaN, and whether the float-truncated convergence
 * test (:41) passes. */
__device__ __forceinline__ double e_newton_iter(const DevEos &E, double e0, double M0, double M, double Pi,
                                                bool &nan_step, bool &conv)
{
    double pp = eos_p<1>(E, e0);
    double cs2 = eos_cs2<1>(E, e0);
    double cst2 = pp / e0;
    double A = M0 * (1.0 - cst2) + Pi;
    double B = M0 * (M0 + Pi) - M;
    double H = (double)sqrtf(fabsf(__double2float_rn(A * A + 4 * cst2 * B)));
    double D = (A - H) / (2 * cst2);
    double f = e0 + D;
    double fp = 1.0 - ((cs2 - cst2) * (B + D * H - ((cs2 - cst2) * cst2 * D * M0) / e0)) / (cst2 * e0 * H);
    double q = f / fp;
    double e = e0 - q;
    nan_step = isnan(q);
    conv = (double)fabsf(__double2float_rn(e - e0)) <= 1.0e-3 * (double)fabsf(__double2float_rn(e));
    return e;
}

/* EnergyMomentumTensor.cpp:22-111, the tabulated-EoS root solve: Newton from
 * ePrev, bisection if Newton does not converge. */
__device__ __forceinline__ double e_newton_table_body(const DevEos &E, double ePrev, double M0, double M, double Pi, bool &bad)
{
    double e0 = ePrev;
    for (int j = 0; j < 10000; ++j) {                              /* MAX_ITERS_NR */
        bool nan_step, conv;
        double e = e_newton_iter(E, e0, M0, M, Pi, nan_step, conv);
        if (nan_step) { bad = true; return ePrev; }
        if (conv) return e;
        e0 = e;
    }
    return e_bisect_table(E, ePrev, M0, M, Pi);
}

/* The root solve as a call (one copy of the loop for a long kernel whose
 * instruction footprint matters) or inlined (short phase kernels). */
static __device__ __noinline__ double e_newton_table(const DevEos &E, double ePrev, double M0, double M, double Pi, bool &bad)
{
    return e_newton_table_body(E, ePrev, M0, M, Pi, bad);
}

/* EnergyMomentumTensor.cpp:22-115: energy density from M0, M, Pi; the
 * conformal closed form (:113) truncates through float. */
template <int EOS, bool INL = false>
__device__ __forceinline__ double e_from_conserved(const DevEos &E, double ePrev, double M0, double M, double Pi, bool &bad)
{
    if (EOS == 0) {
        float h = sqrtf(fabsf(__double2float_rn(4 * M0 * M0 - 3 * M)));
        return (double)fabsf(__double2float_rn((double)h - M0));
    }
    if (INL) return e_newton_table_body(E, ePrev, M0, M, Pi, bad);
    return e_newton_table(E, ePrev, M0, M, Pi, bad);
}

struct Prim { double e, p, ut, ux, uy, un; };

/* EnergyMomentumTensor.cpp:117-233, from the five combinations it uses
 * (M0 = ttt - pitt, M1..M3 = tt^i - pit^i, Pi). */
template <int EOS, bool INL = false>
__device__ __forceinline__ Prim infer(const DevEos &E, double t, double M0, double M1, double M2, double M3,
                                      double Pi, double ePrev, bool &bad)
{
    Prim r;
    double M = M1 * M1 + M2 * M2 + t * t * M3 * M3;
    if (ePrev <= 0.1) r.e = M0 - M / M0;
    else r.e = e_from_conserved<EOS, INL>(E, ePrev, M0, M, Pi, bad);
    if (isnan(r.e)) bad = true;
    r.p = eos_p<EOS>(E, r.e);
    if (r.e < 1.e-7) { r.e = 1.e-7; r.p = 1.e-7; }
    double P = r.p + Pi;
    double Einv = 1.0 / (r.e + P);
    r.ut = (double)sqrtf(fabsf(__double2float_rn((M0 + P) * Einv)));
    double E2 = Einv / r.ut;
    r.ux = M1 * E2;
    r.uy = M2 * E2;
    r.un = M3 * E2;
    if (r.ut > 1.0e3) { r.ut = 1.0; r.ux = 0.0; r.uy = 0.0; r.un = 0.0; }
    return r;
}

/* --------------------------------------------------- bulk viscosity */
struct Zeta { int law; double norm, T0, w; };

/* SourceTerms.cpp:40-48 (T in fm^-1) or a Gaussian in T [GeV] */
__device__ __forceinline__ double zeta_over_s(const Zeta &Z, double T)
{
    if (Z.law == 1) {
        double z = (T * 0.197326938 - Z.T0) / Z.w;
        return Z.norm * exp(-(z * z));
    }
    double x = T / 1.01355;
    if (x > 1.05) return 0.9 * exp(-(x - 1) / 0.025) + 0.25 * exp(-(x - 1) / 0.13) + 0.001;
    else if (x < 0.995) return 0.9 * exp((x - 1) / 0.0025) + 0.22 * exp((x - 1) / 0.022) + 0.03;
    return -13.77 * x * x + 27.55 * x - 13.45;
}

/* a / b with y = RN(1/b): exact (div_rcp) in FP64, a * y in FP32 */
__device__ __forceinline__ double dvr(double a, double b, double y) { return div_rcp(a, b, y); }
__device__ __forceinline__ float dvr(float a, float, float y) { return a * y; }

/* SourceTerms.cpp:55-313, the right-hand side of the pi^{mu nu} (and Pi)
 * relaxation equations divided by u^tau.  yt = RN(1/t); every division by
 * t, 2t, t^2 and 5 goes through the shared reciprocal (dvr: the same
 * quotient in FP64, a product in FP32). */
template <typename R, int EOS, bool BULK>
__device__ void pimunu_rhs(const DevEos &E, const Zeta &Z, R *rhs, R t, R yt, double e_d, double p_d,
    double ut_d, double ux_d, double uy_d, double un_d, double utp, double uxp, double uyp, double unp,
    const R *pv, R Pi,
    R dxut, R dyut, R dnut, R dxux, R dyux, R dnux,
    R dxuy, R dyuy, R dnuy, R dxun, R dyun, R dnun, R dkvk,
    R d_etabar, R d_dt)
{
    const R ut = R(ut_d), ux = R(ux_d), uy = R(uy_d), un = R(un_d), e = R(e_d), p = R(p_d);
    const R delta_pipi = R(1.33333), tau_pipi = R(1.42857), delta_PiPi = R(0.666667), lambda_piPi = R(1.2);
    const R pitt = pv[0], pitx = pv[1], pity = pv[2], pitn = pv[3], pixx = pv[4];
    const R pixy = pv[5], pixn = pv[6], piyy = pv[7], piyn = pv[8], pinn = pv[9];
    R T = R(eos_T<EOS>(E, e_d));
    R taupiInv = T / 5 / d_etabar;
    R beta_pi = dvr(e + p, R(5), R(0.2));
    R cs2 = R(eos_cs2<EOS>(E, e_d));
    R a = R(1.0) / R(3.0) - cs2;
    R a2 = a * a;
    R beta_Pi = 15 * a2 * (e + p);
    R lambda_Pipi = dvr(8 * a, R(5), R(0.2));
    R tauPiInv = R(0.0);
    /* in FP64 for both precisions: zeta/s underflows FP32 far from its peak
     * while a2 = 0 for both EoS kinds, and 0/0 must not appear */
    if (BULK) tauPiInv = R(15 * double(a2) * double(T) / zeta_over_s(Z, double(T)));
    R ut2 = ut * ut, un2 = un * un, t2 = t * t, t3 = t * t2;
    const R yt2 = R(1.0) / t2, y2t = yt * R(0.5);   /* RN(1/t^2); RN(1/(2t)) = RN(1/t) / 2 */
    const R kThird = R(1.0) / R(3.0), yut = R(1.0) / ut, ydt = R(1.0) / d_dt;
    R dtut = dvr(R(ut_d - utp), d_dt, ydt), dtux = dvr(R(ux_d - uxp), d_dt, ydt), dtuy = dvr(R(uy_d - uyp), d_dt, ydt), dtun = dvr(R(un_d - unp), d_dt, ydt);
    R Dut = ut * dtut + ux * dxut + uy * dyut + un * dnut + t * un * un;
    R DuxUpper = ut * dtux + ux * dxux + uy * dyux + un * dnux;
    R Dux = -DuxUpper;
    R DuyUpper = ut * dtuy + ux * dxuy + uy * dyuy + un * dnuy;
    R Duy = -DuyUpper;
    R DunUpper = ut * dtun + ux * dxun + uy * dyun + un * dnun + dvr(2 * ut * un, t, yt);
    R Dun = -t2 * DunUpper;
    R dut = Dut - t * un * un;
    R dux = ut * dtux + ux * dxux + uy * dyux + un * dnux;
    R duy = ut * dtuy + ux * dxuy + uy * dyuy + un * dnuy;
    R dun = ut * dtun + ux * dxun + uy * dyun + un * dnun;
    R theta = dvr(ut, t, yt) + dtut + dxux + dyuy + dnun;
    R stt = -t * ut * un2 + (dtut - ut * dut) + dvr((ut2 - 1) * theta, R(3.0), kThird);
    R stx = -(t * un2 * ux) / R(2.0) + (dtux - dxut) / R(2.0) - (ux * dut + ut * dux) / R(2.0) + dvr(ut * ux * theta, R(3.0), kThird);
    R sty = -(t * un2 * uy) / R(2.0) + (dtuy - dyut) / R(2.0) - (uy * dut + ut * duy) / R(2.0) + dvr(ut * uy * theta, R(3.0), kThird);
    R stn = dvr(-un * (R(2.0) * ut2 + t2 * un2), R(2.0) * t, y2t) + (dtun - dvr(dnut, t2, yt2)) / R(2.0) - (un * dut + ut * dun) / R(2.0) + dvr(ut * un * theta, R(3.0), kThird);
    R sxx = -(dxux + ux * dux) + dvr((R(1.0) + ux * ux) * theta, R(3.0), kThird);
    R sxy = -(dxuy + dyux) / R(2.0) - (uy * dux + ux * duy) / R(2.0) + dvr(ux * uy * theta, R(3.0), kThird);
    R sxn = dvr(-ut * ux * un, t, yt) - (dxun + dvr(dnux, t2, yt2)) / R(2.0) - (un * dux + ux * dun) / R(2.0) + dvr(ux * un * theta, R(3.0), kThird);
    R syy = -(dyuy + uy * duy) + dvr((R(1.0) + uy * uy) * theta, R(3.0), kThird);
    R syn = dvr(-ut * uy * un, t, yt) - (dyun + dvr(dnuy, t2, yt2)) / R(2.0) - (un * duy + uy * dun) / R(2.0) + dvr(uy * un * theta, R(3.0), kThird);
    R snn = -ut * (R(1.0) + R(2.0) * t2 * un2) / t3 - dvr(dnun, t2, yt2) - un * dun + dvr((yt2 + un2) * theta, R(3.0), kThird);
    R wtx = (-dtux - dxut + ut * dux - ux * dut - t * un2 * ux) / R(2.0);
    R wty = (-dtuy - dyut + ut * duy - uy * dut - t * un2 * uy) / R(2.0);
    R wtn = (-t2 * dtun - R(2.0) * t * un - dnut - ut * Dun - t2 * un * dut - t3 * un * un2) / R(2.0);
    R wxy = (dxuy - dyux + ux * duy - uy * dux) / R(2.0);
    R wxn = (t2 * dxun - dnux - ux * Dun - t2 * un * dux) / R(2.0);
    R wyn = (t2 * dyun - dnuy - uy * Dun - t2 * un * duy) / R(2.0);
    R wxt = wtx, wyt = wty, wnt = dvr(wtn, t2, yt2), wyx = -wxy, wnx = dvr(-wxn, t2, yt2), wny = dvr(-wyn, t2, yt2);
    R I1tt = R(2.0) * ut * (pitt * Dut + pitx * Dux + pity * Duy + pitn * Dun);
    R I1tx = (pitt * ux + pitx * ut) * Dut + (pitx * ux + pixx * ut) * Dux + (pity * ux + pixy * ut) * Duy + (pitn * ux + pixn * ut) * Dun;
    R I1ty = (pitt * uy + pity * ut) * Dut + (pitx * uy + pixy * ut) * Dux + (pity * uy + piyy * ut) * Duy + (pitn * uy + piyn * ut) * Dun;
    R I1tn = (pitt * un + pitn * ut) * Dut + (pitx * un + pixn * ut) * Dux + (pity * un + piyn * ut) * Duy + (pitn * un + pinn * ut) * Dun;
    R I1xx = R(2.0) * ux * (pitx * Dut + pixx * Dux + pixy * Duy + pixn * Dun);
    R I1xy = (pitx * uy + pity * ux) * Dut + (pixx * uy + pixy * ux) * Dux + (pixy * uy + piyy * ux) * Duy + (pixn * uy + piyn * ux) * Dun;
    R I1xn = (pitx * un + pitn * ux) * Dut + (pixx * un + pixn * ux) * Dux + (pixy * un + piyn * ux) * Duy + (pixn * un + pinn * ux) * Dun;
    R I1yy = R(2.0) * uy * (pity * Dut + pixy * Dux + piyy * Duy + piyn * Dun);
    R I1yn = (pity * un + pitn * uy) * Dut + (pixy * un + pixn * uy) * Dux + (piyy * un + piyn * uy) * Duy + (piyn * un + pinn * uy) * Dun;
    R I1nn = R(2.0) * un * (pitn * Dut + pixn * Dux + piyn * Duy + pinn * Dun);
    R I2tt = theta * pitt, I2tx = theta * pitx, I2ty = theta * pity, I2tn = theta * pitn, I2xx = theta * pixx;
    R I2xy = theta * pixy, I2xn = theta * pixn, I2yy = theta * piyy, I2yn = theta * piyn, I2nn = theta * pinn;
    R I3tt = R(2.0) * (pitx * wtx + pity * wty + pitn * wtn);
    R I3tx = pitt * wxt + pity * wxy + pitn * wxn + pixx * wtx + pixy * wty + pixn * wtn;
    R I3ty = pitt * wyt + pitx * wyx + pitn * wyn + pixy * wtx + piyy * wty + piyn * wtn;
    R I3tn = pitt * wnt + pitx * wnx + pity * wny + pixn * wtx + piyn * wty + pinn * wtn;
    R I3xx = R(2.0) * (pitx * wxt + pixy * wxy + pixn * wxn);
    R I3xy = pitx * wyt + pity * wxt + pixx * wyx + piyy * wxy + pixn * wyn + piyn * wxn;
    R I3xn = pitx * wnt + pitn * wxt + pixx * wnx + pixy * wny + piyn * wxy + pinn * wxn;
    R I3yy = R(2.0) * (pity * wyt + pixy * wyx + piyn * wyn);
    R I3yn = pity * wnt + pitn * wyt + pixy * wnx + pixn * wyx + piyy * wny + pinn * wyn;
    R I3nn = R(2.0) * (pitn * wnt + pixn * wnx + piyn * wny);
    R ux2 = ux * ux, uy2 = uy * uy;
    R ps = pitt * stt - R(2.0) * pitx * stx - R(2.0) * pity * sty + pixx * sxx + R(2.0) * pixy * sxy + piyy * syy - R(2.0) * pitn * stn * t2 + R(2.0) * pixn * sxn * t2 + R(2.0) * piyn * syn * t2 + pinn * snn * t2 * t2;
    R I4tt = (pitt * stt - pitx * stx - pity * sty - t2 * pitn * stn) - dvr((R(1.0) - ut2) * ps, R(3.0), kThird);
    R I4tx = (pitt * stx + pitx * stt) / R(2.0) - (pitx * sxx + pixx * stx) / R(2.0) - (pity * sxy + pixy * sty) / R(2.0) - t2 * (pitn * sxn + pixn * stn) / R(2.0) + dvr((ut * ux) * ps, R(3.0), kThird);
    R I4ty = (pitt * sty + pity * stt) / R(2.0) - (pitx * sxy + pixy * stx) / R(2.0) - (pity * syy + piyy * sty) / R(2.0) - t2 * (pitn * syn + piyn * stn) / R(2.0) + dvr((ut * uy) * ps, R(3.0), kThird);
    R I4tn = (pitt * stn + pitn * stt) / R(2.0) - (pitx * sxn + pixn * stx) / R(2.0) - (pity * syn + piyn * sty) / R(2.0) - t2 * (pitn * snn + pinn * stn) / R(2.0) + dvr((ut * un) * ps, R(3.0), kThird);
    R I4xx = (pitx * stx - pixx * sxx - pixy * sxy - t2 * pixn * sxn) + dvr((R(1.0) + ux2) * ps, R(3.0), kThird);
    R I4xy = (pitx * sty + pity * stx) / R(2.0) - (pixx * sxy + pixy * sxx) / R(2.0) - (pixy * syy + piyy * sxy) / R(2.0) - t2 * (pixn * syn + piyn * sxn) / R(2.0) + dvr((ux * uy) * ps, R(3.0), kThird);
    R I4xn = (pitx * stn + pitn * stx) / R(2.0) - (pixx * sxn + pixn * sxx) / R(2.0) - (pixy * syn + piyn * sxy) / R(2.0) - t2 * (pixn * snn + pinn * sxn) / R(2.0) + dvr((ux * un) * ps, R(3.0), kThird);
    R I4yy = (pity * sty - pixy * sxy - piyy * syy - t2 * piyn * syn) + dvr((R(1.0) + uy2) * ps, R(3.0), kThird);
    R I4yn = (pity * stn + pitn * sty) / R(2.0) - (pixy * sxn + pixn * sxy) / R(2.0) - (piyy * syn + piyn * syy) / R(2.0) - t2 * (piyn * snn + pinn * syn) / R(2.0) + dvr((uy * un) * ps, R(3.0), kThird);
    R I4nn = (pitn * stn - pixn * sxn - piyn * syn - t2 * pinn * snn) + dvr((yt2 + un2) * ps, R(3.0), kThird);
    R Itt = I1tt + delta_pipi * I2tt - I3tt + tau_pipi * I4tt - lambda_piPi * Pi * stt;
    R Itx = I1tx + delta_pipi * I2tx - I3tx + tau_pipi * I4tx - lambda_piPi * Pi * stx;
    R Ity = I1ty + delta_pipi * I2ty - I3ty + tau_pipi * I4ty - lambda_piPi * Pi * sty;
    R Itn = I1tn + delta_pipi * I2tn - I3tn + tau_pipi * I4tn - lambda_piPi * Pi * stn;
    R Ixx = I1xx + delta_pipi * I2xx - I3xx + tau_pipi * I4xx - lambda_piPi * Pi * sxx;
    R Ixy = I1xy + delta_pipi * I2xy - I3xy + tau_pipi * I4xy - lambda_piPi * Pi * sxy;
    R Ixn = I1xn + delta_pipi * I2xn - I3xn + tau_pipi * I4xn - lambda_piPi * Pi * sxn;
    R Iyy = I1yy + delta_pipi * I2yy - I3yy + tau_pipi * I4yy - lambda_piPi * Pi * syy;
    R Iyn = I1yn + delta_pipi * I2yn - I3yn + tau_pipi * I4yn - lambda_piPi * Pi * syn;
    R Inn = I1nn + delta_pipi * I2nn - I3nn + tau_pipi * I4nn - lambda_piPi * Pi * snn;
    R dpitt = R(2.0) * beta_pi * stt - pitt * taupiInv - Itt - R(2.0) * un * t * pitn;
    R dpitx = R(2.0) * beta_pi * stx - pitx * taupiInv - Itx - un * t * pixn;
    R dpity = R(2.0) * beta_pi * sty - pity * taupiInv - Ity - un * t * piyn;
    R dpitn = R(2.0) * beta_pi * stn - pitn * taupiInv - Itn - un * t * pinn - dvr(ut * pitn + un * pitt, t, yt);
    R dpixx = R(2.0) * beta_pi * sxx - pixx * taupiInv - Ixx;
    R dpixy = R(2.0) * beta_pi * sxy - pixy * taupiInv - Ixy;
    R dpixn = R(2.0) * beta_pi * sxn - pixn * taupiInv - Ixn - dvr(ut * pixn + un * pitx, t, yt);
    R dpiyy = R(2.0) * beta_pi * syy - piyy * taupiInv - Iyy;
    R dpiyn = R(2.0) * beta_pi * syn - piyn * taupiInv - Iyn - dvr(ut * piyn + un * pity, t, yt);
    R dpinn = R(2.0) * beta_pi * snn - pinn * taupiInv - Inn - dvr(2 * (ut * pinn + un * pitn), t, yt);
    rhs[0] = dvr(dpitt, ut, yut) + pitt * dkvk;
    rhs[1] = dvr(dpitx, ut, yut) + pitx * dkvk;
    rhs[2] = dvr(dpity, ut, yut) + pity * dkvk;
    rhs[3] = dvr(dpitn, ut, yut) + pitn * dkvk;
    rhs[4] = dvr(dpixx, ut, yut) + pixx * dkvk;
    rhs[5] = dvr(dpixy, ut, yut) + pixy * dkvk;
    rhs[6] = dvr(dpixn, ut, yut) + pixn * dkvk;
    rhs[7] = dvr(dpiyy, ut, yut) + piyy * dkvk;
    rhs[8] = dvr(dpiyn, ut, yut) + piyn * dkvk;
    rhs[9] = dvr(dpinn, ut, yut) + pinn * dkvk;
    if (BULK) {
        R dPi = -beta_Pi * theta - Pi * tauPiInv - delta_PiPi * Pi * theta + lambda_Pipi * ps;
        rhs[10] = dvr(dPi, ut, yut) + Pi * dkvk;
    }
}

} // namespace vh

#endif

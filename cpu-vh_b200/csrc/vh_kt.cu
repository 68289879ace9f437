/*
 * vh_kt.cu -- the Kurganov-Tadmor RK2 stage as one fused sm_100a kernel.
 *
 * The reference runs each RK stage as seven OpenMP loop nests over the lattice
 * (source, x, y, eta flux passes, inference, regulation, ghost cells;
 * FullyDiscreteKurganovTadmorScheme.cpp:895-923), each re-reading and
 * re-writing the full state.  Here one thread owns one interior cell for the
 * whole stage: it evaluates the source term, the six half-site fluxes and the
 * direction sources, accumulates them in registers in the reference's order,
 * applies the stage-2 convex combination, recovers (e, p, u) from the new
 * T^{tau mu}, regulates pi^{mu nu} and Pi, and writes the cell and its ghost
 * copies once.  e, p and u are double-buffered (read *_in, write *_out) so
 * that no thread overwrites a value a neighbour still reads; that is what lets
 * the inference move into the stencil kernel.  Per step the state crosses HBM
 * twice (the algorithmic minimum for two stages), in 2 launches instead of 14
 * loop nests.
 *
 * Arithmetic is the reference's, operation for operation, in FP64 with float
 * truncations where the reference has them; the library is compiled with
 * --fmad=false so no multiply-add is fused behind the reference's back.
 */
#include <cuda_runtime.h>
#include <cstdlib>
#include "vh_kernels.h"

namespace vh {

/* Half-site states at the face between cells b and b+st (HalfSiteExtrapolation.cpp:12-26):
 * for the forward face of cell s, b = s; for its backward face, b = s - st. */
__device__ __forceinline__ void extrapolate(const double *__restrict__ qn, long long b, long long st, double th,
                                            double &qR, double &qL)
{
    double A = __ldg(qn + b - st), B = __ldg(qn + b), C = __ldg(qn + b + st), D = __ldg(qn + b + 2 * st);
    qR = C - approx_deriv(th, B, C, D) / 2;
    qL = B + approx_deriv(th, A, B, C) / 2;
}

/* SemiDiscreteKurganovTadmorScheme.cpp:14-62 with LocalPropagationSpeed.cpp:14-22,
 * SpectralRadius.cpp:14-24 and FluxFunctions.cpp:15-25, for the face between
 * cells b and b+st along axis dir (1 x, 2 y, 3 eta).  fwd: r = -H, else r += H.
 * dir and fwd are runtime values so that the six faces of a cell share one copy
 * of this code (the fully unrolled form overflowed the instruction cache). */
template <int NQ, int EOS, bool INL = false>
__device__ __forceinline__ void face_flux(const StageArgs &A, long long b, long long st, int dir, bool fwd,
                                          double ePrev, double *__restrict__ r, bool &bad)
{
    const double th = A.theta;
    const long long L = A.L;
    const double *__restrict__ q = A.qin;
    double qRs[8], qLs[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) extrapolate(q + c * L, b, st, th, qRs[c], qLs[c]);
    double PiR = 0, PiL = 0;
    if (NQ == 15) extrapolate(q + 14 * L, b, st, th, PiR, PiL);
    Prim R = infer<EOS, INL>(A.eos, A.t, qRs[0] - qRs[4], qRs[1] - qRs[5], qRs[2] - qRs[6], qRs[3] - qRs[7], PiR, ePrev, bad);
    Prim Lf = infer<EOS, INL>(A.eos, A.t, qLs[0] - qLs[4], qLs[1] - qLs[5], qLs[2] - qLs[6], qLs[3] - qLs[7], PiL, ePrev, bad);
    const double vR = (dir == 1) ? R.ux : (dir == 2) ? R.uy : R.un;
    const double vL = (dir == 1) ? Lf.ux : (dir == 2) ? Lf.uy : Lf.un;
    const double rhoLeft = fabs(vL / Lf.ut);
    const double rhoRight = fabs(vR / R.ut);
    const double a = fmax(rhoLeft, rhoRight);
    const double yR = 1.0 / R.ut, yL = 1.0 / Lf.ut;   /* one reciprocal per state, exact quotients via div_rcp */
#pragma unroll
    for (int n = 0; n < NQ; ++n) {
        double qR, qL;
        if (n < 8) { qR = qRs[n]; qL = qLs[n]; }
        else if (n == 14) { qR = PiR; qL = PiL; }
        else extrapolate(q + n * L, b, st, th, qR, qL);
        double FqR = div_rcp(vR * qR, R.ut, yR);
        double FqL = div_rcp(vL * qL, Lf.ut, yL);
        double res = FqR + FqL - a * (qR - qL);
        res /= 2;
        r[n] = fwd ? -res : r[n] + res;
    }
}

/* SourceTerms.cpp:316-419: sources from d(pi^{tau mu})/dx^i of the T^{tau mu} rows. */
template <int NQ>
__device__ __forceinline__ void dir_sources(const StageArgs &A, long long s, long long st, double d, int dir, double *S)
{
    const long long L = A.L;
    const double *__restrict__ q = A.qin;
    const double fac = 1 / d / 2;
    const double ut = __ldg(A.uin + s);
    const double v = __ldg(A.uin + dir * L + s);
    const double vv = v / ut;
#define DER(n) ((__ldg(q + (n) * L + s + st) - __ldg(q + (n) * L + s - st)) * fac)
    const double dpitt = DER(4), dpitx = DER(5), dpity = DER(6), dpitn = DER(7);
    if (dir == 1) {
        double dpixx = DER(8), dpixy = DER(9), dpixn = DER(10);
        if (NQ == 15) { double dPi = DER(14); S[0] = dpitt * vv - dpitx - vv * dPi; S[1] = dpitx * vv - dpixx - dPi; }
        else { S[0] = dpitt * vv - dpitx; S[1] = dpitx * vv - dpixx; }
        S[2] = dpity * vv - dpixy;
        S[3] = dpitn * vv - dpixn;
    } else if (dir == 2) {
        double dpixy = DER(9), dpiyy = DER(11), dpiyn = DER(12);
        if (NQ == 15) { double dPi = DER(14); S[0] = dpitt * vv - dpity - vv * dPi; S[2] = dpity * vv - dpiyy - dPi; }
        else { S[0] = dpitt * vv - dpity; S[2] = dpity * vv - dpiyy; }
        S[1] = dpitx * vv - dpixy;
        S[3] = dpitn * vv - dpiyn;
    } else {
        double dpixn = DER(10), dpiyn = DER(12), dpinn = DER(13);
        if (NQ == 15) { double dPi = DER(14); S[0] = dpitt * vv - dpitn - vv * dPi; S[3] = dpitn * vv - dpinn - dPi / A.t2pow; }
        else { S[0] = dpitt * vv - dpitn; S[3] = dpitn * vv - dpinn; }
        S[1] = dpitx * vv - dpixn;
        S[2] = dpity * vv - dpiyn;
    }
#undef DER
}

/* eulerStepKernelX/Y/Z (FullyDiscreteKurganovTadmorScheme.cpp:300-634), the
 * axes in the reference's order x, y, eta. */
template <int NQ, int EOS, bool HAS_Z>
__device__ __forceinline__ void flux_update(const StageArgs &A, long long s, double ePrev, double *__restrict__ acc, bool &bad)
{
#pragma unroll 1
    for (int dir = 1; dir <= (HAS_Z ? 3 : 2); ++dir) {
        const long long st = (dir == 1) ? 1 : (dir == 2) ? (long long)A.ncx : (long long)A.ncx * A.ncy;
        const double d = (dir == 1) ? A.dx : (dir == 2) ? A.dy : A.dz;
        const double yd = (dir == 1) ? A.inv_dx : (dir == 2) ? A.inv_dy : A.inv_dz;
        double r[NQ];
#pragma unroll 1
        for (int f = 0; f < 2; ++f) face_flux<NQ, EOS>(A, f == 0 ? s : s - st, st, dir, f == 0, ePrev, r, bad);
#pragma unroll
        for (int n = 0; n < NQ; ++n) r[n] = div_rcp(r[n], d, yd);
        double S[4];
        dir_sources<NQ>(A, s, st, d, dir, S);
#pragma unroll
        for (int n = 0; n < 4; ++n) { r[n] += S[n]; r[n] *= A.dt; }
#pragma unroll
        for (int n = 4; n < NQ; ++n) r[n] *= A.dt;
#pragma unroll
        for (int n = 0; n < NQ; ++n) acc[n] += r[n];
    }
}

/* SourceTerms.cpp:421-612 (USE_APPROX_DERIVATIVE; the dynamical-source arrays
 * are zero, DynamicalVariables.cpp:47-52), then Q + dt S
 * (FullyDiscreteKurganovTadmorScheme.cpp:264-273). */
template <int NQ, int EOS>
__device__ __forceinline__ void source_update(const StageArgs &A, long long s, double *__restrict__ acc)
{
    const long long L = A.L;
    const double th = A.theta;
    const long long sx = 1, sy = A.ncx, sz = (long long)A.ncx * A.ncy;
    double Qv[NQ];
#pragma unroll
    for (int n = 0; n < NQ; ++n) Qv[n] = __ldg(A.qin + n * L + s);
    const double Pi = (NQ == 15) ? Qv[14] : 0;
    const double *__restrict__ utv = A.uin, *__restrict__ uxv = A.uin + L, *__restrict__ uyv = A.uin + 2 * L,
                 *__restrict__ unv = A.uin + 3 * L, *__restrict__ pv = A.pin;
    const double e = __ldg(A.ein + s), p = __ldg(pv + s);
    const double ut = __ldg(utv + s), ux = __ldg(uxv + s), uy = __ldg(uyv + s), un = __ldg(unv + s);
    const double dxut = div_rcp(approx_deriv(th, __ldg(utv + s - sx), ut, __ldg(utv + s + sx)), A.dx, A.inv_dx);
    const double dxux = div_rcp(approx_deriv(th, __ldg(uxv + s - sx), ux, __ldg(uxv + s + sx)), A.dx, A.inv_dx);
    const double dxuy = div_rcp(approx_deriv(th, __ldg(uyv + s - sx), uy, __ldg(uyv + s + sx)), A.dx, A.inv_dx);
    const double dxun = div_rcp(approx_deriv(th, __ldg(unv + s - sx), un, __ldg(unv + s + sx)), A.dx, A.inv_dx);
    const double dyut = div_rcp(approx_deriv(th, __ldg(utv + s - sy), ut, __ldg(utv + s + sy)), A.dy, A.inv_dy);
    const double dyux = div_rcp(approx_deriv(th, __ldg(uxv + s - sy), ux, __ldg(uxv + s + sy)), A.dy, A.inv_dy);
    const double dyuy = div_rcp(approx_deriv(th, __ldg(uyv + s - sy), uy, __ldg(uyv + s + sy)), A.dy, A.inv_dy);
    const double dyun = div_rcp(approx_deriv(th, __ldg(unv + s - sy), un, __ldg(unv + s + sy)), A.dy, A.inv_dy);
    const double dnut = div_rcp(approx_deriv(th, __ldg(utv + s - sz), ut, __ldg(utv + s + sz)), A.dz, A.inv_dz);
    const double dnux = div_rcp(approx_deriv(th, __ldg(uxv + s - sz), ux, __ldg(uxv + s + sz)), A.dz, A.inv_dz);
    const double dnuy = div_rcp(approx_deriv(th, __ldg(uyv + s - sz), uy, __ldg(uyv + s + sz)), A.dz, A.inv_dz);
    const double dnun = div_rcp(approx_deriv(th, __ldg(unv + s - sz), un, __ldg(unv + s + sz)), A.dz, A.inv_dz);
    const double dxp = div_rcp(approx_deriv(th, __ldg(pv + s - sx), p, __ldg(pv + s + sx)), A.dx, A.inv_dx);
    const double dyp = div_rcp(approx_deriv(th, __ldg(pv + s - sy), p, __ldg(pv + s + sy)), A.dy, A.inv_dy);
    const double dnp = div_rcp(approx_deriv(th, __ldg(pv + s - sz), p, __ldg(pv + s + sz)), A.dz, A.inv_dz);
    const double t = A.t;
    /* Tnn(e, p + Pi, un, pinn, t), EnergyMomentumTensor.cpp:328-330 */
    const double pP = p + Pi;
    const double yt = A.inv_t;
    const double tnn = (e + pP) * un * un + div_rcp(div_rcp(pP, t, yt), t, yt) + Qv[13];
    const double yut = 1.0 / ut;
    const double vx = div_rcp(ux, ut, yut), vy = div_rcp(uy, ut, yut), vn = div_rcp(un, ut, yut);
    const double dxvx = div_rcp(dxux - vx * dxut, ut, yut);
    const double dyvy = div_rcp(dyuy - vy * dyut, ut, yut);
    const double dnvn = div_rcp(dnun - vn * dnut, ut, yut);
    const double dkvk = dxvx + dyvy + dnvn;
    double S[NQ];
    S[0] = 0.0 - (div_rcp(Qv[0], t, yt) + t * tnn) + dkvk * (Qv[4] - p - Pi) - vx * dxp - vy * dyp - vn * dnp;
    S[1] = 0.0 - div_rcp(Qv[1], t, yt) - dxp + dkvk * Qv[5];
    S[2] = 0.0 - div_rcp(Qv[2], t, yt) - dyp + dkvk * Qv[6];
    S[3] = 0.0 - div_rcp(3 * Qv[3], t, yt) - dnp / A.t2pow + dkvk * Qv[7];
    pimunu_rhs<EOS, NQ == 15>(A.eos, A.zeta, S + 4, t, e, p, ut, ux, uy, un,
                              __ldg(A.upin + s), __ldg(A.upin + L + s), __ldg(A.upin + 2 * L + s), __ldg(A.upin + 3 * L + s),
                              Qv + 4, Pi, dxut, dyut, dnut, dxux, dyux, dnux, dxuy, dyuy, dnuy, dxun, dyun, dnun, dkvk,
                              A.etabar, A.dt);
#pragma unroll
    for (int n = 0; n < NQ; ++n) acc[n] = Qv[n] + A.dt * S[n];
}

/* regulateDissipativeCurrents, REG_SCHEME_1 (FullyDiscreteKurganovTadmorScheme.cpp:690-859).
 * When e > e_reg both factors are exactly 1 and the reference's multiplies are
 * identities, so the block is skipped. */
template <int NQ>
__device__ __forceinline__ void regulate(const StageArgs &A, double *__restrict__ acc, const Prim &P, bool &bad)
{
    if (P.e > A.e_reg) return;
    const double t = A.t_inf, t2 = t * t;
    const double pitt = acc[4], pitx = acc[5], pity = acc[6], pitn = acc[7], pixx = acc[8];
    const double pixy = acc[9], pixn = acc[10], piyy = acc[11], piyn = acc[12], pinn = acc[13];
    const double Pi = (NQ == 15) ? acc[14] : 0;
    const double ut = P.ut, ux = P.ux, uy = P.uy, un = P.un;
    const double xi0 = 0.1, rhomax = 1.0;
    double pipi = pitt * pitt - 2 * pitx * pitx - 2 * pity * pity + pixx * pixx + 2 * pixy * pixy + piyy * piyy - 2 * pitn * pitn * t2 + 2 * pixn * pixn * t2 + 2 * piyn * piyn * t2 + pinn * pinn * t2 * t2;
    double spipi = sqrt(fabs(pipi));
    double pimumu = pitt - pixx - piyy - pinn * t * t;
    double piu0 = -(pitn * t2 * un) + pitt * ut - pitx * ux - pity * uy;
    double piu1 = -(pixn * t2 * un) + pitx * ut - pixx * ux - pixy * uy;
    double piu2 = -(piyn * t2 * un) + pity * ut - pixy * ux - piyy * uy;
    double piu3 = -(pinn * t2 * un) + pitn * ut - pixn * ux - piyn * uy;
    double a1 = spipi / rhomax / (double)sqrtf(__double2float_rn(P.e * P.e + 3 * P.p * P.p));
    double a2 = pimumu / xi0 / rhomax / spipi;
    double a3 = piu0 / xi0 / rhomax / spipi;
    double a4 = piu1 / xi0 / rhomax / spipi;
    double a5 = piu2 / xi0 / rhomax / spipi;
    double a6 = piu3 / xi0 / rhomax / spipi;
    double a12 = fmax(a1, a2), a34 = fmax(a3, a4), a56 = fmax(a5, a6), a3456 = fmax(a34, a56);
    double rho = fmax(a12, a3456);
    double facShear = vh_tanh(rho) / rho;
    if (fabs(rho) < 1.e-7) facShear = 1.0;
#pragma unroll
    for (int n = 4; n < 14; ++n) acc[n] *= facShear;
    if (isnan(facShear)) bad = true;
    if (NQ == 15) {
        double rhoBulk = fabs(Pi) / P.p;
        double facBulk = vh_tanh(rhoBulk) / rhoBulk;
        if (fabs(rhoBulk) < 1.e-7) facBulk = 1.0;
        acc[14] *= facBulk;
        if (isnan(facBulk)) bad = true;
    }
}

template <int NQ>
__device__ __forceinline__ void put_cell(const StageArgs &A, long long d, const double *__restrict__ acc, const Prim &P)
{
    const long long L = A.L;
#pragma unroll
    for (int n = 0; n < NQ; ++n) A.qout[n * L + d] = acc[n];
    A.eout[d] = P.e;
    A.pout[d] = P.p;
    A.uout[d] = P.ut;
    A.uout[L + d] = P.ux;
    A.uout[2 * L + d] = P.uy;
    A.uout[3 * L + d] = P.un;
}

#ifndef VH_STAGE_MIN_BLOCKS
#define VH_STAGE_MIN_BLOCKS 4   /* 128 registers: 16 warps/SM; measured faster than 2-3 blocks at 168-255 */
#endif

template <int NQ, int EOS, bool HAS_Z, bool STAGE2>
__global__ void __launch_bounds__(128, VH_STAGE_MIN_BLOCKS) kt_stage_kernel(const __grid_constant__ StageArgs A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
    const int k = blockIdx.z + 2;
    if (i >= A.nx + 2 || j >= A.ny + 2) return;
    const long long sxy = (long long)A.ncx * A.ncy;
    const long long s = i + (long long)A.ncx * j + sxy * k;
    const double ePrev = __ldg(A.ein + s);
    bool bad = false;
    double acc[NQ];
    source_update<NQ, EOS>(A, s, acc);
    flux_update<NQ, EOS, HAS_Z>(A, s, ePrev, acc, bad);
    if (!HAS_Z) {
        /* nz = 1: the eta ghosts equal the cell, every eta slope is 0 and the
         * reference's eta pass adds exactly +0.0 (which turns a -0 into +0). */
#pragma unroll
        for (int n = 0; n < NQ; ++n) acc[n] += 0.0;
    }
    if (STAGE2) {
#pragma unroll
        for (int n = 0; n < NQ; ++n) { acc[n] += __ldg(A.qbase + n * A.L + s); acc[n] /= 2; }
    }
    /* setInferredVariablesKernel (EnergyMomentumTensor.cpp:235-287) with ePrev = e[s] */
    Prim P = infer<EOS>(A.eos, A.t_inf, acc[0] - acc[4], acc[1] - acc[5], acc[2] - acc[6], acc[3] - acc[7],
                        (NQ == 15) ? acc[14] : 0.0, ePrev, bad);
    regulate<NQ>(A, acc, P, bad);
    if (bad) raise_error(A.err, kErrNan, s, A.step);
    put_cell<NQ>(A, s, acc, P);
    /* zero-gradient ghost faces (DynamicalVariables.cpp:220-378) */
    if (i == 2) { put_cell<NQ>(A, s - 1, acc, P); put_cell<NQ>(A, s - 2, acc, P); }
    if (i == A.nx + 1) { put_cell<NQ>(A, s + 1, acc, P); put_cell<NQ>(A, s + 2, acc, P); }
    if (j == 2) { put_cell<NQ>(A, s - A.ncx, acc, P); put_cell<NQ>(A, s - 2 * A.ncx, acc, P); }
    if (j == A.ny + 1) { put_cell<NQ>(A, s + A.ncx, acc, P); put_cell<NQ>(A, s + 2 * A.ncx, acc, P); }
    if (k == 2) { put_cell<NQ>(A, s - sxy, acc, P); put_cell<NQ>(A, s - 2 * sxy, acc, P); }
    if (k == A.nz + 1) { put_cell<NQ>(A, s + sxy, acc, P); put_cell<NQ>(A, s + 2 * sxy, acc, P); }
}

/* ---------------------------------------------------------------------
 * Phase-split form of the same stage: five short kernels instead of one long
 * one, in the reference's own phase order (FullyDiscreteKurganovTadmorScheme.cpp:
 * eulerStepKernelSource, X, Y, Z, then inference/regulation/ghosts).  The
 * partial sums live in qout between phases; FP64 stores are exact, so the
 * result is bit-identical to the fused kernel.  Each phase's code is a
 * fraction of the fused kernel's, which fits the instruction cache: the fused
 * kernel spends most of its stall time waiting for instruction fetch.
 * --------------------------------------------------------------------- */
__device__ __forceinline__ bool stage_cell(const StageArgs &A, int &i, int &j, int &k, long long &s)
{
    i = blockIdx.x * blockDim.x + threadIdx.x + 2;
    j = blockIdx.y * blockDim.y + threadIdx.y + 2;
    k = blockIdx.z + 2;
    if (i >= A.nx + 2 || j >= A.ny + 2) return false;
    s = i + (long long)A.ncx * j + (long long)A.ncx * A.ncy * k;
    return true;
}

template <int NQ, int EOS>
__global__ void __launch_bounds__(128, VH_STAGE_MIN_BLOCKS) kt_source_kernel(const __grid_constant__ StageArgs A)
{
    int i, j, k;
    long long s;
    if (!stage_cell(A, i, j, k, s)) return;
    double acc[NQ];
    source_update<NQ, EOS>(A, s, acc);
#pragma unroll
    for (int n = 0; n < NQ; ++n) A.qout[n * A.L + s] = acc[n];
}

template <int NQ, int EOS, int DIR>
__global__ void __launch_bounds__(128, VH_STAGE_MIN_BLOCKS) kt_flux_kernel(const __grid_constant__ StageArgs A)
{
    int i, j, k;
    long long s;
    if (!stage_cell(A, i, j, k, s)) return;
    const double ePrev = __ldg(A.ein + s);
    bool bad = false;
    const long long st = (DIR == 1) ? 1 : (DIR == 2) ? (long long)A.ncx : (long long)A.ncx * A.ncy;
    const double d = (DIR == 1) ? A.dx : (DIR == 2) ? A.dy : A.dz;
    const double yd = (DIR == 1) ? A.inv_dx : (DIR == 2) ? A.inv_dy : A.inv_dz;
    double r[NQ];
#pragma unroll 1
    for (int f = 0; f < 2; ++f) face_flux<NQ, EOS, true>(A, f == 0 ? s : s - st, st, DIR, f == 0, ePrev, r, bad);
#pragma unroll
    for (int n = 0; n < NQ; ++n) r[n] = div_rcp(r[n], d, yd);
    double S[4];
    dir_sources<NQ>(A, s, st, d, DIR, S);
#pragma unroll
    for (int n = 0; n < 4; ++n) { r[n] += S[n]; r[n] *= A.dt; }
#pragma unroll
    for (int n = 4; n < NQ; ++n) r[n] *= A.dt;
#pragma unroll
    for (int n = 0; n < NQ; ++n) A.qout[n * A.L + s] += r[n];
    if (bad) raise_error(A.err, kErrNan, s, A.step);
}

template <int NQ, int EOS, bool HAS_Z, bool STAGE2>
__global__ void __launch_bounds__(128, VH_STAGE_MIN_BLOCKS) kt_final_kernel(const __grid_constant__ StageArgs A)
{
    int i, j, k;
    long long s;
    if (!stage_cell(A, i, j, k, s)) return;
    const long long sxy = (long long)A.ncx * A.ncy;
    const double ePrev = __ldg(A.ein + s);
    bool bad = false;
    double acc[NQ];
#pragma unroll
    for (int n = 0; n < NQ; ++n) acc[n] = A.qout[n * A.L + s];
    if (!HAS_Z) {
#pragma unroll
        for (int n = 0; n < NQ; ++n) acc[n] += 0.0;
    }
    if (STAGE2) {
#pragma unroll
        for (int n = 0; n < NQ; ++n) { acc[n] += __ldg(A.qbase + n * A.L + s); acc[n] /= 2; }
    }
    Prim P = infer<EOS, true>(A.eos, A.t_inf, acc[0] - acc[4], acc[1] - acc[5], acc[2] - acc[6], acc[3] - acc[7],
                        (NQ == 15) ? acc[14] : 0.0, ePrev, bad);
    regulate<NQ>(A, acc, P, bad);
    if (bad) raise_error(A.err, kErrNan, s, A.step);
    put_cell<NQ>(A, s, acc, P);
    if (i == 2) { put_cell<NQ>(A, s - 1, acc, P); put_cell<NQ>(A, s - 2, acc, P); }
    if (i == A.nx + 1) { put_cell<NQ>(A, s + 1, acc, P); put_cell<NQ>(A, s + 2, acc, P); }
    if (j == 2) { put_cell<NQ>(A, s - A.ncx, acc, P); put_cell<NQ>(A, s - 2 * A.ncx, acc, P); }
    if (j == A.ny + 1) { put_cell<NQ>(A, s + A.ncx, acc, P); put_cell<NQ>(A, s + 2 * A.ncx, acc, P); }
    if (k == 2) { put_cell<NQ>(A, s - sxy, acc, P); put_cell<NQ>(A, s - 2 * sxy, acc, P); }
    if (k == A.nz + 1) { put_cell<NQ>(A, s + sxy, acc, P); put_cell<NQ>(A, s + 2 * sxy, acc, P); }
}

/* DynamicalVariables.cpp:169-218 (T^{tau mu} from e, p+Pi, u, pi) and the
 * ghost faces; the previous-step velocity starts equal to u. */
__global__ void init_kernel(const __grid_constant__ InitArgs A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= A.nx || j >= A.ny) return;
    const long long N = (long long)A.nx * A.ny * A.nz;
    const long long m = i + (long long)A.nx * (j + (long long)A.ny * k);
    const long long L = A.L, sxy = (long long)A.ncx * A.ncy;
    const long long s = (i + 2) + (long long)A.ncx * (j + 2) + sxy * (k + 2);
    double qv[15];
    const double e = A.e[m], p = A.p[m];
    const double ut = A.u[m], ux = A.u[N + m], uy = A.u[2 * N + m], un = A.u[3 * N + m];
    for (int c = 0; c < 10; ++c) qv[4 + c] = A.pi ? A.pi[c * N + m] : 0.0;
    const double Pi = (A.nq == 15 && A.Pi) ? A.Pi[m] : 0.0;
    if (A.nq == 15) qv[14] = Pi;
    const double P = p + Pi;
    qv[0] = (e + P) * ut * ut - P + qv[4];
    qv[1] = (e + P) * ut * ux + qv[5];
    qv[2] = (e + P) * ut * uy + qv[6];
    qv[3] = (e + P) * ut * un + qv[7];
    auto put = [&](long long d) {
        for (int n = 0; n < A.nq; ++n) A.q[n * L + d] = qv[n];
        A.eo[d] = e; A.po[d] = p;
        A.uo[d] = ut; A.uo[L + d] = ux; A.uo[2 * L + d] = uy; A.uo[3 * L + d] = un;
    };
    put(s);
    A.upo[s] = ut; A.upo[L + s] = ux; A.upo[2 * L + s] = uy; A.upo[3 * L + s] = un;
    const int ii = i + 2, jj = j + 2, kk = k + 2;
    if (ii == 2) { put(s - 1); put(s - 2); }
    if (ii == A.nx + 1) { put(s + 1); put(s + 2); }
    if (jj == 2) { put(s - A.ncx); put(s - 2 * A.ncx); }
    if (jj == A.ny + 1) { put(s + A.ncx); put(s + 2 * A.ncx); }
    if (kk == 2) { put(s - sxy); put(s - 2 * sxy); }
    if (kk == A.nz + 1) { put(s + sxy); put(s + 2 * sxy); }
}

/* device math self-check: 0 vh_tanh(a), 1 div_rcp(a, b, RN(1/b)), 2 IEEE a/b,
 * 3 powf_quarter(float(a)) */
__global__ void math_check_kernel(int which, const double *a, const double *b, int n, double *out, PowfTab pq)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double x = a[i], r;
    if (which == 0) r = vh_tanh(x);
    else if (which == 1) { double y = b[i]; r = div_rcp(x, y, 1.0 / y); }
    else if (which == 2) r = x / b[i];
    else r = (double)powf_quarter(__double2float_rn(x), pq);
    out[i] = r;
}

void launch_math_check(int which, const double *a, const double *b, int n, double *out, const PowfTab &pq, cudaStream_t s)
{
    math_check_kernel<<<(n + 255) / 256, 256, 0, s>>>(which, a, b, n, out, pq);
}

void launch_init(const InitArgs &a, cudaStream_t s)
{
    dim3 block(32, 4, 1);
    dim3 grid((a.nx + 31) / 32, (a.ny + 3) / 4, a.nz);
    init_kernel<<<grid, block, 0, s>>>(a);
}

/* Fused for small lattices (launch- and latency-bound: one wave of threads,
 * each carrying a whole stage), phase-split from 2^18 interior cells up
 * (measured on B200: 131x131x61 split 5.43 ms/step vs fused 6.82; 101x101x1
 * fused 0.120 ms vs split 0.163).  VH_STAGE_MODE=fused|split overrides. */
static bool use_split(const StageArgs &a)
{
    static int forced = [] {
        const char *e = getenv("VH_STAGE_MODE");
        return !e ? -1 : (e[0] == 'f' ? 0 : 1);
    }();
    if (forced >= 0) return forced == 1;
    return (long long)a.nx * a.ny * a.nz >= (1LL << 18);
}

template <int NQ, int EOS>
static void launch_stage_t(const StageArgs &a, cudaStream_t s, StageMarks *m)
{
    dim3 block(32, 4, 1);
    dim3 grid((a.nx + 31) / 32, (a.ny + 3) / 4, a.nz);
    const bool z = a.nz > 1, st2 = a.qbase != nullptr;
    if (m) { m->n = 0; cudaEventRecord(m->ev[0], s); }
    auto mark = [&](int phase) {
        if (!m) return;
        m->phase[m->n] = phase;
        cudaEventRecord(m->ev[++m->n], s);
    };
    if (!use_split(a)) {
        if (z && st2) kt_stage_kernel<NQ, EOS, true, true><<<grid, block, 0, s>>>(a);
        else if (z) kt_stage_kernel<NQ, EOS, true, false><<<grid, block, 0, s>>>(a);
        else if (st2) kt_stage_kernel<NQ, EOS, false, true><<<grid, block, 0, s>>>(a);
        else kt_stage_kernel<NQ, EOS, false, false><<<grid, block, 0, s>>>(a);
        mark(5);
        return;
    }
    kt_source_kernel<NQ, EOS><<<grid, block, 0, s>>>(a);
    mark(0);
    kt_flux_kernel<NQ, EOS, 1><<<grid, block, 0, s>>>(a);
    mark(1);
    kt_flux_kernel<NQ, EOS, 2><<<grid, block, 0, s>>>(a);
    mark(2);
    if (z) { kt_flux_kernel<NQ, EOS, 3><<<grid, block, 0, s>>>(a); mark(3); }
    if (z && st2) kt_final_kernel<NQ, EOS, true, true><<<grid, block, 0, s>>>(a);
    else if (z) kt_final_kernel<NQ, EOS, true, false><<<grid, block, 0, s>>>(a);
    else if (st2) kt_final_kernel<NQ, EOS, false, true><<<grid, block, 0, s>>>(a);
    else kt_final_kernel<NQ, EOS, false, false><<<grid, block, 0, s>>>(a);
    mark(4);
}

int stage_launches(int nx, int ny, int nz)
{
    StageArgs a{};
    a.nx = nx; a.ny = ny; a.nz = nz;
    if (!use_split(a)) return 1;
    return nz > 1 ? 5 : 4;
}

void launch_stage(const StageArgs &a, int nq, int eos_kind, cudaStream_t s, StageMarks *m)
{
    if (nq == 15) {
        if (eos_kind == 1) launch_stage_t<15, 1>(a, s, m); else launch_stage_t<15, 0>(a, s, m);
    } else {
        if (eos_kind == 1) launch_stage_t<14, 1>(a, s, m); else launch_stage_t<14, 0>(a, s, m);
    }
}

} // namespace vh

/*
 * vh_stage.cuh -- per-cell bodies of the KT RK2 stage, shared by the
 * single-event kernels (vh_kt.cu) and the batched kernels (vh_batch.cu).
 *
 * Every body takes the stage's arguments by reference and the cell it owns;
 * the arithmetic is the reference's, operation for operation, in FP64 with
 * float truncations where the reference has them.  Because both launch forms
 * run these same functions, a cell's result does not depend on which form
 * (fused or phase-split, single event or batch) computed it.
 */
#ifndef VH_STAGE_CUH
#define VH_STAGE_CUH

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

/* ---------------------------------------------------------------------
 * The flux phase reading q from a tile staged in shared memory: the same
 * arithmetic as face_flux / dir_sources, with every read of the conserved
 * variables going to the tile (index = position in the tile, stride along
 * the axis = the tile's stride), so the results are bit-identical.
 * --------------------------------------------------------------------- */
struct QTile {
    const double *__restrict__ q;
    int P;                   /* doubles per component plane of the tile */
    __device__ __forceinline__ double operator()(int n, int i) const { return q[n * P + i]; }
};

__device__ __forceinline__ void extrapolate_t(const QTile &qt, int n, int b, int st, double th, double &qR, double &qL)
{
    double A = qt(n, b - st), B = qt(n, b), C = qt(n, b + st), D = qt(n, b + 2 * st);
    qR = C - approx_deriv(th, B, C, D) / 2;
    qL = B + approx_deriv(th, A, B, C) / 2;
}

template <int NQ, int EOS>
__device__ __forceinline__ void face_flux_t(const StageArgs &A, const QTile &qt, int b, int st, int dir, bool fwd,
                                            double ePrev, double *__restrict__ r, bool &bad)
{
    const double th = A.theta;
    double qRs[8], qLs[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) extrapolate_t(qt, c, b, st, th, qRs[c], qLs[c]);
    double PiR = 0, PiL = 0;
    if (NQ == 15) extrapolate_t(qt, 14, b, st, th, PiR, PiL);
    /* the two half-site root solves as one loop: one copy of the inlined
     * Newton solve instead of two (smaller instruction footprint, measured
     * 5 % faster on the phase-split stage; the same arithmetic) */
    Prim R, Lf;
#pragma unroll 1
    for (int side = 0; side < 2; ++side) {
        const bool l = side == 1;
        Prim P = infer<EOS, true>(A.eos, A.t, l ? qLs[0] - qLs[4] : qRs[0] - qRs[4], l ? qLs[1] - qLs[5] : qRs[1] - qRs[5],
                                  l ? qLs[2] - qLs[6] : qRs[2] - qRs[6], l ? qLs[3] - qLs[7] : qRs[3] - qRs[7],
                                  l ? PiL : PiR, ePrev, bad);
        if (l) Lf = P; else R = P;
    }
    const double vR = (dir == 1) ? R.ux : (dir == 2) ? R.uy : R.un;
    const double vL = (dir == 1) ? Lf.ux : (dir == 2) ? Lf.uy : Lf.un;
    const double rhoLeft = fabs(vL / Lf.ut);
    const double rhoRight = fabs(vR / R.ut);
    const double a = fmax(rhoLeft, rhoRight);
    const double yR = 1.0 / R.ut, yL = 1.0 / Lf.ut;
#pragma unroll
    for (int n = 0; n < NQ; ++n) {
        double qR, qL;
        if (n < 8) { qR = qRs[n]; qL = qLs[n]; }
        else if (n == 14) { qR = PiR; qL = PiL; }
        else extrapolate_t(qt, n, b, st, th, qR, qL);
        double FqR = div_rcp(vR * qR, R.ut, yR);
        double FqL = div_rcp(vL * qL, Lf.ut, yL);
        double res = FqR + FqL - a * (qR - qL);
        res /= 2;
        r[n] = fwd ? -res : r[n] + res;
    }
}

/* dir_sources with q from the tile at ts +- tst and u^tau, u^dir of the
 * padded cell given (dir_sources_t below reads them at s) */
template <int NQ>
__device__ __forceinline__ void dir_sources_uv(const StageArgs &A, const QTile &qt, int ts, int tst, double ut, double v,
                                               double d, int dir, double *S)
{
    const double fac = 1 / d / 2;
    const double vv = v / ut;
#define DER(n) ((qt(n, ts + tst) - qt(n, ts - tst)) * fac)
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

template <int NQ>
__device__ __forceinline__ void dir_sources_t(const StageArgs &A, const QTile &qt, int ts, int tst, long long s,
                                              double d, int dir, double *S)
{
    dir_sources_uv<NQ>(A, qt, ts, tst, __ldg(A.uin + s), __ldg(A.uin + dir * A.L + s), d, dir, S);
}

/* copy 8 bytes global -> shared without staging through registers */
__device__ __forceinline__ void cp_async8(double *smem, const double *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

/* Programmatic dependent launch (kernels launched with
 * cudaLaunchAttributeProgrammaticStreamSerialization).  pdl_trigger lets the
 * next kernel on the stream start once every block of this one has issued
 * it; pdl_wait returns once the previous kernel on the stream has completed
 * and its writes are visible.  A kernel launched without the attribute
 * passes both at once. */
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

/* hint: bring the line holding *p into L2 */
__device__ __forceinline__ void prefetch_l2(const double *p)
{
    asm volatile("prefetch.global.L2 [%0];\n" ::"l"(__cvta_generic_to_global(p)));
}

/* the values a flux launch along dir reads for cell s only after its root
 * solves -- the accumulator it adds to, u^tau and u^dir of the direction
 * sources -- requested into L2 when the block starts (no registers held) */
template <int NQ>
__device__ __forceinline__ void prefetch_flux_cell(const StageArgs &A, long long s, int dir)
{
#pragma unroll 1
    for (int n = 0; n < NQ; ++n) prefetch_l2(A.qout + n * A.L + s);
    prefetch_l2(A.uin + s);
    prefetch_l2(A.uin + dir * A.L + s);
}

/* One block of the staged flux along DIR: TX x TY cells (x by y for DIR 1
 * and 2, x by eta for DIR 3, at the block's fixed third coordinate) and the
 * 2-cell halo along DIR, all NQ components, copied asynchronously into sm
 * (NQ * (TX + 4 [DIR 1]) * (TY + 4 [DIR 2, 3]) doubles), then the flux of
 * every interior cell of the tile as flux_body computes it. */
template <int NQ, int EOS, int DIR, int TX, int TY>
__device__ __forceinline__ void flux_staged_tile(const StageArgs &A, int i0, int j0, int k0, double *__restrict__ sm)
{
    constexpr int BX = TX + (DIR == 1 ? 4 : 0), BY = TY + (DIR == 1 ? 0 : 4), P = BX * BY;
    const int tid = threadIdx.x + TX * threadIdx.y;
    const long long sxy = (long long)A.ncx * A.ncy;
    /* padded coordinates of the tile's first box element; the box's second
     * axis is y (DIR 1, 2) or eta (DIR 3) */
    const int bx0 = i0 + 2 - (DIR == 1 ? 2 : 0);
    const int by0 = (DIR == 3) ? k0 : j0;            /* = first cell - 2 for DIR 2, 3 */
    const int b2lim = (DIR == 3) ? A.nz + 4 : A.ny + 4;
    const int by_first = (DIR == 1) ? j0 + 2 : by0;
    for (int e = tid; e < NQ * P; e += TX * TY) {
        const int n = e / P, rr = e - n * P, bxi = rr % BX, byi = rr / BX;
        const int x = bx0 + bxi, yk = by_first + byi;
        if (x < A.ncx && yk < b2lim) {
            const long long g = (DIR == 3) ? x + (long long)A.ncx * (j0 + 2) + sxy * yk
                                           : x + (long long)A.ncx * yk + sxy * (k0 + 2);
            cp_async8(sm + e, A.qin + n * A.L + g);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    const int i = i0 + threadIdx.x + 2;
    const int j = (DIR == 3) ? j0 + 2 : j0 + threadIdx.y + 2;
    const int k = (DIR == 3) ? k0 + threadIdx.y + 2 : k0 + 2;
    if (i >= A.nx + 2 || j >= A.ny + 2 || k >= A.nz + 2) return;
    const long long s = i + (long long)A.ncx * j + sxy * k;
    const int ts = (threadIdx.x + (DIR == 1 ? 2 : 0)) + BX * (threadIdx.y + (DIR == 1 ? 0 : 2));
    const int tst = (DIR == 1) ? 1 : BX;
    const QTile qt{sm, P};
    const double ePrev = __ldg(A.ein + s);
    bool bad = false;
    const double d = (DIR == 1) ? A.dx : (DIR == 2) ? A.dy : A.dz;
    const double yd = (DIR == 1) ? A.inv_dx : (DIR == 2) ? A.inv_dy : A.inv_dz;
    double r[NQ];
#pragma unroll 1
    for (int f = 0; f < 2; ++f) face_flux_t<NQ, EOS>(A, qt, f == 0 ? ts : ts - tst, tst, DIR, f == 0, ePrev, r, bad);
#pragma unroll
    for (int n = 0; n < NQ; ++n) r[n] = div_rcp(r[n], d, yd);
    double S[4];
    dir_sources_t<NQ>(A, qt, ts, tst, s, d, DIR, S);
#pragma unroll
    for (int n = 0; n < 4; ++n) { r[n] += S[n]; r[n] *= A.dt; }
#pragma unroll
    for (int n = 4; n < NQ; ++n) r[n] *= A.dt;
#pragma unroll
    for (int n = 0; n < NQ; ++n) A.qout[n * A.L + s] += r[n];
    if (bad) raise_error(A.err, kErrNan, s, A.step);
}

/* Geometry of the flux tile along DIR: TX x TY cells, their values with a
 * 2-cell halo along DIR (BX x BY per component) and the half slopes of
 * HalfSiteExtrapolation.cpp:12-26 at every position one cell in from the
 * halo's ends (HX x HY per component). */
template <int DIR, int TX, int TY>
struct FluxTile {
    static constexpr int BX = TX + (DIR == 1 ? 4 : 0), BY = TY + (DIR == 1 ? 0 : 4), P = BX * BY;
    static constexpr int HX = TX + (DIR == 1 ? 2 : 0), HY = TY + (DIR == 1 ? 0 : 2), H = HX * HY;
    static constexpr int kDoubles(int nq) { return nq * (P + H); }
};

/* The staged flux along DIR with each half slope computed once per tile.
 * A face's half-site states are qR = q(b+1) - d(b+1)/2 and qL = q(b) + d(b)/2
 * with d the minmod-limited slope at a cell (approx_deriv); the reference
 * evaluates every slope at a cell for each of the four faces around its two
 * neighbours along the axis, with identical arguments and so an identical
 * value.  Here the block computes the half slope d/2 of every tile position
 * once into shared memory; each thread then forms its cell's four states
 * (two faces, two sides), runs their root solves (one inlined copy of infer,
 * in a rolled loop) and updates q* one component at a time.  Every value is
 * the reference's arithmetic on the same operands, so the results are
 * bit-identical to flux_staged_tile.  sm: FluxTile::kDoubles(NQ) doubles. */
template <int NQ, int EOS, int DIR, int TX, int TY>
__device__ __forceinline__ void flux_slopes_tile(const StageArgs &A, int i0, int j0, int k0, double *__restrict__ sm)
{
    using G = FluxTile<DIR, TX, TY>;
    constexpr int BX = G::BX, P = G::P, HX = G::HX, H = G::H;
    double *__restrict__ hs = sm + NQ * P;
    const int tid = threadIdx.x + TX * threadIdx.y;
    const long long sxy = (long long)A.ncx * A.ncy;
    const int bx0 = i0 + 2 - (DIR == 1 ? 2 : 0);
    const int b2lim = (DIR == 3) ? A.nz + 4 : A.ny + 4;
    const int by_first = (DIR == 1) ? j0 + 2 : (DIR == 3) ? k0 : j0;
    for (int e = tid; e < NQ * P; e += TX * TY) {
        const int n = e / P, rr = e - n * P, bxi = rr % BX, byi = rr / BX;
        const int x = bx0 + bxi, yk = by_first + byi;
        if (x < A.ncx && yk < b2lim) {
            const long long g = (DIR == 3) ? x + (long long)A.ncx * (j0 + 2) + sxy * yk
                                           : x + (long long)A.ncx * yk + sxy * (k0 + 2);
            cp_async8(sm + e, A.qin + n * A.L + g);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    const double th = A.theta;
    constexpr int tst = (DIR == 1) ? 1 : BX;
    for (int e = tid; e < NQ * H; e += TX * TY) {
        const int n = e / H, rr = e - n * H, hx = rr % HX, hy = rr / HX;
        const int tp = (hx + (DIR == 1 ? 1 : 0)) + BX * (hy + (DIR == 1 ? 0 : 1));
        const double *q = sm + n * P + tp;
        hs[e] = approx_deriv(th, q[-tst], q[0], q[tst]) / 2;
    }
    __syncthreads();
    const int i = i0 + threadIdx.x + 2;
    const int j = (DIR == 3) ? j0 + 2 : j0 + threadIdx.y + 2;
    const int k = (DIR == 3) ? k0 + threadIdx.y + 2 : k0 + 2;
    if (i >= A.nx + 2 || j >= A.ny + 2 || k >= A.nz + 2) return;
    const long long s = i + (long long)A.ncx * j + sxy * k;
    const int ts = (threadIdx.x + (DIR == 1 ? 2 : 0)) + BX * (threadIdx.y + (DIR == 1 ? 0 : 2));
    const int hp = (threadIdx.x + (DIR == 1 ? 1 : 0)) + HX * (threadIdx.y + (DIR == 1 ? 0 : 1));
    constexpr int hst = (DIR == 1) ? 1 : HX;
    const QTile qt{sm, P};
    const double ePrev = __ldg(A.ein + s);
    bool bad = false;
    /* states m = 0..3: forward face R, L; backward face R, L */
    double ut0 = 0, ut1 = 0, ut2 = 0, ut3 = 0, v0 = 0, v1 = 0, v2 = 0, v3 = 0;
#pragma unroll 1
    for (int m = 0; m < 4; ++m) {
        const int vo = (m == 0) ? ts + tst : (m == 3) ? ts - tst : ts;
        const int ho = (m == 0) ? hp + hst : (m == 3) ? hp - hst : hp;
        const bool minus = (m & 1) == 0;        /* R states subtract the half slope */
        double st[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            const int n = (c < 8) ? c : 14;
            if (n >= NQ) { st[c] = 0; continue; }
            const double qv = sm[n * P + vo], hv = hs[n * H + ho];
            st[c] = minus ? qv - hv : qv + hv;
        }
        const Prim Pm = infer<EOS, true>(A.eos, A.t, st[0] - st[4], st[1] - st[5], st[2] - st[6], st[3] - st[7],
                                         st[8], ePrev, bad);
        const double vm = (DIR == 1) ? Pm.ux : (DIR == 2) ? Pm.uy : Pm.un;
        if (m == 0) { ut0 = Pm.ut; v0 = vm; }
        else if (m == 1) { ut1 = Pm.ut; v1 = vm; }
        else if (m == 2) { ut2 = Pm.ut; v2 = vm; }
        else { ut3 = Pm.ut; v3 = vm; }
    }
    const double y0 = 1.0 / ut0, y1 = 1.0 / ut1, y2 = 1.0 / ut2, y3 = 1.0 / ut3;
    /* spectral radius of each face, max(|vL / utL|, |vR / utR|) */
    const double af = fmax(fabs(div_rcp(v1, ut1, y1)), fabs(div_rcp(v0, ut0, y0)));
    const double ab = fmax(fabs(div_rcp(v3, ut3, y3)), fabs(div_rcp(v2, ut2, y2)));
    const double d = (DIR == 1) ? A.dx : (DIR == 2) ? A.dy : A.dz;
    const double yd = (DIR == 1) ? A.inv_dx : (DIR == 2) ? A.inv_dy : A.inv_dz;
    double S[4];
    dir_sources_t<NQ>(A, qt, ts, tst, s, d, DIR, S);
    /* H(s-1/2) - H(s+1/2) component by component, added to q* */
#pragma unroll 1
    for (int n = 0; n < NQ; ++n) {
        const double *q = sm + n * P + ts, *h = hs + n * H + hp;
        const double Rf = q[tst] - h[hst], Lf = q[0] + h[0], Rb = q[0] - h[0], Lb = q[-tst] + h[-hst];
        double rf = div_rcp(v0 * Rf, ut0, y0) + div_rcp(v1 * Lf, ut1, y1) - af * (Rf - Lf);
        rf /= 2;
        double rb = div_rcp(v2 * Rb, ut2, y2) + div_rcp(v3 * Lb, ut3, y3) - ab * (Rb - Lb);
        rb /= 2;
        double r = -rf;
        r = r + rb;
        r = div_rcp(r, d, yd);
        if (n < 4) r += (n == 0) ? S[0] : (n == 1) ? S[1] : (n == 2) ? S[2] : S[3];
        r *= A.dt;
        A.qout[n * A.L + s] += r;
    }
    if (bad) raise_error(A.err, kErrNan, s, A.step);
}

/* ---------------------------------------------------------------------
 * The flux along DIR over lines: the lattice is cut into lines along DIR,
 * and the lines into bundles of W = 4 adjacent lines (x-columns for DIR 2
 * and 3, so that a warp's loads cover whole 32-byte sectors, 8 columns
 * measured slower; y-rows for DIR 1, where a warp's 4 x 8 patch of cells
 * is more compact than 32 cells of one row and its root solves diverge
 * less: 27 % fewer Newton iterations per warp on the 131x131x61 Glauber
 * event, x flux 0.639 -> 0.624 ms per step).  Run positions R = pos + nd *
 * bundle enumerate (position along DIR, bundle); a block takes PB = 128 / W
 * consecutive run positions times W columns, which may span the end of one
 * line and the start of the next.  Every thread therefore has a cell (131
 * cells a line no longer leave 29 of 160 lanes idle as 32-wide tiles do).
 * Shared memory holds, per component, each line piece the block touches
 * with its 2-cell halo at both ends (a "slot"), W values per position, and
 * the half slopes at the same indices.
 * --------------------------------------------------------------------- */
#ifndef VH_FLUX_XW
#define VH_FLUX_XW 4      /* lines per bundle along x (1: a warp is 32 cells of one row) */
#endif
template <int DIR, int WW = (DIR == 1) ? VH_FLUX_XW : 4>
struct FluxLines {
    static constexpr int W = WW;
    static constexpr int PB = 128 / W;
    /* line pieces one block can touch, for lines of nd cells */
    static __host__ __device__ int max_slots(int nd) { return (PB - 1) / nd + 2; }
    /* doubles per component of the staged values (and of the half slopes) */
    static __host__ __device__ int plane(int nd) { return (PB + 4 * max_slots(nd)) * W; }
    static __host__ __device__ long long bundles(int nx, int ny, int nz)
    {
        const long long nxq = (nx + W - 1) / W, nyq = (ny + W - 1) / W;
        return (DIR == 1) ? nyq * nz : (DIR == 2) ? nxq * nz : nxq * ny;
    }
};

/* blk: the block's index among the event's line blocks (runs blk * PB on) */
/* the face-once flux's line bundles (mixed precision): 8 adjacent x-columns
 * along y and eta (a warp's loads are 4 rows of 64 bytes; 4 columns, 8 rows
 * of 32 bytes, measured 10-11 % slower), the FP64 flux's along x */
template <int DIR>
using FaceLinesG = FluxLines<DIR, (DIR == 1) ? VH_FLUX_XW : 8>;

template <int NQ, int EOS, int DIR, int UNR = 1, bool PDL = false>
__device__ __forceinline__ void flux_lines_block(const StageArgs &A, double *__restrict__ sm, long long blk)
{
    /* with PDL, only the update of the accumulator (written by the previous
     * phase) waits for the previous kernel; the staged stencil, e and u are
     * the stage's inputs, complete before the stage's first kernel started */
    if (PDL) pdl_trigger();
    using G = FluxLines<DIR>;
    constexpr int W = G::W, PB = G::PB;
    const int nd = (DIR == 1) ? A.nx : (DIR == 2) ? A.ny : A.nz;
    const int PS = G::plane(nd);
    double *__restrict__ hs = sm + NQ * PS;
    const long long sxy = (long long)A.ncx * A.ncy;
    const long long gst = (DIR == 1) ? 1 : (DIR == 2) ? (long long)A.ncx : sxy;
    const int nxq = (A.nx + W - 1) / W;
    const long long nbund = G::bundles(A.nx, A.ny, A.nz);
    const long long Rtot = (long long)nd * nbund;
    /* line and bundle indices in 32-bit arithmetic: an event's cell count
     * is far below 2^31 (its 61 FP64 planes alone would need 1 TB) */
    const unsigned und = (unsigned)nd;
    const long long R0 = blk * PB;
    const long long b0 = (unsigned)R0 / und;
    const int p0 = (int)((unsigned)R0 - (unsigned)b0 * und);
    const int tid = threadIdx.x;
    /* padded address of bundle b's column w at position -2 along DIR, or -1
     * if that column is outside the lattice */
    auto base = [&](long long b, int w) -> long long {
        if (DIR == 1) {
            const unsigned nyq = (unsigned)(A.ny + W - 1) / W, k = (unsigned)b / nyq, jq = (unsigned)b - k * nyq;
            const int y = (int)jq * W + w;
            if (y >= A.ny) return -1;
            return A.ncx * (y + 2) + sxy * (k + 2);
        }
        const unsigned o = (unsigned)b / (unsigned)nxq, xq = (unsigned)b - o * (unsigned)nxq;
        const int x = (int)xq * W + w;
        if (x >= A.nx) return -1;
        return (DIR == 2) ? (x + 2) + sxy * (o + 2) : (x + 2) + A.ncx * (o + 2);
    };
    /* this thread's cell (valid: inside the lattice) */
    const int w = tid % W, pr = tid / W;
    const long long R = R0 + pr;
    long long b = 0, bb = -1;
    int pos = 0;
    if (R < Rtot) {
        b = (unsigned)R / und;
        pos = (int)((unsigned)R - (unsigned)b * und);
        bb = base(b, w);
    }
    const bool valid = bb >= 0;
    const long long s = valid ? bb + (long long)(pos + 2) * gst : 0;
    if (valid) prefetch_flux_cell<NQ>(A, s, DIR);
    /* the root solves' start, read while the stencil is staged */
    const double ePrev = valid ? __ldg(A.ein + s) : 0.0;
    /* staging: slot l covers positions [first_l - 2, first_l + len_l + 2) of
     * bundle b0 + l at shared indices [M_l, M_l + len_l + 4) */
    const int mlen_max = PS / W;
    for (int r = tid; r < mlen_max * W; r += 128) {
        const int m = r / W, w = r - m * W;
        int l = 0, M = 0, first = p0, left = PB;
        long long off = -1;
        for (; l < G::max_slots(nd) && left > 0; ++l) {
            const int len = (nd - first < left) ? nd - first : left;
            if (m < M + len + 4) {
                if (b0 + l < nbund) {
                    const long long bb = base(b0 + l, w);
                    if (bb >= 0) off = bb + (long long)(first + (m - M)) * gst;
                }
                break;
            }
            M += len + 4;
            left -= len;
            first = 0;
        }
        if (off >= 0) {
#pragma unroll 1
            for (int n = 0; n < NQ; ++n) cp_async8(sm + n * PS + r, A.qin + n * A.L + off);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    const double th = A.theta;
    for (int r = tid + W; r < (mlen_max - 1) * W; r += 128) {
#pragma unroll 1
        for (int n = 0; n < NQ; ++n) {
            const double *q = sm + n * PS + r;
            hs[n * PS + r] = approx_deriv(th, q[-W], q[0], q[W]) / 2;
        }
    }
    __syncthreads();
    if (!valid) return;
    const int ts = ((int)(R - R0) + 2 + 4 * (int)(b - b0)) * W + w;
    constexpr int tst = W;
    const QTile qt{sm, PS};
    bool bad = false;
    /* states m = 0..3: forward face R, L; backward face R, L */
    double ut0 = 0, ut1 = 0, ut2 = 0, ut3 = 0, v0 = 0, v1 = 0, v2 = 0, v3 = 0;
#pragma unroll 1
    for (int mm = 0; mm < 4; ++mm) {
        const int o = (mm == 0) ? ts + tst : (mm == 3) ? ts - tst : ts;
        const bool minus = (mm & 1) == 0;        /* R states subtract the half slope */
        double st[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            const int n = (c < 8) ? c : 14;
            if (n >= NQ) { st[c] = 0; continue; }
            const double qv = sm[n * PS + o], hv = hs[n * PS + o];
            st[c] = minus ? qv - hv : qv + hv;
        }
        const Prim Pm = infer<EOS, true>(A.eos, A.t, st[0] - st[4], st[1] - st[5], st[2] - st[6], st[3] - st[7],
                                         st[8], ePrev, bad);
        const double vm = (DIR == 1) ? Pm.ux : (DIR == 2) ? Pm.uy : Pm.un;
        if (mm == 0) { ut0 = Pm.ut; v0 = vm; }
        else if (mm == 1) { ut1 = Pm.ut; v1 = vm; }
        else if (mm == 2) { ut2 = Pm.ut; v2 = vm; }
        else { ut3 = Pm.ut; v3 = vm; }
    }
    /* u of the direction sources, read while the reciprocals run */
    const double uts = __ldg(A.uin + s), uds = __ldg(A.uin + DIR * A.L + s);
    const double y0 = 1.0 / ut0, y1 = 1.0 / ut1, y2 = 1.0 / ut2, y3 = 1.0 / ut3;
    const double af = fmax(fabs(div_rcp(v1, ut1, y1)), fabs(div_rcp(v0, ut0, y0)));
    const double ab = fmax(fabs(div_rcp(v3, ut3, y3)), fabs(div_rcp(v2, ut2, y2)));
    const double d = (DIR == 1) ? A.dx : (DIR == 2) ? A.dy : A.dz;
    const double yd = (DIR == 1) ? A.inv_dx : (DIR == 2) ? A.inv_dy : A.inv_dz;
    double S[4];
    dir_sources_uv<NQ>(A, qt, ts, tst, uts, uds, d, DIR, S);
    if (PDL) pdl_wait();
#pragma unroll UNR
    for (int n = 0; n < NQ; ++n) {
        const double *q = sm + n * PS + ts, *h = hs + n * PS + ts;
        const double Rf = q[tst] - h[tst], Lf = q[0] + h[0], Rb = q[0] - h[0], Lb = q[-tst] + h[-tst];
        double rf = div_rcp(v0 * Rf, ut0, y0) + div_rcp(v1 * Lf, ut1, y1) - af * (Rf - Lf);
        rf /= 2;
        double rb = div_rcp(v2 * Rb, ut2, y2) + div_rcp(v3 * Lb, ut3, y3) - ab * (Rb - Lb);
        rb /= 2;
        double r = -rf;
        r = r + rb;
        r = div_rcp(r, d, yd);
        if (n < 4) r += (n == 0) ? S[0] : (n == 1) ? S[1] : (n == 2) ? S[2] : S[3];
        r *= A.dt;
        A.qout[n * A.L + s] += r;
    }
    if (bad) raise_error(A.err, kErrNan, s, A.step);
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
    /* nz = 1: the eta neighbours are the cell itself (see put_with_ghosts) */
    const long long sx = 1, sy = A.ncx, sz = (A.nz > 1) ? (long long)A.ncx * A.ncy : 0;
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
    /* the dynamical sources, SourceTerms.cpp:584-587 (0 without them) */
    const double *__restrict__ sv = A.src;
    const double s0 = sv ? __ldg(sv + s) : 0.0, s1 = sv ? __ldg(sv + L + s) : 0.0;
    const double s2 = sv ? __ldg(sv + 2 * L + s) : 0.0, s3 = sv ? __ldg(sv + 3 * L + s) : 0.0;
    S[0] = s0 - (div_rcp(Qv[0], t, yt) + t * tnn) + dkvk * (Qv[4] - p - Pi) - vx * dxp - vy * dyp - vn * dnp;
    S[1] = s1 - div_rcp(Qv[1], t, yt) - dxp + dkvk * Qv[5];
    S[2] = s2 - div_rcp(Qv[2], t, yt) - dyp + dkvk * Qv[6];
    S[3] = s3 - div_rcp(3 * Qv[3], t, yt) - dnp / A.t2pow + dkvk * Qv[7];
    pimunu_rhs<double, EOS, NQ == 15>(A.eos, A.zeta, S + 4, t, yt, e, p, ut, ux, uy, un,
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
__device__ __forceinline__ void regulate(const StageArgs &A, double *__restrict__ acc, const Prim &P, bool &bad,
                                         long long s)
{
    if (P.e > A.e_reg) {
        /* regFacShear / regFacBulk of the reference (kept only when asked for) */
        if (A.regfac) { A.regfac[s] = 1.0; if (NQ == 15) A.regfac[A.L + s] = 1.0; }
        return;
    }
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
    if (A.regfac) A.regfac[s] = facShear;
    if (NQ == 15) {
        double rhoBulk = fabs(Pi) / P.p;
        double facBulk = vh_tanh(rhoBulk) / rhoBulk;
        if (fabs(rhoBulk) < 1.e-7) facBulk = 1.0;
        acc[14] *= facBulk;
        if (isnan(facBulk)) bad = true;
        if (A.regfac) A.regfac[A.L + s] = facBulk;
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

/* the cell and its zero-gradient ghost copies (DynamicalVariables.cpp:220-378).
 * A 2+1D event (nz = 1) keeps no eta ghost planes while it evolves: nothing
 * in the step reads them (the eta pass is skipped, and the eta differences of
 * the source terms and of the vorticity take the cell itself, which is what
 * the ghost copies hold), so the four copies of every cell -- 4/5 of the
 * phase's stores -- are left out and written only when a field is read
 * (launch_eta_ghost_fill). */
template <int NQ>
__device__ __forceinline__ void put_with_ghosts(const StageArgs &A, int i, int j, int k, long long s,
                                                const double *__restrict__ acc, const Prim &P)
{
    const long long sxy = (long long)A.ncx * A.ncy;
    put_cell<NQ>(A, s, acc, P);
    if (i == 2) { put_cell<NQ>(A, s - 1, acc, P); put_cell<NQ>(A, s - 2, acc, P); }
    if (i == A.nx + 1) { put_cell<NQ>(A, s + 1, acc, P); put_cell<NQ>(A, s + 2, acc, P); }
    if (j == 2) { put_cell<NQ>(A, s - A.ncx, acc, P); put_cell<NQ>(A, s - 2 * A.ncx, acc, P); }
    if (j == A.ny + 1) { put_cell<NQ>(A, s + A.ncx, acc, P); put_cell<NQ>(A, s + 2 * A.ncx, acc, P); }
    if (A.nz > 1) {
        if (k == 2) { put_cell<NQ>(A, s - sxy, acc, P); put_cell<NQ>(A, s - 2 * sxy, acc, P); }
        if (k == A.nz + 1) { put_cell<NQ>(A, s + sxy, acc, P); put_cell<NQ>(A, s + 2 * sxy, acc, P); }
    }
}

/* One whole stage for cell (i, j, k) at padded index s. */
template <int NQ, int EOS, bool HAS_Z, bool STAGE2>
__device__ __forceinline__ void stage_body(const StageArgs &A, int i, int j, int k, long long s)
{
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
    regulate<NQ>(A, acc, P, bad, s);
    if (bad) raise_error(A.err, kErrNan, s, A.step);
    put_with_ghosts<NQ>(A, i, j, k, s, acc, P);
}

/* Phase bodies of the split stage, in the reference's phase order
 * (eulerStepKernelSource, X, Y, Z, then inference/regulation/ghosts).  The
 * partial sums live in qout between phases; FP64 stores are exact, so the
 * split stage is bit-identical to stage_body. */
template <int NQ, int EOS>
__device__ __forceinline__ void source_body(const StageArgs &A, long long s)
{
    double acc[NQ];
    source_update<NQ, EOS>(A, s, acc);
#pragma unroll
    for (int n = 0; n < NQ; ++n) A.qout[n * A.L + s] = acc[n];
}

template <int NQ, int EOS, int DIR>
__device__ __forceinline__ void flux_body(const StageArgs &A, long long s)
{
    prefetch_flux_cell<NQ>(A, s, DIR);
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
__device__ __forceinline__ void final_body(const StageArgs &A, int i, int j, int k, long long s)
{
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
    regulate<NQ>(A, acc, P, bad, s);
    if (bad) raise_error(A.err, kErrNan, s, A.step);
    put_with_ghosts<NQ>(A, i, j, k, s, acc, P);
}

/* =====================================================================
 * Mixed precision (vh_config.precision = VH_PREC_MIXED): the limiter, the
 * flux arithmetic and the source terms in FP32; the conserved variables,
 * their RK accumulation, the half-site states fed to the root solve, the
 * root solve itself (infer) and the EoS stay FP64.  Differences of stored
 * FP64 values are taken in FP64 before rounding to FP32, so no cancellation
 * happens in FP32.  These bodies are instantiated only by the mixed
 * translation unit (vh_mixed.cu, compiled with fast FP32 division).
 * ===================================================================== */
__device__ __forceinline__ float minmod_f(float x, float y)
{
    const float sx = (x < 0.f) ? -1.f : 1.f, sy = (y < 0.f) ? -1.f : 1.f;
    return (sx + sy) * fminf(fabsf(x), fabsf(y)) * 0.5f;
}

/* FluxLimiter.cpp:14-32 on the FP64 differences y - x, z - x, z - y */
__device__ __forceinline__ float slope_f(float th, double x, double y, double z)
{
    const float l = th * (float)(y - x), c = (float)(z - x) * 0.5f, r = th * (float)(z - y);
    return minmod_f(l, minmod_f(c, r));
}

__device__ __forceinline__ void extrapolate_m(const double *__restrict__ qn, long long b, long long st, float th,
                                              double &qR, double &qL)
{
    const double A = __ldg(qn + b - st), B = __ldg(qn + b), C = __ldg(qn + b + st), D = __ldg(qn + b + 2 * st);
    qR = C - (double)(0.5f * slope_f(th, B, C, D));
    qL = B + (double)(0.5f * slope_f(th, A, B, C));
}

/* face_flux with FP32 slopes and flux arithmetic; FP64 half-site states and root solve */
template <int NQ, int EOS>
__device__ __forceinline__ void face_flux_m(const StageArgs &A, long long b, long long st, int dir, bool fwd,
                                            double ePrev, double *__restrict__ r, bool &bad)
{
    const float th = (float)A.theta;
    const long long L = A.L;
    const double *__restrict__ q = A.qin;
    double qRs[8], qLs[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) extrapolate_m(q + c * L, b, st, th, qRs[c], qLs[c]);
    double PiR = 0, PiL = 0;
    if (NQ == 15) extrapolate_m(q + 14 * L, b, st, th, PiR, PiL);
    Prim R = infer<EOS, true>(A.eos, A.t, qRs[0] - qRs[4], qRs[1] - qRs[5], qRs[2] - qRs[6], qRs[3] - qRs[7], PiR, ePrev, bad);
    Prim Lf = infer<EOS, true>(A.eos, A.t, qLs[0] - qLs[4], qLs[1] - qLs[5], qLs[2] - qLs[6], qLs[3] - qLs[7], PiL, ePrev, bad);
    const float vR = (float)((dir == 1) ? R.ux : (dir == 2) ? R.uy : R.un);
    const float vL = (float)((dir == 1) ? Lf.ux : (dir == 2) ? Lf.uy : Lf.un);
    const float sR = vR / (float)R.ut, sL = vL / (float)Lf.ut;
    const float a = fmaxf(fabsf(sL), fabsf(sR));
#pragma unroll
    for (int n = 0; n < NQ; ++n) {
        double qR, qL;
        if (n < 8) { qR = qRs[n]; qL = qLs[n]; }
        else if (n == 14) { qR = PiR; qL = PiL; }
        else extrapolate_m(q + n * L, b, st, th, qR, qL);
        const float res = 0.5f * (sR * (float)qR + sL * (float)qL - a * (float)(qR - qL));
        r[n] = fwd ? -(double)res : r[n] + (double)res;
    }
}

/* source_update in FP32 (SourceTerms.cpp:421-612), accumulated onto the FP64 q */
template <int NQ, int EOS>
__device__ __forceinline__ void source_update_m(const StageArgs &A, long long s, double *__restrict__ acc)
{
    const long long L = A.L;
    const float th = (float)A.theta;
    /* nz = 1: the eta neighbours are the cell itself (see put_with_ghosts) */
    const long long sx = 1, sy = A.ncx, sz = (A.nz > 1) ? (long long)A.ncx * A.ncy : 0;
    double Qv[NQ];
#pragma unroll
    for (int n = 0; n < NQ; ++n) Qv[n] = __ldg(A.qin + n * L + s);
    const double *__restrict__ utv = A.uin, *__restrict__ uxv = A.uin + L, *__restrict__ uyv = A.uin + 2 * L,
                 *__restrict__ unv = A.uin + 3 * L, *__restrict__ pv = A.pin;
    const double e = __ldg(A.ein + s), p = __ldg(pv + s);
    const double utd = __ldg(utv + s), uxd = __ldg(uxv + s), uyd = __ldg(uyv + s), und = __ldg(unv + s);
    const float ydx = (float)A.inv_dx, ydy = (float)A.inv_dy, ydz = (float)A.inv_dz;
#define SLOPE(v, c, st, y) (slope_f(th, __ldg((v) + s - (st)), (c), __ldg((v) + s + (st))) * (y))
    const float dxut = SLOPE(utv, utd, sx, ydx), dxux = SLOPE(uxv, uxd, sx, ydx), dxuy = SLOPE(uyv, uyd, sx, ydx), dxun = SLOPE(unv, und, sx, ydx);
    const float dyut = SLOPE(utv, utd, sy, ydy), dyux = SLOPE(uxv, uxd, sy, ydy), dyuy = SLOPE(uyv, uyd, sy, ydy), dyun = SLOPE(unv, und, sy, ydy);
    const float dnut = SLOPE(utv, utd, sz, ydz), dnux = SLOPE(uxv, uxd, sz, ydz), dnuy = SLOPE(uyv, uyd, sz, ydz), dnun = SLOPE(unv, und, sz, ydz);
    const float dxp = SLOPE(pv, p, sx, ydx), dyp = SLOPE(pv, p, sy, ydy), dnp = SLOPE(pv, p, sz, ydz);
#undef SLOPE
    const float t = (float)A.t, yt = (float)A.inv_t;
    const float Pi = (NQ == 15) ? (float)Qv[14] : 0.f;
    const float ut = (float)utd, ux = (float)uxd, uy = (float)uyd, un = (float)und;
    const float pP = (float)p + Pi;
    const float tnn = ((float)e + pP) * un * un + pP * yt * yt + (float)Qv[13];
    const float yut = 1.f / ut;
    const float vx = ux * yut, vy = uy * yut, vn = un * yut;
    const float dkvk = (dxux - vx * dxut) * yut + (dyuy - vy * dyut) * yut + (dnun - vn * dnut) * yut;
    float S[NQ];
    const double *__restrict__ sv = A.src;
    const float s0 = sv ? (float)__ldg(sv + s) : 0.f, s1 = sv ? (float)__ldg(sv + L + s) : 0.f;
    const float s2 = sv ? (float)__ldg(sv + 2 * L + s) : 0.f, s3 = sv ? (float)__ldg(sv + 3 * L + s) : 0.f;
    S[0] = s0 - ((float)Qv[0] * yt + t * tnn) + dkvk * ((float)Qv[4] - (float)p - Pi) - vx * dxp - vy * dyp - vn * dnp;
    S[1] = s1 - (float)Qv[1] * yt - dxp + dkvk * (float)Qv[5];
    S[2] = s2 - (float)Qv[2] * yt - dyp + dkvk * (float)Qv[6];
    S[3] = s3 - 3.f * (float)Qv[3] * yt - dnp / (float)A.t2pow + dkvk * (float)Qv[7];
    float pvf[10];
#pragma unroll
    for (int n = 0; n < 10; ++n) pvf[n] = (float)Qv[4 + n];
    pimunu_rhs<float, EOS, NQ == 15>(A.eos, A.zeta, S + 4, t, yt, e, p, utd, uxd, uyd, und,
                                     __ldg(A.upin + s), __ldg(A.upin + L + s), __ldg(A.upin + 2 * L + s), __ldg(A.upin + 3 * L + s),
                                     pvf, Pi, dxut, dyut, dnut, dxux, dyux, dnux, dxuy, dyuy, dnuy, dxun, dyun, dnun, dkvk,
                                     (float)A.etabar, (float)A.dt);
#pragma unroll
    for (int n = 0; n < NQ; ++n) acc[n] = Qv[n] + A.dt * (double)S[n];
}

template <int NQ, int EOS>
__device__ __forceinline__ void source_body_m(const StageArgs &A, long long s)
{
    double acc[NQ];
    source_update_m<NQ, EOS>(A, s, acc);
#pragma unroll
    for (int n = 0; n < NQ; ++n) A.qout[n * A.L + s] = acc[n];
}

template <int NQ, int EOS, int DIR>
__device__ __forceinline__ void flux_body_m(const StageArgs &A, long long s)
{
    const double ePrev = __ldg(A.ein + s);
    bool bad = false;
    const long long st = (DIR == 1) ? 1 : (DIR == 2) ? (long long)A.ncx : (long long)A.ncx * A.ncy;
    const double d = (DIR == 1) ? A.dx : (DIR == 2) ? A.dy : A.dz;
    const double yd = (DIR == 1) ? A.inv_dx : (DIR == 2) ? A.inv_dy : A.inv_dz;
    double r[NQ];
#pragma unroll 1
    for (int f = 0; f < 2; ++f) face_flux_m<NQ, EOS>(A, f == 0 ? s : s - st, st, DIR, f == 0, ePrev, r, bad);
    double S[4];
    dir_sources<NQ>(A, s, st, d, DIR, S);
#pragma unroll
    for (int n = 0; n < 4; ++n) r[n] = (r[n] * yd + S[n]) * A.dt;
#pragma unroll
    for (int n = 4; n < NQ; ++n) r[n] *= yd * A.dt;
#pragma unroll
    for (int n = 0; n < NQ; ++n) A.qout[n * A.L + s] += r[n];
    if (bad) raise_error(A.err, kErrNan, s, A.step);
}

/* the fused stage in mixed precision */
template <int NQ, int EOS, bool HAS_Z, bool STAGE2>
__device__ __forceinline__ void stage_body_m(const StageArgs &A, int i, int j, int k, long long s)
{
    const double ePrev = __ldg(A.ein + s);
    bool bad = false;
    double acc[NQ];
    source_update_m<NQ, EOS>(A, s, acc);
#pragma unroll 1
    for (int dir = 1; dir <= (HAS_Z ? 3 : 2); ++dir) {
        const long long st = (dir == 1) ? 1 : (dir == 2) ? (long long)A.ncx : (long long)A.ncx * A.ncy;
        const double d = (dir == 1) ? A.dx : (dir == 2) ? A.dy : A.dz;
        const double yd = (dir == 1) ? A.inv_dx : (dir == 2) ? A.inv_dy : A.inv_dz;
        double r[NQ];
#pragma unroll 1
        for (int f = 0; f < 2; ++f) face_flux_m<NQ, EOS>(A, f == 0 ? s : s - st, st, dir, f == 0, ePrev, r, bad);
        double S[4];
        dir_sources<NQ>(A, s, st, d, dir, S);
#pragma unroll
        for (int n = 0; n < 4; ++n) acc[n] += (r[n] * yd + S[n]) * A.dt;
#pragma unroll
        for (int n = 4; n < NQ; ++n) acc[n] += r[n] * yd * A.dt;
    }
    if (STAGE2) {
#pragma unroll
        for (int n = 0; n < NQ; ++n) acc[n] = (acc[n] + __ldg(A.qbase + n * A.L + s)) * 0.5;
    }
    Prim P = infer<EOS>(A.eos, A.t_inf, acc[0] - acc[4], acc[1] - acc[5], acc[2] - acc[6], acc[3] - acc[7],
                        (NQ == 15) ? acc[14] : 0.0, ePrev, bad);
    regulate<NQ>(A, acc, P, bad, s);
    if (bad) raise_error(A.err, kErrNan, s, A.step);
    put_with_ghosts<NQ>(A, i, j, k, s, acc, P);
}

/* ---------------------------------------------------------------------
 * Face-once flux (mixed precision).  The reference evaluates every face twice
 * -- once for each adjacent cell, each time with that cell's e as the root
 * solve's starting point (SemiDiscreteKurganovTadmorScheme.cpp:14-62 called
 * from both neighbours) -- which bit parity requires.  The mixed path
 * evaluates each face once, starting the root solve from the e of the cell on
 * the face's upper side, and hands the face flux to both cells through shared
 * memory: half the root solves and extrapolations, and the flux leaving one
 * cell is exactly the flux entering its neighbour.  Where the two cells lie
 * on different sides of the root solve's e <= 0.1 branch (the dilute edge)
 * the lower cell evaluates its forward face itself, as the reference does.
 *
 * A block of TX x TY threads covers a tile of faces: along x the faces
 * i0 - 1/2 .. i0 + TX - 3/2 of TY rows and the cells i0 .. i0 + TX - 2; along
 * y (eta) the block's second index runs along y (eta) and the last row of
 * threads only computes faces.
 * --------------------------------------------------------------------- */
template <int NQ, int EOS>
__device__ __forceinline__ void face_H_m(const StageArgs &A, long long b, long long st, int dir, double ePrev,
                                         double *__restrict__ H, bool &bad)
{
#pragma unroll
    for (int n = 0; n < NQ; ++n) H[n] = 0.0;
    face_flux_m<NQ, EOS>(A, b, st, dir, false, ePrev, H, bad);
}

/* one tile of the face-once flux along DIR; (i0, j0, k0) interior coordinates
 * of the block's first face-owning cell; sm holds NQ * TX * TY doubles */
template <int NQ, int EOS, int DIR, int TX, int TY, bool PDL = false>
__device__ __forceinline__ void flux_faces_tile(const StageArgs &A, int i0, int j0, int k0, double *__restrict__ sm)
{
    if (PDL) pdl_trigger();   /* see flux_lines_block */
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty;
    const int i = i0 + tx + 2;
    const int j = (DIR == 3) ? j0 + 2 : j0 + ty + 2;
    const int k = (DIR == 3) ? k0 + ty + 2 : k0 + 2;
    const long long sxy = (long long)A.ncx * A.ncy;
    const long long st = (DIR == 1) ? 1 : (DIR == 2) ? (long long)A.ncx : sxy;
    const int along = (DIR == 1) ? i : (DIR == 2) ? j : k;             /* padded index along DIR */
    const int n_along = (DIR == 1) ? A.nx : (DIR == 2) ? A.ny : A.nz;
    const bool across_ok = (DIR == 1) ? (j < A.ny + 2 && k < A.nz + 2)
                         : (DIR == 2) ? (i < A.nx + 2 && k < A.nz + 2)
                                      : (i < A.nx + 2 && j < A.ny + 2);
    /* this thread's face lies between cells along - 1 and along; the faces up
     * to the one after the last interior cell are needed (its stencil reaches
     * the second ghost layer, index n_along + 3) */
    const bool face_ok = across_ok && along <= n_along + 2;
    const long long s = i + (long long)A.ncx * j + sxy * k;
    bool bad = false;
    double H[NQ];
    if (face_ok) {
        prefetch_flux_cell<NQ>(A, s, DIR);
        face_H_m<NQ, EOS>(A, s - st, st, DIR, __ldg(A.ein + s), H, bad);
        if constexpr (DIR != 1) {
#pragma unroll
            for (int n = 0; n < NQ; ++n) sm[n * (TX * TY) + tid] = H[n];
        }
    } else {
#pragma unroll
        for (int n = 0; n < NQ; ++n) H[n] = 0.0;
    }
    /* along x a row of faces is one warp: the next face comes by shuffle, no
     * block barrier; along y and eta it comes through shared memory */
    double Hn[NQ];
    if constexpr (DIR == 1) {
        static_assert(TX == 32, "a row of x faces is one warp");
#pragma unroll
        for (int n = 0; n < NQ; ++n) Hn[n] = __shfl_down_sync(0xffffffffu, H[n], 1);
    } else {
        __syncthreads();
    }
    const bool last = (DIR == 1) ? (tx == TX - 1) : (ty == TY - 1);
    if (face_ok && !last && along <= n_along + 1) {
        const int nxt = (DIR == 1) ? tid + 1 : tid + TX;
        const double d = (DIR == 1) ? A.dx : (DIR == 2) ? A.dy : A.dz;
        const double yd = (DIR == 1) ? A.inv_dx : (DIR == 2) ? A.inv_dy : A.inv_dz;
        double r[NQ];
        const double e_self = __ldg(A.ein + s), e_next = __ldg(A.ein + s + st);
        if ((e_self <= 0.1) != (e_next <= 0.1)) {
            double F[NQ];
            face_H_m<NQ, EOS>(A, s, st, DIR, e_self, F, bad);
#pragma unroll
            for (int n = 0; n < NQ; ++n) r[n] = H[n] - F[n];
        } else {
#pragma unroll
            for (int n = 0; n < NQ; ++n) r[n] = H[n] - ((DIR == 1) ? Hn[n] : sm[n * (TX * TY) + nxt]);
        }
        double S[4];
        dir_sources<NQ>(A, s, st, d, DIR, S);
#pragma unroll
        for (int n = 0; n < 4; ++n) r[n] = (r[n] * yd + S[n]) * A.dt;
#pragma unroll
        for (int n = 4; n < NQ; ++n) r[n] *= yd * A.dt;
        if (PDL) pdl_wait();
#pragma unroll
        for (int n = 0; n < NQ; ++n) A.qout[n * A.L + s] += r[n];
    }
    if (bad) raise_error(A.err, kErrNan, s, A.step);
    if constexpr (DIR != 1) __syncthreads();
}

/* The face-once flux over line pieces (mixed precision, single events):
 * the faces of each line along DIR (nd + 1 of them, face f between cells
 * f - 1 and f) enumerated like FluxLines' cells, R = f + (nd + 1) * bundle,
 * one face per thread, the W columns of a bundle side by side.  A block
 * takes PB consecutive faces and updates the cells of all but its last face
 * (the next block starts there: blocks overlap by one face), so no lane
 * idles at line ends and only one face in PB is computed twice.  The face
 * arithmetic, the next face through shared memory and the recomputation
 * across the root solve's e <= 0.1 branch are those of flux_faces_tile, so
 * a cell's update is the same.  sm: NQ * 128 doubles. */
template <int NQ, int EOS, int DIR, bool PDL = false>
__device__ __forceinline__ void flux_faces_lines(const StageArgs &A, double *__restrict__ sm, long long blk)
{
    if (PDL) pdl_trigger();   /* see flux_lines_block */
    using G = FaceLinesG<DIR>;
    constexpr int W = G::W, PB = G::PB;
    const int nd = (DIR == 1) ? A.nx : (DIR == 2) ? A.ny : A.nz;
    const int nf = nd + 1;
    const long long sxy = (long long)A.ncx * A.ncy;
    const long long st = (DIR == 1) ? 1 : (DIR == 2) ? (long long)A.ncx : sxy;
    const int nxq = (A.nx + W - 1) / W;
    const long long Rtot = (long long)nf * G::bundles(A.nx, A.ny, A.nz);
    const int tid = threadIdx.x, w = tid % W, pr = tid / W;
    const long long R = blk * (PB - 1) + pr;
    bool face_ok = R < Rtot;
    int f = 0;
    long long s = 0;
    if (face_ok) {
        /* 32-bit index arithmetic, as in flux_lines_block */
        const unsigned b = (unsigned)R / (unsigned)nf;
        f = (int)((unsigned)R - b * (unsigned)nf);
        long long base;
        if (DIR == 1) {
            const unsigned nyq = (unsigned)(A.ny + W - 1) / W, k = b / nyq, jq = b - k * nyq;
            const int y = (int)jq * W + w;
            face_ok = y < A.ny;
            base = A.ncx * (y + 2) + sxy * (k + 2);
        } else {
            const unsigned o = b / (unsigned)nxq, xq = b - o * (unsigned)nxq;
            const int x = (int)xq * W + w;
            face_ok = x < A.nx;
            base = (DIR == 2) ? (x + 2) + sxy * (o + 2) : (x + 2) + A.ncx * (o + 2);
        }
        s = base + (long long)(f + 2) * st;       /* the face's upper cell (a ghost for f = nd) */
    }
    bool bad = false;
    double H[NQ];
    if (face_ok) {
        prefetch_flux_cell<NQ>(A, s, DIR);
        face_H_m<NQ, EOS>(A, s - st, st, DIR, __ldg(A.ein + s), H, bad);
    } else {
#pragma unroll
        for (int n = 0; n < NQ; ++n) H[n] = 0.0;
    }
#pragma unroll
    for (int n = 0; n < NQ; ++n) sm[n * 128 + tid] = H[n];
    __syncthreads();
    if (face_ok && f < nd && pr < PB - 1) {
        const int nxt = tid + W;                  /* face f + 1 of the same line */
        const double d = (DIR == 1) ? A.dx : (DIR == 2) ? A.dy : A.dz;
        const double yd = (DIR == 1) ? A.inv_dx : (DIR == 2) ? A.inv_dy : A.inv_dz;
        double r[NQ];
        const double e_self = __ldg(A.ein + s), e_next = __ldg(A.ein + s + st);
        if ((e_self <= 0.1) != (e_next <= 0.1)) {
            double F[NQ];
            face_H_m<NQ, EOS>(A, s, st, DIR, e_self, F, bad);
#pragma unroll
            for (int n = 0; n < NQ; ++n) r[n] = H[n] - F[n];
        } else {
#pragma unroll
            for (int n = 0; n < NQ; ++n) r[n] = H[n] - sm[n * 128 + nxt];
        }
        double S[4];
        dir_sources<NQ>(A, s, st, d, DIR, S);
#pragma unroll
        for (int n = 0; n < 4; ++n) r[n] = (r[n] * yd + S[n]) * A.dt;
#pragma unroll
        for (int n = 4; n < NQ; ++n) r[n] *= yd * A.dt;
        if (PDL) pdl_wait();
#pragma unroll
        for (int n = 0; n < NQ; ++n) A.qout[n * A.L + s] += r[n];
    }
    if (bad) raise_error(A.err, kErrNan, s, A.step);
}

/* ---------------------------------------------------------------------
 * Face-parallel stage for small lattices.  A single event of ~10^4 cells is
 * latency-bound: one thread per cell carries the whole stage.  Here each cell
 * gets 1 + 2 * ndir threads: thread 0 evaluates the source term, thread 1 +
 * 2 (dir - 1) + f the face f (0 forward, 1 backward) of axis dir, all with the
 * cell's e as the root solve's start; the face results go through shared
 * memory and thread 0 combines them in flux_update's order -- r = (-H_fwd) +
 * H_bwd per axis, the same operations as the one-thread stage, so the result
 * is bit-identical (the backward face is accumulated onto -0.0, which leaves
 * every value, signed zeros included, unchanged).
 * --------------------------------------------------------------------- */
template <int NQ, int EOS, bool HAS_Z, bool STAGE2, bool MIXED>
__device__ __forceinline__ void stage_faces_cell(const StageArgs &A, int i, int j, int k, bool valid,
                                                 double *__restrict__ sm /* [2 ndir][NQ][TX] */, int TX)
{
    constexpr int ND = HAS_Z ? 3 : 2;
    const int tx = threadIdx.x, role = threadIdx.y;
    const long long sxy = (long long)A.ncx * A.ncy;
    const long long s = i + (long long)A.ncx * j + sxy * k;
    bool bad = false;
    double acc[NQ];
    if (valid && role > 0) {
        const int dir = 1 + (role - 1) / 2;
        const bool fwd = ((role - 1) % 2) == 0;
        const long long st = (dir == 1) ? 1 : (dir == 2) ? (long long)A.ncx : sxy;
        const double ePrev = __ldg(A.ein + s);
        double r[NQ];
#pragma unroll
        for (int n = 0; n < NQ; ++n) r[n] = -0.0;
        if constexpr (MIXED) face_flux_m<NQ, EOS>(A, fwd ? s : s - st, st, dir, fwd, ePrev, r, bad);
        else face_flux<NQ, EOS>(A, fwd ? s : s - st, st, dir, fwd, ePrev, r, bad);
#pragma unroll
        for (int n = 0; n < NQ; ++n) sm[((role - 1) * NQ + n) * TX + tx] = r[n];
    } else if (valid) {
        if constexpr (MIXED) source_update_m<NQ, EOS>(A, s, acc);
        else source_update<NQ, EOS>(A, s, acc);
    }
    __syncthreads();
    if (valid && role == 0) {
        const double ePrev = __ldg(A.ein + s);
#pragma unroll 1
        for (int dir = 1; dir <= ND; ++dir) {
            const long long st = (dir == 1) ? 1 : (dir == 2) ? (long long)A.ncx : sxy;
            const double d = (dir == 1) ? A.dx : (dir == 2) ? A.dy : A.dz;
            const double yd = (dir == 1) ? A.inv_dx : (dir == 2) ? A.inv_dy : A.inv_dz;
            const double *hf = sm + (2 * (dir - 1)) * NQ * TX, *hb = sm + (2 * (dir - 1) + 1) * NQ * TX;
            double r[NQ];
#pragma unroll
            for (int n = 0; n < NQ; ++n) r[n] = hf[n * TX + tx] + hb[n * TX + tx];
            double S[4];
            dir_sources<NQ>(A, s, st, d, dir, S);
            if constexpr (MIXED) {
#pragma unroll
                for (int n = 0; n < 4; ++n) acc[n] += (r[n] * yd + S[n]) * A.dt;
#pragma unroll
                for (int n = 4; n < NQ; ++n) acc[n] += r[n] * yd * A.dt;
            } else {
#pragma unroll
                for (int n = 0; n < NQ; ++n) r[n] = div_rcp(r[n], d, yd);
#pragma unroll
                for (int n = 0; n < 4; ++n) { r[n] += S[n]; r[n] *= A.dt; }
#pragma unroll
                for (int n = 4; n < NQ; ++n) r[n] *= A.dt;
#pragma unroll
                for (int n = 0; n < NQ; ++n) acc[n] += r[n];
            }
        }
        if (!HAS_Z && !MIXED) {
#pragma unroll
            for (int n = 0; n < NQ; ++n) acc[n] += 0.0;
        }
        if (STAGE2) {
            if constexpr (MIXED) {
#pragma unroll
                for (int n = 0; n < NQ; ++n) acc[n] = (acc[n] + __ldg(A.qbase + n * A.L + s)) * 0.5;
            } else {
#pragma unroll
                for (int n = 0; n < NQ; ++n) { acc[n] += __ldg(A.qbase + n * A.L + s); acc[n] /= 2; }
            }
        }
        Prim P = infer<EOS, true>(A.eos, A.t_inf, acc[0] - acc[4], acc[1] - acc[5], acc[2] - acc[6], acc[3] - acc[7],
                                  (NQ == 15) ? acc[14] : 0.0, ePrev, bad);
        regulate<NQ>(A, acc, P, bad, s);
        put_with_ghosts<NQ>(A, i, j, k, s, acc, P);
    }
    if (bad) raise_error(A.err, kErrNan, s, A.step);
}

/* launch-form independent selection of the per-cell bodies: MIXED picks the
 * mixed-precision source, flux and fused bodies; finalize is FP64 in both */
template <int NQ, int EOS, bool MIXED>
__device__ __forceinline__ void source_phase(const StageArgs &A, long long s)
{
    if constexpr (MIXED) source_body_m<NQ, EOS>(A, s);
    else source_body<NQ, EOS>(A, s);
}
template <int NQ, int EOS, int DIR, bool MIXED>
__device__ __forceinline__ void flux_phase(const StageArgs &A, long long s)
{
    if constexpr (MIXED) flux_body_m<NQ, EOS, DIR>(A, s);
    else flux_body<NQ, EOS, DIR>(A, s);
}
template <int NQ, int EOS, bool HAS_Z, bool STAGE2, bool MIXED>
__device__ __forceinline__ void stage_phase(const StageArgs &A, int i, int j, int k, long long s)
{
    if constexpr (MIXED) stage_body_m<NQ, EOS, HAS_Z, STAGE2>(A, i, j, k, s);
    else stage_body<NQ, EOS, HAS_Z, STAGE2>(A, i, j, k, s);
}

} // namespace vh

#endif

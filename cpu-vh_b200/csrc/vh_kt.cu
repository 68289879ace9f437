/*
 * vh_kt.cu -- single-event launch forms of the Kurganov-Tadmor RK2 stage.
 *
 * The reference runs each RK stage as seven OpenMP loop nests over the lattice
 * (source, x, y, eta flux passes, inference, regulation, ghost cells;
 * FullyDiscreteKurganovTadmorScheme.cpp:895-923), each re-reading and
 * re-writing the full state.  Here one thread owns one interior cell:
 *  - fused (small lattices): one kernel per stage evaluates the source term,
 *    the six half-site fluxes and the direction sources, accumulates them in
 *    registers in the reference's order, applies the stage-2 convex
 *    combination, recovers (e, p, u), regulates pi^{mu nu} and Pi and writes
 *    the cell and its ghost copies once;
 *  - phase-split (large lattices): the same work as source, x, y, eta flux and
 *    finalize kernels, partial sums in the stage's output planes.
 * e, p and u are double-buffered (read *_in, write *_out) so that no thread
 * overwrites a value a neighbour still reads; that is what lets the inference
 * move into the stencil kernels.  The per-cell bodies live in vh_stage.cuh.
 *
 * Arithmetic is the reference's, operation for operation, in FP64 with float
 * truncations where the reference has them; the library is compiled with
 * --fmad=false so no multiply-add is fused behind the reference's back.
 */
#include <cuda_runtime.h>
#include <cstdlib>
#include "vh_stage_kernels.cuh"

namespace vh {

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

/* Vorticity.cpp:6-171 for one interior cell: beta_mu = u_mu / T with
 * u_mu = (u^t, -u^x, -u^y, -u^eta) and T = T(e) of the cell (the neighbours'
 * velocities are divided by this cell's T too), a backward time difference
 * against the previous step's velocity and central spatial differences;
 * w_{mu nu} = -(d_mu beta_nu - d_nu beta_mu) / 2.  Every quotient by T uses
 * the cell's rounded reciprocal through div_rcp, which equals the IEEE
 * quotient bit for bit. */
template <int EOS>
__global__ void vorticity_kernel(const __grid_constant__ VortArgs A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
    const int k = blockIdx.z + 2;
    if (i >= A.nx + 2 || j >= A.ny + 2) return;
    const long long L = A.L, sxy = (long long)A.ncx * A.ncy;
    const long long s = i + (long long)A.ncx * j + sxy * k;
    const double T = eos_T<EOS>(A.eos, __ldg(A.e + s));
    const double yT = 1.0 / T;
    const long long sz = (A.nz > 1) ? sxy : 0;      /* nz = 1: no eta ghost planes are kept */
    const long long nb[6] = {s - 1, s + 1, s - A.ncx, s + A.ncx, s - sz, s + sz};
    double b[4], ddt[4], dd[3][4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const double *uc = A.u + c * L, *upc = A.up + c * L;
        const double u0 = (c == 0) ? __ldg(uc + s) : __ldg(uc + s) * -1.0;
        const double p0 = (c == 0) ? __ldg(upc + s) : __ldg(upc + s) * -1.0;
        double bn[6];
#pragma unroll
        for (int m = 0; m < 6; ++m) {
            const double un = (c == 0) ? __ldg(uc + nb[m]) : __ldg(uc + nb[m]) * -1.0;
            bn[m] = div_rcp(un, T, yT);
        }
        b[c] = div_rcp(u0, T, yT);
        const double bp = div_rcp(p0, T, yT);
        ddt[c] = (b[c] - bp) / A.dt;
        dd[0][c] = (bn[1] - bn[0]) / (2.0 * A.dx);
        dd[1][c] = (bn[3] - bn[2]) / (2.0 * A.dy);
        dd[2][c] = (bn[5] - bn[4]) / (2.0 * A.dz);
    }
    double *w = A.w;
    w[0 * L + s] = (-1.0 / 2.0) * (ddt[1] - dd[0][0]);
    w[1 * L + s] = (-1.0 / 2.0) * (ddt[2] - dd[1][0]);
    w[2 * L + s] = (-1.0 / 2.0) * (ddt[3] - dd[2][0]);
    w[3 * L + s] = (-1.0 / 2.0) * (dd[0][2] - dd[1][1]);
    w[4 * L + s] = (-1.0 / 2.0) * (dd[0][3] - dd[2][1]);
    w[5 * L + s] = (-1.0 / 2.0) * (dd[1][3] - dd[2][2]);
#pragma unroll
    for (int c = 0; c < 4; ++c) w[(6 + c) * L + s] = b[c];
}

/* the four eta ghost planes of one field plane of a 2+1D event, copied from
 * its interior plane (what DynamicalVariables.cpp:220-378 leaves there) */
__global__ void eta_ghost_fill_kernel(double *plane, int nx, int ny, int ncx, long long sxy)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
    if (i >= nx + 2 || j >= ny + 2) return;
    const long long s = i + (long long)ncx * j + 2 * sxy;
    const double v = plane[s];
    plane[s - sxy] = v;
    plane[s - 2 * sxy] = v;
    plane[s + sxy] = v;
    plane[s + 2 * sxy] = v;
}

void launch_eta_ghost_fill(double *plane, int nx, int ny, int ncx, int ncy, cudaStream_t s)
{
    dim3 block(32, 4, 1);
    dim3 grid((nx + 31) / 32, (ny + 3) / 4, 1);
    eta_ghost_fill_kernel<<<grid, block, 0, s>>>(plane, nx, ny, ncx, (long long)ncx * ncy);
}

void launch_vorticity(const VortArgs &a, cudaStream_t s)
{
    dim3 block(32, 4, 1);
    dim3 grid((a.nx + 31) / 32, (a.ny + 3) / 4, a.nz);
    if (a.eos_kind == 1) vorticity_kernel<1><<<grid, block, 0, s>>>(a);
    else vorticity_kernel<0><<<grid, block, 0, s>>>(a);
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

__global__ void scatter_interior_kernel(const double *in, double *out, int nplanes, long long L, int nx, int ny, int nz,
                                        int ncx, int ncy)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= nx || j >= ny) return;
    const long long N = (long long)nx * ny * nz;
    const long long m = i + (long long)nx * (j + (long long)ny * k);
    const long long s = (i + 2) + (long long)ncx * ((j + 2) + (long long)ncy * (k + 2));
    for (int c = 0; c < nplanes; ++c) out[c * L + s] = in[c * N + m];
}

void launch_scatter_interior(const double *in, double *out, int nplanes, long long L, int nx, int ny, int nz,
                             int ncx, int ncy, cudaStream_t s)
{
    dim3 block(32, 4, 1);
    dim3 grid((nx + 31) / 32, (ny + 3) / 4, nz);
    scatter_interior_kernel<<<grid, block, 0, s>>>(in, out, nplanes, L, nx, ny, nz, ncx, ncy);
}

void launch_init(const InitArgs &a, cudaStream_t s)
{
    dim3 block(32, 4, 1);
    dim3 grid((a.nx + 31) / 32, (a.ny + 3) / 4, a.nz);
    init_kernel<<<grid, block, 0, s>>>(a);
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
        if (eos_kind == 1) launch_stage_t<15, 1, false>(a, s, m); else launch_stage_t<15, 0, false>(a, s, m);
    } else {
        if (eos_kind == 1) launch_stage_t<14, 1, false>(a, s, m); else launch_stage_t<14, 0, false>(a, s, m);
    }
}

} // namespace vh

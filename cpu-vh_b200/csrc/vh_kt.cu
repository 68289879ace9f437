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

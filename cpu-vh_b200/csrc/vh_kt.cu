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
#include "vh_stage.cuh"

namespace vh {

#ifndef VH_STAGE_MIN_BLOCKS
#define VH_STAGE_MIN_BLOCKS 4   /* 128 registers: 16 warps/SM; measured faster than 2-3 blocks at 168-255 */
#endif

/* interior cell (i, j, k) of this thread, at padded index s */
__device__ __forceinline__ bool stage_cell(const StageArgs &A, int &i, int &j, int &k, long long &s)
{
    i = blockIdx.x * blockDim.x + threadIdx.x + 2;
    j = blockIdx.y * blockDim.y + threadIdx.y + 2;
    k = blockIdx.z + 2;
    if (i >= A.nx + 2 || j >= A.ny + 2) return false;
    s = i + (long long)A.ncx * j + (long long)A.ncx * A.ncy * k;
    return true;
}

template <int NQ, int EOS, bool HAS_Z, bool STAGE2>
__global__ void __launch_bounds__(128, VH_STAGE_MIN_BLOCKS) kt_stage_kernel(const __grid_constant__ StageArgs A)
{
    int i, j, k;
    long long s;
    if (!stage_cell(A, i, j, k, s)) return;
    stage_body<NQ, EOS, HAS_Z, STAGE2>(A, i, j, k, s);
}

/* Phase-split form of the same stage: five short kernels instead of one long
 * one.  Each phase's code is a fraction of the fused kernel's and fits the
 * instruction cache: the fused kernel spends most of its stall time waiting
 * for instruction fetch on large lattices. */
template <int NQ, int EOS>
__global__ void __launch_bounds__(128, VH_STAGE_MIN_BLOCKS) kt_source_kernel(const __grid_constant__ StageArgs A)
{
    int i, j, k;
    long long s;
    if (!stage_cell(A, i, j, k, s)) return;
    source_body<NQ, EOS>(A, s);
}

template <int NQ, int EOS, int DIR>
__global__ void __launch_bounds__(128, VH_STAGE_MIN_BLOCKS) kt_flux_kernel(const __grid_constant__ StageArgs A)
{
    int i, j, k;
    long long s;
    if (!stage_cell(A, i, j, k, s)) return;
    flux_body<NQ, EOS, DIR>(A, s);
}

template <int NQ, int EOS, bool HAS_Z, bool STAGE2>
__global__ void __launch_bounds__(128, VH_STAGE_MIN_BLOCKS) kt_final_kernel(const __grid_constant__ StageArgs A)
{
    int i, j, k;
    long long s;
    if (!stage_cell(A, i, j, k, s)) return;
    final_body<NQ, EOS, HAS_Z, STAGE2>(A, i, j, k, s);
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

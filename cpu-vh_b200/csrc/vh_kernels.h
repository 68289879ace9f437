/*
 * vh_kernels.h -- launch interface between the C ABI (vh_capi.cu) and the
 * kernels (vh_kt.cu, vh_fo.cu).  Internal to the library.
 */
#ifndef VH_KERNELS_H
#define VH_KERNELS_H

#include <cuda_runtime.h>
#include "vh_physics.cuh"
#include "vh_b200.h"

namespace vh {

/* Arguments of one fused RK stage (FullyDiscreteKurganovTadmorScheme.cpp:895-906
 * for stage 1, :912-923 for stage 2). */
struct StageArgs {
    const double *qin;     /* conserved variables the stage differentiates (NQ planes) */
    double *qout;          /* updated conserved variables (NQ planes)                  */
    const double *qbase;   /* stage 2: q^n for the convex combination; stage 1: null   */
    const double *ein, *pin;
    double *eout, *pout;
    const double *uin;     /* 4 planes, read on the 7-point stencil                    */
    const double *upin;    /* 4 planes, previous velocity, read at the centre          */
    double *uout;          /* 4 planes                                                 */
    long long L;           /* plane stride in doubles                                  */
    int nx, ny, nz, ncx, ncy;
    double t;              /* time the stage's fluxes and sources are evaluated at     */
    double t2pow;          /* pow(t, 2) from the host libm (SourceTerms.cpp:415, :587) */
    double t_inf;          /* time of the inference and regulation (t after t += dt)   */
    double dt, dx, dy, dz, theta, etabar, e_reg;
    double inv_dx, inv_dy, inv_dz;   /* RN(1/dx) etc. for div_rcp                      */
    double inv_t;          /* RN(1/t)                                                  */
    const double *src;     /* dynamical sources t, x, y, eta (4 planes) or null        */
    double *regfac;        /* regulation factors shear, bulk (2 planes) or null        */
    int step;              /* step index for error reports                             */
    DevEos eos;
    Zeta zeta;
    DevErr err;
};

/* Interior initial condition -> padded state (DynamicalVariables.cpp:169-218
 * and the ghost faces). */
struct InitArgs {
    const double *e, *p, *u, *pi, *Pi;   /* interior planes, u: 4, pi: 10 (pi, Pi nullable) */
    double *q, *eo, *po, *uo, *upo;      /* padded planes */
    long long L;
    int nx, ny, nz, ncx, ncy, nq;
};

void launch_init(const InitArgs &a, cudaStream_t s);
/* interior arrays (nplanes x nx*ny*nz) -> the interior of padded planes */
void launch_scatter_interior(const double *in, double *out, int nplanes, long long L, int nx, int ny, int nz,
                             int ncx, int ncy, cudaStream_t s);

/* Initial conditions on the device (vh_ic.cu) into interior planes e, p, u */
struct GlauberArgs {
    int nx, ny, nz;
    double dx, dy, dz;
    double R, a, sigma_nn, b, e0, eta_flat, eta_sigma;   /* e0 in fm^-4 */
    DevEos eos;
    int eos_kind;
};
struct HotspotArgs {
    int nx, ny;
    double dx, dy, w;
    const double *spots;     /* device: x[n], y[n], amplitude[n] (fm^-4) */
    int nspots;
    DevEos eos;
    int eos_kind;
};
void launch_glauber_ic(const GlauberArgs &g, double *npart, unsigned long long *mx, double *e, double *p, double *u,
                       cudaStream_t s);
void launch_hotspot_ic(const HotspotArgs &h, double *e, double *p, double *u, cudaStream_t s);

/* Thermal vorticity of the current state (Vorticity.cpp:6-171) */
struct VortArgs {
    const double *u, *up, *e;           /* current u, previous-step u, e (padded planes) */
    double *w;                          /* 6 planes wtx wty wtn wxy wxn wyn, then 4 planes beta t x y n */
    long long L;
    int nx, ny, nz, ncx, ncy;
    double dt, dx, dy, dz;
    DevEos eos;
    int eos_kind;
};
void launch_vorticity(const VortArgs &a, cudaStream_t s);
void launch_math_check(int which, const double *a, const double *b, int n, double *out, const PowfTab &pq, cudaStream_t s);
/* Optional per-phase timing marks of one stage: ev[0] is recorded before the
 * first kernel, ev[n+1] after kernel n, whose phase id is phase[n]
 * (0 source, 1-3 x/y/eta flux, 4 finalize, 5 fused stage). */
struct StageMarks {
    cudaEvent_t ev[6];
    int phase[5];
    int n;
};
void launch_stage(const StageArgs &a, int nq, int eos_kind, cudaStream_t s, StageMarks *m = nullptr);
int stage_launches(int nx, int ny, int nz);   /* kernel launches per RK stage */
/* the same stage in mixed precision (vh_mixed.cu) */
void launch_stage_mixed(const StageArgs &a, int nq, int eos_kind, cudaStream_t s, StageMarks *m = nullptr);

/* ---- batched phase kernels (vh_batch_kernels.cuh) ---- */
struct BatchLaunch {
    const StageArgs *args; /* this stage's arguments, one per member */
    const int4 *tiles;     /* (member, i0, j0, k) in interior coordinates */
    int ntiles;
};
using BatchKernel = void (*)(BatchLaunch);
/* phase: VH_PHASE_*; zm: 0 all members 2+1D, 1 all 3+1D, 2 mixed */
BatchKernel batch_kernel(int nq, int eos_kind, int phase, bool st2, int zm, bool mixed);
BatchKernel batch_kernel_mixed(int nq, int eos_kind, int phase, bool st2, int zm);
/* mixed precision: the face-once flux along dir (1-3) over face tiles of
 * 32 x 8 faces (block 32 x 8) */
BatchKernel batch_face_kernel_mixed(int nq, int eos_kind, int dir);
/* FP64: the flux along dir (1-3) over line blocks (member, block); 128
 * threads, dynamic shared memory batch_lines_smem(nq, dir, nd) bytes for
 * the smallest extent nd along dir among the members */
BatchKernel batch_lines_kernel(int nq, int eos_kind, int dir);
size_t batch_lines_smem(int nq, int dir, int nd);
int batch_lines_per_block(int dir);
long long batch_line_blocks(int dir, int nx, int ny, int nz);
/* mixed precision along y or eta (dir 2, 3): the face-once flux over face
 * line blocks (member, block), 128 threads; the blocks of one member */
BatchKernel batch_face_lines_kernel_mixed(int nq, int eos_kind, int dir);
long long batch_face_line_blocks(int dir, int nx, int ny, int nz);

/* ---- freezeout ---- */
struct FoArgs {
    /* current state (padded) */
    const double *q;         /* NQ planes */
    const double *e;
    const double *u;         /* 4 planes */
    long long L;
    int nx, ny, nz, ncx, ncy, nq;
    /* coarse slabs, interior layout i + nx*(j + ny*k): [2][11][N] = e, ux, uy, un, e, pixx, pixy, pixn, piyy, piyn, Pi */
    double *slab_prev, *slab_cur;
    double eF;
    double dtau_c, dx, dy, dz;   /* lattice_spacing of HydroPlugin.cpp:137-152 */
    double t0, dt, t;            /* cell_tau = t0 + n dt, normals scaled by t (FreezeOut.cpp:228, :243) */
    int n;                       /* loop index of the freezeout block */
    DevEos eos;
    DevErr err;
    int *counts;                 /* per (hyper)cube element counts, then offsets */
    int *block_sums;
    int *n_above;                /* cells above eF */
    double *elems;               /* output, VH_FO_COLUMNS per element */
    int cap;                     /* capacity of elems in elements */
    double *slots;               /* centroids and normals of the first slot_cap crossed cubes */
    int slot_cap;
    int *n_total;
};

/* doubles of one crossed cube's element slot: up to 10 elements (Cornelius
 * MAX_ELEMENTS), centroid and normal (4 + 4) each */
constexpr int kFoSlotDoubles = 80;
/* the freezeout scratch ends with its header: crossed cubes, cells above
 * e_F, elements */
constexpr int kFoHeaderInts = 3;

/* Runs the whole freezeout block; returns the number of elements through
 * *a.n_total (device) and leaves elements in a.elems. */
void launch_freezeout(const FoArgs &a, cudaStream_t s);
/* nz = 1: write the eta ghost planes of one padded field plane (ncz = 5) */
void launch_eta_ghost_fill(double *plane, int nx, int ny, int ncx, int ncy, cudaStream_t s);
void launch_freezeout_emit(const FoArgs &a, cudaStream_t s);
void launch_cornelius_batch(int dim, const double *cubes, int n, double v0, const double *dx,
                            double *slots, int *counts, int *err, cudaStream_t st);
size_t freezeout_scratch_ints(int nx, int ny, int nz);

/* exclusive prefix sum of data[0..n) in place, data[n] = total (and *total
 * if non-null); bsum needs (n + kScanChunk) / kScanChunk + 1 ints */
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanChunk = kScanThreads * kScanItems;
void exclusive_scan(int *data, long long n, int *bsum, int *total, cudaStream_t st);

} // namespace vh

#endif

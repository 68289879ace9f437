/*
 * vh_fo.cu -- freezeout block on the device: the reference's
 * swapAndSetHydroVariables + callFOFinder2p1D/3p1D + checkForCellsAboveTc
 * (freezeout/FreezeOut.cpp:57-381), which it runs serially over every cube.
 *
 * Pipeline (all on the event's stream):
 *   gather    current state -> coarse slab (11 planes over the interior) and
 *             the count of cells above e_F (warp-aggregated)
 *   classify  one thread per (hyper)cube between the previous and current
 *             slab: the above/below corner count; only cubes the surface
 *             crosses go on
 *   compact   exclusive scan of the flags -> dense list of crossed cubes, in
 *             the reference's loop order (ix outermost, then iy, then iz)
 *   count     Cornelius on each crossed cube -> number of elements
 *   scan      -> output offset of every cube's elements
 *   emit      Cornelius again, then the tri-/quadri-linear interpolation of
 *             the ten hydro fields at each centroid, T and P from the EoS,
 *             and the 20 surface.dat columns written at the cube's offset
 * The output is therefore in exactly the order the reference writes it.
 * Cubes crossed by the surface are a small fraction of the lattice, so
 * Cornelius runs twice on them rather than staging geometry in memory.
 */
#include <cuda_runtime.h>
#include "vh_kernels.h"
#include "vh_cornelius.cuh"

namespace vh {


static long long cube_count(int nx, int ny, int nz)
{
    return (long long)(nx - 1) * (ny - 1) * (nz > 1 ? nz - 1 : 1);
}

size_t freezeout_scratch_ints(int nx, int ny, int nz)
{
    long long nc = cube_count(nx, ny, nz);
    long long nb = (nc + 1 + kScanChunk - 1) / kScanChunk + 1;
    /* flags/offsets, list, counts/offsets, block sums, header (n_straddle, n_above, n_total) */
    return (size_t)((nc + 1) + nc + (nc + 1) + nb + 3);
}

struct FoScratch {
    int *flags, *list, *counts, *bsum, *hdr;   /* hdr: [0] crossed cubes, [1] cells above, [2] elements */
    long long nc, nb;
};

static FoScratch carve(const FoArgs &a)
{
    FoScratch s;
    s.nc = cube_count(a.nx, a.ny, a.nz);
    s.nb = (s.nc + 1 + kScanChunk - 1) / kScanChunk + 1;
    s.flags = a.counts;
    s.list = s.flags + s.nc + 1;
    s.counts = s.list + s.nc;
    s.bsum = s.counts + s.nc + 1;
    s.hdr = s.bsum + s.nb;
    return s;
}

/* ------------------------------------------------------------ gather */
__global__ void fo_gather_kernel(const __grid_constant__ FoArgs a, int *above)
{
    const long long N = (long long)a.nx * a.ny * a.nz;
    const long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    bool up = false;
    if (m < N) {
        const int ix = (int)(m % a.nx), iy = (int)((m / a.nx) % a.ny), iz = (int)(m / ((long long)a.nx * a.ny));
        const long long L = a.L;
        const long long s = (ix + 2) + (long long)a.ncx * ((iy + 2) + (long long)a.ncy * (iz + 2));
        const double e = a.e[s];
        double *c = a.slab_cur;
        c[0 * N + m] = e;
        c[1 * N + m] = a.u[1 * L + s];
        c[2 * N + m] = a.u[2 * L + s];
        c[3 * N + m] = a.u[3 * L + s];
        c[4 * N + m] = e;
        c[5 * N + m] = a.q[8 * L + s];
        c[6 * N + m] = a.q[9 * L + s];
        c[7 * N + m] = a.q[10 * L + s];
        c[8 * N + m] = a.q[11 * L + s];
        c[9 * N + m] = a.q[12 * L + s];
        c[10 * N + m] = (a.nq == 15) ? a.q[14 * L + s] : 0.0;
        up = e > a.eF;
    }
    unsigned b = __ballot_sync(0xffffffffu, up);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(above, __popc(b));
}

/* cube index c enumerates (ix, iy, iz) with iz fastest, ix slowest: the
 * reference's loop nest order */
__device__ __forceinline__ void cube_coords(const FoArgs &a, long long c, int &ix, int &iy, int &iz)
{
    const int mz = a.nz > 1 ? a.nz - 1 : 1;
    iz = (int)(c % mz);
    iy = (int)((c / mz) % (a.ny - 1));
    ix = (int)(c / ((long long)mz * (a.ny - 1)));
}

__device__ __forceinline__ double slab(const FoArgs &a, int which, int v, int ix, int iy, int iz)
{
    const long long N = (long long)a.nx * a.ny * a.nz;
    const double *S = which ? a.slab_cur : a.slab_prev;
    return S[v * N + ix + (long long)a.nx * (iy + (long long)a.ny * iz)];
}

/* ----------------------------------------------------------- classify */
__global__ void fo_classify_kernel(const __grid_constant__ FoArgs a, FoScratch sc)
{
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= sc.nc) return;
    int ix, iy, iz;
    cube_coords(a, c, ix, iy, iz);
    const bool four = a.nz > 1;
    int above = 0;
    for (int t = 0; t < 2; t++)
        for (int bx = 0; bx < 2; bx++)
            for (int by = 0; by < 2; by++)
                for (int bz = 0; bz < (four ? 2 : 1); bz++)
                    if (slab(a, t, 0, ix + bx, iy + by, iz + bz) >= a.eF) above++;
    const int all = four ? 16 : 8;
    sc.flags[c] = (above != 0 && above != all) ? 1 : 0;
}

/* -------------------------------------------------------------- scan */
/* exclusive scan of data[0..n) in place, data[n] = total; three passes */
__global__ void scan_reduce_kernel(const int *data, long long n, int *bsum)
{
    __shared__ int red[kScanThreads / 32];
    long long base = blockIdx.x * (long long)kScanChunk;
    int v = 0;
    for (int k = 0; k < kScanItems; k++) {
        long long i = base + threadIdx.x * (long long)kScanItems + k;
        if (i < n) v += data[i];
    }
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        int w = red[threadIdx.x];
        for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
        if (threadIdx.x == 0) bsum[blockIdx.x] = w;
    }
}

__global__ void scan_blocks_kernel(int *bsum, long long nb)
{
    /* one block of 1024 threads, sequential over tiles of 1024 block sums */
    __shared__ int tile[kScanThreads];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (long long t0 = 0; t0 < nb; t0 += kScanThreads) {
        long long i = t0 + threadIdx.x;
        int v = (i < nb) ? bsum[i] : 0;
        tile[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < kScanThreads; off <<= 1) {
            int add = (threadIdx.x >= off) ? tile[threadIdx.x - off] : 0;
            __syncthreads();
            tile[threadIdx.x] += add;
            __syncthreads();
        }
        int incl = tile[threadIdx.x];
        if (i < nb) bsum[i] = carry + incl - v;
        __syncthreads();
        if (threadIdx.x == kScanThreads - 1) carry += incl;
        __syncthreads();
    }
}

__global__ void scan_apply_kernel(int *data, long long n, const int *bsum, int *total)
{
    __shared__ int tile[kScanThreads];
    long long base = blockIdx.x * (long long)kScanChunk;
    int loc[kScanItems], s = 0;
    for (int k = 0; k < kScanItems; k++) {
        long long i = base + threadIdx.x * (long long)kScanItems + k;
        loc[k] = (i < n) ? data[i] : 0;
        s += loc[k];
    }
    tile[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < kScanThreads; off <<= 1) {
        int add = (threadIdx.x >= off) ? tile[threadIdx.x - off] : 0;
        __syncthreads();
        tile[threadIdx.x] += add;
        __syncthreads();
    }
    int run = bsum[blockIdx.x] + tile[threadIdx.x] - s;
    for (int k = 0; k < kScanItems; k++) {
        long long i = base + threadIdx.x * (long long)kScanItems + k;
        if (i < n) data[i] = run;
        if (i == n - 1) { data[n] = run + loc[k]; if (total) *total = run + loc[k]; }
        run += loc[k];
    }
    if (n == 0 && blockIdx.x == 0 && threadIdx.x == 0) { data[0] = 0; if (total) *total = 0; }
}

void exclusive_scan(int *data, long long n, int *bsum, int *total, cudaStream_t st)
{
    long long nb = (n + kScanChunk - 1) / kScanChunk;
    if (nb == 0) nb = 1;
    scan_reduce_kernel<<<(unsigned)nb, kScanThreads, 0, st>>>(data, n, bsum);
    scan_blocks_kernel<<<1, kScanThreads, 0, st>>>(bsum, nb);
    scan_apply_kernel<<<(unsigned)nb, kScanThreads, 0, st>>>(data, n, bsum, total);
}

__global__ void fo_compact_kernel(FoScratch sc)
{
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= sc.nc) return;
    if (sc.flags[c + 1] != sc.flags[c]) sc.list[sc.flags[c]] = (int)c;
}

/* --------------------------------------------------------- Cornelius */
__device__ int cube_surface(const FoArgs &a, int ix, int iy, int iz, cor::Work &w, double cen[][4], double nor[][4])
{
    if (a.nz > 1) {
        double h[2][2][2][2];
        for (int t = 0; t < 2; t++) for (int bx = 0; bx < 2; bx++) for (int by = 0; by < 2; by++) for (int bz = 0; bz < 2; bz++)
            h[t][bx][by][bz] = slab(a, t, 0, ix + bx, iy + by, iz + bz);
        const double dx[4] = {a.dtau_c, a.dx, a.dy, a.dz};
        return cor::surface_4d(w, h, a.eF, dx, cen, nor);
    }
    double cb[2][2][2];
    for (int t = 0; t < 2; t++) for (int bx = 0; bx < 2; bx++) for (int by = 0; by < 2; by++)
        cb[t][bx][by] = slab(a, t, 0, ix + bx, iy + by, 0);
    const double dx3[3] = {a.dtau_c, a.dx, a.dy};
    return cor::surface_3d(w, cb, a.eF, dx3, cen, nor);
}

/* element slots: the centroids and normals the count step finds for the
 * first slot_cap crossed cubes, kept for the emit step (8 doubles per
 * element, kMaxElements per cube) so that it need not run Cornelius again:
 * the per-thread Cornelius work area (~13 KB) is what the emit step's DRAM
 * traffic was made of */
static_assert(cor::kMaxHedra <= cor::kMaxElements && cor::kMaxElements * 8 == kFoSlotDoubles,
              "a cube's elements fit its slot");
constexpr int kSlotDoubles = kFoSlotDoubles;

__global__ void __launch_bounds__(128) fo_count_kernel(const __grid_constant__ FoArgs a, FoScratch sc)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= sc.nc) return;
    const int nst = sc.hdr[0];
    if (i >= nst) { sc.counts[i] = 0; return; }
    int ix, iy, iz;
    cube_coords(a, sc.list[i], ix, iy, iz);
    cor::Work w;
    double cen[cor::kMaxHedra][4], nor[cor::kMaxHedra][4];
    int ne = cube_surface(a, ix, iy, iz, w, cen, nor);
    if (ne < 0) { raise_error(a.err, 5, sc.list[i], a.n); ne = 0; }
    sc.counts[i] = ne;
    if (i < a.slot_cap) {
        double *o = a.slots + i * kSlotDoubles;
        for (int k = 0; k < ne; k++)
            for (int d = 0; d < 4; d++) { o[8 * k + d] = cen[k][d]; o[8 * k + 4 + d] = nor[k][d]; }
    }
}

/* FreezeOut.cpp:40-55 */
__device__ __forceinline__ double interp3(double x0, double x1, double x2, double a000, double a100, double a010,
                                          double a001, double a110, double a101, double a011, double a111)
{
    return ((1 - x0) * (1 - x1) * (1 - x2) * a000) + ((x0) * (1 - x1) * (1 - x2) * a100) + ((1 - x0) * (x1) * (1 - x2) * a010) +
           ((1 - x0) * (1 - x1) * (x2) * a001) + ((x0) * (x1) * (1 - x2) * a110) + ((x0) * (1 - x1) * (x2) * a101) +
           ((1 - x0) * (x1) * (x2) * a011) + ((x0) * (x1) * (x2) * a111);
}

/* FreezeOut.cpp:13-38 (the a1011 term is summed before a0111, as there) */
__device__ __forceinline__ double interp4(double x0, double x1, double x2, double x3, const double *c)
{
    /* c: corners indexed [t][x][y][z] -> t*8 + x*4 + y*2 + z */
    return ((1 - x0) * (1 - x1) * (1 - x2) * (1 - x3) * c[0]) + ((x0) * (1 - x1) * (1 - x2) * (1 - x3) * c[8]) +
           ((1 - x0) * (x1) * (1 - x2) * (1 - x3) * c[4]) + ((1 - x0) * (1 - x1) * (x2) * (1 - x3) * c[2]) +
           ((1 - x0) * (1 - x1) * (1 - x2) * (x3) * c[1]) + ((x0) * (x1) * (1 - x2) * (1 - x3) * c[12]) +
           ((x0) * (1 - x1) * (x2) * (1 - x3) * c[10]) + ((x0) * (1 - x1) * (1 - x2) * (x3) * c[9]) +
           ((1 - x0) * (x1) * (x2) * (1 - x3) * c[6]) + ((1 - x0) * (x1) * (1 - x2) * (x3) * c[5]) +
           ((1 - x0) * (1 - x1) * (x2) * (x3) * c[3]) + ((x0) * (x1) * (x2) * (1 - x3) * c[14]) +
           ((x0) * (x1) * (1 - x2) * (x3) * c[13]) + ((x0) * (1 - x1) * (x2) * (x3) * c[11]) +
           ((1 - x0) * (x1) * (x2) * (x3) * c[7]) + ((x0) * (x1) * (x2) * (x3) * c[15]);
}

/* FreezeOut.cpp:200-361, per element: position, tau-scaled normal, the ten
 * interpolated fields, T and P */
template <int EOS>
__device__ __forceinline__ void emit_element(const FoArgs &a, int ix, int iy, int iz, const double *cen,
                                             const double *nor, double *__restrict__ o)
{
    const bool four = a.nz > 1;
    const double cell_tau = a.t0 + ((double)a.n) * a.dt;
    const double cell_x = (double)ix * a.dx - (((double)(a.nx - 1)) / 2.0 * a.dx);
    const double cell_y = (double)iy * a.dy - (((double)(a.ny - 1)) / 2.0 * a.dy);
    double f[10];
    if (four) {
        const double cell_z = (double)iz * a.dz - (((double)(a.nz - 1)) / 2.0 * a.dz);
        const double tf = cen[0] / a.dtau_c, xf = cen[1] / a.dx, yf = cen[2] / a.dy, zf = cen[3] / a.dz;
        for (int v = 0; v < 10; v++) {
            double c[16];
            for (int t = 0; t < 2; t++) for (int bx = 0; bx < 2; bx++) for (int by = 0; by < 2; by++) for (int bz = 0; bz < 2; bz++)
                c[t * 8 + bx * 4 + by * 2 + bz] = slab(a, t, v + 1, ix + bx, iy + by, iz + bz);
            f[v] = interp4(tf, xf, yf, zf, c);
        }
        o[0] = cen[0] + cell_tau; o[1] = cen[1] + cell_x; o[2] = cen[2] + cell_y; o[3] = cen[3] + cell_z;
        o[4] = a.t * nor[0]; o[5] = a.t * nor[1]; o[6] = a.t * nor[2]; o[7] = a.t * nor[3];
    } else {
        const double tf = cen[1] / a.dtau_c, xf = cen[2] / a.dx, yf = cen[3] / a.dy;
        for (int v = 0; v < 10; v++)
            f[v] = interp3(tf, xf, yf, slab(a, 0, v + 1, ix, iy, 0), slab(a, 1, v + 1, ix, iy, 0),
                           slab(a, 0, v + 1, ix + 1, iy, 0), slab(a, 0, v + 1, ix, iy + 1, 0),
                           slab(a, 1, v + 1, ix + 1, iy, 0), slab(a, 1, v + 1, ix, iy + 1, 0),
                           slab(a, 0, v + 1, ix + 1, iy + 1, 0), slab(a, 1, v + 1, ix + 1, iy + 1, 0));
        o[0] = cen[1] + cell_tau; o[1] = cen[2] + cell_x; o[2] = cen[3] + cell_y; o[3] = 0.0;
        o[4] = a.t * nor[1]; o[5] = a.t * nor[2]; o[6] = a.t * nor[3]; o[7] = 0.0;
    }
    o[8] = f[0]; o[9] = f[1]; o[10] = f[2];
    o[11] = f[3];
    o[12] = eos_T<EOS>(a.eos, f[3]);
    o[13] = eos_p<EOS>(a.eos, f[3]);
    o[14] = f[4]; o[15] = f[5]; o[16] = f[6]; o[17] = f[7]; o[18] = f[8];
    o[19] = f[9];
}

/* a crossed cube beyond the slots: Cornelius again, as the count step ran it */
template <int EOS>
static __device__ __noinline__ void emit_recompute(const FoArgs &a, int ix, int iy, int iz, long long off)
{
    cor::Work w;
    double cen[cor::kMaxHedra][4], nor[cor::kMaxHedra][4];
    const int ne = cube_surface(a, ix, iy, iz, w, cen, nor);
    for (int k = 0; k < ne; k++) {
        if (off + k >= a.cap) return;
        emit_element<EOS>(a, ix, iy, iz, cen[k], nor[k], a.elems + (off + k) * VH_FO_COLUMNS);
    }
}

template <int EOS>
__global__ void __launch_bounds__(128) fo_emit_kernel(const __grid_constant__ FoArgs a, FoScratch sc)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= sc.nc || i >= sc.hdr[0]) return;
    int ix, iy, iz;
    cube_coords(a, sc.list[i], ix, iy, iz);
    const long long off = sc.counts[i];
    if (i >= a.slot_cap) { emit_recompute<EOS>(a, ix, iy, iz, off); return; }
    const int ne = sc.counts[i + 1] - sc.counts[i];
    const double *sl = a.slots + i * kSlotDoubles;
    for (int k = 0; k < ne; k++) {
        if (off + k >= a.cap) return;
        emit_element<EOS>(a, ix, iy, iz, sl + 8 * k, sl + 8 * k + 4, a.elems + (off + k) * VH_FO_COLUMNS);
    }
}

__global__ void fo_header_kernel(FoScratch sc)
{
    /* hdr[0] = number of crossed cubes (flags scanned in place: flags[nc]) */
    sc.hdr[0] = sc.flags[sc.nc];
}

void launch_freezeout(const FoArgs &a, cudaStream_t st)
{
    FoScratch sc = carve(a);
    const long long N = (long long)a.nx * a.ny * a.nz;
    cudaMemsetAsync(sc.hdr, 0, 3 * sizeof(int), st);
    fo_gather_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(a, sc.hdr + 1);
    const unsigned gc = (unsigned)((sc.nc + 255) / 256);
    fo_classify_kernel<<<gc, 256, 0, st>>>(a, sc);
    exclusive_scan(sc.flags, sc.nc, sc.bsum, nullptr, st);
    fo_compact_kernel<<<gc, 256, 0, st>>>(sc);
    fo_header_kernel<<<1, 1, 0, st>>>(sc);
    const unsigned gk = (unsigned)((sc.nc + 127) / 128);
    fo_count_kernel<<<gk, 128, 0, st>>>(a, sc);
    exclusive_scan(sc.counts, sc.nc, sc.bsum, sc.hdr + 2, st);
    launch_freezeout_emit(a, st);
}

/* the emit step alone, from the offsets the last launch_freezeout left in the
 * scratch: the elements of a block that did not fit, into a larger buffer */
void launch_freezeout_emit(const FoArgs &a, cudaStream_t st)
{
    if (!a.elems || a.cap <= 0) return;
    FoScratch sc = carve(a);
    const unsigned gk = (unsigned)((sc.nc + 127) / 128);
    if (a.eos.kind == 1) fo_emit_kernel<1><<<gk, 128, 0, st>>>(a, sc);
    else fo_emit_kernel<0><<<gk, 128, 0, st>>>(a, sc);
}

} // namespace vh

namespace vh {

/* Cornelius on caller-supplied cubes (dim 3: 8 corner values per cube,
 * [t][x][y]; dim 4: 16 values, [t][x][y][z]).  Each thread handles one
 * cube and writes up to kMaxElements elements of 2*dim doubles (centroid
 * then normal, the trailing dim components as Cornelius::get_centroid_elem
 * returns them) into its fixed slot, and its element count. */
__global__ void __launch_bounds__(128) cornelius_batch_kernel(int dim, const double *cubes, int n, double v0,
                                                              double d0, double d1, double d2, double d3,
                                                              double *slots, int *counts, int *err)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    cor::Work w;
    double cen[cor::kMaxHedra][4], nor[cor::kMaxHedra][4];
    int ne;
    if (dim == 3) {
        double cb[2][2][2];
        for (int i = 0; i < 8; i++) (&cb[0][0][0])[i] = cubes[8LL * c + i];
        const double dx3[3] = {d0, d1, d2};
        ne = cor::surface_3d(w, cb, v0, dx3, cen, nor);
    } else {
        double h[2][2][2][2];
        for (int i = 0; i < 16; i++) (&h[0][0][0][0])[i] = cubes[16LL * c + i];
        const double dx[4] = {d0, d1, d2, d3};
        ne = cor::surface_4d(w, h, v0, dx, cen, nor);
    }
    if (ne < 0) { atomicExch(err, 1); ne = 0; }
    counts[c] = ne;
    for (int k = 0; k < ne; k++) {
        double *o = slots + ((long long)c * cor::kMaxElements + k) * 8;
        for (int j = 0; j < dim; j++) o[j] = cen[k][j + 4 - dim];
        for (int j = 0; j < dim; j++) o[dim + j] = nor[k][j + 4 - dim];
    }
}

void launch_cornelius_batch(int dim, const double *cubes, int n, double v0, const double *dx,
                            double *slots, int *counts, int *err, cudaStream_t st)
{
    cornelius_batch_kernel<<<(n + 127) / 128, 128, 0, st>>>(dim, cubes, n, v0, dx[0], dx[1], dx[2], dim == 4 ? dx[3] : 0.0,
                                                            slots, counts, err);
}

} // namespace vh

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
    /* flags/offsets, list, counts/offsets, block sums, header (n_straddle,
     * n_above, n_total) */
    return (size_t)((nc + 1) + nc + (nc + 1) + nb + kFoHeaderInts);
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
/* threads run over the cubes in the slab's memory order (x fastest, so a
 * warp's corner loads are contiguous); each flag goes to the cube's index
 * in the reference's order (cube_coords) */
__global__ void fo_classify_kernel(const __grid_constant__ FoArgs a, FoScratch sc)
{
    const long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (m >= sc.nc) return;
    const int mz = a.nz > 1 ? a.nz - 1 : 1;
    const int ix = (int)(m % (a.nx - 1));
    const int iy = (int)((m / (a.nx - 1)) % (a.ny - 1));
    const int iz = (int)(m / ((long long)(a.nx - 1) * (a.ny - 1)));
    const long long c = iz + (long long)mz * (iy + (long long)(a.ny - 1) * ix);
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

/* ---------------------------------------------- count, 4D, grouped lanes
 * The per-thread count above leaves ~4 warps per SM on a 131x131x61 event
 * (one thread per crossed hypercube, ~17 k of them), each thread a long
 * serial chain through the work area in local memory.  Here eight lanes take
 * one hypercube and a 128-thread block sixteen:
 *   cubes     lane c builds the c-th of the hypercube's eight 3-cubes
 *             (surface_4d's order), its lines and polygons and the polygon
 *             centroids, into a pool in shared memory; the pool is allotted
 *             by a block-wide scan of the line and polygon counts known from
 *             the corner comparisons (cube_line_count), so lines and polygons
 *             keep the reference's order and indices stay in it;
 *   hedra     one lane per hypercube assembles the polyhedra (all polygons in
 *             one when nothing is ambiguous, the reference's search loop
 *             otherwise);
 *   geometry  the sums of Polyhedron::calculate_centroid/normal in rounds of
 *             eight tetrahedra, one per lane, each term added to the running
 *             sums in the reference's order through width-8 shuffles.
 * Every value is computed by the same expression as in surface_4d, in the
 * same order: the elements are bit-identical.  A block whose hypercubes need
 * more than the pool holds takes them in rounds (one hypercube, at most 96
 * lines, always fits): no hypercube is left to a slower path, whose serial
 * latency alone would be that of the whole per-thread count. */
constexpr int kG4 = 16;                     /* hypercubes per 128-thread block */
constexpr int kPoolLines = 512, kPoolPolys = 128;

struct Count4Shared {
    double p[kPoolLines][2][4];
    double out[kPoolLines][4];
    unsigned char flip[kPoolLines];
    cor::Poly poly[kPoolPolys];
    unsigned short tl[kPoolLines];           /* tetrahedra of the polyhedron being measured: its line */
    unsigned char tp[kPoolLines];            /*   and the polygon the line belongs to */
    cor::Hedron hed[kG4][cor::kMaxHedra];
    int lbase[128], pbase[128], nl[128], np[128];
    unsigned char amb[128], err[128];
    int nh[kG4];
    int wsum[4];
    int next_l, next_p;                      /* the next round's pool offsets */
};

/* the centroid and normal of polyhedron h (Polyhedron::calculate_centroid and
 * calculate_normal, cornelius.cpp:842-987), its tetrahedra listed in
 * S.tl/S.tp from index base; the eight lanes of gmask cooperate */
__device__ void hedron_geometry_group(const cor::WorkRef &w, Count4Shared &S, int base, int T, int q,
                                      unsigned gmask, double *centroid, double *normal)
{
    double mean[4] = {0, 0, 0, 0};
    for (int r = 0; r < T; r += 8) {
        const int t = r + q;
        double s[4] = {0, 0, 0, 0};
        if (t < T) {
            const int l = S.tl[base + t];
            const double *p1 = cor::lstart(w, l), *p2 = cor::lend(w, l);
            for (int k = 0; k < 4; k++) s[k] = p1[k] + p2[k];
        }
        for (int u = 0; u < 8; u++) {
            double v[4];
            for (int k = 0; k < 4; k++) v[k] = __shfl_sync(gmask, s[k], u, 8);
            if (r + u < T)
                for (int k = 0; k < 4; k++) mean[k] += v[k];
        }
    }
    for (int j = 0; j < 4; j++) mean[j] = mean[j] / (double)(2.0 * T);
    double up[4] = {0, 0, 0, 0}, down = 0;
    for (int r = 0; r < T; r += 8) {
        const int t = r + q;
        double s[5] = {0, 0, 0, 0, 0};
        if (t < T) {
            const int l = S.tl[base + t];
            const double *cent = S.poly[S.tp[base + t]].cen;
            const double *p1 = cor::lstart(w, l), *p2 = cor::lend(w, l);
            double cm[4], a4[4], b4[4], c4[4], n[4];
            for (int k = 0; k < 4; k++) cm[k] = (p1[k] + p2[k] + cent[k] + mean[k]) / 4.0;
            for (int k = 0; k < 4; k++) { a4[k] = p1[k] - mean[k]; b4[k] = p2[k] - mean[k]; c4[k] = cent[k] - mean[k]; }
            cor::tetravolume(a4, b4, c4, n);
            double V = 0;
            for (int k = 0; k < 4; k++) V += n[k] * n[k];
            V = sqrt(V);
            for (int k = 0; k < 4; k++) s[k] = cm[k] * V;
            s[4] = V;
        }
        for (int u = 0; u < 8; u++) {
            double v[5];
            for (int k = 0; k < 5; k++) v[k] = __shfl_sync(gmask, s[k], u, 8);
            if (r + u < T) {
                for (int k = 0; k < 4; k++) up[k] += v[k];
                down += v[4];
            }
        }
    }
    for (int i = 0; i < 4; i++) centroid[i] = up[i] / down;
    for (int i = 0; i < 4; i++) normal[i] = 0;
    for (int r = 0; r < T; r += 8) {
        const int t = r + q;
        double n[4] = {0, 0, 0, 0};
        if (t < T) {
            const int l = S.tl[base + t];
            const double *cent = S.poly[S.tp[base + t]].cen;
            const double *p1 = cor::lstart(w, l), *p2 = cor::lend(w, l);
            double a4[4], b4[4], c4[4], vout[4];
            for (int k = 0; k < 4; k++) { a4[k] = p1[k] - centroid[k]; b4[k] = p2[k] - centroid[k]; c4[k] = cent[k] - centroid[k]; }
            cor::tetravolume(a4, b4, c4, n);
            for (int k = 0; k < 4; k++) vout[k] = w.out[l][k] - centroid[k];
            cor::orient(n, vout);
        }
        for (int u = 0; u < 8; u++) {
            double v[4];
            for (int k = 0; k < 4; k++) v[k] = __shfl_sync(gmask, n[k], u, 8);
            if (r + u < T)
                for (int k = 0; k < 4; k++) normal[k] += v[k];
        }
    }
}

__global__ void __launch_bounds__(128, 3) fo_count4_kernel(const __grid_constant__ FoArgs a, FoScratch sc)
{
    extern __shared__ __align__(16) unsigned char count4_smem[];
    Count4Shared &S = *reinterpret_cast<Count4Shared *>(count4_smem);
    const int tid = threadIdx.x, g = tid >> 3, q = tid & 7, lane = tid & 31, wid = tid >> 5;
    const unsigned gmask = 0xFFu << (lane & ~7);
    const int nst = sc.hdr[0];
    /* the uncrossed entries of the counts the offsets are scanned from */
    for (long long i = nst + (long long)blockIdx.x * 128 + tid; i < sc.nc; i += (long long)gridDim.x * 128)
        sc.counts[i] = 0;
    const double dx[4] = {a.dtau_c, a.dx, a.dy, a.dz};
    const double E0 = a.eF;
    const cor::WorkRef pool{S.p, S.out, S.flip, S.poly, 0, 0, kPoolLines, kPoolPolys, false};
    for (long long hb = blockIdx.x; hb * kG4 < nst; hb += gridDim.x) {
        const long long hidx = hb * kG4 + g;
        const bool valid = hidx < nst;
        /* this lane's 3-cube: axis ci held at cj (surface_4d's enumeration) */
        const int ci = q >> 1, cj = q & 1;
        double cu[2][2][2];
        int nlc = 0, ambsq = 0, npm = 0, below = 0;
        bool errc = false;
        if (valid) {
            int ix, iy, iz;
            cube_coords(a, sc.list[hidx], ix, iy, iz);
            for (int A = 0; A < 2; A++)
                for (int B = 0; B < 2; B++)
                    for (int C = 0; C < 2; C++) {
                        const int t = (ci == 0) ? cj : A;
                        const int bx = (ci == 0) ? A : (ci == 1) ? cj : B;
                        const int by = (ci <= 1) ? B : (ci == 2) ? cj : C;
                        const int bz = (ci <= 2) ? C : cj;
                        cu[A][B][C] = slab(a, t, 0, ix + bx, iy + by, iz + bz);
                        if (cu[A][B][C] < E0) below++;
                    }
            nlc = cor::cube_line_count(cu, ci, E0, ambsq, errc);
            if (nlc > 0) {
                const bool ambc = ambsq > 0 || nlc == 6;     /* cube_polygons' ambiguity */
                npm = ambc ? (nlc > 3 ? nlc - 2 : 1) : 1;    /* the most polygons it can make */
            }
        }
        /* block-wide exclusive scan of the line and polygon counts, in lane
         * order (hypercube order, then surface_4d's cube order) */
        const int packed = nlc | (npm << 16);
        int incl = packed;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) S.wsum[wid] = incl;
        __syncthreads();
        int before = 0;
        for (int k = 0; k < wid; k++) before += S.wsum[k];
        const int excl = before + incl - packed;
        const int lb = excl & 0xffff, pb = excl >> 16;
        /* the group's range: from its first cube's start to its last cube's end */
        const int g_lbeg = __shfl_sync(0xffffffffu, lb, lane & ~7);
        const int g_pbeg = __shfl_sync(0xffffffffu, pb, lane & ~7);
        const int g_lend = __shfl_sync(0xffffffffu, lb + nlc, (lane & ~7) + 7);
        const int g_pend = __shfl_sync(0xffffffffu, pb + npm, (lane & ~7) + 7);
        /* rounds: each takes the next run of groups whose ranges fit the pool
         * from offset (off_l, off_p); one hypercube (at most 96 lines and 80
         * polygons reserved) always fits alone, so every round advances */
        int off_l = 0, off_p = 0;
        bool done = !valid;
        for (;;) {
            const bool mine = !done && g_lend - off_l <= kPoolLines && g_pend - off_p <= kPoolPolys;
            if (tid == 0) { S.next_l = 1 << 30; S.next_p = 1 << 30; }
            /* cubes: lines, polygons, polygon centroids */
            int npc = 0;
            bool ambb = false, errb = errc;
            const int rl = lb - off_l, rp = pb - off_p;
            if (mine && nlc > 0 && !errc) {
                cor::WorkRef w{S.p, S.out, S.flip, S.poly, rl, rp, rl + nlc, rp + npm, false};
                const int n = cor::cube_polygons(w, cu, ci, cj * dx[ci], E0, dx, &ambb);
                if (w.error || n != nlc || w.nl != rl + nlc) errb = true;
                else {
                    npc = w.np - rp;
                    for (int k = rp; k < w.np; k++) cor::poly_centroid(w, S.poly[k]);
                }
            }
            S.lbase[tid] = rl;
            S.pbase[tid] = rp;
            S.nl[tid] = nlc;
            S.np[tid] = npc;
            S.amb[tid] = (nlc > 0 && ambb) ? 1 : 0;
            S.err[tid] = errb ? 1 : 0;
            __syncthreads();
            if (mine) {
                const int g0 = g * 8;
                int gnl = 0, gnp = 0, gamb = 0;
                bool gerr = false;
                for (int c = 0; c < 8; c++) {
                    gnl += S.nl[g0 + c];
                    gnp += S.np[g0 + c];
                    gamb += S.amb[g0 + c];
                    gerr |= S.err[g0 + c] != 0;
                }
                if (gnp > cor::kMaxPoly) gerr = true;             /* the per-thread work area's polygon cap */
                /* surface_4d: 24 lines and 2 (or 14) corners below make it ambiguous */
                int points = __shfl_sync(gmask, below, 0, 8) + __shfl_sync(gmask, below, 1, 8);
                if (points > 8) points = 16 - points;
                const bool ambiguous = gamb > 0 || (gnl == 24 && points == 2);
                if (q == 0) {
                    int nh = 0;
                    if (!gerr) {
                        cor::WorkRef w = pool;
                        unsigned char list[cor::kMaxPoly];
                        int npolys = 0;
                        for (int c = 0; c < 8; c++)
                            for (int k = 0; k < S.np[g0 + c]; k++) list[npolys++] = (unsigned char)(S.pbase[g0 + c] + k);
                        cor::Hedron *hed = S.hed[g];
                        if (ambiguous) {
                            bool not_used[cor::kMaxPoly];
                            int used = 0;
                            for (int i = 0; i < npolys; i++) not_used[i] = true;
                            do {
                                if (nh >= cor::kMaxHedra) { w.error = true; break; }
                                hed[nh].npoly = 0; hed[nh].ntet = 0;
                                for (int i = 0; i < npolys; i++)
                                    if (not_used[i] && cor::hedron_add(w, hed[nh], list[i], false)) { not_used[i] = false; used++; i = 0; }
                                if (w.error) break;
                                nh++;
                            } while (used < npolys);
                        } else {
                            hed[0].npoly = 0; hed[0].ntet = 0;
                            for (int i = 0; i < npolys; i++) cor::hedron_add(w, hed[0], list[i], true);
                            nh = 1;
                        }
                        if (w.error) nh = -1;
                    } else {
                        nh = -1;
                    }
                    S.nh[g] = nh;
                }
                __syncwarp(gmask);
                const int nh = S.nh[g];
                const int base = S.lbase[g0];
                for (int hh = 0; hh < nh; hh++) {
                    const cor::Hedron &h = S.hed[g][hh];
                    if (q == 0) {
                        int t = 0;
                        for (int i = 0; i < h.npoly; i++) {
                            const cor::Poly &pg = S.poly[h.poly[i]];
                            for (int j = 0; j < pg.nlines; j++) { S.tl[base + t] = pg.line[j]; S.tp[base + t] = h.poly[i]; t++; }
                        }
                    }
                    __syncwarp(gmask);
                    double cen[4], nor[4];
                    hedron_geometry_group(pool, S, base, h.ntet, q, gmask, cen, nor);
                    if (q == 0 && hidx < a.slot_cap) {
                        double *o = a.slots + hidx * kSlotDoubles + 8 * hh;
                        for (int d = 0; d < 4; d++) { o[d] = cen[d]; o[4 + d] = nor[d]; }
                    }
                    __syncwarp(gmask);
                }
                if (q == 0) {
                    int ne = nh;
                    if (ne < 0) { raise_error(a.err, 5, sc.list[hidx], a.n); ne = 0; }
                    sc.counts[hidx] = ne;
                }
                done = true;
            } else if (!done && q == 0) {
                atomicMin(&S.next_l, g_lbeg);
                atomicMin(&S.next_p, g_pbeg);
            }
            __syncthreads();
            if (S.next_l == (1 << 30)) break;                    /* every group of the block is done */
            off_l = S.next_l;
            off_p = S.next_p;
            __syncthreads();                                     /* next_l / next_p are reset next round */
        }
    }
}

static void launch_count4(const FoArgs &a, FoScratch sc, cudaStream_t st)
{
    static int blocks = [] {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(fo_count4_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Count4Shared));
        int per_sm = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fo_count4_kernel, 128, sizeof(Count4Shared));
        return sms * (per_sm > 0 ? per_sm : 1);
    }();
    const long long need = (sc.nc + kG4 - 1) / kG4;
    const unsigned grid = (unsigned)(need < blocks ? (need > 0 ? need : 1) : blocks);
    fo_count4_kernel<<<grid, 128, sizeof(Count4Shared), st>>>(a, sc);
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
    cudaMemsetAsync(sc.hdr, 0, kFoHeaderInts * sizeof(int), st);
    fo_gather_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(a, sc.hdr + 1);
    const unsigned gc = (unsigned)((sc.nc + 255) / 256);
    fo_classify_kernel<<<gc, 256, 0, st>>>(a, sc);
    exclusive_scan(sc.flags, sc.nc, sc.bsum, nullptr, st);
    fo_compact_kernel<<<gc, 256, 0, st>>>(sc);
    fo_header_kernel<<<1, 1, 0, st>>>(sc);
    const unsigned gk = (unsigned)((sc.nc + 127) / 128);
    if (a.nz > 1) launch_count4(a, sc, st);
    else fo_count_kernel<<<gk, 128, 0, st>>>(a, sc);
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

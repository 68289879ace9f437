/*
 * vh_batch.cu -- many events of different lattice sizes advanced together.
 *
 * The reference evolves one event per process (HydroPlugin.cpp:226-307); a
 * small 2+1D event (81^2..201^2 cells) cannot fill a B200, so a batch advances
 * any number of resident events with one launch per phase for all of them:
 *
 *  - every member keeps its own vh_event state (planes, EoS, error flags,
 *    freezeout), so everything the single-event API offers still works on it;
 *  - a per-step prep kernel writes each member's two StageArgs (stage 1 and
 *    stage 2 buffer roles, times from a host-computed table) into device
 *    memory from the member's step counter, so one captured CUDA graph of a
 *    whole RK2 step replays unchanged step after step;
 *  - the phase kernels walk a tile table (member, i0, j0, k) — one 128-thread
 *    block per tile, or a persistent grid of resident blocks striding through
 *    the table — and run the same per-cell bodies as the single-event kernels
 *    (vh_stage.cuh), with the member's arguments staged in shared memory;
 *  - the tile shape, the grid form and fused-versus-split are chosen per
 *    phase by timing stage 1 (which writes only scratch planes) for every
 *    candidate on the batch's own members.
 *
 * Results are bit-identical to stepping each member alone.
 */
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "vh_batch_kernels.cuh"
#include "vh_event.h"

namespace vh {

/* one member's step-independent description, device-resident */
struct BatchMember {
    StageArgs base;        /* static fields of the member's stage arguments */
    double *q[3];
    double *ep[2];
    double *u[3];
    const double *ttab;    /* 4 doubles per step n: t, t + dt, pow(t, 2), pow(t + dt, 2) */
    int tcap;              /* steps covered by ttab */
    int active;
};

struct BatchPrep {
    const BatchMember *mem;
    int *nstep;            /* per member: steps done */
    StageArgs *args;       /* [2][nmem]: stage 1 then stage 2 */
    int nmem;
    int advance;           /* 1: count the step (graph replay); 0: arguments only */
};

/* Buffer roles of step n exactly as vh_event_step assigns them (qc = uc = n
 * mod 2, qs = us = 2, e/p: stage 1 reads ep[0] and writes ep[1]). */
__global__ void batch_prep_kernel(const __grid_constant__ BatchPrep P)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= P.nmem) return;
    const BatchMember &M = P.mem[e];
    const int n = P.nstep[e];
    StageArgs a = M.base, b = M.base;
    /* an inactive member is not advanced: every tile of it is skipped, the
     * phase kernels testing nx before any access (the state pointers of
     * M.base are null) */
    if (!M.active || n >= M.tcap) {
        a.nx = 0;
        b.nx = 0;
        P.args[e] = a;
        P.args[P.nmem + e] = b;
        return;
    }
    /* a member whose device has flagged an error is not computed either --
     * its state is invalid (the reference exits at its first NaN), and in
     * garbage cells the root solves would run their 10^4 Newton and 10^6
     * bisection iterations every step until the host reads the error -- but
     * its step count advances as the host counts it, so that the buffer
     * roles of host and device stay the same */
    if (M.base.err.code && *M.base.err.code != 0) {
        a.nx = 0;
        b.nx = 0;
        P.args[e] = a;
        P.args[P.nmem + e] = b;
        if (P.advance) P.nstep[e] = n + 1;
        return;
    }
    const long long L = M.base.L;
    const double *tt = M.ttab + 4 * (long long)n;
    const int c = n & 1;
    a.step = n;
    a.qin = M.q[c]; a.qout = M.q[2]; a.qbase = nullptr;
    a.ein = M.ep[0]; a.pin = M.ep[0] + L; a.eout = M.ep[1]; a.pout = M.ep[1] + L;
    a.uin = M.u[c]; a.upin = M.u[1 - c]; a.uout = M.u[2];
    a.t = tt[0]; a.t2pow = tt[2]; a.t_inf = tt[1]; a.inv_t = 1.0 / tt[0];
    b.step = n;
    b.qin = M.q[2]; b.qout = M.q[1 - c]; b.qbase = M.q[c];
    b.ein = M.ep[1]; b.pin = M.ep[1] + L; b.eout = M.ep[0]; b.pout = M.ep[0] + L;
    b.uin = M.u[2]; b.upin = M.u[c]; b.uout = M.u[1 - c];
    b.t = tt[1]; b.t2pow = tt[3]; b.t_inf = tt[1]; b.inv_t = 1.0 / tt[1];
    P.args[e] = a;
    P.args[P.nmem + e] = b;
    if (P.advance) P.nstep[e] = n + 1;
}

BatchKernel batch_kernel(int nq, int eos_kind, int phase, bool st2, int zm, bool mixed)
{
    return mixed ? batch_kernel_mixed(nq, eos_kind, phase, st2, zm) : batch_kernel_of<false>(nq, eos_kind, phase, st2, zm);
}

template <int NQ, int EOS>
static BatchKernel batch_lines_t(int dir)
{
    return dir == 1 ? kt_batch_lines_kernel<NQ, EOS, 1> : dir == 2 ? kt_batch_lines_kernel<NQ, EOS, 2>
                                                              : kt_batch_lines_kernel<NQ, EOS, 3>;
}

BatchKernel batch_lines_kernel(int nq, int eos_kind, int dir)
{
    if (nq == 15) return eos_kind == 1 ? batch_lines_t<15, 1>(dir) : batch_lines_t<15, 0>(dir);
    return eos_kind == 1 ? batch_lines_t<14, 1>(dir) : batch_lines_t<14, 0>(dir);
}

size_t batch_lines_smem(int nq, int dir, int nd)
{
    const int plane = dir == 1 ? FluxLines<1>::plane(nd) : dir == 2 ? FluxLines<2>::plane(nd) : FluxLines<3>::plane(nd);
    return sizeof(double) * 2 * (size_t)nq * plane;
}

int batch_lines_per_block(int dir) { return dir == 1 ? FluxLines<1>::PB : dir == 2 ? FluxLines<2>::PB : FluxLines<3>::PB; }

long long batch_line_blocks(int dir, int nx, int ny, int nz)
{
    const int nd = dir == 1 ? nx : dir == 2 ? ny : nz;
    const long long bund = dir == 1 ? FluxLines<1>::bundles(nx, ny, nz) : dir == 2 ? FluxLines<2>::bundles(nx, ny, nz)
                                                                        : FluxLines<3>::bundles(nx, ny, nz);
    const int pb = batch_lines_per_block(dir);
    return ((long long)nd * bund + pb - 1) / pb;
}

long long batch_face_line_blocks(int dir, int nx, int ny, int nz)
{
    const int nd = dir == 2 ? ny : nz;
    const long long bund = dir == 2 ? FaceLinesG<2>::bundles(nx, ny, nz) : FaceLinesG<3>::bundles(nx, ny, nz);
    const int pb = dir == 2 ? FaceLinesG<2>::PB : FaceLinesG<3>::PB;
    return ((long long)(nd + 1) * bund + pb - 2) / (pb - 1);
}

/* resident 128-thread blocks per SM of a batch kernel (persistent grid size) */
static int resident_blocks(BatchKernel k)
{
    static std::mutex mu;
    static std::map<BatchKernel, int> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(k);
    if (it != cache.end()) return it->second;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, 128, 0) != cudaSuccess || nb < 1) nb = 1;
    cache[k] = nb;
    return nb;
}

} // namespace vh

namespace {

constexpr int kShapes[][2] = {{32, 4}, {64, 2}, {16, 8}, {128, 1}, {8, 16}};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

struct Tiles {
    int4 *all = nullptr;   /* every (member, tile) */
    int n_all = 0;
    int4 *z = nullptr;     /* tiles of 3+1D members (eta flux) */
    int n_z = 0;
};

struct TimeTable {
    double t0 = 0, dt = 0;
    double *d = nullptr;
    int cap = 0;
};

} // namespace

struct vh_batch {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t sync = nullptr;
    std::vector<vh_event *> mem;
    int nq = 14, eos_kind = 0;
    bool mixed = false;              /* members evolve in mixed precision */
    bool any_z = false;
    int zmode = 0;                   /* 0 all 2+1D, 1 all 3+1D, 2 mixed */
    std::vector<vh::BatchMember> h_mem;
    vh::BatchMember *d_mem = nullptr;
    int *d_nstep = nullptr;
    vh::StageArgs *d_args = nullptr;
    std::vector<TimeTable> ttabs;
    std::vector<int> mem_ttab;
    std::map<int, Tiles> tiles;      /* key: tile_x */
    int4 *ftiles[3] = {};            /* mixed precision: face tiles per axis */
    int n_ftiles[3] = {};
    int4 *fltiles[3] = {};           /* mixed precision: face line blocks along y, eta */
    int n_fltiles[3] = {};
    int4 *ltiles[3] = {};            /* FP64: line blocks (member, block) per axis */
    int n_ltiles[3] = {};
    size_t lsmem[3] = {};            /* their dynamic shared memory */
    bool tuned = false;
    vh_batch_tuning tune{};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool timing = false;
    std::vector<vh::StageMarks> marks;
    size_t marks_used = 0;
};

namespace {

int bfail(int code, const std::string &msg) { return vh::set_error(code, msg); }

#define BTRY(x)                                                                                        \
    do {                                                                                               \
        cudaError_t e__ = (x);                                                                         \
        if (e__ != cudaSuccess)                                                                        \
            return bfail(e__ == cudaErrorMemoryAllocation ? VH_ERR_NOMEM : VH_ERR_CUDA,                \
                         std::string(#x) + ": " + cudaGetErrorString(e__));                            \
    } while (0)

int build_tiles(vh_batch *b, int tx)
{
    if (b->tiles.count(tx)) return VH_OK;
    const int ty = 128 / tx;
    std::vector<int4> all, z;
    for (size_t m = 0; m < b->mem.size(); ++m) {
        const vh_config &c = b->mem[m]->cfg;
        for (int k = 0; k < c.nz; ++k)
            for (int j0 = 0; j0 < c.ny; j0 += ty)
                for (int i0 = 0; i0 < c.nx; i0 += tx) {
                    int4 t = make_int4((int)m, i0, j0, k);
                    all.push_back(t);
                    if (c.nz > 1) z.push_back(t);
                }
    }
    Tiles T;
    T.n_all = (int)all.size();
    T.n_z = (int)z.size();
    BTRY(cudaMalloc(&T.all, std::max<size_t>(all.size(), 1) * sizeof(int4)));
    BTRY(cudaMemcpy(T.all, all.data(), all.size() * sizeof(int4), cudaMemcpyHostToDevice));
    if (!z.empty()) {
        BTRY(cudaMalloc(&T.z, z.size() * sizeof(int4)));
        BTRY(cudaMemcpy(T.z, z.data(), z.size() * sizeof(int4), cudaMemcpyHostToDevice));
    }
    b->tiles[tx] = T;
    return VH_OK;
}

/* mixed precision: the face tiles of kt_batch_face_kernel, per axis (x
 * tiles cover 31 cells of 8 rows, y tiles 32 cells of 7 rows, eta tiles 32
 * cells of 7 planes of one row, of the 3+1D members) */
int build_face_tiles(vh_batch *b)
{
    constexpr int TX = vh::kBatchFaceTX, TY = vh::kBatchFaceTY;
    std::vector<int4> f[3];
    for (size_t m = 0; m < b->mem.size(); ++m) {
        const vh_config &c = b->mem[m]->cfg;
        for (int k = 0; k < c.nz; ++k) {
            for (int j0 = 0; j0 < c.ny; j0 += TY)
                for (int i0 = 0; i0 < c.nx; i0 += TX - 1) f[0].push_back(make_int4((int)m, i0, j0, k));
            for (int j0 = 0; j0 < c.ny; j0 += TY - 1)
                for (int i0 = 0; i0 < c.nx; i0 += TX) f[1].push_back(make_int4((int)m, i0, j0, k));
        }
        if (c.nz > 1)
            for (int j = 0; j < c.ny; ++j)
                for (int k0 = 0; k0 < c.nz; k0 += TY - 1)
                    for (int i0 = 0; i0 < c.nx; i0 += TX) f[2].push_back(make_int4((int)m, i0, j, k0));
    }
    for (int d = 0; d < 3; ++d) {
        b->n_ftiles[d] = (int)f[d].size();
        if (f[d].empty()) continue;
        BTRY(cudaMalloc(&b->ftiles[d], f[d].size() * sizeof(int4)));
        BTRY(cudaMemcpy(b->ftiles[d], f[d].data(), f[d].size() * sizeof(int4), cudaMemcpyHostToDevice));
    }
    /* face line blocks along y and eta (the 3+1D members) */
    std::vector<int4> fl[3];
    for (size_t m = 0; m < b->mem.size(); ++m) {
        const vh_config &c = b->mem[m]->cfg;
        for (int d = 2; d <= (c.nz > 1 ? 3 : 2); ++d) {
            const long long nb = vh::batch_face_line_blocks(d, c.nx, c.ny, c.nz);
            for (long long k = 0; k < nb; ++k) fl[d - 1].push_back(make_int4((int)m, (int)k, 0, 0));
        }
    }
    for (int d = 1; d < 3; ++d) {
        b->n_fltiles[d] = (int)fl[d].size();
        if (fl[d].empty()) continue;
        BTRY(cudaMalloc(&b->fltiles[d], fl[d].size() * sizeof(int4)));
        BTRY(cudaMemcpy(b->fltiles[d], fl[d].data(), fl[d].size() * sizeof(int4), cudaMemcpyHostToDevice));
    }
    return VH_OK;
}

/* mixed batches run their y and eta flux over face line pieces (the
 * single-event form); VH_BATCH_FACE_LINES=0 keeps the 32 x 8 face tiles */
bool batch_face_lines_on()
{
    static int on = [] {
        const char *e = getenv("VH_BATCH_FACE_LINES");
        return (e && e[0] == '0') ? 0 : 1;
    }();
    return on == 1;
}

/* FP64 batches run their flux over line pieces (the single-event form);
 * VH_BATCH_LINES=0 keeps the per-cell flux of kt_batch_kernel */
bool batch_lines_on()
{
    static int on = [] {
        const char *e = getenv("VH_BATCH_LINES");
        return (e && e[0] == '0') ? 0 : 1;
    }();
    return on == 1;
}

/* FP64: the line blocks of kt_batch_lines_kernel per axis, every member's
 * blocks in member order (eta: the 3+1D members) */
int build_line_tiles(vh_batch *b)
{
    std::vector<int4> f[3];
    for (size_t m = 0; m < b->mem.size(); ++m) {
        const vh_config &c = b->mem[m]->cfg;
        for (int d = 1; d <= (c.nz > 1 ? 3 : 2); ++d) {
            const long long nb = vh::batch_line_blocks(d, c.nx, c.ny, c.nz);
            for (long long k = 0; k < nb; ++k) f[d - 1].push_back(make_int4((int)m, (int)k, 0, 0));
            const int nd = d == 1 ? c.nx : d == 2 ? c.ny : c.nz;
            b->lsmem[d - 1] = std::max(b->lsmem[d - 1], vh::batch_lines_smem(b->nq, d, nd));
        }
    }
    for (int d = 0; d < 3; ++d) {
        b->n_ltiles[d] = (int)f[d].size();
        if (f[d].empty()) continue;
        BTRY(cudaMalloc(&b->ltiles[d], f[d].size() * sizeof(int4)));
        BTRY(cudaMemcpy(b->ltiles[d], f[d].data(), f[d].size() * sizeof(int4), cudaMemcpyHostToDevice));
        vh::BatchKernel k = vh::batch_lines_kernel(b->nq, b->eos_kind, d + 1);
        BTRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->lsmem[d]));
        /* shared memory for 5 resident blocks, the rest to L1 (the EoS table) */
        const int pct = (int)((5 * (b->lsmem[d] + sizeof(vh::StageArgs) + 1024) * 100 + 228 * 1024 - 1) / (228 * 1024));
        BTRY(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, std::min(pct, 100)));
    }
    return VH_OK;
}

/* host libm values of the times of steps [0, cap): t = t0 + n dt exactly as
 * vh_event_step advances it, pow(t, 2) as SourceTerms.cpp:415, :587 */
int ensure_times(vh_batch *b, int need)
{
    bool changed = false;
    for (size_t i = 0; i < b->ttabs.size(); ++i) {
        TimeTable &T = b->ttabs[i];
        if (T.cap >= need) continue;
        int cap = std::max(need, std::max(2 * T.cap, 1024));
        std::vector<double> h(4 * (size_t)cap);
        for (int n = 0; n < cap; ++n) {
            const double t = T.t0 + n * T.dt;
            const double t1 = t + T.dt;
            h[4 * (size_t)n] = t;
            h[4 * (size_t)n + 1] = t1;
            h[4 * (size_t)n + 2] = pow(t, 2);
            h[4 * (size_t)n + 3] = pow(t1, 2);
        }
        double *d = nullptr;
        BTRY(cudaStreamSynchronize(b->stream));   /* in-flight steps may still read the old table */
        BTRY(cudaMalloc(&d, h.size() * sizeof(double)));
        BTRY(cudaMemcpy(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
        cudaFree(T.d);
        T.d = d;
        T.cap = cap;
        changed = true;
    }
    if (changed) {
        for (size_t m = 0; m < b->mem.size(); ++m) {
            b->h_mem[m].ttab = b->ttabs[b->mem_ttab[m]].d;
            b->h_mem[m].tcap = b->ttabs[b->mem_ttab[m]].cap;
        }
        BTRY(cudaMemcpyAsync(b->d_mem, b->h_mem.data(), b->h_mem.size() * sizeof(vh::BatchMember),
                             cudaMemcpyHostToDevice, b->stream));
        BTRY(cudaStreamSynchronize(b->stream));
    }
    return VH_OK;
}

vh::StageMarks *next_marks(vh_batch *b)
{
    if (!b->timing) return nullptr;
    if (b->marks_used == b->marks.size()) {
        vh::StageMarks m{};
        for (cudaEvent_t &e : m.ev)
            if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        b->marks.push_back(m);
    }
    return &b->marks[b->marks_used++];
}

void launch_prep(vh_batch *b, int advance)
{
    vh::BatchPrep P;
    P.mem = b->d_mem;
    P.nstep = b->d_nstep;
    P.args = b->d_args;
    P.nmem = (int)b->mem.size();
    P.advance = advance;
    vh::batch_prep_kernel<<<(P.nmem + 127) / 128, 128, 0, b->stream>>>(P);
}

/* one phase over the batch with the given tile shape and grid form */
void launch_phase(vh_batch *b, int stage, int phase, int tx, int persistent)
{
    const Tiles &T = b->tiles[tx];
    vh::BatchLaunch B;
    B.args = b->d_args + (size_t)stage * b->mem.size();
    B.tiles = phase == 3 ? T.z : T.all;
    B.ntiles = phase == 3 ? T.n_z : T.n_all;
    if (B.ntiles == 0) return;
    vh::BatchKernel k = vh::batch_kernel(b->nq, b->eos_kind, phase, stage == 1, b->zmode, b->mixed);
    int grid = B.ntiles;
    if (persistent) grid = std::min(grid, vh::resident_blocks(k) * b->sms);
    dim3 block(tx, 128 / tx, 1);
    k<<<grid, block, 0, b->stream>>>(B);
}

/* FP64: one axis of the flux over the line blocks */
void launch_lines(vh_batch *b, int stage, int dir)
{
    vh::BatchLaunch B;
    B.args = b->d_args + (size_t)stage * b->mem.size();
    B.tiles = b->ltiles[dir - 1];
    B.ntiles = b->n_ltiles[dir - 1];
    if (B.ntiles == 0) return;
    vh::BatchKernel k = vh::batch_lines_kernel(b->nq, b->eos_kind, dir);
    k<<<B.ntiles, 128, b->lsmem[dir - 1], b->stream>>>(B);
}

/* mixed precision: one axis of the face-once flux over the face tiles */
void launch_face(vh_batch *b, int stage, int dir)
{
    vh::BatchLaunch B;
    B.args = b->d_args + (size_t)stage * b->mem.size();
    if (dir >= 2 && batch_face_lines_on()) {
        B.tiles = b->fltiles[dir - 1];
        B.ntiles = b->n_fltiles[dir - 1];
        if (B.ntiles == 0) return;
        vh::BatchKernel k = vh::batch_face_lines_kernel_mixed(b->nq, b->eos_kind, dir);
        k<<<B.ntiles, 128, 0, b->stream>>>(B);
        return;
    }
    B.tiles = b->ftiles[dir - 1];
    B.ntiles = b->n_ftiles[dir - 1];
    if (B.ntiles == 0) return;
    vh::BatchKernel k = vh::batch_face_kernel_mixed(b->nq, b->eos_kind, dir);
    k<<<B.ntiles, dim3(vh::kBatchFaceTX, vh::kBatchFaceTY, 1), 0, b->stream>>>(B);
}

void launch_stage(vh_batch *b, int stage, const vh_batch_tuning &t, vh::StageMarks *m)
{
    if (m) { m->n = 0; cudaEventRecord(m->ev[0], b->stream); }
    auto run = [&](int phase) {
        /* the split stage's flux is face-once in mixed precision, as on
         * single events (the tile shape of these phases is then unused) */
        const bool flux = phase >= VH_PHASE_FLUX_X && phase <= VH_PHASE_FLUX_ETA;
        if (flux && b->mixed) launch_face(b, stage, phase - VH_PHASE_FLUX_X + 1);
        else if (flux && batch_lines_on()) launch_lines(b, stage, phase - VH_PHASE_FLUX_X + 1);
        else launch_phase(b, stage, phase, t.tile_x[phase], t.persistent[phase]);
        if (m) { m->phase[m->n] = phase; cudaEventRecord(m->ev[++m->n], b->stream); }
    };
    if (t.fused) { run(VH_PHASE_FUSED); return; }
    run(VH_PHASE_SOURCE);
    run(VH_PHASE_FLUX_X);
    run(VH_PHASE_FLUX_Y);
    if (b->any_z) run(VH_PHASE_FLUX_ETA);
    run(VH_PHASE_FINAL);
}

int check_members(vh_batch *b)
{
    for (size_t m = 0; m < b->mem.size(); ++m) {
        vh_event *ev = b->mem[m];
        if (!ev->initialised) return bfail(VH_ERR_STATE, "batch member " + std::to_string(m) + " has no initial state");
        if (ev->fo_pending) return bfail(VH_ERR_STATE, "batch member " + std::to_string(m) + " has a freezeout block pending");
        const int c = ev->n & 1;
        if (ev->qc != c || ev->qn != 1 - c || ev->qs != 2 || ev->uc != c || ev->up != 1 - c || ev->us != 2 || ev->ec != 0)
            return bfail(VH_ERR_STATE, "batch member " + std::to_string(m) + ": unexpected buffer roles");
    }
    return VH_OK;
}

/* order the batch stream after every member's queued work */
int join_members(vh_batch *b)
{
    for (vh_event *ev : b->mem) {
        BTRY(cudaEventRecord(b->sync, ev->stream));
        BTRY(cudaStreamWaitEvent(b->stream, b->sync, 0));
    }
    return VH_OK;
}

/* order every member's later work after the batch stream */
int release_members(vh_batch *b)
{
    BTRY(cudaEventRecord(b->sync, b->stream));
    for (vh_event *ev : b->mem) BTRY(cudaStreamWaitEvent(ev->stream, b->sync, 0));
    return VH_OK;
}

int upload_steps(vh_batch *b)
{
    std::vector<int> n(b->mem.size());
    for (size_t m = 0; m < b->mem.size(); ++m) n[m] = b->mem[m]->n;
    BTRY(cudaMemcpyAsync(b->d_nstep, n.data(), n.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
    BTRY(cudaStreamSynchronize(b->stream));
    return VH_OK;
}

void drop_graph(vh_batch *b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

/* Time stage 1 of the current step for every (tile shape, grid form), fused
 * and split (split only for a mixed batch, whose forms round differently);
 * stage 1 writes only the scratch planes (qS, e/p[1], uS), which the real
 * step rewrites, so the members' state is untouched. */
int autotune(vh_batch *b)
{
    for (int s = 0; s < kNumShapes; ++s) {
        int rc = build_tiles(b, kShapes[s][0]);
        if (rc != VH_OK) return rc;
    }
    launch_prep(b, 0);
    /* a second timing round only where a stage is short enough for launch
     * noise to matter (under 2 ms); large batches are timed once */
    const int max_rounds = 2;
    const int ncand = kNumShapes * 2;
    /* the timing events, destroyed on every return (value-initialised, so an
     * event that was never created is null) */
    struct Marks {
        std::vector<vh::StageMarks> v;
        explicit Marks(size_t n) : v(n) {}
        ~Marks()
        {
            for (auto &m : v)
                for (cudaEvent_t e : m.ev)
                    if (e) cudaEventDestroy(e);
        }
    } marks((size_t)max_rounds * ncand * 2);
    std::vector<vh::StageMarks> &mk = marks.v;
    for (auto &m : mk)
        for (cudaEvent_t &e : m.ev) BTRY(cudaEventCreate(&e));
    double best[VH_NPHASES];
    int best_c[VH_NPHASES];
    for (int ph = 0; ph < VH_NPHASES; ++ph) { best[ph] = 1e30; best_c[ph] = 0; }
    size_t used = 0;
    for (int r = 0; r < max_rounds; ++r) {
        const size_t first = used;
        for (int s = 0; s < kNumShapes; ++s)
            for (int p = 0; p < 2; ++p) {
                vh_batch_tuning t{};
                for (int ph = 0; ph < VH_NPHASES; ++ph) { t.tile_x[ph] = kShapes[s][0]; t.tile_y[ph] = kShapes[s][1]; t.persistent[ph] = p; }
                t.fused = 0;
                launch_stage(b, 0, t, &mk[used++]);
                t.fused = 1;
                if (!b->mixed) launch_stage(b, 0, t, &mk[used++]);
            }
        BTRY(cudaGetLastError());
        BTRY(cudaStreamSynchronize(b->stream));
        /* best[phase] over candidates: min over rounds */
        size_t k = first;
        for (int cnd = 0; cnd < ncand; ++cnd)
            for (int f = 0; f < (b->mixed ? 1 : 2); ++f) {
                const vh::StageMarks &m = mk[k++];
                for (int n = 0; n < m.n; ++n) {
                    float ms = 0;
                    BTRY(cudaEventElapsedTime(&ms, m.ev[n], m.ev[n + 1]));
                    if (ms < best[m.phase[n]]) { best[m.phase[n]] = ms; best_c[m.phase[n]] = cnd; }
                }
            }
        const double split_ms = best[VH_PHASE_SOURCE] + best[VH_PHASE_FLUX_X] + best[VH_PHASE_FLUX_Y] +
                                best[VH_PHASE_FINAL] + (b->any_z ? best[VH_PHASE_FLUX_ETA] : 0.0);
        if (std::min(best[VH_PHASE_FUSED], split_ms) > 2.0) break;
    }
    double split = best[VH_PHASE_SOURCE] + best[VH_PHASE_FLUX_X] + best[VH_PHASE_FLUX_Y] + best[VH_PHASE_FINAL] +
                   (b->any_z ? best[VH_PHASE_FLUX_ETA] : 0.0);
    vh_batch_tuning t{};
    /* a mixed batch keeps the split stage: its face-once flux and the fused
     * stage's per-cell flux round differently, and a batch's results must not
     * depend on which of two close timings won */
    t.fused = (!b->mixed && best[VH_PHASE_FUSED] < split) ? 1 : 0;
    for (int ph = 0; ph < VH_NPHASES; ++ph) {
        const int c = best_c[ph];
        t.tile_x[ph] = kShapes[c / 2][0];
        t.tile_y[ph] = kShapes[c / 2][1];
        t.persistent[ph] = c % 2;
    }
    t.stage_ms = t.fused ? best[VH_PHASE_FUSED] : split;
    b->tune = t;
    b->tuned = true;
    drop_graph(b);
    return VH_OK;
}

/* load every kernel the step uses (and size its persistent grid) before the
 * capture, so that no module loading happens while the stream is captured */
int preload(vh_batch *b)
{
    cudaFuncAttributes attr;
    BTRY(cudaFuncGetAttributes(&attr, vh::batch_prep_kernel));
    for (int stage = 0; stage < 2; ++stage)
        for (int ph = 0; ph < VH_NPHASES; ++ph) {
            vh::BatchKernel k = vh::batch_kernel(b->nq, b->eos_kind, ph, stage == 1, b->zmode, b->mixed);
            BTRY(cudaFuncGetAttributes(&attr, k));
            vh::resident_blocks(k);
        }
    if (b->mixed) {
        for (int d = 1; d <= 3; ++d) BTRY(cudaFuncGetAttributes(&attr, vh::batch_face_kernel_mixed(b->nq, b->eos_kind, d)));
        for (int d = 2; d <= 3; ++d) BTRY(cudaFuncGetAttributes(&attr, vh::batch_face_lines_kernel_mixed(b->nq, b->eos_kind, d)));
    }
    else
        for (int d = 1; d <= 3; ++d) BTRY(cudaFuncGetAttributes(&attr, vh::batch_lines_kernel(b->nq, b->eos_kind, d)));
    return VH_OK;
}

int ensure_graph(vh_batch *b)
{
    if (b->exec) return VH_OK;
    int rc = preload(b);
    if (rc != VH_OK) return rc;
    BTRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    launch_prep(b, 1);
    launch_stage(b, 0, b->tune, nullptr);
    launch_stage(b, 1, b->tune, nullptr);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (e != cudaSuccess) return bfail(VH_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    b->graph = g;
    BTRY(cudaGraphInstantiate(&b->exec, g, 0));
    return VH_OK;
}

int valid_tuning(const vh_batch_tuning *t)
{
    for (int ph = 0; ph < VH_NPHASES; ++ph) {
        bool ok = false;
        for (int s = 0; s < kNumShapes; ++s) ok |= (t->tile_x[ph] == kShapes[s][0] && t->tile_y[ph] == kShapes[s][1]);
        if (!ok) return 0;
    }
    return 1;
}

} // namespace

extern "C" {

int vh_batch_create(vh_event *const *events, int n_events, vh_batch **out)
{
    if (!events || n_events < 1 || !out) return bfail(VH_ERR_ARG, "bad argument");
    *out = nullptr;
    vh_batch *b = new vh_batch;
    int rc = VH_OK;
#define CTRY(x) do { cudaError_t e__ = (x); if (e__ != cudaSuccess) { rc = bfail(e__ == cudaErrorMemoryAllocation ? VH_ERR_NOMEM : VH_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e__)); vh_batch_destroy(b); return rc; } } while (0)
    for (int i = 0; i < n_events; ++i) {
        vh_event *ev = events[i];
        if (!ev) { vh_batch_destroy(b); return bfail(VH_ERR_ARG, "null member"); }
        for (int j = 0; j < i; ++j)
            if (events[j] == ev) { vh_batch_destroy(b); return bfail(VH_ERR_ARG, "event listed twice"); }
        const bool mixed = ev->cfg.precision == VH_PREC_MIXED;
        if (i > 0 && (ev->nq != b->nq || ev->cfg.eos_kind != b->eos_kind || ev->device != b->device || mixed != b->mixed)) {
            vh_batch_destroy(b);
            return bfail(VH_ERR_ARG, "batch members must share the EoS kind, bulk on/off, the precision and the device");
        }
        if (i == 0) { b->nq = ev->nq; b->eos_kind = ev->cfg.eos_kind; b->device = ev->device; b->mixed = mixed; }
        b->mem.push_back(ev);
        b->any_z |= ev->cfg.nz > 1;
    }
    bool all_z = true;
    for (vh_event *ev : b->mem) all_z &= ev->cfg.nz > 1;
    b->zmode = all_z ? 1 : (b->any_z ? 2 : 0);
    int cur = 0;
    CTRY(cudaGetDevice(&cur));
    if (cur != b->device) { vh_batch_destroy(b); return bfail(VH_ERR_ARG, "members live on another device"); }
    CTRY(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device));
    CTRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    CTRY(cudaEventCreateWithFlags(&b->sync, cudaEventDisableTiming));
    const size_t nm = b->mem.size();
    b->h_mem.resize(nm);
    b->mem_ttab.resize(nm);
    for (size_t m = 0; m < nm; ++m) {
        vh_event *ev = b->mem[m];
        vh::BatchMember &M = b->h_mem[m];
        std::memset(&M, 0, sizeof M);
        M.base = vh::stage_args_base(ev);
        for (int i = 0; i < 3; ++i) { M.q[i] = ev->q[i]; M.u[i] = ev->u[i]; }
        for (int i = 0; i < 2; ++i) M.ep[i] = ev->ep[i];
        M.active = 1;
        int found = -1;
        for (size_t i = 0; i < b->ttabs.size(); ++i)
            if (b->ttabs[i].t0 == ev->cfg.t0 && b->ttabs[i].dt == ev->cfg.dt) found = (int)i;
        if (found < 0) {
            TimeTable T;
            T.t0 = ev->cfg.t0;
            T.dt = ev->cfg.dt;
            b->ttabs.push_back(T);
            found = (int)b->ttabs.size() - 1;
        }
        b->mem_ttab[m] = found;
    }
    CTRY(cudaMalloc(&b->d_mem, nm * sizeof(vh::BatchMember)));
    CTRY(cudaMalloc(&b->d_nstep, nm * sizeof(int)));
    CTRY(cudaMalloc(&b->d_args, 2 * nm * sizeof(vh::StageArgs)));
    CTRY(cudaMemcpy(b->d_mem, b->h_mem.data(), nm * sizeof(vh::BatchMember), cudaMemcpyHostToDevice));
    CTRY(cudaMemset(b->d_nstep, 0, nm * sizeof(int)));
#undef CTRY
    rc = ensure_times(b, 1024);
    if (rc == VH_OK && b->mixed) rc = build_face_tiles(b);
    if (rc == VH_OK && !b->mixed) rc = build_line_tiles(b);
    if (rc != VH_OK) { vh_batch_destroy(b); return rc; }
    *out = b;
    return VH_OK;
}

int vh_batch_destroy(vh_batch *b)
{
    if (!b) return VH_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(b);
    for (auto &kv : b->tiles) { cudaFree(kv.second.all); cudaFree(kv.second.z); }
    for (int4 *f : b->ftiles) cudaFree(f);
    for (int4 *f : b->ltiles) cudaFree(f);
    for (int4 *f : b->fltiles) cudaFree(f);
    for (auto &T : b->ttabs) cudaFree(T.d);
    for (auto &m : b->marks)
        for (cudaEvent_t e : m.ev) cudaEventDestroy(e);
    cudaFree(b->d_mem);
    cudaFree(b->d_nstep);
    cudaFree(b->d_args);
    if (b->sync) cudaEventDestroy(b->sync);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return VH_OK;
}

int vh_batch_size(vh_batch *b, int *n_events)
{
    if (!b || !n_events) return bfail(VH_ERR_ARG, "null argument");
    *n_events = (int)b->mem.size();
    return VH_OK;
}

int vh_batch_set_active(vh_batch *b, int member, int active)
{
    if (!b || member < 0 || member >= (int)b->mem.size()) return bfail(VH_ERR_ARG, "bad member index");
    b->h_mem[member].active = active ? 1 : 0;
    BTRY(cudaMemcpyAsync(&b->d_mem[member].active, &b->h_mem[member].active, sizeof(int), cudaMemcpyHostToDevice,
                         b->stream));
    BTRY(cudaStreamSynchronize(b->stream));
    return VH_OK;
}

int vh_batch_autotune(vh_batch *b, vh_batch_tuning *out)
{
    if (!b) return bfail(VH_ERR_ARG, "null batch");
    int rc = check_members(b);
    if (rc == VH_OK) rc = upload_steps(b);
    if (rc == VH_OK) rc = join_members(b);
    if (rc == VH_OK) rc = autotune(b);
    if (rc == VH_OK) rc = release_members(b);
    if (rc == VH_OK && out) *out = b->tune;
    return rc;
}

int vh_batch_get_tuning(vh_batch *b, vh_batch_tuning *out)
{
    if (!b || !out) return bfail(VH_ERR_ARG, "null argument");
    if (!b->tuned) return bfail(VH_ERR_STATE, "batch not tuned yet (vh_batch_autotune or a first vh_batch_step)");
    *out = b->tune;
    return VH_OK;
}

int vh_batch_set_tuning(vh_batch *b, const vh_batch_tuning *t)
{
    if (!b || !t) return bfail(VH_ERR_ARG, "null argument");
    if (!valid_tuning(t)) return bfail(VH_ERR_ARG, "tile shape not among 32x4, 64x2, 16x8, 128x1, 8x16");
    for (int ph = 0; ph < VH_NPHASES; ++ph) {
        int rc = build_tiles(b, t->tile_x[ph]);
        if (rc != VH_OK) return rc;
    }
    b->tune = *t;
    b->tuned = true;
    drop_graph(b);
    return VH_OK;
}

int vh_batch_step(vh_batch *b, int nsteps)
{
    if (!b || nsteps < 0) return bfail(VH_ERR_ARG, "bad argument");
    if (nsteps == 0) return VH_OK;
    int rc = check_members(b);
    if (rc != VH_OK) return rc;
    int need = 0;
    for (vh_event *ev : b->mem) need = std::max(need, ev->n + nsteps + 1);
    if ((rc = ensure_times(b, need)) != VH_OK) return rc;
    /* a member's dynamical sources may have been set or removed since */
    bool changed = false;
    for (size_t m = 0; m < b->mem.size(); ++m) {
        const double *src = b->mem[m]->src_on ? b->mem[m]->src : nullptr;
        if (b->h_mem[m].base.src != src) { b->h_mem[m].base.src = src; changed = true; }
    }
    if (changed)
        BTRY(cudaMemcpyAsync(b->d_mem, b->h_mem.data(), b->h_mem.size() * sizeof(vh::BatchMember),
                             cudaMemcpyHostToDevice, b->stream));
    if ((rc = upload_steps(b)) != VH_OK) return rc;
    if ((rc = join_members(b)) != VH_OK) return rc;
    if (!b->tuned && (rc = autotune(b)) != VH_OK) return rc;
    if (b->timing) {
        for (int it = 0; it < nsteps; ++it) {
            launch_prep(b, 1);
            launch_stage(b, 0, b->tune, next_marks(b));
            launch_stage(b, 1, b->tune, next_marks(b));
        }
    } else {
        if ((rc = ensure_graph(b)) != VH_OK) return rc;
        for (int it = 0; it < nsteps; ++it) BTRY(cudaGraphLaunch(b->exec, b->stream));
    }
    BTRY(cudaGetLastError());
    if ((rc = release_members(b)) != VH_OK) return rc;
    for (size_t m = 0; m < b->mem.size(); ++m) {
        if (!b->h_mem[m].active) continue;
        vh_event *ev = b->mem[m];
        ev->n += nsteps;
        ev->t = ev->cfg.t0 + ev->n * ev->cfg.dt;
        if (nsteps & 1) { std::swap(ev->qc, ev->qn); std::swap(ev->uc, ev->up); }
    }
    return VH_OK;
}

int vh_batch_kernel_launches(vh_batch *b, int *per_step)
{
    if (!b || !per_step) return bfail(VH_ERR_ARG, "null argument");
    if (!b->tuned) return bfail(VH_ERR_STATE, "batch not tuned yet");
    const int stage = b->tune.fused ? 1 : (b->any_z ? 5 : 4);
    *per_step = 1 + 2 * stage;   /* prep + two stages */
    return VH_OK;
}

int vh_batch_phase_timing(vh_batch *b, int enable)
{
    if (!b) return bfail(VH_ERR_ARG, "null batch");
    b->timing = enable != 0;
    b->marks_used = 0;
    return VH_OK;
}

int vh_batch_phase_times(vh_batch *b, double *ms, long long *launches)
{
    if (!b || !ms || !launches) return bfail(VH_ERR_ARG, "null argument");
    BTRY(cudaStreamSynchronize(b->stream));
    for (int p = 0; p < VH_NPHASES; ++p) { ms[p] = 0; launches[p] = 0; }
    for (size_t i = 0; i < b->marks_used; ++i) {
        const vh::StageMarks &m = b->marks[i];
        for (int n = 0; n < m.n; ++n) {
            float t = 0;
            BTRY(cudaEventElapsedTime(&t, m.ev[n], m.ev[n + 1]));
            ms[m.phase[n]] += t;
            launches[m.phase[n]] += 1;
        }
    }
    b->marks_used = 0;
    return VH_OK;
}

int vh_batch_stream(vh_batch *b, void **stream)
{
    if (!b || !stream) return bfail(VH_ERR_ARG, "null argument");
    *stream = (void *)b->stream;
    return VH_OK;
}

} /* extern "C" */

/*
 * vh_capi.cu -- the C ABI event implementation (include/vh_b200.h).
 *
 * The event object and its state layout are described in vh_event.h.  One
 * RK2 step is two RK stages (vh_kt.cu), each either one fused kernel or the
 * phase-split kernels; buffer roles rotate by index on the host.
 */
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <map>
#include <string>
#include <vector>

#include "vh_b200.h"
#include "vh_internal.h"
#include "vh_kernels.h"
#include "vh_event.h"

static thread_local std::string g_err;

static int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

int vh::set_error(int code, const std::string &msg) { return fail(code, msg); }
#define CUDA_TRY(x)                                                                                   \
    do {                                                                                              \
        cudaError_t e__ = (x);                                                                        \
        if (e__ != cudaSuccess) return fail(e__ == cudaErrorMemoryAllocation ? VH_ERR_NOMEM : VH_ERR_CUDA, \
                                            std::string(#x) + ": " + cudaGetErrorString(e__));        \
    } while (0)

namespace {

std::mutex g_powf_mu;
std::map<int, vh::DevPowf> g_powf;

int device_powf(int dev, vh::DevPowf *out)
{
    std::lock_guard<std::mutex> lk(g_powf_mu);
    auto it = g_powf.find(dev);
    if (it != g_powf.end()) { *out = it->second; return VH_OK; }
    const vh::PowfQuarterTable &T = vh::powf_quarter_table();
    vh::DevPowf d;
    unsigned lob, hib;
    std::memcpy(&lob, &T.lo, 4);
    std::memcpy(&hib, &T.hi, 4);
    d.hb0 = lob >> 16;
    d.hb1 = hib >> 16;
    size_t nk = std::max<size_t>(T.keys.size(), 1);
    CUDA_TRY(cudaMalloc(&d.keys, nk * sizeof(unsigned)));
    CUDA_TRY(cudaMalloc(&d.vals, nk * sizeof(float)));
    CUDA_TRY(cudaMalloc(&d.bucket, T.bucket.size() * sizeof(unsigned)));
    if (!T.keys.empty()) {
        CUDA_TRY(cudaMemcpy(d.keys, T.keys.data(), T.keys.size() * sizeof(unsigned), cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(d.vals, T.vals.data(), T.vals.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    CUDA_TRY(cudaMemcpy(d.bucket, T.bucket.data(), T.bucket.size() * sizeof(unsigned), cudaMemcpyHostToDevice));
    g_powf[dev] = d;
    *out = d;
    return VH_OK;
}

/* Device memory of events comes from a stream-ordered pool per device that
 * keeps freed memory mapped: events that come and go (the server retires
 * and admits them continually) reuse it, without cudaFree's unmapping and
 * device-wide synchronisation.  The pool is trimmed when the last event on
 * the device is destroyed and no server holds it (a server keeps the memory
 * through its idle gaps), so an idle process holds nothing. */
struct EventPool {
    cudaMemPool_t pool = nullptr;
    int live = 0;
    int holds = 0;
};
std::mutex g_pool_mu;
std::map<int, EventPool> g_pools;

cudaError_t pool_of(int dev, cudaMemPool_t *out)
{
    std::lock_guard<std::mutex> lk(g_pool_mu);
    EventPool &P = g_pools[dev];
    if (!P.pool) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaError_t e = cudaMemPoolCreate(&P.pool, &props);
        if (e != cudaSuccess) { P.pool = nullptr; return e; }
        unsigned long long keep = ~0ULL;
        e = cudaMemPoolSetAttribute(P.pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) return e;
    }
    *out = P.pool;
    return cudaSuccess;
}

void pool_live(int dev, int delta)
{
    std::lock_guard<std::mutex> lk(g_pool_mu);
    EventPool &P = g_pools[dev];
    P.live += delta;
    if (P.live == 0 && P.holds == 0 && P.pool) cudaMemPoolTrimTo(P.pool, 0);
}

/* an event buffer, ordered on the event's stream.  A diagnostic, off by
 * default: VH_POISON_ALLOC=1 fills every new buffer with all-ones bytes (a
 * NaN in every double), =2 with 0x7E bytes (1.4e301 in every double, 2.1e38
 * in every float: finite, so fmin/fmax-based limiters and wave speeds do not
 * discard it as they discard a NaN), before the library's own
 * initialisation, so that a value read before any kernel wrote it changes the
 * results the tests compare. */
cudaError_t ev_alloc(vh_event *ev, void *ptr, size_t bytes)
{
    cudaMemPool_t pool = nullptr;
    cudaError_t e = pool_of(ev->device, &pool);
    if (e != cudaSuccess) return e;
    e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(ptr), bytes, pool, ev->stream);
    if (e == cudaSuccess) {
        const char *p = getenv("VH_POISON_ALLOC");
        if (p && (p[0] == '1' || p[0] == '2'))
            e = cudaMemsetAsync(*reinterpret_cast<void **>(ptr), p[0] == '1' ? 0xFF : 0x7E, bytes, ev->stream);
    }
    return e;
}

void ev_free(vh_event *ev, void *p)
{
    if (p) cudaFreeAsync(p, ev->stream);
}

} // namespace



void vh::event_pool_hold(int dev, int delta)
{
    std::lock_guard<std::mutex> lk(g_pool_mu);
    EventPool &P = g_pools[dev];
    P.holds += delta;
    if (P.live == 0 && P.holds == 0 && P.pool) cudaMemPoolTrimTo(P.pool, 0);
}

vh::StageArgs vh::stage_args_base(const vh_event *ev)
{
    const vh_config &c = ev->cfg;
    vh::StageArgs A{};
    A.L = ev->L;
    A.nx = c.nx; A.ny = c.ny; A.nz = c.nz; A.ncx = ev->ncx; A.ncy = ev->ncy;
    A.dt = c.dt; A.dx = c.dx; A.dy = c.dy; A.dz = c.dz; A.theta = c.theta; A.etabar = c.etabar;
    A.inv_dx = 1.0 / c.dx; A.inv_dy = 1.0 / c.dy; A.inv_dz = 1.0 / c.dz;
    A.e_reg = ev->e_reg;
    A.eos = dev_eos(ev);
    A.zeta.law = c.zeta_law; A.zeta.norm = c.zeta_norm; A.zeta.T0 = c.zeta_T0_GeV; A.zeta.w = c.zeta_width_GeV;
    A.err.code = ev->err; A.err.step = ev->err + 1; A.err.cell = ev->err_cell;
    A.src = ev->src_on ? ev->src : nullptr;
    A.regfac = ev->regfac_on ? ev->regfac : nullptr;
    return A;
}

extern "C" {

const char *vh_last_error(void) { return g_err.c_str(); }

int vh_device_available(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); return 0; }
    return n > 0 ? 1 : 0;
}

int vh_event_destroy(vh_event *ev)
{
    if (!ev) return VH_OK;
    if (ev->stream) {
        for (double *p : {ev->slab, ev->tables, ev->ic, ev->fo_slabs, ev->fo_elems, ev->fo_slots, ev->vort, ev->src,
                          ev->regfac})
            ev_free(ev, p);
        for (void *p : {(void *)ev->err, (void *)ev->err_cell, (void *)ev->powf_miss, (void *)ev->fo_scratch})
            ev_free(ev, p);
        cudaStreamSynchronize(ev->stream);
    }
    if (ev->fo_hdr) cudaFreeHost(ev->fo_hdr);
    if (ev->fo_done) cudaEventDestroy(ev->fo_done);
    for (auto &m : ev->marks)
        for (cudaEvent_t e : m.ev) cudaEventDestroy(e);
    if (ev->stream) cudaStreamDestroy(ev->stream);
    if (ev->pooled) pool_live(ev->device, -1);
    delete ev;
    return VH_OK;
}

int vh_event_create(const vh_config *cfg, const double *eos_rows, int eos_nrows, vh_event **out)
{
    if (!cfg || !out) return fail(VH_ERR_ARG, "null argument");
    *out = nullptr;
    if (cfg->nx < 2 || cfg->ny < 2 || cfg->nz < 1) return fail(VH_ERR_ARG, "lattice must be at least 2x2x1");
    /* the kernels index cells and lines in 32-bit arithmetic */
    if ((long long)(cfg->nx + 4) * (cfg->ny + 4) * (cfg->nz + 4) >= (1LL << 31))
        return fail(VH_ERR_ARG, "lattice too large (2^31 padded cells or more)");
    if (!(cfg->dx > 0 && cfg->dy > 0 && cfg->dz > 0 && cfg->dt > 0 && cfg->t0 > 0))
        return fail(VH_ERR_ARG, "spacings and t0 must be positive");
    if (cfg->eos_kind == VH_EOS_TABLE && (!eos_rows || eos_nrows < 2 || eos_nrows > 100000))
        return fail(VH_ERR_ARG, "tabulated EoS needs 2..100000 rows");
    if (cfg->precision != VH_PREC_FP64 && cfg->precision != VH_PREC_MIXED) return fail(VH_ERR_ARG, "unknown precision mode");
    if (!vh_device_available()) return fail(VH_ERR_NODEVICE, "no CUDA device");
    vh_event *ev = new vh_event();
    ev->cfg = *cfg;
    ev->nq = cfg->bulk ? 15 : 14;
    ev->ncx = cfg->nx + 4; ev->ncy = cfg->ny + 4; ev->ncz = cfg->nz + 4;
    long long len = (long long)ev->ncx * ev->ncy * ev->ncz;
    ev->L = (len + 31) / 32 * 32;
    ev->N = (long long)cfg->nx * cfg->ny * cfg->nz;
    ev->heos.init(*cfg, eos_rows, eos_nrows);
    ev->e_reg = ev->heos.energy_of_T(cfg->T_reg_GeV / vh::kHbarc);
    ev->e_fo = ev->heos.energy_of_T(cfg->T_freezeout_GeV / vh::kHbarc);
    int rc;
#define TRY(x) do { cudaError_t e__ = (x); if (e__ != cudaSuccess) { rc = fail(e__ == cudaErrorMemoryAllocation ? VH_ERR_NOMEM : VH_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e__)); vh_event_destroy(ev); return rc; } } while (0)
    TRY(cudaGetDevice(&ev->device));
    TRY(cudaStreamCreateWithFlags(&ev->stream, cudaStreamNonBlocking));
    pool_live(ev->device, 1);
    ev->pooled = true;
    const long long planes = 3LL * ev->nq + 2 * 2 + 3 * 4;
    TRY(ev_alloc(ev, &ev->slab, (size_t)(planes * ev->L) * sizeof(double)));
    TRY(cudaMemsetAsync(ev->slab, 0, (size_t)(planes * ev->L) * sizeof(double), ev->stream));
    double *p = ev->slab;
    for (int b = 0; b < 3; ++b) { ev->q[b] = p; p += ev->nq * ev->L; }
    for (int b = 0; b < 2; ++b) { ev->ep[b] = p; p += 2 * ev->L; }
    for (int b = 0; b < 3; ++b) { ev->u[b] = p; p += 4 * ev->L; }
    if (cfg->eos_kind == VH_EOS_TABLE) {
        TRY(ev_alloc(ev, &ev->tables, 2 * (size_t)eos_nrows * sizeof(double)));
        TRY(cudaMemcpyAsync(ev->tables, ev->heos.p_tb.data(), eos_nrows * sizeof(double), cudaMemcpyHostToDevice, ev->stream));
        TRY(cudaMemcpyAsync(ev->tables + eos_nrows, ev->heos.T_tb.data(), eos_nrows * sizeof(double), cudaMemcpyHostToDevice, ev->stream));
    } else {
        rc = device_powf(ev->device, &ev->powf);
        if (rc != VH_OK) { vh_event_destroy(ev); return rc; }
    }
    TRY(ev_alloc(ev, &ev->err, 2 * sizeof(int)));
    TRY(ev_alloc(ev, &ev->err_cell, sizeof(long long)));
    TRY(ev_alloc(ev, &ev->powf_miss, sizeof(unsigned long long)));
    TRY(cudaMemsetAsync(ev->err, 0, 2 * sizeof(int), ev->stream));
    TRY(cudaMemsetAsync(ev->err_cell, 0, sizeof(long long), ev->stream));
    TRY(cudaMemsetAsync(ev->powf_miss, 0, sizeof(unsigned long long), ev->stream));
    TRY(ev_alloc(ev, &ev->ic, (size_t)(17 * ev->N) * sizeof(double)));
    TRY(cudaStreamSynchronize(ev->stream));
#undef TRY
    *out = ev;
    return VH_OK;
}

static int do_init(vh_event *ev, const double *d_e, const double *d_p, const double *d_u, const double *d_pi, const double *d_Pi)
{
    if (ev->fo_pending) return fail(VH_ERR_STATE, "new initial state with a freezeout block pending");
    vh::InitArgs a;
    a.e = d_e; a.p = d_p; a.u = d_u; a.pi = d_pi; a.Pi = d_Pi;
    ev->qc = 0; ev->qn = 1; ev->qs = 2; ev->ec = 0; ev->uc = 0; ev->up = 1; ev->us = 2;
    a.q = ev->q[ev->qc];
    a.eo = ev->ep[ev->ec];
    a.po = ev->ep[ev->ec] + ev->L;
    a.uo = ev->u[ev->uc];
    a.upo = ev->u[ev->up];
    a.L = ev->L;
    a.nx = ev->cfg.nx; a.ny = ev->cfg.ny; a.nz = ev->cfg.nz;
    a.ncx = ev->ncx; a.ncy = ev->ncy; a.nq = ev->nq;
    vh::launch_init(a, ev->stream);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemsetAsync(ev->err, 0, 2 * sizeof(int), ev->stream));
    CUDA_TRY(cudaMemsetAsync(ev->err_cell, 0, sizeof(long long), ev->stream));
    if (ev->fo_slabs) CUDA_TRY(cudaMemsetAsync(ev->fo_slabs, 0, (size_t)(2 * 11 * ev->N) * sizeof(double), ev->stream));
    ev->fo_prev = 0;
    ev->fo_count = 0;
    ev->n = 0;
    ev->t = ev->cfg.t0;
    ev->initialised = true;
    return VH_OK;
}

int vh_event_set_initial(vh_event *ev, const double *e, const double *p, const double *u, const double *pi, const double *Pi)
{
    if (!ev || !e || !p || !u) return fail(VH_ERR_ARG, "null argument");
    const size_t N = (size_t)ev->N, B = N * sizeof(double);
    double *d = ev->ic;
    CUDA_TRY(cudaMemcpyAsync(d, e, B, cudaMemcpyHostToDevice, ev->stream));
    CUDA_TRY(cudaMemcpyAsync(d + N, p, B, cudaMemcpyHostToDevice, ev->stream));
    CUDA_TRY(cudaMemcpyAsync(d + 2 * N, u, 4 * B, cudaMemcpyHostToDevice, ev->stream));
    if (pi) CUDA_TRY(cudaMemcpyAsync(d + 6 * N, pi, 10 * B, cudaMemcpyHostToDevice, ev->stream));
    if (Pi) CUDA_TRY(cudaMemcpyAsync(d + 16 * N, Pi, B, cudaMemcpyHostToDevice, ev->stream));
    return do_init(ev, d, d + N, d + 2 * N, pi ? d + 6 * N : nullptr, Pi ? d + 16 * N : nullptr);
}

int vh_event_init_glauber(vh_event *ev, double R, double a, double sigma_nn, double b, double e0_GeV,
                          double eta_flat, double eta_sigma)
{
    if (!ev) return fail(VH_ERR_ARG, "null event");
    if (!(R > 0 && a > 0 && sigma_nn > 0 && e0_GeV > 0 && eta_sigma > 0)) return fail(VH_ERR_ARG, "bad Glauber parameters");
    const size_t N = (size_t)ev->N;
    double *d = ev->ic;
    vh::GlauberArgs g;
    g.nx = ev->cfg.nx; g.ny = ev->cfg.ny; g.nz = ev->cfg.nz;
    g.dx = ev->cfg.dx; g.dy = ev->cfg.dy; g.dz = ev->cfg.dz;
    g.R = R; g.a = a; g.sigma_nn = sigma_nn; g.b = b; g.e0 = e0_GeV / vh::kHbarc;
    g.eta_flat = eta_flat; g.eta_sigma = eta_sigma;
    g.eos = dev_eos(ev);
    g.eos_kind = ev->cfg.eos_kind;
    /* staging: e, p, u(4) as vh_event_set_initial; the participant density and
     * its maximum borrow the (unused) pi and Pi slots */
    vh::launch_glauber_ic(g, d + 6 * N, reinterpret_cast<unsigned long long *>(d + 16 * N), d, d + N, d + 2 * N,
                          ev->stream);
    CUDA_TRY(cudaGetLastError());
    return do_init(ev, d, d + N, d + 2 * N, nullptr, nullptr);
}

int vh_event_init_hotspots(vh_event *ev, unsigned long long seed, double mean_spots, double w, double k_gamma,
                           double amp_mean_GeV, double R, double a)
{
    if (!ev) return fail(VH_ERR_ARG, "null event");
    if (ev->cfg.nz != 1 || k_gamma < 1.0 || !(w > 0) || !(mean_spots >= 0))
        return fail(VH_ERR_ARG, "hotspot events are 2+1D, with k_gamma >= 1 and w > 0");
    std::vector<double> cx, cy, amp;
    vh::draw_hotspots(seed, mean_spots, k_gamma, amp_mean_GeV, R, a, cx, cy, amp);
    const size_t N = (size_t)ev->N, ns = cx.size();
    if (3 * ns > 10 * N) return fail(VH_ERR_ARG, "lattice too small for the number of hotspots drawn");
    std::vector<double> spots(3 * ns);
    for (size_t k = 0; k < ns; ++k) { spots[k] = cx[k]; spots[ns + k] = cy[k]; spots[2 * ns + k] = amp[k]; }
    double *d = ev->ic;
    if (ns) CUDA_TRY(cudaMemcpyAsync(d + 6 * N, spots.data(), 3 * ns * sizeof(double), cudaMemcpyHostToDevice, ev->stream));
    vh::HotspotArgs h;
    h.nx = ev->cfg.nx; h.ny = ev->cfg.ny; h.dx = ev->cfg.dx; h.dy = ev->cfg.dy; h.w = w;
    h.spots = d + 6 * N;
    h.nspots = (int)ns;
    h.eos = dev_eos(ev);
    h.eos_kind = ev->cfg.eos_kind;
    vh::launch_hotspot_ic(h, d, d + N, d + 2 * N, ev->stream);
    CUDA_TRY(cudaGetLastError());
    return do_init(ev, d, d + N, d + 2 * N, nullptr, nullptr);
}

int vh_event_set_initial_device(vh_event *ev, const double *d_e, const double *d_p, const double *d_u, const double *d_pi, const double *d_Pi)
{
    if (!ev || !d_e || !d_p || !d_u) return fail(VH_ERR_ARG, "null argument");
    return do_init(ev, d_e, d_p, d_u, d_pi, d_Pi);
}

static void launch_vort(vh_event *ev)
{
    vh::VortArgs a;
    a.u = ev->u[ev->uc]; a.up = ev->u[ev->up]; a.e = ev->ep[ev->ec];
    a.w = ev->vort; a.L = ev->L;
    a.nx = ev->cfg.nx; a.ny = ev->cfg.ny; a.nz = ev->cfg.nz; a.ncx = ev->ncx; a.ncy = ev->ncy;
    a.dt = ev->cfg.dt; a.dx = ev->cfg.dx; a.dy = ev->cfg.dy; a.dz = ev->cfg.dz;
    a.eos = dev_eos(ev);
    a.eos_kind = ev->cfg.eos_kind;
    vh::launch_vorticity(a, ev->stream);
}

static vh::StageMarks *next_marks(vh_event *ev)
{
    if (!ev->timing) return nullptr;
    if (ev->marks_used == ev->marks.size()) {
        vh::StageMarks m{};
        for (cudaEvent_t &e : m.ev)
            if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        ev->marks.push_back(m);
    }
    return &ev->marks[ev->marks_used++];
}

int vh_event_step(vh_event *ev, int nsteps)
{
    if (!ev || nsteps < 0) return fail(VH_ERR_ARG, "bad argument");
    if (!ev->initialised) return fail(VH_ERR_STATE, "vh_event_step before vh_event_set_initial");
    if (ev->fo_pending) return fail(VH_ERR_STATE, "vh_event_step with a freezeout block pending");
    const vh_config &c = ev->cfg;
    vh::StageArgs A = vh::stage_args_base(ev);
    const bool mixed = c.precision == VH_PREC_MIXED;
    auto launch = [&](const vh::StageArgs &a, vh::StageMarks *m) {
        if (mixed) vh::launch_stage_mixed(a, ev->nq, c.eos_kind, ev->stream, m);
        else vh::launch_stage(a, ev->nq, c.eos_kind, ev->stream, m);
    };
    for (int it = 0; it < nsteps; ++it) {
        const double t = ev->t;
        const double t1 = t + c.dt;           /* `t += dt` of rungeKutta2 */
        A.step = ev->n;
        /* stage 1: q -> qS, (e,p)[ec] -> (e,p)[1-ec], u/up -> uS */
        A.qin = ev->q[ev->qc]; A.qout = ev->q[ev->qs]; A.qbase = nullptr;
        A.ein = ev->ep[ev->ec]; A.pin = ev->ep[ev->ec] + ev->L;
        A.eout = ev->ep[1 - ev->ec]; A.pout = ev->ep[1 - ev->ec] + ev->L;
        A.uin = ev->u[ev->uc]; A.upin = ev->u[ev->up]; A.uout = ev->u[ev->us];
        A.t = t; A.t2pow = pow(t, 2); A.t_inf = t1; A.inv_t = 1.0 / t;
        launch(A, next_marks(ev));
        /* stage 2: qS -> Q, convex with q; u(new) goes to the old up buffer */
        A.qin = ev->q[ev->qs]; A.qout = ev->q[ev->qn]; A.qbase = ev->q[ev->qc];
        A.ein = ev->ep[1 - ev->ec]; A.pin = ev->ep[1 - ev->ec] + ev->L;
        A.eout = ev->ep[ev->ec]; A.pout = ev->ep[ev->ec] + ev->L;
        A.uin = ev->u[ev->us]; A.upin = ev->u[ev->uc]; A.uout = ev->u[ev->up];
        A.t = t1; A.t2pow = pow(t1, 2); A.t_inf = t1; A.inv_t = 1.0 / t1;
        launch(A, next_marks(ev));
        std::swap(ev->qc, ev->qn);
        std::swap(ev->uc, ev->up);
        if (ev->vort_on) launch_vort(ev);        /* HydroPlugin.cpp:302-305 */
        ev->n += 1;
        ev->t = c.t0 + ev->n * c.dt;
    }
    CUDA_TRY(cudaGetLastError());
    return VH_OK;
}

int vh_event_status(vh_event *ev, int *err_step, long long *err_cell)
{
    if (!ev) return fail(VH_ERR_ARG, "null event");
    CUDA_TRY(cudaStreamSynchronize(ev->stream));
    int h[2];
    long long cell;
    CUDA_TRY(cudaMemcpy(h, ev->err, sizeof(h), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(&cell, ev->err_cell, sizeof(cell), cudaMemcpyDeviceToHost));
    if (err_step) *err_step = h[1];
    if (err_cell) *err_cell = cell;
    if (h[0] != 0) {
        char buf[160];
        std::snprintf(buf, sizeof buf, "device error %d at step %d, cell %lld", h[0], h[1], cell);
        return fail(h[0], buf);
    }
    return VH_OK;
}

int vh_event_progress(vh_event *ev, int *steps_done, double *t)
{
    if (!ev) return fail(VH_ERR_ARG, "null event");
    if (steps_done) *steps_done = ev->n;
    if (t) *t = ev->t;
    return VH_OK;
}

static const double *field_ptr(const vh_event *ev, int field)
{
    if (field >= 0 && field < ev->nq) return ev->q[ev->qc] + (long long)field * ev->L;
    if (field >= VH_F_UT && field < VH_F_UT + 4) return ev->u[ev->uc] + (long long)(field - VH_F_UT) * ev->L;
    if (field >= VH_F_UPT && field < VH_F_UPT + 4) return ev->u[ev->up] + (long long)(field - VH_F_UPT) * ev->L;
    if (field == VH_F_E) return ev->ep[ev->ec];
    if (field == VH_F_P) return ev->ep[ev->ec] + ev->L;
    if (ev->vort && field >= VH_F_W && field < VH_F_W + 6) return ev->vort + (long long)(field - VH_F_W) * ev->L;
    if (ev->vort && field >= VH_F_BETA && field < VH_F_BETA + 4) return ev->vort + (long long)(6 + field - VH_F_BETA) * ev->L;
    if (ev->regfac && field >= VH_F_REGFAC && field < VH_F_REGFAC + 2) return ev->regfac + (long long)(field - VH_F_REGFAC) * ev->L;
    return nullptr;
}

/* A 2+1D event's state planes carry no eta ghost copies while it evolves
 * (put_with_ghosts); a read writes them first, so every read sees the
 * reference's padded layout. */
static void fill_eta_ghosts(vh_event *ev, int field, const double *plane)
{
    if (ev->cfg.nz != 1) return;
    const bool state = (field >= 0 && field < ev->nq) || (field >= VH_F_UT && field < VH_F_UT + 4) ||
                       (field >= VH_F_UPT && field < VH_F_UPT + 4) || field == VH_F_E || field == VH_F_P;
    if (state)
        vh::launch_eta_ghost_fill(const_cast<double *>(plane), ev->cfg.nx, ev->cfg.ny, ev->ncx, ev->ncy, ev->stream);
}

int vh_event_get_field(vh_event *ev, int field, double *host_out)
{
    if (!ev || !host_out) return fail(VH_ERR_ARG, "null argument");
    const double *src = field_ptr(ev, field);
    if (!src) return fail(VH_ERR_ARG, "unknown field id");
    fill_eta_ghosts(ev, field, src);
    size_t len = (size_t)ev->ncx * ev->ncy * ev->ncz;
    CUDA_TRY(cudaMemcpyAsync(host_out, src, len * sizeof(double), cudaMemcpyDeviceToHost, ev->stream));
    CUDA_TRY(cudaStreamSynchronize(ev->stream));
    return VH_OK;
}

int vh_event_device_field(vh_event *ev, int field, double **d_ptr)
{
    if (!ev || !d_ptr) return fail(VH_ERR_ARG, "null argument");
    const double *src = field_ptr(ev, field);
    if (!src) return fail(VH_ERR_ARG, "unknown field id");
    fill_eta_ghosts(ev, field, src);
    CUDA_TRY(cudaGetLastError());
    *d_ptr = const_cast<double *>(src);
    return VH_OK;
}

int vh_event_set_sources(vh_event *ev, const double *st, const double *sx, const double *sy, const double *sn)
{
    if (!ev) return fail(VH_ERR_ARG, "null event");
    if (!st) { ev->src_on = false; return VH_OK; }
    if (!sx || !sy || !sn) return fail(VH_ERR_ARG, "all four source components are needed");
    const size_t N = (size_t)ev->N, B = N * sizeof(double);
    if (!ev->src) {
        const size_t P = (size_t)4 * ev->L * sizeof(double);
        CUDA_TRY(ev_alloc(ev, &ev->src, P));
        CUDA_TRY(cudaMemsetAsync(ev->src, 0, P, ev->stream));
    }
    /* through the initial-condition staging planes (free between initial states) */
    double *d = ev->ic;
    CUDA_TRY(cudaMemcpyAsync(d, st, B, cudaMemcpyHostToDevice, ev->stream));
    CUDA_TRY(cudaMemcpyAsync(d + N, sx, B, cudaMemcpyHostToDevice, ev->stream));
    CUDA_TRY(cudaMemcpyAsync(d + 2 * N, sy, B, cudaMemcpyHostToDevice, ev->stream));
    CUDA_TRY(cudaMemcpyAsync(d + 3 * N, sn, B, cudaMemcpyHostToDevice, ev->stream));
    vh::launch_scatter_interior(d, ev->src, 4, ev->L, ev->cfg.nx, ev->cfg.ny, ev->cfg.nz, ev->ncx, ev->ncy, ev->stream);
    CUDA_TRY(cudaGetLastError());
    ev->src_on = true;
    return VH_OK;
}

int vh_event_keep_regulation(vh_event *ev, int enable)
{
    if (!ev) return fail(VH_ERR_ARG, "null event");
    ev->regfac_on = enable != 0;
    if (ev->regfac_on && !ev->regfac) {
        const size_t P = (size_t)2 * ev->L * sizeof(double);
        CUDA_TRY(ev_alloc(ev, &ev->regfac, P));
        CUDA_TRY(cudaMemsetAsync(ev->regfac, 0, P, ev->stream));   /* as calloc'd before the first step */
    }
    return VH_OK;
}

int vh_event_vorticity(vh_event *ev, int enable)
{
    if (!ev) return fail(VH_ERR_ARG, "null event");
    if (!ev->initialised) return fail(VH_ERR_STATE, "vh_event_vorticity before vh_event_set_initial");
    ev->vort_on = enable != 0;
    if (!ev->vort_on) return VH_OK;
    if (!ev->vort) {
        const size_t B = (size_t)10 * ev->L * sizeof(double);
        CUDA_TRY(ev_alloc(ev, &ev->vort, B));
        CUDA_TRY(cudaMemsetAsync(ev->vort, 0, B, ev->stream));
    }
    launch_vort(ev);                              /* HydroPlugin.cpp:197-199 */
    CUDA_TRY(cudaGetLastError());
    return VH_OK;
}

int vh_event_phase_timing(vh_event *ev, int enable)
{
    if (!ev) return fail(VH_ERR_ARG, "null event");
    ev->timing = enable != 0;
    ev->marks_used = 0;
    return VH_OK;
}

int vh_event_phase_times(vh_event *ev, double *ms, long long *launches)
{
    if (!ev || !ms || !launches) return fail(VH_ERR_ARG, "null argument");
    CUDA_TRY(cudaStreamSynchronize(ev->stream));
    for (int p = 0; p < VH_NPHASES; ++p) { ms[p] = 0; launches[p] = 0; }
    for (size_t i = 0; i < ev->marks_used; ++i) {
        const vh::StageMarks &m = ev->marks[i];
        for (int n = 0; n < m.n; ++n) {
            float t = 0;
            CUDA_TRY(cudaEventElapsedTime(&t, m.ev[n], m.ev[n + 1]));
            ms[m.phase[n]] += t;
            launches[m.phase[n]] += 1;
        }
    }
    ev->marks_used = 0;
    return VH_OK;
}

int vh_event_kernel_launches(vh_event *ev, int *per_step)
{
    if (!ev || !per_step) return fail(VH_ERR_ARG, "null argument");
    *per_step = 2 * vh::stage_launches(ev->cfg.nx, ev->cfg.ny, ev->cfg.nz);
    return VH_OK;
}

int vh_event_stream(vh_event *ev, void **stream)
{
    if (!ev || !stream) return fail(VH_ERR_ARG, "null argument");
    *stream = (void *)ev->stream;
    return VH_OK;
}

int vh_event_energy_of_T(vh_event *ev, double T, double *e_out)
{
    if (!ev || !e_out) return fail(VH_ERR_ARG, "null argument");
    *e_out = ev->heos.energy_of_T(T);
    return VH_OK;
}

/* powf calibration diagnostics: inputs seen outside the calibrated range */
int vh_event_powf_misses(vh_event *ev, unsigned long long *misses)
{
    if (!ev || !misses) return fail(VH_ERR_ARG, "null argument");
    CUDA_TRY(cudaMemcpy(misses, ev->powf_miss, sizeof(*misses), cudaMemcpyDeviceToHost));
    return VH_OK;
}

/* ------------------------------------------------------------ freezeout */
static void fo_args(vh_event *ev, vh::FoArgs &a)
{
    const vh_config &c = ev->cfg;
    const size_t N = (size_t)ev->N;
    a.q = ev->q[ev->qc]; a.e = ev->ep[ev->ec]; a.u = ev->u[ev->uc];
    a.L = ev->L; a.nx = c.nx; a.ny = c.ny; a.nz = c.nz; a.ncx = ev->ncx; a.ncy = ev->ncy; a.nq = ev->nq;
    a.slab_prev = ev->fo_slabs + (size_t)ev->fo_prev * 11 * N;
    a.slab_cur = ev->fo_slabs + (size_t)(1 - ev->fo_prev) * 11 * N;
    a.eF = ev->e_fo;
    a.dtau_c = c.dt * c.fo_factor; a.dx = c.dx; a.dy = c.dy; a.dz = c.dz;
    a.t0 = c.t0; a.dt = c.dt; a.t = ev->t; a.n = ev->n + 1;
    a.eos = dev_eos(ev);
    a.err.code = ev->err; a.err.step = ev->err + 1; a.err.cell = ev->err_cell;
    /* scratch: [counts: ncubes+1][block sums][n_above][n_total] */
    a.counts = ev->fo_scratch;
    a.block_sums = nullptr;
    a.n_above = nullptr;
    a.n_total = nullptr;
    a.elems = ev->fo_elems;
    a.cap = ev->fo_cap;
    a.slots = ev->fo_slots;
    a.slot_cap = ev->fo_slot_cap;
}

int vh_event_freezeout_launch(vh_event *ev)
{
    if (!ev) return fail(VH_ERR_ARG, "null event");
    if (!ev->initialised) return fail(VH_ERR_STATE, "freezeout before vh_event_set_initial");
    if (ev->fo_pending) return fail(VH_ERR_STATE, "a freezeout block is already pending");
    const vh_config &c = ev->cfg;
    const size_t N = (size_t)ev->N;
    if (!ev->fo_slabs) {
        CUDA_TRY(ev_alloc(ev, &ev->fo_slabs, 2 * 11 * N * sizeof(double)));
        CUDA_TRY(cudaMemsetAsync(ev->fo_slabs, 0, 2 * 11 * N * sizeof(double), ev->stream));
        ev->fo_scratch_ints = vh::freezeout_scratch_ints(c.nx, c.ny, c.nz);
        CUDA_TRY(ev_alloc(ev, &ev->fo_scratch, ev->fo_scratch_ints * sizeof(int)));
        CUDA_TRY(cudaMallocHost(&ev->fo_hdr, 2 * sizeof(int)));
        CUDA_TRY(cudaEventCreateWithFlags(&ev->fo_done, cudaEventDisableTiming));
        /* a first element buffer sized for a surface crossing the lattice
         * (twice its cross sections in 3+1D, eight times its edges in 2+1D),
         * so that blocks seldom overflow it; VH_FO_INITIAL_CAP overrides the
         * size (tests of the overflow path) */
        if (!ev->fo_elems) {
            const long long nx = c.nx, ny = c.ny, nz = c.nz;
            long long cap = (nz > 1 ? 2 * (nx * ny + ny * nz + nx * nz) : 8 * (nx + ny)) + 1024;
            if (const char *env = getenv("VH_FO_INITIAL_CAP")) cap = std::max(1LL, atoll(env));
            ev->fo_cap = (int)std::min<long long>(cap, 1LL << 28);
            CUDA_TRY(ev_alloc(ev, &ev->fo_elems, (size_t)ev->fo_cap * VH_FO_COLUMNS * sizeof(double)));
            /* element slots for as many crossed cubes as the first buffer has
             * elements (a cube beyond them runs Cornelius again in the emit step) */
            ev->fo_slot_cap = ev->fo_cap;
            CUDA_TRY(ev_alloc(ev, &ev->fo_slots, (size_t)ev->fo_slot_cap * vh::kFoSlotDoubles * sizeof(double)));
        }
    }
    vh::FoArgs a;
    fo_args(ev, a);
    vh::launch_freezeout(a, ev->stream);
    CUDA_TRY(cudaGetLastError());
    /* header words 1 and 2: cells above e_F, elements */
    CUDA_TRY(cudaMemcpyAsync(ev->fo_hdr, ev->fo_scratch + ev->fo_scratch_ints - vh::kFoHeaderInts + 1, 2 * sizeof(int),
                             cudaMemcpyDeviceToHost, ev->stream));
    CUDA_TRY(cudaEventRecord(ev->fo_done, ev->stream));
    ev->fo_pending = true;
    return VH_OK;
}

int vh_event_freezeout_finish(vh_event *ev, int *n_elements, int *n_above)
{
    if (!ev) return fail(VH_ERR_ARG, "null event");
    if (!ev->fo_pending) return fail(VH_ERR_STATE, "no freezeout block pending");
    ev->fo_pending = false;
    CUDA_TRY(cudaEventSynchronize(ev->fo_done));
    int above = ev->fo_hdr[0], total = ev->fo_hdr[1];
    if (total > ev->fo_cap) {
        /* not enough room: a buffer with room to grow, and the emit step
         * again from the offsets the block left in the scratch */
        ev_free(ev, ev->fo_elems);
        ev->fo_elems = nullptr;
        ev->fo_cap = total + total / 2 + 1024;
        CUDA_TRY(ev_alloc(ev, &ev->fo_elems, (size_t)ev->fo_cap * VH_FO_COLUMNS * sizeof(double)));
        vh::FoArgs a;
        fo_args(ev, a);
        vh::launch_freezeout_emit(a, ev->stream);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaStreamSynchronize(ev->stream));
    }
    ev->fo_prev = 1 - ev->fo_prev;
    ev->fo_count = total;
    if (n_elements) *n_elements = total;
    if (n_above) *n_above = above;
    return VH_OK;
}

int vh_event_freezeout(vh_event *ev, int *n_elements, int *n_above)
{
    int rc = vh_event_freezeout_launch(ev);
    if (rc != VH_OK) return rc;
    return vh_event_freezeout_finish(ev, n_elements, n_above);
}

int vh_event_fetch_surface(vh_event *ev, double *host_out, int cap_elements, int *n_elements)
{
    if (!ev) return fail(VH_ERR_ARG, "null event");
    if (n_elements) *n_elements = ev->fo_count;
    if (ev->fo_count > cap_elements) return fail(VH_ERR_CAPACITY, "surface buffer too small");
    if (ev->fo_count == 0) return VH_OK;
    if (!host_out) return fail(VH_ERR_ARG, "null output");
    CUDA_TRY(cudaMemcpyAsync(host_out, ev->fo_elems, (size_t)ev->fo_count * VH_FO_COLUMNS * sizeof(double),
                             cudaMemcpyDeviceToHost, ev->stream));
    CUDA_TRY(cudaStreamSynchronize(ev->stream));
    return VH_OK;
}

/* ------------------------------------------------- device math check */
int vh_device_math_check(int which, const double *a, const double *b, int n, double *out)
{
    if (which < 0 || which > 3 || n < 0 || !a || !out || ((which == 1 || which == 2) && !b)) return fail(VH_ERR_ARG, "bad argument");
    if (n == 0) return VH_OK;
    if (!vh_device_available()) return fail(VH_ERR_NODEVICE, "no CUDA device");
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    vh::DevPowf pw;
    vh::PowfTab pq{};
    if (which == 3) {
        int rc = device_powf(dev, &pw);
        if (rc != VH_OK) return rc;
        pq.keys = pw.keys; pq.vals = pw.vals; pq.bucket = pw.bucket; pq.hb0 = pw.hb0; pq.hb1 = pw.hb1; pq.miss = nullptr;
    }
    double *d = nullptr;
    const size_t B = (size_t)n * sizeof(double);
    CUDA_TRY(cudaMalloc(&d, 3 * B));
    cudaError_t e = cudaMemcpy(d, a, B, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && b) e = cudaMemcpy(d + n, b, B, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        vh::launch_math_check(which, d, d + n, n, d + 2 * (size_t)n, pq, 0);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d + 2 * (size_t)n, B, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(VH_ERR_CUDA, std::string("vh_device_math_check: ") + cudaGetErrorString(e));
    return VH_OK;
}

/* ------------------------------------------------- Cornelius service */
int vh_cornelius_surfaces(int dim, const double *cubes, int n_cubes, double value0, const double *dx,
                          double *elements, int cap_elements, int *counts, int *n_elements)
{
    if ((dim != 3 && dim != 4) || n_cubes < 0 || !cubes || !dx || !counts) return fail(VH_ERR_ARG, "bad argument");
    if (n_elements) *n_elements = 0;
    if (n_cubes == 0) return VH_OK;
    if (!vh_device_available()) return fail(VH_ERR_NODEVICE, "no CUDA device");
    const int per = dim == 3 ? 8 : 16;
    const size_t slot_doubles = (size_t)n_cubes * 10 * 8;
    double *d_cubes = nullptr, *d_slots = nullptr;
    int *d_counts = nullptr, *d_err = nullptr;
    cudaStream_t st = nullptr;
    int rc = VH_OK;
    std::vector<double> slots;
    std::vector<int> cnt;
#define GO(x) do { cudaError_t e__ = (x); if (e__ != cudaSuccess) { rc = fail(VH_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e__)); goto done; } } while (0)
    GO(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    GO(cudaMalloc(&d_cubes, (size_t)n_cubes * per * sizeof(double)));
    GO(cudaMalloc(&d_slots, slot_doubles * sizeof(double)));
    GO(cudaMalloc(&d_counts, (size_t)n_cubes * sizeof(int)));
    GO(cudaMalloc(&d_err, sizeof(int)));
    GO(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    GO(cudaMemcpyAsync(d_cubes, cubes, (size_t)n_cubes * per * sizeof(double), cudaMemcpyHostToDevice, st));
    vh::launch_cornelius_batch(dim, d_cubes, n_cubes, value0, dx, d_slots, d_counts, d_err, st);
    GO(cudaGetLastError());
    slots.resize(slot_doubles);
    cnt.resize(n_cubes);
    int herr;
    GO(cudaMemcpyAsync(slots.data(), d_slots, slot_doubles * sizeof(double), cudaMemcpyDeviceToHost, st));
    GO(cudaMemcpyAsync(cnt.data(), d_counts, (size_t)n_cubes * sizeof(int), cudaMemcpyDeviceToHost, st));
    GO(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    GO(cudaStreamSynchronize(st));
    if (herr) { rc = fail(VH_ERR_CORNELIUS, "Cornelius construction error"); goto done; }
    {
        int total = 0;
        for (int c = 0; c < n_cubes; ++c) {
            counts[c] = cnt[c];
            for (int k = 0; k < cnt[c]; ++k) {
                if (total < cap_elements && elements)
                    std::memcpy(elements + (size_t)total * 2 * dim, slots.data() + ((size_t)c * 10 + k) * 8, 2 * dim * sizeof(double));
                total++;
            }
        }
        if (n_elements) *n_elements = total;
        if (total > cap_elements) rc = fail(VH_ERR_CAPACITY, "element buffer too small");
    }
#undef GO
done:
    cudaFree(d_cubes); cudaFree(d_slots); cudaFree(d_counts); cudaFree(d_err);
    if (st) cudaStreamDestroy(st);
    return rc;
}

} /* extern "C" */

/*
 * vh_server.cpp -- an event server over the C ABI (no counterpart in the
 * reference, which evolves one event per process, HydroPlugin.cpp:226-307).
 *
 * Callers submit events (configuration + host initial condition) at any time;
 * one worker thread owns the GPU and runs rounds:
 *
 *   admit   queued events while their estimated device footprint fits the
 *           memory budget (a fraction of the free HBM when the server
 *           started); each becomes a vh_event with its state on the device
 *           until it is done;
 *   step    the active events advanced concurrently: events below
 *           solo_cells interior cells in one vh_batch per kind (precision,
 *           bulk, EoS; rebuilt when its members change, launch configuration
 *           tuned once per kind of batch and reused), larger events -- which
 *           fill the GPU on their own and run faster with the single-event
 *           kernels -- by vh_event_step on their own streams;
 *   freeze  the freezeout blocks of all events queued first, then collected,
 *           at the reference's cadence (a block before loop index n when
 *           n % coarseProperTimeFOFactor == 0, HydroPlugin.cpp:249-266); the
 *           elements of each block are copied to the event's host surface as
 *           soon as the block is done;
 *   retire  an event whose blocks found no cell above e_F three times
 *           (HydroPlugin.cpp:267-281), that reached the step cap, or whose
 *           device status reports an error, frees its device memory and is
 *           reported through vh_server_poll.
 *
 * Admission happens at round boundaries: a round is the steps up to the next
 * freezeout block of the members, so every member's blocks fall on its own
 * cadence.
 */
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "vh_b200.h"
#include "vh_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
    unsigned long long tag = 0;
    vh_config cfg{};
    std::vector<double> e, p, u, pi, Pi;
    int ic_kind = 0;                /* 0 host arrays, 1 device Glauber, 2 device hotspots */
    double icp[8] = {0};            /* generator parameters */
    unsigned long long seed = 0;
    double t_submit = 0, t_admit = 0;
    vh_event *ev = nullptr;
    size_t bytes = 0;
    int steps = 0;
    int last_block = -1;            /* step count of the last freezeout block */
    int zero_blocks = 0;            /* blocks with no cell above e_F (accumulator2) */
    double t_done = 0;
    int status = VH_OK;
    /* VH_FO_COLUMNS per element, one chunk per freezeout block: appending a
     * block copies it once (no regrowth of one large vector) */
    std::vector<std::vector<double>> surface;
    size_t surface_doubles = 0;
    void append(const double *p, size_t n)
    {
        surface.emplace_back(p, p + n);
        surface_doubles += n;
    }
};

size_t estimate_bytes(const vh_config &c)
{
    const size_t nq = c.bulk ? 15 : 14;
    const size_t L = (((size_t)(c.nx + 4) * (c.ny + 4) * (c.nz + 4)) + 31) / 32 * 32;
    const size_t N = (size_t)c.nx * c.ny * c.nz;
    size_t b = (3 * nq + 16) * L * 8;          /* state planes */
    b += 17 * N * 8;                           /* initial-condition staging */
    b += 22 * N * 8 + 8 * N + (1 << 20);       /* freezeout slabs, scratch */
    b += (size_t)16 * (c.nx * c.ny + c.ny * c.nz + c.nx * c.nz + 64) * VH_FO_COLUMNS * 8;  /* surface buffer */
    return b + (2 << 20);
}

} // namespace

struct vh_server {
    vh_server_config cfg{};
    std::vector<double> eos_rows;
    int device = 0;
    Clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv, cv_done;
    std::deque<std::unique_ptr<Job>> queue;
    std::vector<std::unique_ptr<Job>> active;
    std::deque<std::unique_ptr<Job>> done;
    std::map<unsigned long long, std::unique_ptr<Job>> fetched;   /* done, polled, surface not yet taken */
    size_t budget = 0, used = 0;
    bool stop = false;
    int fatal = VH_OK;
    std::string fatal_msg;
    unsigned long long submitted = 0, finished = 0;
    vh_server_stats st{};
    std::map<int, vh_batch_tuning> tunings;    /* per batch kind */
    std::thread worker;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

/* events a vh_batch may hold together (vh_batch_create's requirement) */
int group_key(const vh_config &c) { return (c.bulk ? 1 : 0) + 2 * c.eos_kind + 4 * c.precision; }

/* the tuning cache key: the group and whether its members are 2+1D, 3+1D or both */
int batch_kind(const std::vector<Job *> &members)
{
    bool any3 = false, any2 = false;
    for (Job *j : members) (j->cfg.nz > 1 ? any3 : any2) = true;
    const int z = any3 && any2 ? 2 : (any3 ? 1 : 0);
    return z + 3 * group_key(members.front()->cfg);
}

bool is_solo(const vh_server_config &sc, const vh_config &c)
{
    return sc.solo_cells > 0 && (long long)c.nx * c.ny * c.nz >= sc.solo_cells;
}

struct Group {
    vh_batch *batch = nullptr;
    std::vector<vh_event *> members;      /* the batch's events, in order */
};

/* steps until the next freezeout block of member j (the block happens
 * before loop index n = steps + 1 when n % fac == 0) */
int steps_to_block(const Job &j)
{
    const int fac = std::max(1, j.cfg.fo_factor);
    int k = (j.last_block == j.steps) ? 1 : 0;
    while ((j.steps + k + 1) % fac != 0) ++k;
    return k;
}

void finish_job(vh_server *S, std::unique_ptr<Job> &j, int status)
{
    j->status = status;
    j->t_done = S->now();
    if (j->ev) vh_event_destroy(j->ev);
    j->ev = nullptr;
    std::lock_guard<std::mutex> lk(S->mu);
    S->used -= j->bytes;
    S->st.done += 1;
    S->st.active -= 1;
    S->done.push_back(std::move(j));
    S->finished += 1;
    S->cv_done.notify_all();
}

void worker_main(vh_server *S)
{
    cudaSetDevice(S->device);
    std::map<int, Group> groups;    /* batches by group_key */
    int held_rounds = 0;        /* rounds an admission waited for alignment */
    auto tick = [] { return Clock::now(); };
    auto add = [&](double &acc, Clock::time_point a) {
        const double d = std::chrono::duration<double>(Clock::now() - a).count();
        std::lock_guard<std::mutex> lk(S->mu);
        acc += d;
        return d;
    };
    /* Surfaces come to host memory in two moves: at the block, a device copy
     * into a pinned staging buffer (a pageable destination halves the copy
     * rate); in the next round, while the GPU runs its steps, the append to
     * the event's surface (the host copy and the first touch of its pages
     * cost as much as the device copy).  Staging buffers are reused. */
    struct Staging { double *buf = nullptr; size_t cap = 0; };
    struct Pending { Job *j; Staging s; size_t n; };
    std::vector<Staging> pool;
    std::vector<Pending> pending;
    auto take_staging = [&](size_t need) {
        int best = -1;
        for (int i = 0; i < (int)pool.size(); ++i)
            if (pool[i].cap >= need && (best < 0 || pool[i].cap < pool[best].cap)) best = i;
        Staging st;
        if (best >= 0) {
            st = pool[best];
            pool.erase(pool.begin() + best);
            return st;
        }
        const size_t cap = std::max(need, (size_t)1 << 15);
        if (cudaMallocHost(&st.buf, cap * sizeof(double)) == cudaSuccess) st.cap = cap;
        else st.buf = nullptr;
        return st;
    };
    /* append the staged blocks (of one event, or of all) to their surfaces */
    auto flush = [&](const Job *only) {
        if (pending.empty()) return 0.0;
        const auto t = tick();
        std::vector<Pending> keep;
        for (auto &c : pending) {
            if (only && c.j != only) { keep.push_back(c); continue; }
            c.j->append(c.s.buf, c.n);
            pool.push_back(c.s);
        }
        pending.swap(keep);
        return add(S->st.t_fo_copy_s, t);
    };
    bool waiting = false;       /* events queued after this round's admission */
    auto set_fatal = [&](int rc, const char *where) {
        std::lock_guard<std::mutex> lk(S->mu);
        S->fatal = rc;
        S->fatal_msg = std::string(where) + ": " + vh_last_error();
        S->cv_done.notify_all();
    };
    while (true) {
        /* ---- admit */
        std::vector<std::unique_ptr<Job>> admitted;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            const auto t_w = tick();
            S->cv.wait(lk, [&] { return S->stop || !S->queue.empty() || !S->active.empty(); });
            S->st.t_wait_s += std::chrono::duration<double>(Clock::now() - t_w).count();
            if (S->stop) break;
            /* admit where every member is fo_factor - 1 steps before its next
             * block, as a new event is: all blocks then fall in one round
             * (after two blocked rounds admit anyway: cadences may differ) */
            bool aligned = true;
            for (auto &j : S->active) aligned &= steps_to_block(*j) == std::max(1, j->cfg.fo_factor) - 1;
            const bool admit = aligned || S->queue.empty() || ++held_rounds >= 3;
            if (admit) held_rounds = 0;
            while (admit && !S->queue.empty()) {
                Job &j = *S->queue.front();
                const size_t need = estimate_bytes(j.cfg);
                if (S->used + need > S->budget && !(S->active.empty() && admitted.empty())) break;
                if ((int)(S->active.size() + admitted.size()) >= S->cfg.max_events) break;
                S->used += need;
                j.bytes = need;
                admitted.push_back(std::move(S->queue.front()));
                S->queue.pop_front();
                S->st.queued -= 1;
                S->st.active += 1;
            }
            S->st.bytes_in_use = S->used;
            waiting = !S->queue.empty();
        }
        const auto t_adm = tick();
        for (auto &j : admitted) {
            int rc = vh_event_create(&j->cfg, S->eos_rows.empty() ? nullptr : S->eos_rows.data(),
                                     (int)S->eos_rows.size() / 4, &j->ev);
            if (rc == VH_OK) {
                if (j->ic_kind == 1)
                    rc = vh_event_init_glauber(j->ev, j->icp[0], j->icp[1], j->icp[2], j->icp[3], j->icp[4], j->icp[5],
                                               j->icp[6]);
                else if (j->ic_kind == 2)
                    rc = vh_event_init_hotspots(j->ev, j->seed, j->icp[0], j->icp[1], j->icp[2], j->icp[3], j->icp[4],
                                                j->icp[5]);
                else
                    rc = vh_event_set_initial(j->ev, j->e.data(), j->p.data(), j->u.data(),
                                              j->pi.empty() ? nullptr : j->pi.data(), j->Pi.empty() ? nullptr : j->Pi.data());
            }
            j->t_admit = S->now();
            std::vector<double>().swap(j->e);
            std::vector<double>().swap(j->p);
            std::vector<double>().swap(j->u);
            std::vector<double>().swap(j->pi);
            std::vector<double>().swap(j->Pi);
            if (rc != VH_OK) { finish_job(S, j, rc); continue; }
            S->active.push_back(std::move(j));
        }
        if (!admitted.empty()) add(S->st.t_admit_s, t_adm);
        if (S->active.empty()) continue;

        /* ---- batches of the small events, one per kind (rebuilt when their
         * members changed), and the solo events */
        const auto t_bld = tick();
        std::map<int, std::vector<Job *>> want;
        std::vector<Job *> solo;
        for (auto &j : S->active) {
            if (is_solo(S->cfg, j->cfg)) solo.push_back(j.get());
            else want[group_key(j->cfg)].push_back(j.get());
        }
        for (auto it = groups.begin(); it != groups.end();) {
            if (want.count(it->first)) { ++it; continue; }
            vh_batch_destroy(it->second.batch);
            it = groups.erase(it);
        }
        int brc = VH_OK;
        const char *bwhere = "";
        bool built = false;
        for (auto &kv : want) {
            std::vector<vh_event *> evs;
            for (Job *j : kv.second) evs.push_back(j->ev);
            Group &g = groups[kv.first];
            if (g.batch && g.members == evs) continue;
            if (g.batch) vh_batch_destroy(g.batch);
            g.batch = nullptr;
            g.members = evs;
            built = true;
            if ((brc = vh_batch_create(evs.data(), (int)evs.size(), &g.batch)) != VH_OK) { bwhere = "vh_batch_create"; break; }
            const int kind = batch_kind(kv.second);
            auto it = S->tunings.find(kind);
            if (it != S->tunings.end()) brc = vh_batch_set_tuning(g.batch, &it->second);
            else {
                vh_batch_tuning t;
                brc = vh_batch_autotune(g.batch, &t);
                if (brc == VH_OK) S->tunings[kind] = t;
            }
            if (brc != VH_OK) { bwhere = "batch tuning"; break; }
            std::lock_guard<std::mutex> lk(S->mu);
            S->st.batch_builds += 1;
        }
        if (brc != VH_OK) { set_fatal(brc, bwhere); break; }
        if (built) add(S->st.t_build_s, t_bld);

        /* ---- steps up to the earliest freezeout block (0: a block is due now) */
        int k = 1 << 30;
        for (auto &j : S->active) k = std::min(k, steps_to_block(*j));
        /* events are waiting: stop one step after a block, where they can join */
        if (waiting)
            for (auto &j : S->active)
                if (j->last_block == j->steps) k = std::min(k, 1);
        if (S->cfg.max_steps > 0)
            for (auto &j : S->active) k = std::min(k, std::max(0, S->cfg.max_steps - j->steps));
        if (k > 0) {
            /* everything is queued before anything is waited for: the solo
             * events and the batches run concurrently on their streams */
            const auto t_st = tick();
            for (Job *j : solo)
                if (j->status == VH_OK) j->status = vh_event_step(j->ev, k);
            int rc = VH_OK;
            for (auto &kv : groups)
                if ((rc = vh_batch_step(kv.second.batch, k)) != VH_OK) break;
            if (rc != VH_OK) { set_fatal(rc, "vh_batch_step"); break; }
            const double copy_s = flush(nullptr);
            for (auto &kv : groups) {
                void *bs = nullptr;
                vh_batch_stream(kv.second.batch, &bs);
                cudaStreamSynchronize((cudaStream_t)bs);
            }
            for (Job *j : solo) {
                void *es = nullptr;
                vh_event_stream(j->ev, &es);
                cudaStreamSynchronize((cudaStream_t)es);
            }
            {
                const double d = std::chrono::duration<double>(Clock::now() - t_st).count() - copy_s;
                std::lock_guard<std::mutex> lk(S->mu);
                S->st.t_step_s += d;
            }
            for (auto &j : S->active) j->steps += k;
            std::lock_guard<std::mutex> lk(S->mu);
            S->st.steps += k;
        } else {
            flush(nullptr);
        }

        /* ---- freezeout blocks that are due: queue all, then collect */
        std::vector<Job *> due;
        for (auto &j : S->active)
            if (steps_to_block(*j) == 0) due.push_back(j.get());
        const auto t_fo = tick();
        for (Job *j : due) {
            int rc = vh_event_freezeout_launch(j->ev);
            if (rc != VH_OK) j->status = rc;
        }
        for (Job *j : due) {
            if (j->status != VH_OK) continue;
            j->last_block = j->steps;
            int nel = 0, nab = 0;
            int rc = vh_event_freezeout_finish(j->ev, &nel, &nab);
            if (rc == VH_OK && nel > 0) {
                const auto t_cp = tick();
                const size_t need = (size_t)nel * VH_FO_COLUMNS;
                Staging st = take_staging(need);
                if (st.buf) {
                    rc = vh_event_fetch_surface(j->ev, st.buf, nel, &nel);
                    if (rc == VH_OK) pending.push_back({j, st, need});
                    else pool.push_back(st);
                } else {                                 /* no pinned memory: straight to the surface */
                    std::vector<double> blk(need);
                    rc = vh_event_fetch_surface(j->ev, blk.data(), nel, &nel);
                    if (rc == VH_OK) { j->surface_doubles += need; j->surface.push_back(std::move(blk)); }
                }
                add(S->st.t_fo_copy_s, t_cp);
                std::lock_guard<std::mutex> lk(S->mu);
                S->st.fo_elements += nel;
            }
            if (rc == VH_OK) rc = vh_event_status(j->ev, nullptr, nullptr);
            if (rc != VH_OK) { j->status = rc; continue; }
            if (nab == 0) j->zero_blocks += 1;
        }
        if (!due.empty()) {
            add(S->st.t_fo_s, t_fo);
            std::lock_guard<std::mutex> lk(S->mu);
            S->st.fo_blocks += (long long)due.size();
        }

        /* ---- retire (a batch goes before the events it holds) */
        std::vector<std::unique_ptr<Job>> keep, retire;
        for (auto &j : S->active) {
            const bool capped = S->cfg.max_steps > 0 && j->steps >= S->cfg.max_steps;
            if (j->status != VH_OK || j->zero_blocks >= 3 || capped) retire.push_back(std::move(j));
            else keep.push_back(std::move(j));
        }
        const auto t_ret = tick();
        for (auto &j : retire) {
            auto it = groups.find(group_key(j->cfg));
            if (it != groups.end() &&
                std::find(it->second.members.begin(), it->second.members.end(), j->ev) != it->second.members.end()) {
                vh_batch_destroy(it->second.batch);
                groups.erase(it);
            }
        }
        for (auto &j : retire) {
            flush(j.get());
            finish_job(S, j, j->status);
        }
        if (!retire.empty()) add(S->st.t_retire_s, t_ret);
        S->active.swap(keep);
    }
    for (auto &kv : groups) vh_batch_destroy(kv.second.batch);
    for (auto &c : pending) pool.push_back(c.s);
    for (auto &b : pool) cudaFreeHost(b.buf);
    for (auto &j : S->active)
        if (j->ev) vh_event_destroy(j->ev);
}

} // namespace

extern "C" {

void vh_server_config_default(vh_server_config *c)
{
    if (!c) return;
    std::memset(c, 0, sizeof *c);
    c->hbm_fraction = 0.8;
    c->max_events = 4096;
    c->max_steps = 0;
    c->solo_cells = 1 << 17;
}

int vh_server_create(const vh_server_config *cfg, const double *eos_rows, int eos_nrows, vh_server **out)
{
    if (!out) return vh::set_error(VH_ERR_ARG, "null argument");
    *out = nullptr;
    if (!vh_device_available()) return vh::set_error(VH_ERR_NODEVICE, "no CUDA device");
    vh_server_config c;
    vh_server_config_default(&c);
    if (cfg) c = *cfg;
    if (!(c.hbm_fraction > 0 && c.hbm_fraction <= 1) || c.max_events < 1 || c.max_steps < 0 || c.solo_cells < 0)
        return vh::set_error(VH_ERR_ARG, "bad server configuration");
    auto *S = new vh_server;
    S->cfg = c;
    if (eos_rows && eos_nrows > 0) S->eos_rows.assign(eos_rows, eos_rows + 4 * (size_t)eos_nrows);
    cudaGetDevice(&S->device);
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) { delete S; return vh::set_error(VH_ERR_CUDA, "cudaMemGetInfo"); }
    S->budget = (size_t)(c.hbm_fraction * (double)fr);
    S->st.budget_bytes = S->budget;
    S->t0 = Clock::now();
    vh::event_pool_hold(S->device, 1);      /* keep event memory through idle gaps */
    S->worker = std::thread(worker_main, S);
    *out = S;
    return VH_OK;
}

static int enqueue(vh_server *S, std::unique_ptr<Job> j)
{
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->fatal != VH_OK) return vh::set_error(S->fatal, S->fatal_msg);
    j->t_submit = S->now();
    S->queue.push_back(std::move(j));
    S->submitted += 1;
    S->st.submitted += 1;
    S->st.queued += 1;
    S->cv.notify_all();
    return VH_OK;
}

static int check_submit(vh_server *S, const vh_config *cfg)
{
    if (!S || !cfg) return vh::set_error(VH_ERR_ARG, "null argument");
    if (cfg->eos_kind == VH_EOS_TABLE && S->eos_rows.empty())
        return vh::set_error(VH_ERR_ARG, "tabulated-EoS event on a server created without EoS rows");
    return VH_OK;
}

int vh_server_submit(vh_server *S, const vh_config *cfg, const double *e, const double *p, const double *u,
                     const double *pi, const double *Pi, unsigned long long tag)
{
    if (!e || !p || !u) return vh::set_error(VH_ERR_ARG, "null argument");
    int rc = check_submit(S, cfg);
    if (rc != VH_OK) return rc;
    auto j = std::make_unique<Job>();
    j->tag = tag;
    j->cfg = *cfg;
    const size_t N = (size_t)cfg->nx * cfg->ny * cfg->nz;
    j->e.assign(e, e + N);
    j->p.assign(p, p + N);
    j->u.assign(u, u + 4 * N);
    if (pi) j->pi.assign(pi, pi + 10 * N);
    if (Pi) j->Pi.assign(Pi, Pi + N);
    return enqueue(S, std::move(j));
}

int vh_server_submit_glauber(vh_server *S, const vh_config *cfg, double R, double a, double sigma_nn, double b,
                             double e0_GeV, double eta_flat, double eta_sigma, unsigned long long tag)
{
    int rc = check_submit(S, cfg);
    if (rc != VH_OK) return rc;
    auto j = std::make_unique<Job>();
    j->tag = tag;
    j->cfg = *cfg;
    j->ic_kind = 1;
    const double v[7] = {R, a, sigma_nn, b, e0_GeV, eta_flat, eta_sigma};
    std::copy(v, v + 7, j->icp);
    return enqueue(S, std::move(j));
}

int vh_server_submit_hotspots(vh_server *S, const vh_config *cfg, unsigned long long seed, double mean_spots, double w,
                              double k_gamma, double amp_mean_GeV, double R, double a, unsigned long long tag)
{
    int rc = check_submit(S, cfg);
    if (rc != VH_OK) return rc;
    if (cfg->nz != 1) return vh::set_error(VH_ERR_ARG, "hotspot events are 2+1D");
    auto j = std::make_unique<Job>();
    j->tag = tag;
    j->cfg = *cfg;
    j->ic_kind = 2;
    j->seed = seed;
    const double v[6] = {mean_spots, w, k_gamma, amp_mean_GeV, R, a};
    std::copy(v, v + 6, j->icp);
    return enqueue(S, std::move(j));
}

int vh_server_poll(vh_server *S, vh_server_done *out, int max, int *n)
{
    if (!S || !n || (max > 0 && !out)) return vh::set_error(VH_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    int k = 0;
    while (k < max && !S->done.empty()) {
        auto j = std::move(S->done.front());
        S->done.pop_front();
        vh_server_done &d = out[k++];
        d.tag = j->tag;
        d.status = j->status;
        d.steps = j->steps;
        d.n_elements = (long long)(j->surface_doubles / VH_FO_COLUMNS);
        d.t_submit = j->t_submit;
        d.t_admit = j->t_admit;
        d.t_done = j->t_done;
        S->fetched[j->tag] = std::move(j);
    }
    *n = k;
    if (S->fatal != VH_OK) return vh::set_error(S->fatal, S->fatal_msg);
    return VH_OK;
}

int vh_server_take_surface(vh_server *S, unsigned long long tag, double *out, long long cap_elements, long long *n)
{
    if (!S || !n) return vh::set_error(VH_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->fetched.find(tag);
    if (it == S->fetched.end()) return vh::set_error(VH_ERR_ARG, "no polled event with this tag");
    const Job &j = *it->second;
    const long long m = (long long)(j.surface_doubles / VH_FO_COLUMNS);
    *n = m;
    if (m > cap_elements) return vh::set_error(VH_ERR_CAPACITY, "surface buffer too small");
    if (m > 0) {
        if (!out) return vh::set_error(VH_ERR_ARG, "null output");
        for (const auto &blk : j.surface) {
            std::memcpy(out, blk.data(), blk.size() * sizeof(double));
            out += blk.size();
        }
    }
    S->fetched.erase(it);
    return VH_OK;
}

int vh_server_wait(vh_server *S, double timeout_s)
{
    if (!S) return vh::set_error(VH_ERR_ARG, "null server");
    std::unique_lock<std::mutex> lk(S->mu);
    bool ok = S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                  [&] { return S->finished == S->submitted || S->fatal != VH_OK; });
    if (S->fatal != VH_OK) return vh::set_error(S->fatal, S->fatal_msg);
    return ok ? VH_OK : vh::set_error(VH_ERR_STATE, "timed out waiting for submitted events");
}

int vh_server_stats_get(vh_server *S, vh_server_stats *out)
{
    if (!S || !out) return vh::set_error(VH_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->st;
    out->bytes_in_use = S->used;
    return VH_OK;
}

int vh_server_destroy(vh_server *S)
{
    if (!S) return VH_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        S->cv.notify_all();
    }
    if (S->worker.joinable()) S->worker.join();
    vh::event_pool_hold(S->device, -1);
    delete S;
    return VH_OK;
}

} /* extern "C" */

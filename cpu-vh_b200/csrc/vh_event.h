/*
 * vh_event.h -- the event object behind the C ABI handle (internal).
 *
 * An event owns one device allocation holding every plane of its state:
 *   q[3]  : NQ planes each -- current q, next Q, stage qS
 *           (the reference's q, Q, qS, DynamicalVariables.cpp:21)
 *   ep[2] : (e, p) twice -- read by one stage, written by the other
 *   u[3]  : 4 planes each -- u, up, uS (DynamicalVariables.cpp:23)
 * Buffer roles rotate by index on the host, exactly as the reference swaps
 * pointers (setCurrentConservedVariables, swapFluidVelocity): after n steps
 * qc = uc = n mod 2, qs = us = 2 and ec = 0.
 */
#ifndef VH_EVENT_H
#define VH_EVENT_H

#include <cuda_runtime.h>
#include <cmath>
#include <cstdlib>
#include <vector>
#include "vh_b200.h"
#include "vh_internal.h"
#include "vh_kernels.h"

namespace vh {

/* host-exact powf table, uploaded once per device */
struct DevPowf {
    unsigned *keys = nullptr;
    float *vals = nullptr;
    unsigned *bucket = nullptr;
    unsigned hb0 = 0, hb1 = 0;
};

} // namespace vh

struct vh_event {
    vh_config cfg;
    int nq = 14;
    int ncx = 0, ncy = 0, ncz = 0;
    long long L = 0;          /* plane stride (padded) */
    long long N = 0;          /* interior cells */
    int device = 0;
    cudaStream_t stream = nullptr;
    double *slab = nullptr;
    double *q[3] = {nullptr, nullptr, nullptr};
    double *ep[2] = {nullptr, nullptr};   /* e plane; p plane follows at +L */
    double *u[3] = {nullptr, nullptr, nullptr};
    int qc = 0, qn = 1, qs = 2;          /* current q, next Q, stage qS */
    int ec = 0;                           /* e/p buffer holding the current state */
    int uc = 0, up = 1, us = 2;           /* u, up, uS */
    double *tables = nullptr;             /* p_tb then T_tb */
    bool pooled = false;                  /* counted in the device's event memory pool */
    int *err = nullptr;                   /* [0] code, [1] step */
    long long *err_cell = nullptr;
    unsigned long long *powf_miss = nullptr;
    double *ic = nullptr;                 /* interior staging: e, p, u(4), pi(10), Pi */
    vh::HostEos heos;
    vh::DevPowf powf;
    double e_reg = 0, e_fo = 0;
    int n = 0;
    double t = 0;
    bool initialised = false;
    /* freezeout */
    double *fo_slabs = nullptr;           /* 2 x 11 x N */
    int fo_prev = 0;                      /* which half is the previous slab */
    int *fo_scratch = nullptr;
    size_t fo_scratch_ints = 0;
    double *fo_elems = nullptr;
    int fo_cap = 0;
    double *fo_slots = nullptr;           /* element slots of the count step (vh_fo.cu) */
    int fo_slot_cap = 0;
    int fo_count = 0;
    int *fo_hdr = nullptr;                /* pinned: n_above, n_total of the last block */
    cudaEvent_t fo_done = nullptr;
    bool fo_pending = false;              /* launched, not yet finished */
    /* thermal vorticity (vh_event_vorticity): 6 w planes then 4 beta planes */
    double *vort = nullptr;
    bool vort_on = false;
    /* dynamical sources (vh_event_set_sources): 4 padded planes, ghosts 0 */
    double *src = nullptr;
    bool src_on = false;
    /* regulation factors (vh_event_keep_regulation): shear, bulk planes */
    double *regfac = nullptr;
    bool regfac_on = false;
    /* per-phase timing (vh_event_phase_timing) */
    bool timing = false;
    std::vector<vh::StageMarks> marks;    /* one per stage launched since enabling */
    size_t marks_used = 0;
};

/* an environment switch set to 0 (read on every call; tests of the forms) */
static inline bool vh_env_off(const char *name)
{
    const char *e = getenv(name);
    return e && e[0] == '0';
}

/* VH_CS2_SHORTCUT=0 makes the device evaluate the table sound speed
 * everywhere (the results are the same) */
static inline vh::DevEos dev_eos(const vh_event *ev)
{
    vh::DevEos E;
    E.kind = ev->cfg.eos_kind;
    E.a = ev->cfg.eos_factor;
    E.p_tb = ev->tables;
    E.T_tb = ev->tables ? ev->tables + ev->heos.e_length : nullptr;
    E.e_length = ev->heos.e_length;
    E.e_min = ev->heos.e_min;
    E.e_spacing = ev->heos.e_spacing;
    E.inv_spacing = 1.0 / ev->heos.e_spacing;
    E.cs2_third_hi = (ev->cfg.eos_kind == VH_EOS_TABLE && !vh_env_off("VH_CS2_SHORTCUT")) ? ev->heos.cs2_third_hi : -INFINITY;
    E.pq.keys = ev->powf.keys;
    E.pq.vals = ev->powf.vals;
    E.pq.bucket = ev->powf.bucket;
    E.pq.hb0 = ev->powf.hb0;
    E.pq.hb1 = ev->powf.hb1;
    E.pq.miss = ev->powf_miss;
    E.stop = ev->err;
    return E;
}

namespace vh {
/* the step-independent part of a stage's arguments (pointers and times unset) */
StageArgs stage_args_base(const vh_event *ev);
} // namespace vh

#endif

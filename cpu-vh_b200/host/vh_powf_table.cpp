/*
 * vh_powf_table.cpp -- calibration of the device powf(x, 0.25f) against the
 * host libm.
 *
 * The conformal EoS computes T = powf(e/a, 0.25) (EquationOfState.cpp:196).
 * glibc's powf is accurate to under one ulp but not correctly rounded, and a
 * single differing ulp in T changes the shear relaxation time and, through the
 * float truncations downstream, every later step.  The device therefore
 * evaluates the correctly rounded candidate float(sqrt(sqrt(double x))) and
 * looks the input up in a table of the inputs where the host libm returns
 * something else.  This file builds that table once per process by running the
 * host powf over every float in [2^-60, 2^12) -- the energy densities the
 * evolution can reach (the inference floors e at 1e-7 fm^-4) -- on all host
 * cores.  Outside that range the device keeps the correctly rounded value and
 * counts the input (vh_event_status reports the count through the tests).
 */
#include <cmath>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>
#include <algorithm>

#include "vh_internal.h"

namespace vh {

static const unsigned kLoBits = 67u << 23;    /* 2^-60 */
static const unsigned kHiBits = 139u << 23;   /* 2^12  */

static PowfQuarterTable g_table;
static std::once_flag g_once;

static void build_table()
{
    unsigned nthreads = std::max(1u, std::thread::hardware_concurrency());
    nthreads = std::min(nthreads, 64u);
    const unsigned total = kHiBits - kLoBits;
    std::vector<std::vector<unsigned>> keys(nthreads);
    std::vector<std::vector<float>> vals(nthreads);
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nthreads; ++t) {
        pool.emplace_back([&, t]() {
            unsigned beg = kLoBits + (unsigned)((unsigned long long)total * t / nthreads);
            unsigned end = kLoBits + (unsigned)((unsigned long long)total * (t + 1) / nthreads);
            for (unsigned b = beg; b < end; ++b) {
                float x;
                std::memcpy(&x, &b, 4);
                float g = powf(x, 0.25f);
                float c = (float)std::sqrt(std::sqrt((double)x));
                if (std::memcmp(&g, &c, 4) != 0) { keys[t].push_back(b); vals[t].push_back(g); }
            }
        });
    }
    for (auto &th : pool) th.join();
    PowfQuarterTable &T = g_table;
    std::memcpy(&T.lo, &kLoBits, 4);
    std::memcpy(&T.hi, &kHiBits, 4);
    for (unsigned t = 0; t < nthreads; ++t) {
        T.keys.insert(T.keys.end(), keys[t].begin(), keys[t].end());
        T.vals.insert(T.vals.end(), vals[t].begin(), vals[t].end());
    }
    const unsigned hb0 = kLoBits >> 16, hb1 = kHiBits >> 16;
    T.bucket.assign(hb1 - hb0 + 1, 0);
    size_t pos = 0;
    for (unsigned hb = hb0; hb <= hb1; ++hb) {
        while (pos < T.keys.size() && (T.keys[pos] >> 16) < hb) ++pos;
        T.bucket[hb - hb0] = (unsigned)pos;
    }
}

const PowfQuarterTable &powf_quarter_table()
{
    std::call_once(g_once, build_table);
    return g_table;
}

} // namespace vh

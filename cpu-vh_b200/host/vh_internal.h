/*
 * vh_internal.h -- declarations shared by the host C++ and the CUDA sources
 * of the library (not part of the public ABI).
 */
#ifndef VH_INTERNAL_H
#define VH_INTERNAL_H

#include <cstdint>
#include <string>
#include <cmath>
#include <vector>
#include "vh_b200.h"

namespace vh {

/* HydroPlugin.cpp:111, InitialConditions.cpp:1598 */
constexpr double kHbarc = 0.197326938;

/* Host copy of the reference EoS (EquationOfState.cpp:44-360), used for the
 * scalars the driver computes on the host (freezeout and regulation energy
 * densities, HydroPlugin.cpp:113 and FullyDiscreteKurganovTadmorScheme.cpp:888)
 * and for initial pressures. */
struct HostEos {
    int kind = VH_EOS_CONFORMAL;
    double a = 13.8997;
    int e_length = 0;
    double e_min = 0, e_max = 0, e_spacing = 1;
    std::vector<double> p_tb, T_tb;
    /* the table sound speed is exactly 1/3 for every e <= cs2_third_hi
     * (-inf: no such bound is known for this table); see cs2_third_bound */
    double cs2_third_hi = -INFINITY;

    void init(const vh_config &cfg, const double *rows, int nrows);
    double interp(double ed, const std::vector<double> &tb) const;
    double pressure(double ed) const;
    double cs2(double ed) const;
    double cs2_third_bound() const;
    double temperature(double ed) const;
    double energy_of_T(double T) const;
};

/* powf(x, 0.25f) exactly as the host libm computes it, for every float x in
 * [lo, hi): the correctly rounded value except at the inputs listed in the
 * exception table built by enumerating the host powf (vh_powf_table.cpp). */
struct PowfQuarterTable {
    float lo = 0, hi = 0;
    std::vector<unsigned> keys;     /* float bits of the exceptional inputs, sorted */
    std::vector<float> vals;        /* host powf result at those inputs           */
    std::vector<unsigned> bucket;   /* 65537 offsets into keys by (bits >> 16)    */
};
const PowfQuarterTable &powf_quarter_table();

/* records msg as the calling thread's vh_last_error() and returns code */
int set_error(int code, const std::string &msg);

/* the random draws of the hotspot initial condition (centres, amplitudes in fm^-4) */
void draw_hotspots(uint64_t seed, double mean_spots, double k_gamma, double amp_mean_GeV, double R, double a,
                   std::vector<double> &cx, std::vector<double> &cy, std::vector<double> &amp);

/* keep (delta +1) or release (-1) the device's event memory pool through
 * times without events (vh_capi.cu) */
void event_pool_hold(int dev, int delta);

} // namespace vh

#endif

/*
 * ref_shim.h -- TEST INFRASTRUCTURE ONLY (oracle build of the reference).
 *
 * Force-included (g++ -include) ahead of every translation unit of the
 * unmodified cpu-vh sources when oracle/ref.mk compiles them in place.  The
 * reference fixes three physics knobs with unconditional #defines inside its
 * headers, so a -D on the command line cannot override them:
 *
 *   THETA        rhic/include/FluxLimiter.h:13          (minmod theta, 1.1)
 *   EOS choice   rhic/include/EquationOfState.h:13-15   (CONFORMAL_EOS)
 *   EOS_FACTOR   rhic/include/EquationOfState.h:19      (13.8997)
 *
 * This shim defines those two headers' include guards first and supplies the
 * same declarations with the values chosen by the recipe (VH_THETA,
 * VH_EOS_FACTOR, VH_EOS_TABLE).  The EOS class layout restates
 * EquationOfState.h:27-48 member for member because every reference TU links
 * against it.  The bulk switch PI is only commented out in
 * DynamicalVariables.h:14 (`#ifndef PI` tests follow), so the recipe passes
 * -DPI directly.
 */
#ifndef VH_REF_SHIM_H
#define VH_REF_SHIM_H

#include "DynamicalVariables.h"

#ifndef VH_THETA
#error "VH_THETA must be set by the oracle recipe"
#endif
#ifndef VH_EOS_FACTOR
#error "VH_EOS_FACTOR must be set by the oracle recipe"
#endif

/* FluxLimiter.h replacement (guard name from FluxLimiter.h:8-9). */
#define FLUXLIMITER_H_
#define THETA VH_THETA
PRECISION approximateDerivative(PRECISION x, PRECISION y, PRECISION z);

/* EquationOfState.h replacement (guard name from EquationOfState.h:8-9). */
#define EQUATIONOFSTATE_H_
#ifdef VH_EOS_TABLE
#define HOTQCDHRG_EOS
#else
#define CONFORMAL_EOS
#endif
#define EOS_FACTOR VH_EOS_FACTOR

class EOS
{
 private:
 public:
    double e_min;
    double e_max;
    double e_spacing;
    int e_length;

    double pressure_tb[100000];
    double temperature_tb[100000];

    PRECISION equilibriumPressure(PRECISION e);
    PRECISION speedOfSoundSquared(PRECISION e);
    PRECISION effectiveTemperature(PRECISION e);
    PRECISION equilibriumEnergyDensity(PRECISION T);

    double interpolate1D(double e, double *table);
    void loadEOSHotQCDHRG();
};

extern EOS eqnOfState;

#endif

/*
 * cpu_vh.h -- the C++ plugin surface of cpu-vh, served by the B200 library.
 *
 * Code written against the reference's headers links against
 * libcpu-vh_lib.so from this repository instead: the parameter structs and
 * the HYDRO class keep the reference's member order (ABI-compatible), the
 * functions keep its signatures.
 *
 *   struct LatticeParameters           rhic/include/LatticeParameters.h:17-34
 *   struct HydroParameters             rhic/include/HydroParameters.h:15-23
 *   struct InitialConditionParameters  rhic/include/InitialConditionParameters.h:13-26
 *   class HydroInitialTmunu            rhic/include/HydroInitialTmunu.h:11-31
 *   run(...)                           rhic/include/HydroPlugin.h:13
 *   read*Parameters(dir, params)       LatticeParameters.cpp:68-157, HydroParameters.cpp:207-263,
 *                                      InitialConditionParameters.cpp:65-149
 *   class HYDRO                        rhic/include/HydroWrapper.h:28-91
 *
 * Physics options the reference fixes at compile time (THETA, the EoS kind,
 * EOS_FACTOR, PI) default to its shipped values and can be changed at run
 * time with vh_plugin_set_config() or an optional <configDir>/b200.properties
 * file (named keys: theta, eos, eos_factor, eos_table, bulk, zeta_law,
 * zeta_norm, zeta_T0_GeV, zeta_width_GeV, precision = fp64 | mixed).
 */
#ifndef CPU_VH_H
#define CPU_VH_H

#include <vector>
#include "vh_b200.h"

#define N_GHOST_CELLS_M 2
#define N_GHOST_CELLS_P 2
#define N_GHOST_CELLS 4

struct LatticeParameters {
    int numLatticePointsX;
    int numLatticePointsY;
    int numLatticePointsRapidity;
    int numComputationalLatticePointsX;
    int numComputationalLatticePointsY;
    int numComputationalLatticePointsRapidity;
    int numProperTimePoints;
    int coarseProperTimeFOFactor;
    double latticeSpacingX;
    double latticeSpacingY;
    double latticeSpacingRapidity;
    double latticeSpacingProperTime;
    double fluxLimiterTheta;
};

struct HydroParameters {
    double initialProperTimePoint;
    double shearViscosityToEntropyDensity;
    double freezeoutTemperatureGeV;
    int initializePimunuNavierStokes;
    double regulationTemperatureGeV;
    int doFreezeOut;
};

struct InitialConditionParameters {
    int initialConditionType;
    int numberOfNucleonsPerNuclei;
    int numberOfSourceFiles;
    double initialEnergyDensity;
    double scatteringCrossSectionNN;
    double impactParameter;
    double fractionOfBinaryCollisions;
    double rapidityVariance;
    double rapidityMean;
    int sourceType;
};

class HydroInitialTmunu {
 public:
    std::vector<double> e_in, ut_in, ux_in, uy_in, un_in;
    std::vector<double> pitt_in, pitx_in, pity_in, pitn_in, pixx_in, pixy_in, pixn_in, piyy_in, piyn_in, pinn_in;
    std::vector<double> Pi_in;
};

void readLatticeParameters(const char *configDirectory, void *params);
void readHydroParameters(const char *configDirectory, void *params);
void readInitialConditionParameters(const char *configDirectory, void *params);

void run(void *latticeParams, void *initCondParams, void *hydroParams, const char *rootDirectory,
         const char *outputDir, HydroInitialTmunu init_tmunu);

class HYDRO {
 public:
    HYDRO();
    ~HYDRO();
    std::vector<double> initial_energy_density;
    std::vector<double> initial_ut;
    std::vector<double> initial_ux;
    std::vector<double> initial_uy;
    std::vector<double> initial_un;
    std::vector<double> initial_pitt;
    std::vector<double> initial_pitx;
    std::vector<double> initial_pity;
    std::vector<double> initial_pitn;
    std::vector<double> initial_pixx;
    std::vector<double> initial_pixy;
    std::vector<double> initial_pixn;
    std::vector<double> initial_piyy;
    std::vector<double> initial_piyn;
    std::vector<double> initial_pinn;
    std::vector<double> initial_Pi;
    int run_hydro(int, char **);
    int run_hydro_no_cli();
    void initialize_from_vector(std::vector<double> e);
    void initialize_from_vectors(std::vector<double> e, std::vector<double> ut, std::vector<double> ux,
                                 std::vector<double> uy, std::vector<double> un, std::vector<double> pitt,
                                 std::vector<double> pitx, std::vector<double> pity, std::vector<double> pitn,
                                 std::vector<double> pixx, std::vector<double> pixy, std::vector<double> pixn,
                                 std::vector<double> piyy, std::vector<double> piyn, std::vector<double> pinn,
                                 std::vector<double> Pi);
};

/* Run-time physics options for run() (the reference's compile-time macros).
 * Only theta, eos_kind, eos_factor, bulk, zeta_* and precision are taken from
 * cfg; lattice and hydro values always come from the parameter structs.
 * eos_table_path (nullable) names a binary EoS table (EoS directory format). */
void vh_plugin_set_config(const vh_config *cfg, const char *eos_table_path);

#endif

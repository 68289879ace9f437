/*
 * ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Linked with the unmodified cpu-vh hot-path sources (compiled in place by
 * oracle/ref.mk) into oracle/_ref/libvhref_<variant>.so.  It gives the tests
 * and the CPU baseline a C entry point into the reference's own code:
 *
 *   - it owns the parameter structs the reference reads
 *     (LatticeParameters.h:17-34, HydroParameters.h:15-23,
 *      InitialConditionParameters.h:13-26);
 *   - it injects initial-condition arrays through the three symbols
 *     HydroPlugin.cpp:189-193 expects from InitialConditions.cpp, which cannot
 *     be compiled here (GSL is absent).  The two vector initialisers restate
 *     InitialConditions.cpp:1593-1645 and :1647-1711 line for line;
 *   - it drives rungeKutta2 (FullyDiscreteKurganovTadmorScheme.cpp:867-924)
 *     with the time bookkeeping of the driver loop (HydroPlugin.cpp:226-308);
 *   - it calls the reference freezeout functions (FreezeOut.cpp:57-381, built
 *     inside the HydroPlugin.cpp translation unit) with the output stream
 *     switched to 17 significant digits so every element round-trips exactly.
 *
 * Nothing here is product code: the product never links this library.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <fstream>
#include <vector>
#include <string>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "DynamicalVariables.h"
#include "Vorticity.h"
#include "LatticeParameters.h"
#include "HydroParameters.h"
#include "InitialConditionParameters.h"
#include "HydroInitialTmunu.h"
#include "FullyDiscreteKurganovTadmorScheme.h"
#include "EnergyMomentumTensor.h"
#include "FreezeOut.h"
#include "HydroPlugin.h"
#include "LatticeParameters.h"
#include "HydroParameters.h"
#include "InitialConditionParameters.h"

/* Defined inside the HydroPlugin.cpp TU (FreezeOut.cpp and Memory.cpp are
 * #included there, HydroPlugin.cpp:21-22). */
void swapAndSetHydroVariables(double ****energy_density_evoution, double *****hydrodynamic_evoution,
                              CONSERVED_VARIABLES * const __restrict__ q, PRECISION * const __restrict__ e,
                              FLUID_VELOCITY * const __restrict__ u, int nx, int ny, int nz);
void callFOFinder3p1D(int dim, int nx, int ny, int nz, int n, double t0, double dt, double t, double dx, double dy, double dz, double *lattice_spacing, double freezeoutEnergyDensity,
  double ****hyperCube4D, double ***hyperCube3D, double ****energy_density_evoution, double *****hydrodynamic_evoution,
  std::ofstream& freezeoutSurfaceFile, std::vector<FO_Element>& fo_surf, EOS eqnOfState);
void callFOFinder2p1D(int dim, int nx, int ny, int nz, int n, double t0, double dt, double t, double dx, double dy, double dz, double *lattice_spacing, double freezeoutEnergyDensity,
  double ****hyperCube4D, double ***hyperCube3D, double ****energy_density_evoution, double *****hydrodynamic_evoution,
  std::ofstream& freezeoutSurfaceFile, std::vector<FO_Element>& fo_surf, EOS eqnOfState);
int checkForCellsAboveTc(int nx, int ny, int nz, double freezeoutEnergyDensity, PRECISION *e);
double *** calloc3dArray(double ***array, int dim1, int dim2, int dim3);
double **** calloc4dArray(double ****array, int dim1, int dim2, int dim3, int dim4);
double ***** calloc5dArray(double *****array, int dim1, int dim2, int dim3, int dim4, int dim5);

static struct LatticeParameters g_lat;
static struct HydroParameters g_hydro;
static struct InitialConditionParameters g_ic;
static int g_n = 0;          /* completed RK2 steps */
static double g_t = 0.0;     /* current proper time */
static int g_allocated = 0;   /* padded cells the reference's arrays hold */

/* initial-condition arrays over the interior (column-major i + nx*(j + ny*k)) */
static std::vector<double> ic_e, ic_p, ic_u[4], ic_pi[10], ic_Pi;
static int ic_have = 0;

/* freezeout slabs (HydroPlugin.cpp:158-177) */
static double ****fo_e = NULL;
static double *****fo_h = NULL;
static double ****fo_hc4 = NULL;
static double ***fo_hc3 = NULL;

static PRECISION *qfield(CONSERVED_VARIABLES *c, int n)
{
    switch (n) {
    case 0: return c->ttt; case 1: return c->ttx; case 2: return c->tty; case 3: return c->ttn;
#ifdef PIMUNU
    case 4: return c->pitt; case 5: return c->pitx; case 6: return c->pity; case 7: return c->pitn;
    case 8: return c->pixx; case 9: return c->pixy; case 10: return c->pixn; case 11: return c->piyy;
    case 12: return c->piyn; case 13: return c->pinn;
#endif
#ifdef PI
    case 14: return c->Pi;
#endif
    default: return NULL;
    }
}

static PRECISION *ufield(FLUID_VELOCITY *v, int n)
{
    switch (n) { case 0: return v->ut; case 1: return v->ux; case 2: return v->uy; default: return v->un; }
}

/* Copies the harness IC arrays into the reference globals (the job of
 * setInitialConditions for the built-in types, InitialConditions.cpp:1506-1591). */
static void inject_ic(void)
{
    int nx = g_lat.numLatticePointsX, ny = g_lat.numLatticePointsY, nz = g_lat.numLatticePointsRapidity;
    int ncx = nx + 4, ncy = ny + 4, ncz = nz + 4;
    for (int i = 2; i < nx + 2; ++i)
        for (int j = 2; j < ny + 2; ++j)
            for (int k = 2; k < nz + 2; ++k) {
                int s = columnMajorLinearIndex(i, j, k, ncx, ncy, ncz);
                int m = (i - 2) + nx * ((j - 2) + ny * (k - 2));
                e[s] = ic_e[m];
                p[s] = ic_p[m];
                for (int c = 0; c < 4; ++c) {
                    ufield(u, c)[s] = ic_u[c][m];
                    ufield(up, c)[s] = ic_u[c][m];
                }
#ifdef PIMUNU
                for (int c = 0; c < 10; ++c) qfield(q, 4 + c)[s] = ic_pi[c][m];
#endif
#ifdef PI
                q->Pi[s] = ic_Pi[m];
#endif
            }
}

/* ---- symbols HydroPlugin.cpp needs from InitialConditions.cpp / DynamicalSources.cpp ---- */
void setInitialConditions(void *latticeParams, void *initCondParams, void *hydroParams, const char *rootDirectory)
{
    (void)latticeParams; (void)initCondParams; (void)hydroParams; (void)rootDirectory;
    if (!ic_have) { printf("ref_harness: no IC arrays loaded\n"); exit(-1); }
    inject_ic();
}

/* InitialConditions.cpp:1593-1645 */
void setICFromEnergyDensityVector(void *latticeParams, void *initCondParams, void *hydroParams, const char *rootDirectory, HydroInitialTmunu init_tmunu)
{
    (void)initCondParams; (void)hydroParams; (void)rootDirectory;
    const double hbarc = 0.197326938;
    struct LatticeParameters *lattice = (struct LatticeParameters *)latticeParams;
    int nx = lattice->numLatticePointsX, ny = lattice->numLatticePointsY, nz = lattice->numLatticePointsRapidity;
    for (int i = 2; i < nx + 2; ++i)
        for (int j = 2; j < ny + 2; ++j)
            for (int k = 2; k < nz + 2; ++k) {
                int s = columnMajorLinearIndex(i, j, k, nx + 4, ny + 4, nz + 4);
                int sm = columnMajorLinearIndex(i - 2, j - 2, k - 2, nx, ny, nz);
                e[s] = (PRECISION)(init_tmunu.e_in[sm] / hbarc) + (PRECISION)(1.0e-3);
                p[s] = eqnOfState.equilibriumPressure(e[s]);
                u->ut[s] = 1.0; u->ux[s] = 0.0; u->uy[s] = 0.0; u->un[s] = 0.0;
                up->ut[s] = 1.0; up->ux[s] = 0.0; up->uy[s] = 0.0; up->un[s] = 0.0;
#ifdef PIMUNU
                for (int c = 4; c < 14; ++c) qfield(q, c)[s] = 0.0;
#endif
#ifdef PI
                q->Pi[s] = 0.0;
#endif
            }
}

/* InitialConditions.cpp:1647-1711 (including ut = 1+ux^2+uy^2+un^2 without a sqrt, :1681) */
void setICFromPreequilVectors(void *latticeParams, void *initCondParams, void *hydroParams, const char *rootDirectory, HydroInitialTmunu init_tmunu)
{
    (void)initCondParams; (void)hydroParams; (void)rootDirectory;
    const double hbarc = 0.197326938;
    struct LatticeParameters *lattice = (struct LatticeParameters *)latticeParams;
    int nx = lattice->numLatticePointsX, ny = lattice->numLatticePointsY, nz = lattice->numLatticePointsRapidity;
    for (int i = 2; i < nx + 2; ++i)
        for (int j = 2; j < ny + 2; ++j)
            for (int k = 2; k < nz + 2; ++k) {
                int s = columnMajorLinearIndex(i, j, k, nx + 4, ny + 4, nz + 4);
                int sm = columnMajorLinearIndex(i - 2, j - 2, k - 2, nx, ny, nz);
                e[s] = (PRECISION)(init_tmunu.e_in[sm] / hbarc) + (PRECISION)(1.0e-3);
                p[s] = eqnOfState.equilibriumPressure(e[s]);
                PRECISION ux, uy, un, ut;
                if (fabs(init_tmunu.ux_in[sm]) < 1.0e-7) ux = 0.0; else ux = (PRECISION)init_tmunu.ux_in[sm];
                if (fabs(init_tmunu.uy_in[sm]) < 1.0e-7) uy = 0.0; else uy = (PRECISION)init_tmunu.uy_in[sm];
                if (fabs(init_tmunu.un_in[sm]) < 1.0e-7) un = 0.0; else un = (PRECISION)init_tmunu.un_in[sm];
                ut = 1.0 + ux * ux + uy * uy + un * un;
                u->ux[s] = ux; u->uy[s] = uy; u->un[s] = un; u->ut[s] = ut;
                up->ut[s] = ut; up->ux[s] = ux; up->uy[s] = uy; up->un[s] = un;
#ifdef PIMUNU
                q->pitt[s] = (PRECISION)(init_tmunu.pitt_in[sm] / hbarc);
                q->pitx[s] = (PRECISION)(init_tmunu.pitx_in[sm] / hbarc);
                q->pity[s] = (PRECISION)(init_tmunu.pity_in[sm] / hbarc);
                q->pitn[s] = (PRECISION)(init_tmunu.pitn_in[sm] / hbarc);
                q->pixx[s] = (PRECISION)(init_tmunu.pixx_in[sm] / hbarc);
                q->pixy[s] = (PRECISION)(init_tmunu.pixy_in[sm] / hbarc);
                q->pixn[s] = (PRECISION)(init_tmunu.pixn_in[sm] / hbarc);
                q->piyy[s] = (PRECISION)(init_tmunu.piyy_in[sm] / hbarc);
                q->piyn[s] = (PRECISION)(init_tmunu.piyn_in[sm] / hbarc);
                q->pinn[s] = (PRECISION)(init_tmunu.pinn_in[sm] / hbarc);
#endif
#ifdef PI
                q->Pi[s] = (PRECISION)(init_tmunu.Pi_in[sm] / hbarc);
#endif
            }
}

void readInSource(int n, void *latticeParams, void *initCondParams, void *hydroParams, const char *rootDirectory)
{
    (void)n; (void)latticeParams; (void)initCondParams; (void)hydroParams; (void)rootDirectory;
    printf("ref_harness: dynamical sources (HDF5) are not built\n");
    exit(-1);
}
void noSource(void *latticeParams, void *initCondParams) { (void)latticeParams; (void)initCondParams; }

#ifdef VH_RACE_FREE_GHOSTS
/* DynamicalVariables.cpp:229-276, unchanged, compiled in that file */
void setGhostCellVars(CONSERVED_VARIABLES *const __restrict__ q, PRECISION *const __restrict__ e,
                      PRECISION *const __restrict__ p, FLUID_VELOCITY *const __restrict__ u, int s, int sBC);

/* DynamicalVariables.cpp:220-378 with the loop indices private to each
 * iteration (the original shares s, sBC and iBC/jBC/kBC across OpenMP
 * threads).  Same loop ranges and order, so the result equals the reference
 * run on one thread. */
void setGhostCells(CONSERVED_VARIABLES *const __restrict__ q, PRECISION *const __restrict__ e,
                   PRECISION *const __restrict__ p, FLUID_VELOCITY *const __restrict__ u, void *latticeParams)
{
    struct LatticeParameters *lattice = (struct LatticeParameters *)latticeParams;
    int nx = lattice->numLatticePointsX, ny = lattice->numLatticePointsY, nz = lattice->numLatticePointsRapidity;
    int ncx = lattice->numComputationalLatticePointsX, ncy = lattice->numComputationalLatticePointsY;
    int ncz = lattice->numComputationalLatticePointsRapidity;
#pragma omp parallel for
    for (int j = 2; j < ncy; ++j)
        for (int k = 2; k < ncz; ++k) {
            for (int i = 0; i <= 1; ++i)
                setGhostCellVars(q, e, p, u, columnMajorLinearIndex(i, j, k, ncx, ncy, ncz), columnMajorLinearIndex(2, j, k, ncx, ncy, ncz));
            for (int i = nx + 2; i <= nx + 3; ++i)
                setGhostCellVars(q, e, p, u, columnMajorLinearIndex(i, j, k, ncx, ncy, ncz), columnMajorLinearIndex(nx + 1, j, k, ncx, ncy, ncz));
        }
#pragma omp parallel for
    for (int i = 2; i < ncx; ++i)
        for (int k = 2; k < ncz; ++k) {
            for (int j = 0; j <= 1; ++j)
                setGhostCellVars(q, e, p, u, columnMajorLinearIndex(i, j, k, ncx, ncy, ncz), columnMajorLinearIndex(i, 2, k, ncx, ncy, ncz));
            for (int j = ny + 2; j <= ny + 3; ++j)
                setGhostCellVars(q, e, p, u, columnMajorLinearIndex(i, j, k, ncx, ncy, ncz), columnMajorLinearIndex(i, ny + 1, k, ncx, ncy, ncz));
        }
#pragma omp parallel for
    for (int i = 2; i < ncx; ++i)
        for (int j = 2; j < ncy; ++j) {
            for (int k = 0; k <= 1; ++k)
                setGhostCellVars(q, e, p, u, columnMajorLinearIndex(i, j, k, ncx, ncy, ncz), columnMajorLinearIndex(i, j, 2, ncx, ncy, ncz));
            for (int k = nz + 2; k <= nz + 3; ++k)
                setGhostCellVars(q, e, p, u, columnMajorLinearIndex(i, j, k, ncx, ncy, ncz), columnMajorLinearIndex(i, j, nz + 1, ncx, ncy, ncz));
        }
}
#endif

extern "C" {

int vhref_nq(void) { return NUMBER_CONSERVED_VARIABLES; }
int vhref_is_table_eos(void)
{
#ifdef HOTQCDHRG_EOS
    return 1;
#else
    return 0;
#endif
}
double vhref_theta(void) { return (double)THETA; }

int vhref_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

/* lattice/hydro/ic parameters in the reference's own units */
void vhref_setup(int nx, int ny, int nz, int nt, int fofac,
                 double dx, double dy, double dz, double dt,
                 double t0, double etabar, double TfoGeV, double TregGeV, int ic_type)
{
    memset(&g_lat, 0, sizeof(g_lat));
    memset(&g_hydro, 0, sizeof(g_hydro));
    memset(&g_ic, 0, sizeof(g_ic));
    g_lat.numLatticePointsX = nx; g_lat.numLatticePointsY = ny; g_lat.numLatticePointsRapidity = nz;
    g_lat.numComputationalLatticePointsX = nx + N_GHOST_CELLS;
    g_lat.numComputationalLatticePointsY = ny + N_GHOST_CELLS;
    g_lat.numComputationalLatticePointsRapidity = nz + N_GHOST_CELLS;
    g_lat.numProperTimePoints = nt;
    g_lat.coarseProperTimeFOFactor = fofac;
    g_lat.latticeSpacingX = dx; g_lat.latticeSpacingY = dy; g_lat.latticeSpacingRapidity = dz;
    g_lat.latticeSpacingProperTime = dt;
    g_hydro.initialProperTimePoint = t0;
    g_hydro.shearViscosityToEntropyDensity = etabar;
    g_hydro.freezeoutTemperatureGeV = TfoGeV;
    g_hydro.initializePimunuNavierStokes = 0;
    g_hydro.regulationTemperatureGeV = TregGeV;
    g_hydro.doFreezeOut = 1;
    g_ic.initialConditionType = ic_type;
}

/* Fills the tabulated EoS exactly as EquationOfState.cpp:292-327 does from its
 * binary file (rows of e[GeV/fm^3], P[GeV/fm^3], s, T[GeV]); nrows <= 100000. */
int vhref_load_eos_table(const double *rows, int nrows)
{
    const double hbarc = 0.197326938;
    if (nrows < 2 || nrows > 100000) return -1;
    eqnOfState.e_length = nrows;
    for (int ii = 0; ii < nrows; ii++) {
        double temp = rows[4 * ii + 0];
        temp /= hbarc;
        if (ii == 0) eqnOfState.e_min = temp;
        if (ii == 1) eqnOfState.e_spacing = temp - eqnOfState.e_min;
        if (ii == nrows - 1) eqnOfState.e_max = temp;
        temp = rows[4 * ii + 1];
        eqnOfState.pressure_tb[ii] = temp / hbarc;
        temp = rows[4 * ii + 3];
        eqnOfState.temperature_tb[ii] = temp / hbarc;
    }
    return 0;
}

double vhref_eos_pressure(double ed) { return eqnOfState.equilibriumPressure(ed); }
/* the reference's equilibrium pressure of n energy densities (initial states) */
void vhref_eos_pressure_n(const double *ed, double *p_out, long n)
{
    for (long i = 0; i < n; ++i) p_out[i] = eqnOfState.equilibriumPressure(ed[i]);
}
double vhref_eos_temperature(double ed) { return eqnOfState.effectiveTemperature(ed); }
double vhref_eos_cs2(double ed) { return eqnOfState.speedOfSoundSquared(ed); }
double vhref_eos_energy(double T) { return eqnOfState.equilibriumEnergyDensity(T); }

/* e, p, (ut,ux,uy,un), 10 pi components (pitt..pinn), Pi over the interior. */
void vhref_set_ic_arrays(const double *e_, const double *p_, const double *u_, const double *pi_, const double *Pi_)
{
    int N = g_lat.numLatticePointsX * g_lat.numLatticePointsY * g_lat.numLatticePointsRapidity;
    ic_e.assign(e_, e_ + N);
    ic_p.assign(p_, p_ + N);
    for (int c = 0; c < 4; ++c) ic_u[c].assign(u_ + (size_t)c * N, u_ + (size_t)(c + 1) * N);
    for (int c = 0; c < 10; ++c) {
        if (pi_) ic_pi[c].assign(pi_ + (size_t)c * N, pi_ + (size_t)(c + 1) * N);
        else ic_pi[c].assign(N, 0.0);
    }
    if (Pi_) ic_Pi.assign(Pi_, Pi_ + N); else ic_Pi.assign(N, 0.0);
    ic_have = 1;
}

/* The initialisation part of run() (HydroPlugin.cpp:131, :189-204), plus the
 * freezeout slabs (:158-177). */
void vhref_init(void)
{
    int nx = g_lat.numLatticePointsX, ny = g_lat.numLatticePointsY, nz = g_lat.numLatticePointsRapidity;
    int len = g_lat.numComputationalLatticePointsX * g_lat.numComputationalLatticePointsY * g_lat.numComputationalLatticePointsRapidity;
    if (len > g_allocated) {
        /* the reference sizes its global arrays once per run; a larger event
         * in the same process needs them again at the new size */
        if (g_allocated) freeHostMemory();
        allocateHostMemory(len);
        g_allocated = len;
    }
    /* no dynamical sources unless vhref_set_sources gives them (the arrays
     * outlive an event in this process) */
    memset(Source->sourcet, 0, sizeof(double) * (size_t)len);
    memset(Source->sourcex, 0, sizeof(double) * (size_t)len);
    memset(Source->sourcey, 0, sizeof(double) * (size_t)len);
    memset(Source->sourcen, 0, sizeof(double) * (size_t)len);
    inject_ic();
    g_n = 0;
    g_t = g_hydro.initialProperTimePoint;
    setConservedVariables(g_t, &g_lat);
    setGhostCells(q, e, p, u, &g_lat);
    fo_e = calloc4dArray(fo_e, 2, nx, ny, nz);
    fo_h = calloc5dArray(fo_h, 10, 2, nx, ny, nz);
    fo_hc4 = calloc4dArray(fo_hc4, 2, 2, 2, 2);
    fo_hc3 = calloc3dArray(fo_hc3, 2, 2, 2);
}

/* nsteps iterations of the driver loop body (HydroPlugin.cpp:292-307); the
 * thermal-vorticity update and field dumps are not part of the evolution. */
void vhref_step(int nsteps)
{
    double dt = g_lat.latticeSpacingProperTime;
    double t0 = g_hydro.initialProperTimePoint;
    for (int s = 0; s < nsteps; ++s) {
        rungeKutta2(g_t, dt, q, Q, &g_lat, &g_hydro);
        setCurrentConservedVariables();
        g_n += 1;
        g_t = t0 + g_n * dt;
    }
}

/* wall-clock seconds of nsteps RK2 steps (omp_get_wtime), for the CPU baseline */
double vhref_time_steps(int nsteps)
{
#ifdef _OPENMP
    double a = omp_get_wtime();
    vhref_step(nsteps);
    return omp_get_wtime() - a;
#else
    vhref_step(nsteps);
    return -1.0;
#endif
}

int vhref_steps_done(void) { return g_n; }
double vhref_time(void) { return g_t; }

/* which: 0..NQ-1 -> q component; 100+c -> u^c; 110+c -> up^c; 200 -> e; 201 -> p.
 * Copies the full padded array (ncx*ncy*ncz doubles). */
int vhref_get(int which, double *out)
{
    int len = g_lat.numComputationalLatticePointsX * g_lat.numComputationalLatticePointsY * g_lat.numComputationalLatticePointsRapidity;
    PRECISION *src = NULL;
    if (which >= 0 && which < NUMBER_CONSERVED_VARIABLES) src = qfield(q, which);
    else if (which >= 100 && which < 104) src = ufield(u, which - 100);
    else if (which >= 110 && which < 114) src = ufield(up, which - 110);
    else if (which == 200) src = e;
    else if (which == 201) src = p;
    else if (which == 300) src = wmunu->wtx;
    else if (which == 301) src = wmunu->wty;
    else if (which == 302) src = wmunu->wtn;
    else if (which == 303) src = wmunu->wxy;
    else if (which == 304) src = wmunu->wxn;
    else if (which == 305) src = wmunu->wyn;
    else if (which == 310) src = beta_mu->beta_t;
    else if (which == 311) src = beta_mu->beta_x;
    else if (which == 312) src = beta_mu->beta_y;
    else if (which == 313) src = beta_mu->beta_n;
    else if (which == 400) src = regFacShear;
    else if (which == 401) src = regFacBulk;
    if (!src) return -1;
    memcpy(out, src, sizeof(double) * (size_t)len);
    return 0;
}

/* Fills the reference's dynamical source arrays (Source->sourcet..sourcen,
 * SourceTerms.cpp:584-587) from interior arrays; the ghost cells stay 0. */
void vhref_set_sources(const double *st, const double *sx, const double *sy, const double *sn)
{
    int nx = g_lat.numLatticePointsX, ny = g_lat.numLatticePointsY, nz = g_lat.numLatticePointsRapidity;
    int ncx = nx + 4, ncy = ny + 4;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                int s = (i + 2) + ncx * ((j + 2) + ncy * (k + 2));
                size_t m = i + (size_t)nx * (j + (size_t)ny * k);
                Source->sourcet[s] = st[m];
                Source->sourcex[s] = sx[m];
                Source->sourcey[s] = sy[m];
                Source->sourcen[s] = sn[m];
            }
}

/* The thermal vorticity as the driver computes it after the initial
 * condition and after every step (HydroPlugin.cpp:197-199, :302-305). */
void vhref_vorticity(void)
{
    calculateThermalVorticity(g_t, g_lat.latticeSpacingProperTime, q, Q, &g_lat, &g_hydro);
}

/* One freezeout block of the driver loop (HydroPlugin.cpp:242-266) for loop
 * index n = steps_done + 1, with the surface written to `path` at 17 digits.
 * Returns the number of interior cells above the freezeout energy density. */
int vhref_freezeout(const char *path)
{
    int nx = g_lat.numLatticePointsX, ny = g_lat.numLatticePointsY, nz = g_lat.numLatticePointsRapidity;
    double t0 = g_hydro.initialProperTimePoint, dt = g_lat.latticeSpacingProperTime;
    double dx = g_lat.latticeSpacingX, dy = g_lat.latticeSpacingY, dz = g_lat.latticeSpacingRapidity;
    const double hbarc = 0.197326938;
    const double eF = eqnOfState.equilibriumEnergyDensity(g_hydro.freezeoutTemperatureGeV / hbarc);
    int n = g_n + 1;
    int dim = (nz > 1) ? 4 : 3;
    double ls[4] = {dt * g_lat.coarseProperTimeFOFactor, dx, dy, dz};
    std::vector<FO_Element> fo_surf;
    std::ofstream f;
    f.open(path);
    f.precision(17);
    swapAndSetHydroVariables(fo_e, fo_h, q, e, u, nx, ny, nz);
    if (dim == 4)
        callFOFinder3p1D(dim, nx, ny, nz, n, t0, dt, g_t, dx, dy, dz, ls, eF, fo_hc4, fo_hc3, fo_e, fo_h, f, fo_surf, eqnOfState);
    else
        callFOFinder2p1D(dim, nx, ny, nz, n, t0, dt, g_t, dx, dy, dz, ls, eF, fo_hc4, fo_hc3, fo_e, fo_h, f, fo_surf, eqnOfState);
    f.close();
    return checkForCellsAboveTc(nx, ny, nz, eF, e);
}

/* The reference driver end to end from an energy-density vector, initial
 * condition type 13 (HydroWrapper.cpp:20-23, InitialConditions.cpp:1593). */
void vhref_run_vector(const char *outdir, const double *e_in, int n)
{
    HydroInitialTmunu tm;
    tm.e_in.assign(e_in, e_in + n);
    g_ic.initialConditionType = 13;
    run(&g_lat, &g_ic, &g_hydro, ".", outdir, tm);
}

/* Loads the harness parameter structs with the reference's own parsers. */
void vhref_load_conf(const char *dir)
{
    readLatticeParameters(dir, &g_lat);
    readHydroParameters(dir, &g_hydro);
    readInitialConditionParameters(dir, &g_ic);
}

/* The reference's own positional parsers (LatticeParameters.cpp:68-157,
 * HydroParameters.cpp:207-263, InitialConditionParameters.cpp:65-149). */
void vhref_read_parameters(const char *dir, void *lat, void *hyd, void *ic)
{
    readLatticeParameters(dir, lat);
    readHydroParameters(dir, hyd);
    readInitialConditionParameters(dir, ic);
}

/* The reference driver end to end (HydroPlugin.cpp:74-321) on the harness IC;
 * writes <outdir>/surface.dat at the reference's default 6 digits. */
void vhref_run_full(const char *outdir)
{
    HydroInitialTmunu tm;
    run(&g_lat, &g_ic, &g_hydro, ".", outdir, tm);
}

} /* extern "C" */

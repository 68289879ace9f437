/*
 * hydro_plugin.cpp -- the reference's C++ plugin surface (include/cpu_vh.h)
 * driving the B200 C ABI: the positional rhic-conf parsers, the run() driver
 * loop with its freezeout cadence, stop criterion and surface.dat writer, the
 * initial conditions that need no external data, and the HYDRO wrapper with
 * its command line.
 */
#include <algorithm>
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <fstream>
#include <mutex>
#include <thread>
#include <getopt.h>
#include <iostream>
#include <string>
#include <unistd.h>
#include <vector>

#include "cpu_vh.h"
#include "vh_internal.h"

namespace {

using vh::kHbarc;

struct PluginConfig {
    vh_config phys;
    std::string eos_table;
    PluginConfig()
    {
        vh_config_default(&phys);
        eos_table = "EoS/hrg_hotqcd_eos_binary.dat";   /* EquationOfState.cpp:299 */
    }
};
PluginConfig &plugin()
{
    static PluginConfig p;
    return p;
}

/* The positional reader of LatticeParameters.cpp:78-130: blanks removed, the
 * text after '=' kept, the key itself ignored. */
std::string value_of(std::string line)
{
    line.erase(std::remove_if(line.begin(), line.end(), [](unsigned char c) { return std::isspace(c); }), line.end());
    auto pos = line.find("=");
    return line.substr(pos + 1);
}

/* parser state persists like the reference's file-scope globals */
int g_numLatticePointsX, g_numLatticePointsY, g_numLatticePointsRapidity, g_numProperTimePoints, g_coarseFO;
double g_dx, g_dy, g_dz, g_dt, g_theta;
double g_t0, g_etabar, g_TfoGeV, g_TregGeV;
int g_initPiNS, g_doFO;
int g_icType, g_nSource, g_A, g_sourceType;
double g_e0, g_snn, g_b, g_alpha, g_rapVar, g_rapMean;

std::vector<double> load_eos_table(const std::string &path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        printf("Can not find the EoS file! Exiting!");
        exit(1);
    }
    f.seekg(0, std::ios::end);
    size_t bytes = (size_t)f.tellg();
    f.seekg(0);
    size_t rows = std::min<size_t>(bytes / (4 * sizeof(double)), 100000);
    std::vector<double> r(rows * 4);
    f.read((char *)r.data(), (std::streamsize)(r.size() * sizeof(double)));
    return r;
}

/* optical Glauber thickness T_A(x, y) of GlauberModel.cpp:16-55: Woods-Saxon
 * n0 = 0.17, R = 1.12 A^1/3 - 0.86 A^-1/3, d = 0.54, integrated along z
 * (composite Simpson, converged to ~1e-12 relative) */
double thickness(double x, double y, double A)
{
    const double n0 = 0.17, Rn = 1.12 * pow(A, 1. / 3.) - 0.86 * pow(A, -1. / 3.), d = 0.54;
    const double zmax = Rn + 40 * d;
    const int n = 4000;
    const double h = zmax / n;
    double s = 0;
    for (int k = 0; k <= n; ++k) {
        double z = k * h;
        double f = n0 / (1 + exp((sqrt(x * x + y * y + z * z) - Rn) / d));
        s += (k == 0 || k == n) ? f : (k % 2 ? 4 * f : 2 * f);
    }
    return 2 * s * h / 3;
}

/* GlauberModel.cpp:57-108: mixture of binary collisions and wounded nucleons */
void glauber_transverse(std::vector<double> &eT, int nx, int ny, double dx, double dy, const InitialConditionParameters &ic)
{
    const double A = ic.numberOfNucleonsPerNuclei, snn = ic.scatteringCrossSectionNN, b = ic.impactParameter;
    const double alpha = ic.fractionOfBinaryCollisions;
    auto ncoll = [&](double TAp, double TBm) { return snn * TAp * TBm; };
    auto npart = [&](double TAm, double TAp, double TBm, double TBp) {
        (void)TAm; (void)TBp;
        const double f2mb = 0.1;
        double part = 1 - snn * TBm * f2mb / A;
        double res = TAp * (1 - pow(1 - part, A));
        part = 1 - snn * TAp * f2mb / A;
        res += TBm * (1 - pow(1 - part, A));
        return res;
    };
    const double T0 = thickness(0, 0, A);
    const double nbcNorm = 1. / ncoll(T0, T0), wnNorm = 1. / npart(T0, T0, T0, T0);
    eT.assign((size_t)nx * ny, 0.0);
    for (int i = 0; i < nx; ++i) {
        double x = (i - (nx - 1) / 2.) * dx;
        for (int j = 0; j < ny; ++j) {
            double y = (j - (ny - 1) / 2.) * dy;
            double TAm = thickness(x - b / 2, y, A), TAp = thickness(x + b / 2, y, A);
            double ed = nbcNorm * ncoll(TAp, TAm);
            ed *= alpha;
            ed += (1 - alpha) * wnNorm * npart(TAm, TAp, TAm, TAp);
            eT[i + (size_t)j * nx] = ed;
        }
    }
}

/* reference bulk viscosity law (SourceTerms.cpp:40-48) */
double zeta_ref(double T)
{
    double x = T / 1.01355;
    if (x > 1.05) return 0.9 * exp(-(x - 1) / 0.025) + 0.25 * exp(-(x - 1) / 0.13) + 0.001;
    if (x < 0.995) return 0.9 * exp((x - 1) / 0.0025) + 0.22 * exp((x - 1) / 0.022) + 0.03;
    return -13.77 * x * x + 27.55 * x - 13.45;
}

struct IC {
    std::vector<double> e, p, u, pi, Pi;
};

/* setPimunuInitialCondition / setPimunuNavierStokesInitialCondition
 * (InitialConditions.cpp:530-648), Bjorken Navier-Stokes values */
void pimunu_ic(IC &ic, size_t N, const HydroParameters &h, const vh::HostEos &eos, bool bulk)
{
    ic.pi.assign(10 * N, 0.0);
    ic.Pi.assign(N, 0.0);
    if (h.initializePimunuNavierStokes != 1) return;
    const double t = h.initialProperTimePoint, etabar = h.shearViscosityToEntropyDensity;
    for (size_t m = 0; m < N; ++m) {
        double T = eos.temperature(ic.e[m]);
        if (T == 0) T = 1.e-3;
        double pinn = -4.0 / (3.0 * t * t * t) * etabar * (ic.e[m] + ic.p[m]) / T;
        ic.pi[4 * N + m] = -t * t * pinn / 2;
        ic.pi[7 * N + m] = -t * t * pinn / 2;
        ic.pi[9 * N + m] = pinn;
        if (bulk) ic.Pi[m] = -zeta_ref(T) * (ic.e[m] + ic.p[m]) / T / t;
    }
}

void rest_velocity(IC &ic, size_t N)
{
    ic.u.assign(4 * N, 0.0);
    for (size_t m = 0; m < N; ++m) ic.u[m] = 1.0;
}

/* index of interior cell (i, j, k) in the order the C ABI takes */
inline size_t interior(int i, int j, int k, int nx, int ny) { return i + (size_t)nx * (j + (size_t)ny * k); }

bool build_ic(IC &ic, const LatticeParameters &L, const InitialConditionParameters &icp, const HydroParameters &h,
              const vh::HostEos &eos, bool bulk, const HydroInitialTmunu &tm)
{
    const int nx = L.numLatticePointsX, ny = L.numLatticePointsY, nz = L.numLatticePointsRapidity;
    const size_t N = (size_t)nx * ny * nz;
    ic.e.assign(N, 0.0);
    ic.p.assign(N, 0.0);
    switch (icp.initialConditionType) {
    case 0: {   /* InitialConditions.cpp:953-981 */
        printf("Setting initial conditions: constant energy density.\n");
        double ed = eos.energy_of_T(3.05);
        for (size_t m = 0; m < N; ++m) { ic.e[m] = ed; ic.p[m] = eos.pressure(ed); }
        rest_velocity(ic, N);
        pimunu_ic(ic, N, h, eos, bulk);
        return true;
    }
    case 2: {   /* InitialConditions.cpp:1046-1105 */
        printf("Setting initial conditions: Continous optical Glauber.\n");
        std::vector<double> eT;
        glauber_transverse(eT, nx, ny, L.latticeSpacingX, L.latticeSpacingY, icp);
        std::vector<double> eL(nz);
        for (int k = 0; k < nz; ++k) {
            double eta = (k - (nz - 1) / 2) * L.latticeSpacingRapidity;
            double sc = fabs(eta) - icp.rapidityMean / 2;
            double arg = -sc * sc / icp.rapidityVariance / 2 * (sc < 0 ? 0.0 : 1.0);
            eL[k] = exp(arg);
        }
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int k = 0; k < nz; ++k) {
                    size_t m = interior(i, j, k, nx, ny);
                    double ed = (icp.initialEnergyDensity * eT[i + (size_t)j * nx] * eL[k]) + 1.e-3;
                    ic.e[m] = ed;
                    ic.p[m] = eos.pressure(ed);
                }
        rest_velocity(ic, N);
        pimunu_ic(ic, N, h, eos, bulk);
        return true;
    }
    case 3: {   /* InitialConditions.cpp:1146-1194 (u is 0/0 at r = 0 there too) */
        printf("Setting initial conditions: Ideal hydrodynamic Gubser flow test.\n");
        ic.u.assign(4 * N, 0.0);
        ic.pi.assign(10 * N, 0.0);
        ic.Pi.assign(N, 0.0);
        for (int i = 0; i < nx; ++i) {
            double x = (i - (nx - 1) / 2.) * L.latticeSpacingX;
            for (int j = 0; j < ny; ++j) {
                double y = (j - (ny - 1) / 2.) * L.latticeSpacingY;
                double T = 1.9048812623618392 / pow(1 + pow(1 - pow(x, 2) - pow(y, 2), 2) + 2 * (1 + pow(x, 2) + pow(y, 2)), 0.3333333333333333);
                double r = sqrt(x * x + y * y);
                double phi = atanh(2.0 * r / (1.0 + 1.0 + x * x + y * y));
                for (int k = 0; k < nz; ++k) {
                    size_t m = interior(i, j, k, nx, ny);
                    ic.e[m] = icp.initialEnergyDensity * pow(T, 4);
                    ic.p[m] = ic.e[m] / 3.0;
                    double ux = sinh(phi) * x / r, uy = sinh(phi) * y / r;
                    ic.u[N + m] = ux;
                    ic.u[2 * N + m] = uy;
                    ic.u[3 * N + m] = 0.0;
                    ic.u[m] = sqrt(1 + ux * ux + uy * uy);
                }
            }
        }
        return true;
    }
    case 13:    /* InitialConditions.cpp:1593-1645 */
    case 14: {  /* InitialConditions.cpp:1647-1711 */
        const bool pre = icp.initialConditionType == 14;
        printf(pre ? "Initialize from preequilibrium vectors ...\n" : "Initialize from initial energy density vector ...\n");
        if (tm.e_in.size() < N) { printf("initial vectors hold %zu cells, the lattice %zu\n", tm.e_in.size(), N); exit(-1); }
        ic.u.assign(4 * N, 0.0);
        ic.pi.assign(10 * N, 0.0);
        ic.Pi.assign(N, 0.0);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int k = 0; k < nz; ++k) {
                    size_t m = interior(i, j, k, nx, ny);   /* the reference's sm, same layout */
                    ic.e[m] = (tm.e_in[m] / kHbarc) + (1.0e-3);
                    ic.p[m] = eos.pressure(ic.e[m]);
                    if (!pre) { ic.u[m] = 1.0; continue; }
                    double ux = fabs(tm.ux_in[m]) < 1.0e-7 ? 0.0 : tm.ux_in[m];
                    double uy = fabs(tm.uy_in[m]) < 1.0e-7 ? 0.0 : tm.uy_in[m];
                    double un = fabs(tm.un_in[m]) < 1.0e-7 ? 0.0 : tm.un_in[m];
                    ic.u[m] = 1.0 + ux * ux + uy * uy + un * un;   /* no sqrt, as :1681 */
                    ic.u[N + m] = ux;
                    ic.u[2 * N + m] = uy;
                    ic.u[3 * N + m] = un;
                    const std::vector<double> *pv[10] = {&tm.pitt_in, &tm.pitx_in, &tm.pity_in, &tm.pitn_in, &tm.pixx_in,
                                                         &tm.pixy_in, &tm.pixn_in, &tm.piyy_in, &tm.piyn_in, &tm.pinn_in};
                    for (int c = 0; c < 10; ++c) ic.pi[c * N + m] = pv[c]->size() > m ? (*pv[c])[m] / kHbarc : 0.0;
                    if (bulk) ic.Pi[m] = tm.Pi_in.size() > m ? tm.Pi_in[m] / kHbarc : 0.0;
                }
        return true;
    }
    default:
        printf("Initial condition type %d is not available in this build (types 0, 2, 3, 13, 14 are). Exiting ...\n",
               icp.initialConditionType);
        return false;
    }
}

/* surface.dat on a thread of its own: the run loop hands each freezeout
 * block's elements over (moved, not copied) and goes on stepping while they
 * are formatted with the reference's stream formatting (FreezeOut.cpp:265-270:
 * default precision, space separated, one element per line), so the text
 * formatting is off the evolution's critical path and the file's bytes are
 * the same as when written in line. */
class SurfaceWriter {
 public:
    explicit SurfaceWriter(const std::string &path) : out_(path), th_([this] { loop(); }) {}
    ~SurfaceWriter() { close(); }
    void push(std::vector<double> &&block)
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            q_.push_back(std::move(block));
        }
        cv_.notify_one();
    }
    void close()
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            done_ = true;
        }
        cv_.notify_one();
        if (th_.joinable()) th_.join();
        if (out_.is_open()) out_.close();
    }

 private:
    void loop()
    {
        for (;;) {
            std::vector<double> b;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return done_ || !q_.empty(); });
                if (q_.empty()) return;
                b = std::move(q_.front());
                q_.pop_front();
            }
            for (size_t i = 0; i + VH_FO_COLUMNS <= b.size(); i += VH_FO_COLUMNS) {
                const double *o = &b[i];
                for (int c = 0; c < VH_FO_COLUMNS; ++c) {
                    if (c) out_ << " ";
                    out_ << o[c];
                }
                out_ << '\n';
            }
        }
    }
    std::ofstream out_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::vector<double>> q_;
    bool done_ = false;
    std::thread th_;
};

void dump_field(vh_event *ev, int field, const char *name, double t, const char *dir, const LatticeParameters &L)
{
    const int nx = L.numLatticePointsX, ny = L.numLatticePointsY, nz = L.numLatticePointsRapidity;
    const int ncx = nx + 4, ncy = ny + 4, ncz = nz + 4;
    std::vector<double> v((size_t)ncx * ncy * ncz);
    if (vh_event_get_field(ev, field, v.data()) != VH_OK) return;
    char fname[512];
    snprintf(fname, sizeof fname, "%s/%s_%.3f.dat", dir, name, t);
    FILE *fp = fopen(fname, "w");
    if (!fp) return;
    /* FileIO.cpp:14-59 */
    for (int k = 2; k < nz + 2; ++k) {
        double z = (k - 2 - (nz - 1) / 2.) * L.latticeSpacingRapidity;
        for (int j = 2; j < ny + 2; ++j) {
            double y = (j - 2 - (ny - 1) / 2.) * L.latticeSpacingY;
            for (int i = 2; i < nx + 2; ++i) {
                double x = (i - 2 - (nx - 1) / 2.) * L.latticeSpacingX;
                fprintf(fp, "%.3f\t%.3f\t%.3f\t%.8f\n", x, y, z, v[i + (size_t)ncx * (j + (size_t)ncy * k)]);
            }
        }
    }
    fclose(fp);
}

void die_on(int rc, const char *what)
{
    if (rc == VH_OK) return;
    if (rc == VH_ERR_NAN) printf("\n Found e nan inside getInferredVariables \n");
    printf("%s failed (%d): %s\n", what, rc, vh_last_error());
    exit(-1);
}

} // namespace

/* ------------------------------------------------------------ parsers */
void readLatticeParameters(const char *configDirectory, void *params)
{
    char fname[255];
    snprintf(fname, sizeof fname, "%s/%s", configDirectory, "lattice.properties");
    std::ifstream c(fname);
    if (c.is_open()) {
        std::string l;
        getline(c, l); g_numLatticePointsX = atoi(value_of(l).c_str());
        getline(c, l); g_numLatticePointsY = atoi(value_of(l).c_str());
        getline(c, l); g_numLatticePointsRapidity = atoi(value_of(l).c_str());
        getline(c, l); g_numProperTimePoints = atoi(value_of(l).c_str());
        getline(c, l); g_dx = atof(value_of(l).c_str());
        getline(c, l); g_dy = atof(value_of(l).c_str());
        getline(c, l); g_dz = atof(value_of(l).c_str());
        getline(c, l); g_dt = atof(value_of(l).c_str());
        getline(c, l); g_coarseFO = atoi(value_of(l).c_str());
    } else {
        std::cerr << "No configuration file found for lattice parameters\n";
    }
    LatticeParameters *L = (LatticeParameters *)params;
    L->numLatticePointsX = g_numLatticePointsX;
    L->numLatticePointsY = g_numLatticePointsY;
    L->numLatticePointsRapidity = g_numLatticePointsRapidity;
    L->numComputationalLatticePointsX = g_numLatticePointsX + N_GHOST_CELLS;
    L->numComputationalLatticePointsY = g_numLatticePointsY + N_GHOST_CELLS;
    L->numComputationalLatticePointsRapidity = g_numLatticePointsRapidity + N_GHOST_CELLS;
    L->numProperTimePoints = g_numProperTimePoints;
    L->latticeSpacingX = g_dx;
    L->latticeSpacingY = g_dy;
    L->latticeSpacingRapidity = g_dz;
    L->latticeSpacingProperTime = g_dt;
    L->coarseProperTimeFOFactor = g_coarseFO;
    L->fluxLimiterTheta = g_theta;
}

void readHydroParameters(const char *configDirectory, void *params)
{
    char fname[255];
    snprintf(fname, sizeof fname, "%s/%s", configDirectory, "hydro.properties");
    std::ifstream c(fname);
    if (c.is_open()) {
        std::string l;
        getline(c, l); g_t0 = atof(value_of(l).c_str());
        getline(c, l); g_etabar = atof(value_of(l).c_str());
        getline(c, l); g_TfoGeV = atof(value_of(l).c_str());
        getline(c, l); g_initPiNS = atoi(value_of(l).c_str());
        getline(c, l); g_TregGeV = atof(value_of(l).c_str());
        getline(c, l); g_doFO = atoi(value_of(l).c_str());
    } else {
        std::cerr << "No configuration file found for hydro parameters\n";
    }
    HydroParameters *h = (HydroParameters *)params;
    h->initialProperTimePoint = g_t0;
    h->shearViscosityToEntropyDensity = g_etabar;
    h->freezeoutTemperatureGeV = g_TfoGeV;
    h->initializePimunuNavierStokes = g_initPiNS;
    h->regulationTemperatureGeV = g_TregGeV;
    h->doFreezeOut = g_doFO;
}

void readInitialConditionParameters(const char *configDirectory, void *params)
{
    char fname[255];
    snprintf(fname, sizeof fname, "%s/%s", configDirectory, "ic.properties");
    std::ifstream c(fname);
    if (c.is_open()) {
        std::string l;
        getline(c, l); g_icType = atoi(value_of(l).c_str());
        getline(c, l); g_nSource = atoi(value_of(l).c_str());
        getline(c, l); g_A = atoi(value_of(l).c_str());
        getline(c, l); g_e0 = atof(value_of(l).c_str());
        getline(c, l); g_snn = atof(value_of(l).c_str());
        getline(c, l); g_b = atof(value_of(l).c_str());
        getline(c, l); g_alpha = atof(value_of(l).c_str());
        getline(c, l); g_rapVar = atof(value_of(l).c_str());
        getline(c, l); g_rapMean = atof(value_of(l).c_str());
        getline(c, l); g_sourceType = atoi(value_of(l).c_str());
    } else {
        std::cerr << "No configuration file found for initial condition parameters\n";
    }
    InitialConditionParameters *ic = (InitialConditionParameters *)params;
    ic->initialConditionType = g_icType;
    ic->numberOfSourceFiles = g_nSource;
    ic->numberOfNucleonsPerNuclei = g_A;
    ic->initialEnergyDensity = g_e0;
    ic->scatteringCrossSectionNN = g_snn;
    ic->impactParameter = g_b;
    ic->fractionOfBinaryCollisions = g_alpha;
    ic->rapidityVariance = g_rapVar;
    ic->rapidityMean = g_rapMean;
    ic->sourceType = g_sourceType;
}

/* optional named keys in <configDir>/b200.properties */
static void read_plugin_properties(const char *configDirectory)
{
    char fname[512];
    snprintf(fname, sizeof fname, "%s/%s", configDirectory, "b200.properties");
    std::ifstream c(fname);
    if (!c.is_open()) return;
    PluginConfig &P = plugin();
    std::string l;
    while (getline(c, l)) {
        l.erase(std::remove_if(l.begin(), l.end(), [](unsigned char ch) { return std::isspace(ch); }), l.end());
        auto pos = l.find('=');
        if (l.empty() || l[0] == '#' || pos == std::string::npos) continue;
        std::string k = l.substr(0, pos), v = l.substr(pos + 1);
        if (k == "theta") P.phys.theta = atof(v.c_str());
        else if (k == "eos") P.phys.eos_kind = (v == "table") ? VH_EOS_TABLE : VH_EOS_CONFORMAL;
        else if (k == "eos_factor") P.phys.eos_factor = atof(v.c_str());
        else if (k == "eos_table") P.eos_table = v;
        else if (k == "bulk") P.phys.bulk = atoi(v.c_str());
        else if (k == "zeta_law") P.phys.zeta_law = (v == "gaussian" || v == "1") ? VH_ZETA_GAUSSIAN : VH_ZETA_REFERENCE;
        else if (k == "zeta_norm") P.phys.zeta_norm = atof(v.c_str());
        else if (k == "zeta_T0_GeV") P.phys.zeta_T0_GeV = atof(v.c_str());
        else if (k == "zeta_width_GeV") P.phys.zeta_width_GeV = atof(v.c_str());
        else if (k == "precision") P.phys.precision = (v == "mixed") ? VH_PREC_MIXED : VH_PREC_FP64;
    }
}

void vh_plugin_set_config(const vh_config *cfg, const char *eos_table_path)
{
    if (cfg) plugin().phys = *cfg;
    if (eos_table_path) plugin().eos_table = eos_table_path;
}

/* -------------------------------------------------------------- run() */
/* HydroPlugin.cpp:74-321 */
void run(void *latticeParams, void *initCondParams, void *hydroParams, const char *rootDirectory,
         const char *outputDir, HydroInitialTmunu init_tmunu)
{
    (void)rootDirectory;
    LatticeParameters &L = *(LatticeParameters *)latticeParams;
    InitialConditionParameters &icp = *(InitialConditionParameters *)initCondParams;
    HydroParameters &H = *(HydroParameters *)hydroParams;
    PluginConfig &P = plugin();

    const int nt = L.numProperTimePoints, nx = L.numLatticePointsX, ny = L.numLatticePointsY, nz = L.numLatticePointsRapidity;
    const int fac = L.coarseProperTimeFOFactor;
    const double t0 = H.initialProperTimePoint, dt = L.latticeSpacingProperTime;

    vh_config cfg = P.phys;
    cfg.nx = nx; cfg.ny = ny; cfg.nz = nz;
    cfg.dx = L.latticeSpacingX; cfg.dy = L.latticeSpacingY; cfg.dz = L.latticeSpacingRapidity; cfg.dt = dt;
    cfg.t0 = t0;
    cfg.etabar = H.shearViscosityToEntropyDensity;
    cfg.T_freezeout_GeV = H.freezeoutTemperatureGeV;
    cfg.T_reg_GeV = H.regulationTemperatureGeV;
    cfg.fo_factor = fac;

    std::vector<double> rows;
    if (cfg.eos_kind == VH_EOS_TABLE) rows = load_eos_table(P.eos_table);
    vh::HostEos eos;
    eos.init(cfg, rows.empty() ? nullptr : rows.data(), (int)(rows.size() / 4));

    const double Tfo = H.freezeoutTemperatureGeV / kHbarc;
    const double eF = eos.energy_of_T(Tfo);
    printf("Grid size = %d x %d x %d\n", nx, ny, nz);
    printf("spatial resolution = (%.3f, %.3f, %.3f)\n", L.latticeSpacingX, L.latticeSpacingY, L.latticeSpacingRapidity);
    printf("freezeout temperature = %.3f [fm^-1] (eF = %.3f [fm^-4])\n", Tfo, eF);
    printf("Coarse graining FO surface by factor %d in proper time\n", fac);
    printf("Regulating viscous currents using : Regulation Scheme 1\n");
    if (!((nx > 1) && (ny > 1))) printf("simulation is not in 3+1D or 2+1D; freezeout finder will not work!\n");

    IC ic;
    if (!build_ic(ic, L, icp, H, eos, cfg.bulk != 0, init_tmunu)) exit(-1);

    vh_event *ev = nullptr;
    die_on(vh_event_create(&cfg, rows.empty() ? nullptr : rows.data(), (int)(rows.size() / 4), &ev), "vh_event_create");
    die_on(vh_event_set_initial(ev, ic.e.data(), ic.p.data(), ic.u.data(), ic.pi.data(), cfg.bulk ? ic.Pi.data() : nullptr),
           "vh_event_set_initial");
    /* thermal vorticity after the initial condition and after every step
     * (THERMAL_VORTICITY is on in the reference, HydroPlugin.cpp:197-199, :302-305) */
    die_on(vh_event_vorticity(ev, 1), "vh_event_vorticity");
    /* the regulation factors the reference dumps (regFacShear, regFacBulk) */
    die_on(vh_event_keep_regulation(ev, 1), "vh_event_keep_regulation");

    SurfaceWriter surf(std::string(outputDir) + "/surface.dat");
    const int ncx = nx + 4, ncy = ny + 4, ncz = nz + 4;
    const int ictr = (nx % 2 == 0) ? ncx / 2 : (ncx - 1) / 2, jctr = (ny % 2 == 0) ? ncy / 2 : (ncy - 1) / 2;
    const int kctr = (nz % 2 == 0) ? ncz / 2 : (ncz - 1) / 2;
    const size_t sctr = ictr + (size_t)ncx * (jctr + (size_t)ncy * kctr);
    std::vector<double> fe((size_t)ncx * ncy * ncz), fp(fe.size());

    double t = t0, total_ms = 0;
    int nsteps = 0, acc2 = 0;
    for (int n = 1; n <= nt + 1; ++n) {
        const bool report = (n - 1) % 100 == 0;
        if (report) {
            die_on(vh_event_get_field(ev, VH_F_E, fe.data()), "vh_event_get_field");
            die_on(vh_event_get_field(ev, VH_F_P, fp.data()), "vh_event_get_field");
            printf("n = %d:%d (t = %.3f),\t (e, p) = (%.3f, %.3f) [fm^-4],\t (T = %.3f [GeV]),\t", n - 1, nt, t, fe[sctr], fp[sctr],
                   eos.temperature(fe[sctr]) * kHbarc);
            dump_field(ev, VH_F_E, "e", t, outputDir, L);
            dump_field(ev, VH_F_UT + 1, "ux", t, outputDir, L);
            dump_field(ev, VH_F_UT + 2, "uy", t, outputDir, L);
            dump_field(ev, VH_F_UT, "ut", t, outputDir, L);
            dump_field(ev, 8, "pixx", t, outputDir, L);
            dump_field(ev, 9, "pixy", t, outputDir, L);
            dump_field(ev, 13, "pinn", t, outputDir, L);
            dump_field(ev, VH_F_REGFAC, "regFacShear", t, outputDir, L);
            if (cfg.bulk) {
                dump_field(ev, 14, "Pi", t, outputDir, L);
                dump_field(ev, VH_F_REGFAC + 1, "regFacBulk", t, outputDir, L);
            }
            dump_field(ev, VH_F_W + 3, "wxy", t, outputDir, L);
            dump_field(ev, VH_F_BETA + 1, "beta_x", t, outputDir, L);
            dump_field(ev, VH_F_BETA + 2, "beta_y", t, outputDir, L);
        }
        if (n % fac == 0) {
            int nel = 0, nabove = 0;
            die_on(vh_event_freezeout(ev, &nel, &nabove), "vh_event_freezeout");
            if (H.doFreezeOut && nel > 0) {
                std::vector<double> el((size_t)nel * VH_FO_COLUMNS);
                die_on(vh_event_fetch_surface(ev, el.data(), nel, &nel), "vh_event_fetch_surface");
                surf.push(std::move(el));
            }
            if (nabove == 0) acc2 += 1;
            if (acc2 >= 3 && icp.initialConditionType != 12) {
                printf("\nAll cells have dropped below freezeout energy density\n");
                break;
            }
        }
        auto a = std::chrono::steady_clock::now();
        die_on(vh_event_step(ev, 1), "vh_event_step");
        if (report) die_on(vh_event_status(ev, nullptr, nullptr), "rungeKutta2");
        double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
        if (report) printf("(Elapsed time: %.3f ms)\n", ms);
        total_ms += ms;
        ++nsteps;
        t = t0 + n * dt;
    }
    die_on(vh_event_status(ev, nullptr, nullptr), "rungeKutta2");
    printf("Average time/step: %.3f ms\n", total_ms / (double)nsteps);
    surf.close();
    vh_event_destroy(ev);
}

/* -------------------------------------------------------------- HYDRO */
HYDRO::HYDRO() {}
HYDRO::~HYDRO() {}

void HYDRO::initialize_from_vector(std::vector<double> e) { initial_energy_density = e; }

void HYDRO::initialize_from_vectors(std::vector<double> e, std::vector<double> ut, std::vector<double> ux,
                                    std::vector<double> uy, std::vector<double> un, std::vector<double> pitt,
                                    std::vector<double> pitx, std::vector<double> pity, std::vector<double> pitn,
                                    std::vector<double> pixx, std::vector<double> pixy, std::vector<double> pixn,
                                    std::vector<double> piyy, std::vector<double> piyn, std::vector<double> pinn,
                                    std::vector<double> Pi)
{
    initial_energy_density = e; initial_ut = ut; initial_ux = ux; initial_uy = uy; initial_un = un;
    initial_pitt = pitt; initial_pitx = pitx; initial_pity = pity; initial_pitn = pitn;
    initial_pixx = pixx; initial_pixy = pixy; initial_pixn = pixn; initial_piyy = piyy; initial_piyn = piyn;
    initial_pinn = pinn; initial_Pi = Pi;
}

static HydroInitialTmunu tmunu_of(const HYDRO &h)
{
    HydroInitialTmunu t;
    t.e_in = h.initial_energy_density; t.ut_in = h.initial_ut; t.ux_in = h.initial_ux; t.uy_in = h.initial_uy;
    t.un_in = h.initial_un; t.pitt_in = h.initial_pitt; t.pitx_in = h.initial_pitx; t.pity_in = h.initial_pity;
    t.pitn_in = h.initial_pitn; t.pixx_in = h.initial_pixx; t.pixy_in = h.initial_pixy; t.pixn_in = h.initial_pixn;
    t.piyy_in = h.initial_piyy; t.piyn_in = h.initial_piyn; t.pinn_in = h.initial_pinn; t.Pi_in = h.initial_Pi;
    return t;
}

/* HydroWrapper.cpp:64-136 */
int HYDRO::run_hydro_no_cli()
{
    const char *configDirectory = "rhic-conf", *outputDirectory = "cpu-vh_output";
    LatticeParameters L;
    InitialConditionParameters icp;
    HydroParameters H;
    char cwd[4096];
    const char *root = getcwd(cwd, sizeof cwd);
    printf("configDirectory = %s\n", configDirectory);
    printf("outputDirectory = %s\n", outputDirectory);
    readLatticeParameters(configDirectory, &L);
    readInitialConditionParameters(configDirectory, &icp);
    readHydroParameters(configDirectory, &H);
    read_plugin_properties(configDirectory);
    auto a = std::chrono::steady_clock::now();
    run(&L, &icp, &H, root ? root : ".", outputDirectory, tmunu_of(*this));
    printf("Done hydro.\n");
    printf("Hydro took %f seconds\n", std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count());
    return 0;
}

/* HydroWrapper.cpp:139-211 with the command line of CommandLineArguments.cpp:17-24 */
int HYDRO::run_hydro(int argc, char **argv)
{
    const char *configDirectory = nullptr, *outputDirectory = nullptr;
    bool runHydro = false, runTest = false;
    static struct option opts[] = {{"test", optional_argument, nullptr, 't'},
                                   {"hydro", optional_argument, nullptr, 'h'},
                                   {"output", required_argument, nullptr, 'o'},
                                   {"config", required_argument, nullptr, 'c'},
                                   {nullptr, 0, nullptr, 0}};
    optind = 1;
    int ch;
    while ((ch = getopt_long(argc, argv, "t::h::o:c:", opts, nullptr)) != -1) {
        if (ch == 't') runTest = true;
        else if (ch == 'h') runHydro = true;
        else if (ch == 'o') outputDirectory = optarg;
        else if (ch == 'c') configDirectory = optarg;
    }
    char cwd[4096];
    const char *root = getcwd(cwd, sizeof cwd);
    printf("configDirectory = %s\n", configDirectory ? configDirectory : "(null)");
    printf("outputDirectory = %s\n", outputDirectory ? outputDirectory : "(null)");
    printf(runHydro ? "runHydro = True\n" : "runHydro = False\n");
    printf(runTest ? "runTest = True\n" : "runTest = False\n");
    LatticeParameters L;
    InitialConditionParameters icp;
    HydroParameters H;
    readLatticeParameters(configDirectory ? configDirectory : "", &L);
    readInitialConditionParameters(configDirectory ? configDirectory : "", &icp);
    readHydroParameters(configDirectory ? configDirectory : "", &H);
    if (configDirectory) read_plugin_properties(configDirectory);
    auto a = std::chrono::steady_clock::now();
    if (runHydro) {
        run(&L, &icp, &H, root ? root : ".", outputDirectory ? outputDirectory : ".", HydroInitialTmunu());
        printf("Done hydro.\n");
    }
    printf("Hydro took %f seconds\n", std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count());
    return 0;
}

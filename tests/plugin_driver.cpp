/* Test driver for the C++ drop-in: the embedding path of HydroWrapper.cpp:20-136
 * (HYDRO::initialize_from_vector + run_hydro_no_cli), reading the energy-density
 * vector from a raw binary file of doubles given as argv[1].  Run it in a
 * directory holding rhic-conf/ and an existing cpu-vh_output/. */
#include <cstdio>
#include <fstream>
#include <vector>
#include "cpu_vh.h"

int main(int argc, char **argv)
{
    if (argc < 2) { fprintf(stderr, "usage: plugin_driver e_vector.bin\n"); return 2; }
    std::ifstream f(argv[1], std::ios::binary);
    std::vector<double> e;
    double v;
    while (f.read((char *)&v, sizeof v)) e.push_back(v);
    HYDRO h;
    h.initialize_from_vector(e);
    return h.run_hydro_no_cli();
}

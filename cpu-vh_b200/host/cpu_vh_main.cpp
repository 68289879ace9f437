/* The `cpu-vh` executable: RunHydroWrapper.cpp:9-19 over the B200 library.
 *   cpu-vh --config rhic-conf/ -o output -h */
#include "cpu_vh.h"

int main(int argc, char **argv)
{
    HYDRO vh;
    vh.run_hydro(argc, argv);
    return 0;
}

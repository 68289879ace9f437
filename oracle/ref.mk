# ref.mk -- TEST INFRASTRUCTURE ONLY: builds the reference's own hot path.
#
# Compiles the unmodified cpu-vh sources where they lie (REF, read-only) into
# shared libraries under oracle/_ref/, together with oracle/ref_harness.cpp.
# Nothing is copied out of REF.  The physics macros that the reference fixes
# inside its headers are overridden by force-including oracle/ref_shim.h.
#
#   make -f oracle/ref.mk                 # all variants
#   make -f oracle/ref.mk REF=/path/to/cpu-vh
#
# Variants (one library each, since the reference keeps its state in globals):
#   conf  : conformal EoS a=15.6269, theta=1.8, shear only  (Gubser 2+1D workload)
#   table : tabulated EoS, theta=1.8, shear + bulk (-DPI)   (Glauber 3+1D workload)
#   stock : the shipped macros (conformal a=13.8997, theta=1.1, shear only)
#
# Flags: the shipped ones (CMakeLists.txt:14, -O3 -fopenmp -std=c++11) with
# -ffp-contract=off so the arithmetic is the literal IEEE program of the source
# (GCC would otherwise fuse multiply-adds of its own choosing), and a portable
# x86-64-v3 target instead of -march=native so the binary runs on any AVX2 host.
REF ?= $(if $(VH_REFERENCE),$(VH_REFERENCE),/root/reference)
OUT ?= oracle/_ref
HOSTCXX ?= g++
CXXFLAGS_BASE = -O3 -fopenmp -std=c++11 -march=x86-64-v3 -ffp-contract=off -fPIC -w \
                -I$(REF)/rhic/include -I$(REF)/freezeout -include oracle/ref_shim.h
LDFLAGS = -shared -fopenmp -Wl,-Bsymbolic

SRC_NAMES = DynamicalVariables EnergyMomentumTensor EquationOfState FileIO FluxFunctions \
            FluxLimiter FullyDiscreteKurganovTadmorScheme HalfSiteExtrapolation HydroPlugin \
            LocalPropagationSpeed SemiDiscreteKurganovTadmorScheme SourceTerms SpectralRadius \
            Vorticity FiniteDifference LatticeParameters HydroParameters InitialConditionParameters
SRCS = $(addprefix $(REF)/rhic/src/,$(addsuffix .cpp,$(SRC_NAMES))) oracle/ref_harness.cpp
# the seeded workload generators (C, compiled here as C++): the reference's
# inputs are made without the CUDA library
GEN = oracle/workload_gen.c

DEFS_conf  = -DVH_THETA=1.8 -DVH_EOS_FACTOR=15.6269
DEFS_table = -DVH_THETA=1.8 -DVH_EOS_FACTOR=15.6269 -DVH_EOS_TABLE -DPI
DEFS_stock = -DVH_THETA=1.1 -DVH_EOS_FACTOR=13.8997

# The Glauber workload's variant again as the shipped CMake flags build it
# (CMakeLists.txt:14: -O3 -fopenmp -std=c++11 -march=native, with GCC's own
# multiply-add contraction), for the benchmark's timing only: its arithmetic
# is then compiler-dependent, so no parity test uses it.  -march names the
# GPU hosts' processor family (native to the build host might not run on
# every host the library travels to): the GPU hosts' Xeons (Sapphire and
# Emerald Rapids) run sapphirerapids code; bench.py checks the host's flags
# before it loads this library.
SHIPPED_MARCH ?= sapphirerapids
CXXFLAGS_SHIPPED = -O3 -fopenmp -std=c++11 -march=$(SHIPPED_MARCH) -fPIC -w \
                   -I$(REF)/rhic/include -I$(REF)/freezeout -include oracle/ref_shim.h

all: $(OUT)/libvhref_conf.so $(OUT)/libvhref_table.so $(OUT)/libvhref_stock.so $(OUT)/libvhref_table_shipped.so

# DynamicalVariables.cpp is compiled with its setGhostCells renamed away: the
# reference's version declares its loop indices outside `omp parallel for`
# (DynamicalVariables.cpp:290-291, :324-325, :358-359), a data race that
# corrupts cells when more than one thread runs.  ref_harness.cpp supplies the
# same three loop nests with private indices, so any thread count reproduces
# the single-thread reference exactly.
DV = $(REF)/rhic/src/DynamicalVariables.cpp
SRCS_NO_DV = $(filter-out $(DV),$(SRCS))

$(OUT)/libvhref_%.so: $(SRCS) $(GEN) oracle/ref_shim.h oracle/ref.mk
	@mkdir -p $(OUT)/obj_$*
	$(HOSTCXX) $(CXXFLAGS_BASE) $(DEFS_$*) -DsetGhostCells=vhref_setGhostCells_racy -c $(DV) -o $(OUT)/obj_$*/dv.o
	$(HOSTCXX) -O2 -march=x86-64-v3 -ffp-contract=off -fPIC -x c++ -c $(GEN) -o $(OUT)/obj_$*/gen.o
	$(HOSTCXX) $(CXXFLAGS_BASE) $(DEFS_$*) -DVH_RACE_FREE_GHOSTS $(SRCS_NO_DV) $(OUT)/obj_$*/dv.o $(OUT)/obj_$*/gen.o \
	    $(LDFLAGS) -o $@

$(OUT)/libvhref_table_shipped.so: $(SRCS) $(GEN) oracle/ref_shim.h oracle/ref.mk
	@mkdir -p $(OUT)/obj_table_shipped
	$(HOSTCXX) $(CXXFLAGS_SHIPPED) $(DEFS_table) -DsetGhostCells=vhref_setGhostCells_racy -c $(DV) \
	    -o $(OUT)/obj_table_shipped/dv.o
	$(HOSTCXX) -O2 -march=x86-64-v3 -ffp-contract=off -fPIC -x c++ -c $(GEN) -o $(OUT)/obj_table_shipped/gen.o
	$(HOSTCXX) $(CXXFLAGS_SHIPPED) $(DEFS_table) -DVH_RACE_FREE_GHOSTS $(SRCS_NO_DV) $(OUT)/obj_table_shipped/dv.o \
	    $(OUT)/obj_table_shipped/gen.o $(LDFLAGS) -o $@
	@echo "g++ -O3 -fopenmp -std=c++11 -march=$(SHIPPED_MARCH) (contraction on), race-fixed setGhostCells" \
	    > $(OUT)/shipped_flags.txt

clean:
	rm -rf $(OUT)/libvhref_*.so $(OUT)/obj_*

.PHONY: all clean

# Build recipe for the reference CPU implementation (test infrastructure only).
#
# Compiles MercuryDPM's Kernel straight from its sources under REF (read-only;
# nothing is copied) into oracle/_ref/, in the two variants the reference's own
# CMake produces for the DEM path:
#   serial : default options, MERCURYDPM_TRIANGLE_WALL_CORRECTION on
#            (reference CMakeLists.txt:79-88)
#   omp    : -fopenmp -DMERCURYDPM_USE_OMP, triangle-wall correction off
#            (reference CMakeModules/MercuryDPM_OMP.cmake)
# The Fortran BLAS/LAPACK subset (Kernel/Math/*.f) is replaced by stubs that
# abort: only SmallMatrix uses it and the DEM time step never does.
# The reference-API drivers in oracle/ref_drivers/ are linked against each
# variant into oracle/_ref/libmdpm_ref_{serial,omp}.so (extern "C" entry points
# used by tests/ and by bench.py's reference arm).
#
# Usage:  make -f oracle/ref.mk -j8 REF=<reference checkout>
#         (or with the checkout in $MERCURYDPM_REF)
REF ?= $(MERCURYDPM_REF)
ifeq ($(strip $(REF)),)
$(error give the reference checkout: REF=<path> or MERCURYDPM_REF=<path>)
endif
OUT := oracle/_ref
K   := $(REF)/Kernel

KSRC := BaseObject.cc BaseInteractable.cc BaseCluster.cc Logger.cc File.cc DPMBase.cc \
        MpiContainer.cc MpiDataClass.cc HGrid.cc MercuryBase.cc Mercury2D.cc Mercury3D.cc \
        HGridOptimiser.cc BoundaryHandler.cc PeriodicBoundaryHandler.cc InteractionHandler.cc \
        ParticleHandler.cc SpeciesHandler.cc WallHandler.cc DomainHandler.cc Domain.cc \
        BinaryReader.cc Chute.cc ChuteBottom.cc
KGLOB := Boundaries/*.cc CG/*.cc CG/*/*.cc FMM/*.cc Math/*.cc Math/*/*.cc Mixins/*.cc \
         Particles/*.cc Strings/*.cc VTKWriter/*.cc Walls/*.cc Walls/*/*.cc Interactions/*.cc \
         Interactions/*/*.cc Species/*.cc Species/*/*.cc Nurbs/*.cc Tools/*.cc Controllers/*.cc \
         Helpers/*.cc
SRCS := $(KSRC) $(patsubst $(K)/%,%,$(wildcard $(addprefix $(K)/,$(KGLOB))))

CXX      ?= g++
BASEFLAGS := -std=c++17 -O3 -DNDEBUG -DUNIX -fPIC -w -DMERCURYDPM_LOGLEVEL=Log::DEFAULT \
             -I$(K) -I$(OUT)/gen
SERIALFLAGS := $(BASEFLAGS) -DMERCURYDPM_TRIANGLE_WALL_CORRECTION
OMPFLAGS    := $(BASEFLAGS) -fopenmp -DMERCURYDPM_USE_OMP

SOBJS := $(addprefix $(OUT)/obj/serial/,$(SRCS:.cc=.o)) $(OUT)/obj/serial/CMakeDefinitions.o
OOBJS := $(addprefix $(OUT)/obj/omp/,$(SRCS:.cc=.o)) $(OUT)/obj/omp/CMakeDefinitions.o

DRIVERS := $(wildcard oracle/ref_drivers/*.cpp)

all: $(OUT)/libmdpm_ref_serial.so $(OUT)/libmdpm_ref_omp.so

$(OUT)/gen/CMakeDefinitions.h: $(REF)/Configuration/CMakeDefinitions.h
	@mkdir -p $(@D)
	sed -e 's/@MercuryDPM_BACKTRACE_ENABLE@/OFF/' -e 's/@MercuryDPM_BACKTRACE_DEMANGLE@/OFF/' $< > $@

$(OUT)/gen/CMakeDefinitions.cc: $(REF)/Configuration/CMakeDefinitions.cc
	@mkdir -p $(@D)
	sed -e 's|@MercuryDPM_SOURCE_DIR@|$(REF)|' -e 's|@MercuryDPM_BINARY_DIR@|$(OUT)|' \
	    -e 's/@REVISION@/unknown/' -e 's/@REPOSITORY_URL@/unknown/' \
	    -e 's/@MercuryDPM_VERSION_MAJOR@/1/' -e 's/@MercuryDPM_VERSION_MINOR@/0/' $< > $@

$(OUT)/obj/serial/%.o: $(K)/%.cc $(OUT)/gen/CMakeDefinitions.h
	@mkdir -p $(@D)
	$(CXX) $(SERIALFLAGS) -c $< -o $@

$(OUT)/obj/omp/%.o: $(K)/%.cc $(OUT)/gen/CMakeDefinitions.h
	@mkdir -p $(@D)
	$(CXX) $(OMPFLAGS) -c $< -o $@

$(OUT)/obj/serial/CMakeDefinitions.o: $(OUT)/gen/CMakeDefinitions.cc $(OUT)/gen/CMakeDefinitions.h
	@mkdir -p $(@D)
	$(CXX) $(SERIALFLAGS) -c $< -o $@

$(OUT)/obj/omp/CMakeDefinitions.o: $(OUT)/gen/CMakeDefinitions.cc $(OUT)/gen/CMakeDefinitions.h
	@mkdir -p $(@D)
	$(CXX) $(OMPFLAGS) -c $< -o $@

# The OpenMP runtime is linked by path: some g++ wrappers on this image lack
# the libgomp spec file that a plain `-fopenmp` link needs.
GOMP ?= $(firstword $(wildcard /usr/lib/x86_64-linux-gnu/libgomp.so.1 /usr/lib64/libgomp.so.1))

SDRV := $(patsubst oracle/ref_drivers/%.cpp,$(OUT)/obj/serial/drv_%.o,$(DRIVERS)) $(OUT)/obj/serial/ref_stubs.o
ODRV := $(patsubst oracle/ref_drivers/%.cpp,$(OUT)/obj/omp/drv_%.o,$(DRIVERS)) $(OUT)/obj/omp/ref_stubs.o

$(OUT)/obj/serial/drv_%.o: oracle/ref_drivers/%.cpp oracle/ref_drivers/ref_driver.h include/dem_b200.h $(OUT)/gen/CMakeDefinitions.h
	@mkdir -p $(@D)
	$(CXX) $(SERIALFLAGS) -c $< -o $@

$(OUT)/obj/omp/drv_%.o: oracle/ref_drivers/%.cpp oracle/ref_drivers/ref_driver.h include/dem_b200.h $(OUT)/gen/CMakeDefinitions.h
	@mkdir -p $(@D)
	$(CXX) $(OMPFLAGS) -c $< -o $@

$(OUT)/obj/%/ref_stubs.o: oracle/ref_stubs.cc
	@mkdir -p $(@D)
	$(CXX) -O2 -fPIC -c $< -o $@

# Like the reference's own build, the Kernel is a static archive: only the
# objects a driver needs are linked (some unused classes have undefined members).
$(OUT)/libMercuryBase_serial.a: $(SOBJS)
	rm -f $@ && ar rcs $@ $(SOBJS)

$(OUT)/libMercuryBase_omp.a: $(OOBJS)
	rm -f $@ && ar rcs $@ $(OOBJS)

# The shared libraries are loaded into Python processes: link them against the
# shared libstdc++ (a static copy inside a dlopen'ed library has no
# initialised iostream locale, and the reference prints through std::cout).
LINKCXX ?= $(firstword $(wildcard /usr/bin/g++) $(CXX))

$(OUT)/libmdpm_ref_serial.so: $(OUT)/libMercuryBase_serial.a $(SDRV)
	$(LINKCXX) -shared -o $@ $(SDRV) $(OUT)/libMercuryBase_serial.a

$(OUT)/libmdpm_ref_omp.so: $(OUT)/libMercuryBase_omp.a $(ODRV)
	$(LINKCXX) -shared -o $@ $(ODRV) $(OUT)/libMercuryBase_omp.a $(GOMP) -lpthread

.PHONY: all

# The engine's drop-in base class (mercurydpm_fork_b200/mercury/GpuTimeStep.h)
# compiled into reference drivers, linked against the serial Kernel and the
# engine library (found next to this checkout at run time through $ORIGIN):
#   gpu_tangential_spring_unit_test : the reference's own
#       Drivers/UnitTests/TangentialSpringUnitTest.cpp, unmodified, with its
#       base class DPMBase replaced by GpuDPMBase (oracle/ref_drivers/gpu/)
#   libmdpm_gpu_binding.so : RefDriverT<GpuMercury3D>, the checker's driver on
#       the drop-in base class (solve() with the reference's .ene writer)
ENGINE_LIB := mercurydpm_fork_b200/libdem_b200.so
BINDING := mercurydpm_fork_b200/mercury/GpuTimeStep.h
GPUFLAGS := $(SERIALFLAGS) -I$(REF) -Imercurydpm_fork_b200/mercury -Iinclude -Ioracle/ref_drivers
GPULINK := $(OUT)/libMercuryBase_serial.a $(OUT)/obj/serial/ref_stubs.o -Lmercurydpm_fork_b200 -ldem_b200 \
           -Wl,-rpath,'$$ORIGIN/../../mercurydpm_fork_b200'

SELFTESTS := ForceSelfTest FreeFallSelfTest
SELFTEST_SRC_ForceSelfTest := $(REF)/Drivers/SelfTests/Interactions/ForceSelfTest.cpp
SELFTEST_SRC_FreeFallSelfTest := $(REF)/Drivers/SelfTests/Interactions/FreeFallSelfTest.cpp
SELFTEST_GPU_ForceSelfTest := oracle/ref_drivers/gpu/force_self_test.cpp
SELFTEST_GPU_FreeFallSelfTest := oracle/ref_drivers/gpu/free_fall_self_test.cpp

gpu: $(OUT)/gpu_tangential_spring_unit_test $(OUT)/libmdpm_gpu_binding.so \
     $(foreach t,$(SELFTESTS),$(OUT)/selftest_$(t)_reference $(OUT)/selftest_$(t)_gpu)

# the reference's self tests as they are (the CPU reference run) ...
$(OUT)/selftest_%_reference: $(OUT)/libMercuryBase_serial.a $(OUT)/obj/serial/ref_stubs.o
	$(LINKCXX) $(SERIALFLAGS) $(SELFTEST_SRC_$*) -o $@ $(OUT)/libMercuryBase_serial.a $(OUT)/obj/serial/ref_stubs.o

# ... and with their base class swapped for the engine's
.SECONDEXPANSION:
$(OUT)/selftest_%_gpu: $$(SELFTEST_GPU_$$*) $(BINDING) $(ENGINE_LIB) $(OUT)/libMercuryBase_serial.a \
        $(OUT)/obj/serial/ref_stubs.o
	$(LINKCXX) $(GPUFLAGS) $(SELFTEST_GPU_$*) -o $@ $(GPULINK)

$(OUT)/gpu_tangential_spring_unit_test: oracle/ref_drivers/gpu/tangential_spring_unit_test.cpp $(BINDING) \
        $(ENGINE_LIB) $(OUT)/libMercuryBase_serial.a $(OUT)/obj/serial/ref_stubs.o
	$(LINKCXX) $(GPUFLAGS) $< -o $@ $(GPULINK)

$(OUT)/libmdpm_gpu_binding.so: oracle/ref_drivers/gpu/gpu_binding_driver.cpp oracle/ref_drivers/ref_driver.h \
        $(BINDING) $(ENGINE_LIB) $(OUT)/libMercuryBase_serial.a $(OUT)/obj/serial/ref_stubs.o
	$(LINKCXX) $(GPUFLAGS) -shared $< -o $@ $(GPULINK)

.PHONY: gpu

objs: $(SOBJS) $(OOBJS)
.PHONY: objs

# Builds the reference's own host set-up code (input readers, domain and
# particle initialisation: src/domain.c, src/particle.c, src/rng.c) from the
# reference tree, unmodified, into oracle/_ref/libref_host.so.  The process
# globals normally defined in src/bluebottle.c (which needs MPI) come from a
# translation unit generated from the reference headers' extern
# declarations by oracle/ref_shim.py; src/recorder.h's CGNS include is met
# by an empty stub header.  Test infrastructure only.
#
#   make -f oracle/ref.mk REF=/path/to/reference/src
# (default: $BLUEBOTTLE_REF/src, the checkout at /root/reference otherwise)
BLUEBOTTLE_REF ?= /root/reference
REF ?= $(BLUEBOTTLE_REF)/src
HERE := $(dir $(lastword $(MAKEFILE_LIST)))
OUT := $(HERE)_ref
CC = gcc
CFLAGS = -std=gnu99 -O2 -fPIC -fopenmp -DDOUBLE -w -I$(OUT) -I$(REF)

all: $(OUT)/libref_host.so $(OUT)/libref_host_implicit.so $(OUT)/libref_dropin.so

$(OUT)/cgnslib.h:
	mkdir -p $(OUT)
	: > $@

$(OUT)/ref_globals.c: $(HERE)ref_shim.py | $(OUT)/cgnslib.h
	python3 $(HERE)ref_shim.py $(REF) $@

$(OUT)/%.o: $(REF)/%.c $(OUT)/cgnslib.h
	$(CC) $(CFLAGS) -c $< -o $@

$(OUT)/ref_globals.o: $(OUT)/ref_globals.c
	$(CC) $(CFLAGS) -c $< -o $@

$(OUT)/libref_host.so: $(OUT)/domain.o $(OUT)/particle.o $(OUT)/rng.o $(OUT)/ref_globals.o
	$(CC) -shared -fopenmp -o $@ $^ -lm -Wl,--no-undefined

# the same sources built as the Crank-Nicolson (-DIMPLICIT) program, whose
# restart file omits the diffusion histories (src/domain.c:3242)
$(OUT)/%_i.o: $(REF)/%.c $(OUT)/cgnslib.h
	$(CC) $(CFLAGS) -DIMPLICIT -c $< -o $@

$(OUT)/libref_host_implicit.so: $(OUT)/domain_i.o $(OUT)/particle_i.o $(OUT)/rng_i.o $(OUT)/ref_globals.o
	$(CC) -shared -fopenmp -o $@ $^ -lm -Wl,--no-undefined

clean:
	rm -f $(OUT)/*.o $(OUT)/*.so $(OUT)/ref_globals.c $(OUT)/cgnslib.h

# The drop-in link: the reference's own host files (set-up, readers, the
# VTK writer) compiled unmodified and linked against libbbb200.so, whose
# globals they then use -- the way src/bluebottle.c's program links the
# library.  Built after the library (python -m bluebottle_b200.build).
LIB := $(HERE)../bluebottle_b200
$(OUT)/%_d.o: $(REF)/%.c $(OUT)/cgnslib.h
	$(CC) $(CFLAGS) -c $< -o $@

$(OUT)/libref_dropin.so: $(OUT)/domain_d.o $(OUT)/particle_d.o $(OUT)/rng_d.o $(OUT)/vtk_d.o $(LIB)/libbbb200.so
	$(CC) -shared -fopenmp -o $@ $(OUT)/domain_d.o $(OUT)/particle_d.o $(OUT)/rng_d.o \
	  $(OUT)/vtk_d.o -L$(LIB) -lbbb200 -lm -Wl,--no-undefined \
	  -Wl,-rpath,'$$ORIGIN/../../bluebottle_b200'

# The reference's own CUDA files -- all but src/cuda_bicgstab.cu (it needs
# CUSP, which the reference does not ship) and src/cuda_testing.cu --
# compiled unmodified for sm_100a and linked with the host set-up above
# into oracle/_ref/libref_gpu.so: the reference's GPU kernels behind its
# own cuda_* entry points, which tests/test_gpu_refkernels.py compares this
# library's non-solver entry points with.  `make -f oracle/ref.mk gpu`.
NVCC = nvcc
NVFLAGS = -gencode arch=compute_100a,code=sm_100a -O2 -DDOUBLE -w \
  -Xcompiler -fPIC,-fopenmp -I$(OUT) -I$(REF)
CUSRC = bluebottle_kernel particle_kernel quadrature_kernel entrySearch_kernel \
  cuda_bluebottle cuda_particle cuda_quadrature entrySearch bicgstab_kernel

$(OUT)/%_g.o: $(REF)/%.cu $(OUT)/cgnslib.h
	$(NVCC) $(NVFLAGS) -c $< -o $@

# the assembly half of src/cuda_bicgstab.cu's pressure solve, restated
# (the other half is CUSP)
$(OUT)/ref_pp_shim.o: $(HERE)ref_pp_shim.cu $(OUT)/cgnslib.h
	$(NVCC) $(NVFLAGS) -c $< -o $@

$(OUT)/libref_gpu.so: $(CUSRC:%=$(OUT)/%_g.o) $(OUT)/ref_pp_shim.o $(OUT)/domain.o \
  $(OUT)/particle.o $(OUT)/rng.o $(OUT)/ref_globals.o
	$(NVCC) -gencode arch=compute_100a,code=sm_100a -shared -Xcompiler -fopenmp \
	  -o $@ $^ -lgomp -Xlinker --no-undefined

# the same, built as the Crank-Nicolson (-DIMPLICIT) program
$(OUT)/%_gi.o: $(REF)/%.cu $(OUT)/cgnslib.h
	$(NVCC) $(NVFLAGS) -DIMPLICIT -c $< -o $@

$(OUT)/ref_pp_shim_i.o: $(HERE)ref_pp_shim.cu $(OUT)/cgnslib.h
	$(NVCC) $(NVFLAGS) -DIMPLICIT -c $< -o $@

$(OUT)/libref_gpu_implicit.so: $(CUSRC:%=$(OUT)/%_gi.o) $(OUT)/ref_pp_shim_i.o \
  $(OUT)/domain_i.o $(OUT)/particle_i.o $(OUT)/rng_i.o $(OUT)/ref_globals.o
	$(NVCC) -gencode arch=compute_100a,code=sm_100a -shared -Xcompiler -fopenmp \
	  -o $@ $^ -lgomp -Xlinker --no-undefined

gpu: $(OUT)/libref_gpu.so $(OUT)/libref_gpu_implicit.so

.PHONY: all clean gpu

# Builds the reference SuiteSparse:GraphBLAS v9.3.1 library from its own
# sources (read-only tree given by REF) with plain gcc, no cmake.  Output goes
# only to oracle/_ref/.  The configuration matches a stock release build with
# the CPU JIT off (-DNJIT), OpenMP on and the factory kernels compiled in.
# The cpu_features helper is disabled (-DGBNCPUFEAT); the library then picks
# its AVX paths from compiler macros instead of a run-time probe.  The two
# files cmake would configure (Config/GB_config.h, whose strings only the
# disabled JIT reads, and the no-JIT JITpackage/GB_JITpackage.c) are generated
# from their templates into oracle/_ref/gen when the tree does not hold them.
#
#   make -f oracle/ref.mk -j8        (REF defaults to BASELINE.json's reference_path)
#
# The library is test infrastructure: the parity tests and the CPU-baseline
# leg of bench.py load it as the checker; no product code links it.

REF    ?= $(shell sed -n 's/.*"reference_path": *"\([^"]*\)".*/\1/p' BASELINE.json)
OUT    := oracle/_ref
OBJ    := $(OUT)/obj
GEN    := $(OUT)/gen
CC     := /usr/bin/gcc
INCS   := -I$(GEN) -I$(REF) -I$(REF)/Source -I$(REF)/Include -I$(REF)/Config \
          -I$(REF)/xxHash -I$(REF)/lz4 -I$(REF)/zstd -I$(REF)/zstd/zstd_subset \
          -I$(REF)/JITpackage -I$(REF)/Demo/Include \
          $(foreach d,apply assign builder builtin callback concat convert ewise \
            hyper jit_kernels math memory monoid mxm ok omp print reduce select \
            split slice transpose type wait werk,-I$(REF)/Source/$(d))
CFLAGS := -O3 -DNDEBUG -fPIC -fopenmp -std=c11 -Wno-pragmas -Wundef -w \
          -fexcess-precision=fast -fcx-limited-range -fno-math-errno -fwrapv \
          -DNJIT -DGBNCPUFEAT

SRCS := $(wildcard $(REF)/PreJIT/*.c) $(wildcard $(REF)/Config/*.c) \
        $(wildcard $(REF)/Source/*/*.c) $(wildcard $(REF)/FactoryKernels/*.c)
OBJS := $(patsubst $(REF)/%.c,$(OBJ)/%.o,$(SRCS))

# JIT package: the tree's own file when cmake made one, else the no-JIT one
ifneq ($(wildcard $(REF)/JITpackage/GB_JITpackage.c),)
OBJS += $(OBJ)/JITpackage/GB_JITpackage.o
else
OBJS += $(OBJ)/gen/GB_JITpackage.o
endif
CONFIG_H := $(if $(wildcard $(REF)/Config/GB_config.h),,$(GEN)/GB_config.h)

all: $(OUT)/libgraphblas_ref.so

$(GEN)/GB_config.h: $(REF)/Config/GB_config.h.in
	@mkdir -p $(GEN)
	sed -e 's/@GB_LIB_PREFIX@/lib/' -e 's/@GB_LIB_SUFFIX@/.so/' \
	    -e 's/@GB_OBJ_SUFFIX@/.o/' -e 's/@[A-Z_]*@//g' $< > $@

$(GEN)/GB_JITpackage.c: $(REF)/Config/GB_JITpackage_NJIT.c.in
	@mkdir -p $(GEN)
	cp $< $@

$(OBJ)/gen/GB_JITpackage.o: $(GEN)/GB_JITpackage.c
	@mkdir -p $(dir $@)
	@$(CC) $(CFLAGS) $(INCS) -c $< -o $@

$(OBJ)/%.o: $(REF)/%.c | $(CONFIG_H)
	@mkdir -p $(dir $@)
	@$(CC) $(CFLAGS) $(INCS) -c $< -o $@

$(OUT)/libgraphblas_ref.so: $(OBJS)
	$(CC) -shared -fopenmp -o $@ $(OBJS) -lm -ldl -Wl,-soname,libgraphblas_ref.so

.PHONY: all

# The same reference library with its GB_AxB_dot3 / GB_AxB_saxpy3 calls routed
# to libgrb_b200.so by the maintainer's shim (graphblas_b200/integration/
# gb_b200_gateway.c) through link-time wrapping: the drop-in, demonstrated on
# the real library.  GB_B200=1 in the environment switches the GPU on.
GW      := graphblas_b200/integration/gb_b200_gateway.c
GRBLIB  := graphblas_b200/lib
WRAPPED := $(OUT)/libgraphblas_b200wrap.so

wrap: $(WRAPPED) $(OUT)/libref_runner_wrap.so

$(OBJ)/gb_b200_gateway.o: $(GW) include/grb_b200.h
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) $(INCS) -Iinclude -c $< -o $@

$(WRAPPED): $(OBJS) $(OBJ)/gb_b200_gateway.o $(GRBLIB)/libgrb_b200.so
	$(CC) -shared -fopenmp -o $@ $(OBJS) $(OBJ)/gb_b200_gateway.o \
	    -Wl,--wrap=GB_AxB_dot3 -Wl,--wrap=GB_AxB_saxpy3 \
	    -L$(GRBLIB) -lgrb_b200 -Wl,-rpath,'$$ORIGIN/../../$(GRBLIB)' \
	    -lm -ldl -Wl,-soname,libgraphblas_b200wrap.so

$(OUT)/libref_runner_wrap.so: oracle/ref_runner.c $(WRAPPED)
	$(CC) -O2 -fopenmp -fPIC -shared -std=gnu11 -I$(REF)/Include -o $@ $< \
	    -L$(OUT) -lgraphblas_b200wrap -Wl,-rpath,'$$ORIGIN'

.PHONY: wrap

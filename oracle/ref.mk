# Builds the reference JXFPAMG library from its own C sources into oracle/_ref/
# as a CPU test oracle (FP64: no JXF_SINGLE, as the reference's headers select
# double when it is undefined).  Object files and the shared library go only
# under oracle/_ref/, which is git-ignored.  The reference's own build system
# is not used; this recipe compiles its sources directly with a single-rank
# MPI shim (oracle/mpi_shim) in place of an MPI installation.
#
#   make -f oracle/ref.mk REF=/root/reference -j8
#
REF     ?= /root/reference
override CC := gcc
ORACLE  := $(patsubst %/,%,$(dir $(lastword $(MAKEFILE_LIST))))
OUT     := $(ORACLE)/_ref
SRCROOT := $(REF)/jxfpamg-0220/csrc
SUBDIRS := operation/blas operation/lapack utilities amg krylov mat_vec_data multils apctl \
           diagscale euclid combined cpr ilu communication operation/matops operation/mvops \
           operation/relaxations operation/vecops operation/tmpops
SRCS    := $(foreach d,$(SUBDIRS),$(wildcard $(SRCROOT)/$(d)/*.c))
OBJ64   := $(patsubst $(SRCROOT)/%.c,$(OUT)/obj64/%.o,$(SRCS))
OBJ32   := $(patsubst $(SRCROOT)/%.c,$(OUT)/obj32/%.o,$(SRCS))
DEFS    := -DJXF_USING_OPENMP=1 -DJXF_USING_BIG_INT=0 -DJXF_USING_BIG_DOUBLE=0 -DJXF_USING_MUMPS=0
CFLAGS  := -O2 -fPIC -fopenmp -ffp-contract=off -w -std=gnu99 \
           -I$(ORACLE)/mpi_shim -I$(REF)/jxfpamg-0220/include $(DEFS)

all: $(OUT)/libjxf_ref64.so

$(OUT)/obj64/%.o: $(SRCROOT)/%.c
	@mkdir -p $(dir $@)
	@$(CC) $(CFLAGS) -c $< -o $@

$(OUT)/obj32/%.o: $(SRCROOT)/%.c
	@mkdir -p $(dir $@)
	@$(CC) $(CFLAGS) -DJXF_SINGLE=1 -c $< -o $@

$(OUT)/mpi_shim.o: $(ORACLE)/mpi_shim/mpi_shim.c $(ORACLE)/mpi_shim/mpi.h
	@mkdir -p $(OUT)
	$(CC) -O2 -fPIC -I$(ORACLE)/mpi_shim -c $< -o $@

$(OUT)/ref_driver64.o: $(ORACLE)/ref_driver.c
	@mkdir -p $(OUT)
	$(CC) $(CFLAGS) -c $< -o $@

$(OUT)/ref_stubs.o: $(ORACLE)/ref_stubs.c
	@mkdir -p $(OUT)
	$(CC) -O2 -fPIC -c $< -o $@

$(OUT)/libjxf_ref64.so: $(OBJ64) $(OUT)/mpi_shim.o $(OUT)/ref_stubs.o $(OUT)/ref_driver64.o
	@$(CC) -shared -fopenmp -Wl,--allow-multiple-definition -o $@ $^ -lm

clean:
	rm -rf $(OUT)/obj64 $(OUT)/obj32 $(OUT)/*.o $(OUT)/*.so

.PHONY: all clean

# Builds the reference's own example programs, unchanged, against the
# cabanapd_b200 front end (include/CabanaPD.hpp over the C ABI library):
# the drop-in proof. The sources are read where they lie in the CabanaPD
# tree named by REFERENCE; the binaries go to oracle/_ref/ only (ignored by
# git, shipped with the built library). tests/test_reference_programs.py
# runs them with the reference's regression decks.
#   make -f oracle/reference_programs.mk REFERENCE=<CabanaPD tree>
# (run from the repository root, after the library is built).
REFERENCE ?= /root/reference
NVCC ?= /usr/local/cuda/bin/nvcc
ARCH := -gencode arch=compute_100a,code=sm_100a
OUTDIR := oracle/_ref
LIB := cabanapd_b200/_lib/libcabanapd_b200.so
FLAGS := -x cu --extended-lambda -std=c++17 $(ARCH) -O2 -I include -I include/cabanapd_shim/compat
LINK := -L cabanapd_b200/_lib -lcabanapd_b200 -Xlinker -rpath,'$$ORIGIN/../../cabanapd_b200/_lib'
HDRS := $(wildcard include/*.h include/*.hpp include/cabanapd_shim/*.hpp include/cabanapd_shim/compat/*)

PROGS := $(OUTDIR)/kalthoff_winkler $(OUTDIR)/elastic_wave $(OUTDIR)/powder_fill

all: $(PROGS)

$(OUTDIR)/kalthoff_winkler: $(REFERENCE)/examples/mechanics/kalthoff_winkler.cpp $(HDRS) $(LIB)
	mkdir -p $(OUTDIR)
	$(NVCC) $(FLAGS) $< $(LINK) -o $@

$(OUTDIR)/elastic_wave: $(REFERENCE)/examples/mechanics/elastic_wave.cpp $(HDRS) $(LIB)
	mkdir -p $(OUTDIR)
	$(NVCC) $(FLAGS) $< $(LINK) -o $@

$(OUTDIR)/powder_fill: $(REFERENCE)/examples/dem/powder_fill.cpp $(HDRS) $(LIB)
	mkdir -p $(OUTDIR)
	$(NVCC) $(FLAGS) $< $(LINK) -o $@

.PHONY: all

# Builds the reference implementation from its own sources (read in place
# under REF) into oracle/_ref/ -- test infrastructure and CPU baseline only.
#
#   make -f oracle/ref.mk REF=<reference tree>     (from the repository root)
#
# REF defaults to $TURBOCAT_REFERENCE; with neither set the build stops with a
# message (__graft_entry__.build passes REF explicitly).
#
# Outputs (git-ignored):
#   oracle/_ref/libtcref.so                       probe harness (C entry points)
#   oracle/_ref/_turbocat<ext-suffix>             the reference's pybind11 module
#
# Flags follow the reference's CMakeLists.txt:31-65 (AVX2 + FMA, OpenMP, -O3,
# AVX-512 off).  src/tree/gradtree.cpp is left out (it needs Eigen, which is
# absent; GradTree is off the symmetric path); oracle/refshim supplies a
# stand-in Eigen header for tree.hpp and throwing definitions of the symbols
# whose sources are missing from the reference tree.
REF      ?= $(TURBOCAT_REFERENCE)
ifeq ($(strip $(REF)),)
$(error set REF=<reference source tree> or TURBOCAT_REFERENCE)
endif
OUT      := oracle/_ref
PY       ?= python3
CXX      := /usr/bin/g++
EXT      := $(shell $(PY)-config --extension-suffix 2>/dev/null || echo .so)
PYINC    := $(shell $(PY) -c "import sysconfig;print(sysconfig.get_paths()['include'])")
PBINC    := $(shell $(PY) -c "import pybind11;print(pybind11.get_include())")
CXXFLAGS := -std=c++20 -O3 -DNDEBUG -mavx2 -mfma -funroll-loops -DTURBOCAT_AVX2 -DTURBOCAT_FMA \
            -fopenmp -fPIC -w -I$(REF)/include -Ioracle/refshim

SRCS := core/dataset.cpp core/config.cpp core/types.cpp \
        boosting/loss.cpp boosting/booster.cpp \
        tree/symmetric_tree.cpp tree/tree.cpp tree/histogram.cpp tree/fast_float_ensemble.cpp \
        tree/fast_ensemble.cpp tree/feature_orderings.cpp tree/flat_tree.cpp \
        tree/leaf_wise_tree.cpp tree/feature_bundler.cpp tree/splitter.cpp \
        utils/simd.cpp utils/threading.cpp
OBJS := $(addprefix $(OUT)/obj/,$(subst /,_,$(SRCS:.cpp=.o))) $(OUT)/obj/ref_stubs.o

all: $(OUT)/libtcref.so $(OUT)/_turbocat$(EXT)

$(OUT)/obj:
	mkdir -p $@

define compile_rule
$(OUT)/obj/$(subst /,_,$(1:.cpp=.o)): $(REF)/src/$(1) | $(OUT)/obj
	$(CXX) $(CXXFLAGS) -c $$< -o $$@
endef
$(foreach s,$(SRCS),$(eval $(call compile_rule,$(s))))

$(OUT)/obj/ref_stubs.o: oracle/refshim/ref_stubs.cpp | $(OUT)/obj
	$(CXX) $(CXXFLAGS) -c $< -o $@

$(OUT)/obj/ref_probe.o: oracle/refshim/ref_probe.cpp | $(OUT)/obj
	$(CXX) $(CXXFLAGS) -c $< -o $@

$(OUT)/obj/bindings.o: $(REF)/python/bindings.cpp | $(OUT)/obj
	$(CXX) $(CXXFLAGS) -I$(PYINC) -I$(PBINC) -c $< -o $@

$(OUT)/libtcref.so: $(OBJS) $(OUT)/obj/ref_probe.o
	$(CXX) -shared -fopenmp -o $@ $^

$(OUT)/_turbocat$(EXT): $(OBJS) $(OUT)/obj/bindings.o
	$(CXX) -shared -fopenmp -o $@ $^

.PHONY: all

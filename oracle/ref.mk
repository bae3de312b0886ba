# Builds SymPhas's own CPU solver into oracle/_ref/libsymphas_ref.so, the
# oracle's pin, and oracle/_ref/symphas_binding, SymPhas's models run through
# the SymPhas-side binding of the B200 library (symphas_b200/binding/) beside
# SymPhas's CPU solver.  TEST INFRASTRUCTURE ONLY: tests/ and bench.py's
# reference arm use them; the product never does.
#
#   make -f ref.mk [REF=<SymPhas source dir>]
#
# g++ compiles SymPhas's sources where they lie (lib, datatypes, sym, sol and
# io modules, minus the xdrfile and VTK files) and the pin's driver
# (symphas_ref.cpp, ref_*.cpp); SymPhas's CMake is not run.  Its configuration
# headers are written from SymPhas's own *.in templates by ref_configure.py;
# ref_shim.h is force-included so GCC 13 accepts two of SymPhas's lines
# unedited.  Only oracle/_ref/ is written.  Without the SymPhas sources (a
# machine that only runs the prebuilt library) this makefile does nothing.
REF ?= /root/reference
OUT := _ref
GEN := $(OUT)/gen
OBJ := $(OUT)/obj
LIB := $(OUT)/libsymphas_ref.so
CXX := g++
PY ?= python3

ifeq ($(wildcard $(REF)/sol/inc/solver.h),)
all:
	@echo "ref.mk: no SymPhas sources at $(REF); keeping $(LIB) as it is"
else

MODULES := lib datatypes sym sol io
INC := -include ref_shim.h -I$(GEN) $(foreach m,$(MODULES),-I$(REF)/$(m)/inc) \
       -I$(REF)/examples/solvers -I$(REF) -I.
CXXFLAGS := -std=c++17 -O2 -fPIC -w
REF_SRCS := $(filter-out %/colormap.cpp %xdr.cpp,$(foreach m,$(MODULES),$(wildcard $(REF)/$(m)/src/*.cpp)))
REF_OBJS := $(foreach m,$(MODULES),$(patsubst $(REF)/$(m)/src/%.cpp,$(OBJ)/$(m)_%.o,$(filter $(REF)/$(m)/src/%,$(REF_SRCS))))
DRV_SRCS := symphas_ref.cpp ref_models_2d.cpp ref_models_3d.cpp ref_ops_2d.cpp ref_ops_3d.cpp
DRV_OBJS := $(patsubst %.cpp,$(OBJ)/drv_%.o,$(DRV_SRCS))
BINDING := $(OUT)/symphas_binding
B200_LIB := ../symphas_b200/lib/libsymphas_b200.so
GEN_H := $(GEN)/configured-defs.h
HDRS := ref_shim.h $(GEN_H)

all: $(LIB) $(BINDING)

$(GEN_H): ref_configure.py
	$(PY) ref_configure.py $(REF) $(GEN)

$(OBJ):
	mkdir -p $(OBJ)

define module_rule
$(OBJ)/$(1)_%.o: $(REF)/$(1)/src/%.cpp $(HDRS) | $(OBJ)
	$(CXX) $(CXXFLAGS) $(INC) -c $$< -o $$@
endef
$(foreach m,$(MODULES),$(eval $(call module_rule,$(m))))

$(OBJ)/drv_%.o: %.cpp symphas_ref.h $(HDRS) | $(OBJ)
	$(CXX) $(CXXFLAGS) $(INC) -c $< -o $@

$(LIB): $(DRV_OBJS) $(REF_OBJS)
	$(CXX) -shared -o $@ $^ -lpthread

$(OBJ)/binding_test.o: ../tests/cpp/symphas_binding.cpp ../symphas_b200/binding/solverftb200.h \
                       ../include/symphas_b200.h $(HDRS) | $(OBJ)
	$(CXX) $(CXXFLAGS) $(INC) -I../include -c $< -o $@

# the B200 library is found next to the package at run time ($ORIGIN-relative)
$(BINDING): $(OBJ)/binding_test.o $(REF_OBJS) $(B200_LIB)
	$(CXX) -o $@ $(OBJ)/binding_test.o $(REF_OBJS) -L../symphas_b200/lib -lsymphas_b200 \
	  -Wl,-rpath,'$$ORIGIN/../../symphas_b200/lib' -lpthread

endif

clean:
	rm -rf $(OUT)

.PHONY: all clean

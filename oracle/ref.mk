# Compiles the reference's self-contained math (src/tools.cpp, src/sturm, src/ConfigFile) from
# its sources into oracle/_ref/libnsref.so, with the stand-in headers of ref_shim/ for the two
# external headers that translation unit names.  Test infrastructure only.
# NANOSHAPER_REFERENCE names the root of a NanoShaper source checkout (read only).
ifeq ($(strip $(NANOSHAPER_REFERENCE)),)
$(error set NANOSHAPER_REFERENCE to the root of a NanoShaper source checkout)
endif
REF ?= $(NANOSHAPER_REFERENCE)/src
CXX ?= g++
OUT = _ref
CXXFLAGS = -O2 -std=c++14 -fPIC -ffp-contract=off -fno-fast-math -w \
  -include ref_shim/tbb/global_control.h -Iref_shim -I$(REF) -I$(REF)/ConfigFile -I$(REF)/jama -I$(REF)/tnt -I$(REF)/sturm

all: $(OUT)/libnsref.so

$(OUT)/libnsref.so: ref_shim/ref_wrap.cpp
	mkdir -p $(OUT)
	$(CXX) $(CXXFLAGS) -shared -o $@ ref_shim/ref_wrap.cpp $(REF)/tools.cpp $(REF)/sturm/sturm.cpp \
	  $(REF)/sturm/util.cpp $(REF)/ConfigFile/ConfigFile.cpp -lpthread

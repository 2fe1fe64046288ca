# Reference renderer build recipe -- TEST INFRASTRUCTURE ONLY.
#
#   make -f oracle/rise_ref.mk -j8        (or: make -C oracle rise)
#
# Compiles the reference renderer's library (every .cpp under
# src/Library of the reference tree, read in place, plus the two vendored
# third-party sources it links: stb_image and cgltf) into objects under
# oracle/_ref/rise_obj/, and links them with our harness
# oracle/ref_render_harness.cpp into oracle/_ref/librise_ref.so.
#
# This is our own recipe, not the reference's build system.  Differences
# from the reference's Linux configuration, and why:
#   * -DNO_EXR_SUPPORT -DNO_PNG_SUPPORT -DNO_TIFF_SUPPORT: the OpenEXR,
#     libpng and libtiff headers are not installed here; images are captured
#     in memory by the harness, so no image writer is needed;
#   * no -march=x86-64-v3: the library must also run on the GPU hosts'
#     cores, whatever their ISA level;
#   * -O2 -fPIC: it is linked into a shared library;
#   * forced standard includes: GCC 13 no longer pulls these headers in
#     transitively and some reference sources rely on that;
#   * the generated source RGBToSpectrumTable_LUTData.cpp (absent from the
#     reference tree) is replaced by oracle/ref_lut_data.cpp, which embeds
#     the body of the table that the reference's own generator
#     (tools/JakobHanikaLUTGen.cpp, built and run by oracle/Makefile) writes
#     to oracle/_ref/rec709.coeff.
# Windows-only sources (Win32 console, threads, window output, TLS,
# LoadLibrary), the precompiled-header stub and three sources that the
# reference's own source list does not build either (ManagedJob,
# RayTriangleIntersectionWithDisplacement,
# PixelBasedSpectralIntegratingRasterizerRGB: they no longer compile) are
# left out.

REFERENCE ?= /root/reference
REFLIB     = $(REFERENCE)/src/Library
HERE      := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
OUT        = $(HERE)_ref
OBJDIR     = $(OUT)/rise_obj

CXX ?= g++
# The C++ runtime is linked as the shared system library: a second, static
# copy inside a library that Python loads beside its own crashes the
# reference's iostream reads (its CPU-topology probe).
SHARED_STDCXX ?= $(firstword $(wildcard /usr/lib/x86_64-linux-gnu/libstdc++.so.6 /usr/lib64/libstdc++.so.6))
RISE_FLAGS = -std=gnu++17 -O2 -fPIC -w -fpermissive \
             -DCOLORS_RGB -DMERSENNE53 -DNO_EXR_SUPPORT -DNO_PNG_SUPPORT \
             -DNO_TIFF_SUPPORT -DRISE_ENABLE_MAILBOXING -I$(REFLIB) \
             -include atomic -include mutex -include string -include vector \
             -include map -include set -include memory -include functional \
             -include algorithm -include cstring -include cstdint \
             -include thread -include condition_variable -include limits \
             -include unordered_map -include array -include optional \
             -include chrono -include sstream

EXCLUDE  = %Win32.cpp %Win32Console.cpp %ThreadsWin32.cpp \
           %Win32WindowRasterizerOutput.cpp %TlsTransportWin.cpp %pch.cpp \
           %ManagedJob.cpp %RayTriangleIntersectionWithDisplacement.cpp \
           %PixelBasedSpectralIntegratingRasterizerRGB.cpp
LIB_SRC  = $(filter-out $(EXCLUDE),$(shell find $(REFLIB) -name '*.cpp' | sort))
EXT_SRC  = $(REFERENCE)/extlib/stb/stb_image.cpp $(REFERENCE)/extlib/cgltf/cgltf.cpp
LIB_OBJ  = $(patsubst $(REFLIB)/%.cpp,$(OBJDIR)/lib/%.o,$(LIB_SRC))
EXT_OBJ  = $(patsubst $(REFERENCE)/extlib/%.cpp,$(OBJDIR)/ext/%.o,$(EXT_SRC))

all: $(OUT)/librise_ref.so

$(OBJDIR)/lib/%.o: $(REFLIB)/%.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(RISE_FLAGS) -c $< -o $@

$(OBJDIR)/ext/%.o: $(REFERENCE)/extlib/%.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(RISE_FLAGS) -c $< -o $@

$(OBJDIR)/ref_lut_data.o: $(HERE)ref_lut_data.cpp $(OUT)/rec709.coeff
	@mkdir -p $(dir $@)
	$(CXX) -std=gnu++17 -O2 -fPIC -DRISE_LUT_COEFF='"$(OUT)/rec709.coeff"' -c $< -o $@

$(OBJDIR)/ref_render_harness.o: $(HERE)ref_render_harness.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(RISE_FLAGS) -c $< -o $@

$(OUT)/librise_ref.so: $(LIB_OBJ) $(EXT_OBJ) $(OBJDIR)/ref_lut_data.o $(OBJDIR)/ref_render_harness.o
	$(CXX) -shared -o $@ $^ $(SHARED_STDCXX) -lpthread -lz -ldl

objects: $(LIB_OBJ) $(EXT_OBJ)

# The RISE-side adapter (rise_b200/adapter/: scene extraction and the GPU
# rasterizer, product code compiled against the reference's headers) with
# its test driver tests/cpp/rise_adapter_check.cpp, linked against the
# reference library above and rtb200's; the run paths are relative, so the
# program also runs where the repository is copied.
ROOT       := $(abspath $(HERE)..)
ADAPTER    := $(ROOT)/rise_b200/adapter
ADAPTER_SRC = $(ADAPTER)/rise_extract.cpp $(ADAPTER)/gpu_rasterizer.cpp $(ROOT)/tests/cpp/rise_adapter_check.cpp

adapter: $(OUT)/rise_adapter_check

$(OUT)/rise_adapter_check: $(ADAPTER_SRC) $(ADAPTER)/rise_extract.h $(ADAPTER)/gpu_rasterizer.h $(OUT)/librise_ref.so \
                           $(ROOT)/rise_b200/_lib/librtb200.so $(ROOT)/include/rtb200.h
	$(CXX) $(filter-out -fPIC,$(RISE_FLAGS)) -I$(ROOT)/include -I$(ADAPTER) $(ADAPTER_SRC) -o $@ \
	    -L$(OUT) -lrise_ref -L$(ROOT)/rise_b200/_lib -lrtb200 \
	    -Wl,-rpath,'$$ORIGIN' -Wl,-rpath,'$$ORIGIN/../../rise_b200/_lib' $(SHARED_STDCXX) -lpthread

# Exit status 0 when the reference tree is present.
has-reference:
	@test -d $(REFLIB)

.PHONY: all objects adapter has-reference

# Builds the reference (momokchung/polmdqc) MD library from its own sources into
# oracle/_ref/, for use as a test-only checker.  Nothing here is shipped: the
# product library never links these objects.
#
#   make -f oracle/ref.mk REF=/root/reference -j8
#
# Flags follow the reference's CMakeLists.txt:15 (-O3 -finline-functions
# -ffast-math -fopenmp).  The upstream CMake build is not used: it hard-codes
# homebrew compilers and libint2/OpenBLAS/GMP paths.  The alpha-shape / GMP
# sources and the QM programs are left out (not on the electrostatics path).

REF    ?= /root/reference
OUT    ?= oracle/_ref
REFCXX ?= g++
INC     = -I$(REF)/include -I$(REF)/include/md -I$(REF)/include/oqc -I$(REF)/include/qc
FLAGS   = -std=c++17 -O3 -finline-functions -ffast-math -fopenmp -fPIC -w

EXCLUDE = delcx sosgmp alfcx alphavol alphamol alphamol1 alphamol2 alfmol alforder \
          alfboxsize initalf initalf2 initalfatm spacefill tetrahedron vertex edge face \
          hilbert kalf kdtree multimol
MD_ALL  = $(basename $(notdir $(wildcard $(REF)/src/md/*.cpp)))
MD_SRC  = $(filter-out %Exe $(EXCLUDE),$(MD_ALL))
OBJS    = $(addprefix $(OUT)/obj/md_,$(addsuffix .o,$(MD_SRC))) \
          $(OUT)/obj/mod.o $(OUT)/obj/promo.o $(OUT)/obj/rootdir.o $(OUT)/obj/finalqm.o

# The library without empole.o is what the drop-in shim
# (polmdqc_b200/host/polmdqc_shim.cpp) links against.
CORE_OBJS = $(filter-out $(OUT)/obj/md_empole.o,$(OBJS))
GPULIB    = polmdqc_b200/_lib/libamoeba_gpu.so
SHIM      = polmdqc_b200/host/polmdqc_shim.cpp

all: $(OUT)/libpolmdqc.a $(OUT)/libpolmdqc_noempole.a $(OUT)/ref_dump $(OUT)/ref_time $(OUT)/data.stamp

# The reference's own programs with the shim in place of empole.o: the
# drop-in demonstration (analyze_gpu, testgrad_gpu) and ref_dump_gpu, the
# dump driver running the same path on the GPU (used by the GPU tests).
shim: $(OUT)/ref_dump_gpu $(OUT)/analyze_gpu $(OUT)/testgrad_gpu

$(OUT)/obj/md_%.o: $(REF)/src/md/%.cpp
	@mkdir -p $(dir $@)
	$(REFCXX) $(FLAGS) $(INC) -c $< -o $@

$(OUT)/obj/mod.o: $(REF)/src/mod.cpp
	@mkdir -p $(dir $@)
	$(REFCXX) $(FLAGS) $(INC) -c $< -o $@
$(OUT)/obj/promo.o: $(REF)/src/promo.cpp
	@mkdir -p $(dir $@)
	$(REFCXX) $(FLAGS) $(INC) -c $< -o $@
$(OUT)/obj/rootdir.o: $(REF)/src/rootdir.cpp
	@mkdir -p $(dir $@)
	$(REFCXX) $(FLAGS) $(INC) -c $< -o $@
$(OUT)/obj/finalqm.o: $(REF)/src/qc/finalqm.cpp
	@mkdir -p $(dir $@)
	$(REFCXX) $(FLAGS) $(INC) -c $< -o $@

$(OUT)/libpolmdqc.a: $(OBJS)
	rm -f $@ && ar rcs $@ $^

$(OUT)/libpolmdqc_noempole.a: $(CORE_OBJS)
	rm -f $@ && ar rcs $@ $^

SHIMFLAGS = $(FLAGS) -Iinclude $(SHIM) $(OUT)/libpolmdqc_noempole.a -Lpolmdqc_b200/_lib -lamoeba_gpu \
            -Wl,-rpath,'$$ORIGIN/../../polmdqc_b200/_lib'

$(OUT)/ref_dump_gpu: oracle/ref_dump.cpp $(SHIM) $(OUT)/libpolmdqc_noempole.a $(GPULIB)
	$(REFCXX) $(INC) oracle/ref_dump.cpp $(SHIMFLAGS) -o $@

$(OUT)/analyze_gpu: $(REF)/src/md/analyzeExe.cpp $(SHIM) $(OUT)/libpolmdqc_noempole.a $(GPULIB)
	$(REFCXX) $(INC) $< $(SHIMFLAGS) -o $@

$(OUT)/testgrad_gpu: $(REF)/src/md/testgradExe.cpp $(SHIM) $(OUT)/libpolmdqc_noempole.a $(GPULIB)
	$(REFCXX) $(INC) $< $(SHIMFLAGS) -o $@

# ref_dump: our own driver (oracle/ref_dump.cpp) around the reference library;
# runs initial/getcart/mechanic/energy and prints the globals as JSON.
$(OUT)/ref_dump: oracle/ref_dump.cpp $(OUT)/libpolmdqc.a
	$(REFCXX) $(FLAGS) $(INC) $< $(OUT)/libpolmdqc.a -o $@

# ref_time: our own timing driver (oracle/ref_time.cpp): the reference's
# energy<Gradient>() in its only electrostatics mode, for the benchmark's CPU leg.
$(OUT)/ref_time: oracle/ref_time.cpp $(OUT)/libpolmdqc.a
	$(REFCXX) $(FLAGS) $(INC) $< $(OUT)/libpolmdqc.a -o $@

# Parameter files and test fixtures the reference's own tests read, copied next
# to the build so that runs on another machine can find them.
$(OUT)/data.stamp: $(wildcard $(REF)/params/*.prm)
	@mkdir -p $(OUT)/params $(OUT)/testFiles
	cp $(REF)/params/water03.prm $(REF)/params/amoebabio09.prm $(REF)/params/amoebabio18.prm \
	   $(REF)/params/amoebaplus.prm $(REF)/params/hippoS101.prm $(REF)/params/hippo19.prm \
	   $(REF)/params/water21.prm $(OUT)/params/
	cp -r $(REF)/test/testFiles/amoeba $(REF)/test/testFiles/bounds $(REF)/test/testFiles/rotpole \
	   $(REF)/test/testFiles/amoebap $(REF)/test/testFiles/chkpole $(REF)/test/testFiles/amoebaMisc \
	   $(REF)/test/testFiles/hippo $(OUT)/testFiles/
	touch $@

.PHONY: all shim

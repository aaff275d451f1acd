# Builds the reference's own CPU engine (Pythia `executequery`) from its
# sources where they lie, with outputs only under oracle/_ref/.
#
# This is test infrastructure: the binary is the parity checker that pins the
# C oracle (oracle/pyg_oracle.c) and the CPU arm that bench.py times.  It is
# never part of the product path.
#
#   make -f oracle/ref.mk REF=<path of the reference sources>   (from the repo root)
#
# The reference's own Makefile is not used (its `all` target runs a
# pre-init script that needs a missing hdf5 tarball, and libconfig's
# autoconf build needs bison/flex regeneration).  Instead every translation
# unit of the non-MPI engine is compiled directly with g++/gcc:
#   * libconfig-1.2 (vendored): grammar.c, scanner.c, libconfig.c,
#     libconfigcpp.c++ compiled as shipped; the generated parser sources are
#     in the tree, so no bison/flex run is needed.  -std=gnu++98 because its
#     throw() specifications are rejected by C++17.
#   * bzip2-1.0.5 (vendored): the seven library sources.
#   * the engine: the FILES list of the reference Makefile (non-MPI,
#     non-RDMA, non-HDF5 build).
# One compile-only shim: operators/data_recver_tcp.cpp calls
# TupleBuffer::resetdata, which the snapshot never declares.  That TCP
# receiver is off the join/aggregate path and is never run by the oracle; it
# is compiled with `resetdata(d,l)` mapped to `clear()` on the command line.
# The reference sources are not modified.

ifndef REF
$(error REF is not set: pass REF=<path of the reference sources>)
endif
OUT := oracle/_ref
OBJ := $(OUT)/obj

CXX := g++
CC := gcc
OPT ?= -O2
CXXFLAGS := -std=gnu++98 -m64 $(OPT) -g -w -DSTATS_ALLOCATE -pthread
CFLAGS := -m64 $(OPT) -w

LIBCONFIG := $(REF)/externals/libconfig-1.2
BZIP2 := $(REF)/externals/bzip2-1.0.5
INC := -I$(OUT)/include -I$(REF)

ENGINE := schema hash ProcessorMap Barrier perfcounters query \
	util/hashtable util/buffer \
	visitors/recursivedestroy visitors/recursivefree visitors/prettyprint \
	visitors/threadinit visitors/threadclose \
	operators/base operators/mapwrapper operators/filter operators/sortlimit \
	operators/genericaggregate operators/aggregatecount operators/aggregatesum \
	operators/scan operators/partitionedscan operators/repeatpartitionedscan \
	operators/parallelscan operators/repeatparallelscan operators/merge \
	operators/join operators/shuffle operators/data_sender_shuffle_tcp \
	operators/data_sender_bcast_tcp operators/data_recver_tcp \
	operators/cycleaccountant operators/timeaccountant util/affinitizer \
	operators/project comparator conjunctionevaluator rawcompfns \
	operators/memsegmentwriter operators/loaders/table \
	operators/loaders/parser operators/loaders/loader \
	operators/checker_callstate operators/printer_tuplecount \
	operators/printer_getnextcallcount operators/generator_int \
	operators/generator_zipf operators/printer_perfcnt operators/bitentropy \
	operators/threadidprepend util/numaasserts util/numaallocate \
	operators/consume operators/partition operators/indexjoin util/cpufreq \
	operators/perfcount_scanstart operators/perfcount_getnext \
	operators/perfcount_all operators/sort util/topology util/tcpsocket

ENGINE_OBJS := $(addprefix $(OBJ)/,$(addsuffix .o,$(ENGINE))) $(OBJ)/operators/loaders/sfmt/SFMT.o
LIBCONFIG_OBJS := $(OBJ)/lc/grammar.o $(OBJ)/lc/scanner.o $(OBJ)/lc/libconfig.o $(OBJ)/lc/libconfigcpp.o
BZ_SRCS := blocksort huffman crctable randtable compress decompress bzlib
BZ_OBJS := $(addprefix $(OBJ)/bz/,$(addsuffix .o,$(BZ_SRCS)))

all: $(OUT)/executequery $(OUT)/executemultiplequery

# One recipe run makes all three headers (grouped target): with plain
# targets a parallel make ran the copy once per header and the runs raced.
$(OUT)/include/libconfig.h++ $(OUT)/include/libconfig.h $(OUT)/include/bzlib.h &:
	mkdir -p $(OUT)/include
	cp -f $(LIBCONFIG)/libconfig.h $(LIBCONFIG)/libconfig.h++ $(OUT)/include/
	cp -f $(BZIP2)/bzlib.h $(OUT)/include/

HDRS := $(OUT)/include/libconfig.h++ $(OUT)/include/libconfig.h $(OUT)/include/bzlib.h

$(OBJ)/lc/%.o: $(LIBCONFIG)/%.c $(HDRS)
	mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -I$(LIBCONFIG) -c $< -o $@

$(OBJ)/lc/libconfigcpp.o: $(LIBCONFIG)/libconfigcpp.c++ $(HDRS)
	mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS) -x c++ -I$(LIBCONFIG) -c $< -o $@

$(OBJ)/bz/%.o: $(BZIP2)/%.c
	mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -D_FILE_OFFSET_BITS=64 -c $< -o $@

$(OBJ)/operators/data_recver_tcp.o: $(REF)/operators/data_recver_tcp.cpp $(HDRS)
	mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS) $(INC) '-Dresetdata(d,l)=clear()' -c $< -o $@

$(OBJ)/operators/loaders/sfmt/SFMT.o: $(REF)/operators/loaders/sfmt/SFMT.c $(HDRS)
	mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS) -x c++ $(INC) -c $< -o $@

$(OBJ)/%.o: $(REF)/%.cpp $(HDRS)
	mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS) $(INC) -c $< -o $@

$(OBJ)/timestamp.o:
	mkdir -p $(OBJ)
	echo 'const char* MakefileTimestampSignature="reference engine built by oracle/ref.mk";' > $(OBJ)/timestamp.cpp
	$(CXX) $(CXXFLAGS) -c $(OBJ)/timestamp.cpp -o $@

$(OUT)/libpythia_ref.a: $(ENGINE_OBJS) $(LIBCONFIG_OBJS) $(BZ_OBJS) $(OBJ)/timestamp.o
	rm -f $@
	ar rcs $@ $^

$(OUT)/executequery: $(REF)/drivers/executequery.cpp $(OUT)/libpythia_ref.a
	$(CXX) $(CXXFLAGS) $(INC) $< $(OUT)/libpythia_ref.a -lpthread -lrt -o $@

$(OUT)/executemultiplequery: $(REF)/drivers/executemultiplequery.cpp $(OUT)/libpythia_ref.a
	$(CXX) $(CXXFLAGS) $(INC) $< $(OUT)/libpythia_ref.a -lpthread -lrt -o $@

.PHONY: all

// GpuHashJoinOp: the reference engine's `hashjoin` operator with its build
// and probe run on the GPU through libpyg's C ABI (include/pyg.h).  It is a
// subclass of the reference's own JoinOp (operators/operators.h:3006-3039),
// compiled against the reference headers and linked into the reference
// engine, so plans, scans, merge threads, aggregates and printers stay the
// reference's.  It keeps HashJoinOp's contract (operators/operators.h:
// 3071-3137, operators/join.cpp:367-884):
//
//   init        JoinOp::init parses projection / buildjattr / probejattr /
//               threadgroups and builds the output schema; `hash`,
//               `tuplesperbucket` and `allocpolicy` size the CPU table and
//               are ignored (the GPU table is sized from the build).
//   scanStart   every thread of a group drains its build stream (left
//               threads only, JoinOp::isLeftThread) and its probe stream
//               into its own host buffer, then waits at the group's
//               barrier; the group leader runs pyg_hashjoin_build +
//               pyg_hashjoin_probe_materialize over the group's tuples and
//               copies the joined tuples to pinned host memory (leaders
//               of different groups take turns on the one libpyg context);
//               a second barrier releases the group.
//   getNext     thread t serves slice t (its position in the group) of the
//               group's output, as pages of at most `buffsize` bytes that
//               wrap the output in place.
//   scanStop    closes the probe stream (the build stream was closed in
//               scanStart, as in HashJoinOp::scanStart).
//   threadClose the group leader frees the group's output after a barrier.
//
// Errors of a child or of the GPU are reported as Operator::Error by every
// thread of the group, after both barriers, so no thread is left waiting.
// Columns must be 4 or 8 bytes wide (CT_INTEGER, CT_LONG, CT_DECIMAL,
// CT_DATE, CT_POINTER or CHAR(4)/CHAR(8), copied as bits); join keys must
// be CT_INTEGER or CT_LONG, at most 8 bytes in all.  init throws
// InvalidParameter otherwise.
#ifndef PYG_GPUHASHJOIN_H
#define PYG_GPUHASHJOIN_H

#include <vector>

#include "operators/operators.h"
#include "pyg.h"

class GpuHashJoinOp : public JoinOp {
public:
    GpuHashJoinOp();
    virtual ~GpuHashJoinOp();

    virtual void init(libconfig::Config& root, libconfig::Setting& node);
    virtual void threadInit(unsigned short threadid);
    virtual ResultCode scanStart(unsigned short threadid, Page* indexdatapage, Schema& indexdataschema);
    virtual GetNextResultT getNext(unsigned short threadid);
    virtual ResultCode scanStop(unsigned short threadid);
    virtual void threadClose(unsigned short threadid);
    virtual void destroy();

    // The context every GpuHashJoinOp of the process uses (created on first
    // init on device `gpu.device` of the node, default 0).
    static pyg_ctx* context();

private:
    struct Group {
        char* out;             // pinned host: joined tuples of the group
        long long nout;        // tuples in out
        bool failed;           // a child or the GPU reported an error
        Group() : out(0), nout(0), failed(false) {}
    };
    struct ThreadState {
        std::vector<char> build, probe;  // drained input tuples
        long long pos, end;              // slice of the group output
        Page* page;                      // page handed out by getNext
        bool failed;
        char pad[64];
        ThreadState() : pos(0), end(0), page(0), failed(false) {}
    };

    void join_group(unsigned short groupno);
    static bool drain(Operator* op, unsigned short threadid, std::vector<char>& out, unsigned int tuplesize);
    static pyg_rel as_rel(Schema& s, const std::vector<char>& data);

    std::vector<int32_t> bkeys_, pkeys_, payload_;
    std::vector<pyg_proj> proj_;
    std::vector<Group> groups_;
    std::vector<ThreadState*> threads_;
    float load_factor_;
    static pyg_ctx* ctx_;
};

#endif

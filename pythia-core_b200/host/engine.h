// Plan-level host engine: Operator classes with the reference's contract
// (operators/operators.h:96-203: init / threadInit / scanStart / getNext /
// scanStop / threadClose over pages of fixed-width tuples) for the node
// types of the join / aggregation hot path, each backed by the libpyg C ABI
// (include/pyg*.h).  The GPU provides the data parallelism the reference
// gets from `merge` worker threads, so plans run on logical thread 0 and a
// `merge` node passes its input through.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "../../include/pyg.h"
#include "plan.h"

namespace pyg_host {

struct EngineError : std::runtime_error {
    explicit EngineError(const std::string& m) : std::runtime_error(m) {}
};

// Column layout of a tuple: types PYG_INT32 ("int") / PYG_INT64 ("long"),
// packed back to back (reference Schema::add, schema.cpp).
struct Schema {
    std::vector<int32_t> types;
    std::vector<int32_t> offs;
    int32_t tuple_bytes = 0;

    void add(int32_t type);
    size_t columns() const { return types.size(); }
    int64_t get(const uint8_t* tup, size_t col) const;
    std::string prettyprint(const uint8_t* tup, char sep) const;
    pyg_rel rel(const void* base, int64_t n, bool on_device) const;
    static int32_t type_of(const std::string& name);
};

// A run of packed tuples (the reference's Page / TupleBuffer view).
struct Page {
    const uint8_t* data = nullptr;
    int64_t ntuples = 0;
    int32_t tuple_bytes = 0;
};

// Pinned host buffer holding a whole relation.
struct HostRel {
    uint8_t* data = nullptr;
    int64_t ntuples = 0;
    int64_t cap_bytes = 0;
    int32_t tuple_bytes = 0;
    HostRel() = default;
    HostRel(const HostRel&) = delete;
    HostRel& operator=(const HostRel&) = delete;
    ~HostRel();
    void reserve(int64_t bytes);
    void append(const uint8_t* src, int64_t n);
};

class Operator {
public:
    enum ResultCode { Ready, Finished, Error };
    typedef std::pair<ResultCode, Page*> GetNextResultT;

    virtual ~Operator() = default;
    virtual void init(const Setting& root, const Setting& node);
    virtual void threadInit(unsigned short tid) {}
    virtual ResultCode scanStart(unsigned short tid) = 0;
    virtual GetNextResultT getNext(unsigned short tid) = 0;
    virtual ResultCode scanStop(unsigned short tid) = 0;
    virtual void threadClose(unsigned short tid) {}
    virtual std::vector<Operator*> children() { return {}; }
    // After scanStart: the whole output as a device buffer of n tuples,
    // when the operator produced it on the GPU.  A GPU parent reads it in
    // place instead of pulling pages through host memory.  The buffer stays
    // valid until the operator's next scanStart or its destruction.
    virtual bool device_result(const void** dev, int64_t* n) { return false; }
    Schema& getOutSchema() { return schema; }

    std::string type, name;
    static pyg_ctx* ctx;  // the process-wide GPU context

protected:
    Schema schema;
    int64_t buffsize = 1 << 20;
};

// An operator's materialised output: either a device buffer, kept on the
// device for GPU parents and copied to host only when pages are pulled, or
// host pages filled directly.
struct ResultBuffer {
    HostRel host;
    void* dev = nullptr;
    int64_t n = 0;
    bool host_valid = true;
    int64_t served = 0;
    Page page;
    // Bytes copied device -> host to serve pages, over all operators of
    // the process (the driver prints it).
    static int64_t d2h_bytes;

    ResultBuffer() = default;
    ResultBuffer(const ResultBuffer&) = delete;
    ResultBuffer& operator=(const ResultBuffer&) = delete;
    ~ResultBuffer();
    // Takes ownership of device buffer d (pyg_alloc) holding cnt tuples.
    void keep_device(void* d, int64_t cnt, int32_t tuple_bytes);
    // The host relation was filled directly.
    void keep_host();
    Operator::GetNextResultT next(int64_t buffsize, int32_t tuple_bytes);
    bool device(const void** d, int64_t* cnt) const;
    void rewind() { served = 0; }
};

// Bytes the scans streamed into device memory through the overlapped
// upload ring, and the wall time those loads took (the driver prints both).
struct ScanIngest {
    static int64_t bytes;
    static double seconds;
};

// Serves a materialised relation as pages of buffsize bytes.
class MaterializedOp : public Operator {
public:
    GetNextResultT getNext(unsigned short tid) override;
    ResultCode scanStop(unsigned short tid) override;
    bool device_result(const void** dev, int64_t* n) override { return out.device(dev, n); }

protected:
    ResultBuffer out;
};

class SingleInputOp : public Operator {
public:
    Operator* nextOp = nullptr;
    std::vector<Operator*> children() override { return {nextOp}; }
};

class DualInputOp : public Operator {
public:
    Operator* buildOp = nullptr;
    Operator* probeOp = nullptr;
    std::vector<Operator*> children() override { return {buildOp, probeOp}; }
};

// Reads a whole child into a pinned host relation.
void drain(Operator* op, unsigned short tid, HostRel& out);
// A child's output as a relation: its device buffer when it has one (no
// host round trip), else its pages drained into `host`.
pyg_rel input_rel(Operator* op, unsigned short tid, HostRel& host);

// Builds the operator tree of a plan (reference Query::create, query.cpp:56-326).
struct Query {
    std::vector<std::unique_ptr<Operator>> ops;
    Operator* root = nullptr;
    std::unique_ptr<Setting> plan;
    void create(std::unique_ptr<Setting> plan_root);
    Operator::ResultCode scanStart() { return root->scanStart(0); }
    Operator::GetNextResultT getNext() { return root->getNext(0); }
    Operator::ResultCode scanStop() { return root->scanStop(0); }
    void threadInit();
    void threadClose();
    // "TupleCountPrinter (total=N tuples)" lines of the plan's counters.
    std::vector<std::string> counter_report() const;
};

}  // namespace pyg_host

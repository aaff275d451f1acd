// Operator shims for the join / aggregation hot path over the libpyg C ABI.
#include "engine.h"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>

#include "../../include/pyg_mpsm.h"

namespace pyg_host {

pyg_ctx* Operator::ctx = nullptr;

static void check(int rc, const char* what)
{
    if (rc != PYG_OK) throw EngineError(std::string(what) + ": " + pyg_last_error());
}

// ---------------------------------------------------------------- Schema

void Schema::add(int32_t type)
{
    types.push_back(type);
    offs.push_back(tuple_bytes);
    tuple_bytes += type == PYG_INT32 ? 4 : 8;
}

int64_t Schema::get(const uint8_t* tup, size_t col) const
{
    if (types[col] == PYG_INT32) {
        int32_t v;
        memcpy(&v, tup + offs[col], 4);
        return v;
    }
    int64_t v;
    memcpy(&v, tup + offs[col], 8);
    return v;
}

std::string Schema::prettyprint(const uint8_t* tup, char sep) const
{
    std::string s;
    for (size_t c = 0; c < types.size(); ++c) {
        if (c) s += sep;
        s += std::to_string(get(tup, c));
    }
    return s;
}

pyg_rel Schema::rel(const void* base, int64_t n, bool on_device) const
{
    pyg_rel r;
    memset(&r, 0, sizeof(r));
    r.base = base;
    r.ntuples = n;
    r.tuple_bytes = tuple_bytes;
    r.ncols = (int32_t)types.size();
    for (size_t c = 0; c < types.size(); ++c) {
        r.col_offset[c] = offs[c];
        r.col_type[c] = types[c];
    }
    r.on_device = on_device ? 1 : 0;
    return r;
}

int32_t Schema::type_of(const std::string& name)
{
    if (name == "int" || name == "integer") return PYG_INT32;
    if (name == "long" || name == "date") return PYG_INT64;
    throw EngineError("column type '" + name + "' is not on the GPU join/aggregation path (int, long)");
}

// ---------------------------------------------------------------- HostRel

HostRel::~HostRel()
{
    if (data) pyg_host_free(data);
}

void HostRel::reserve(int64_t bytes)
{
    if (bytes <= cap_bytes) return;
    int64_t cap = cap_bytes ? cap_bytes : (1 << 20);
    while (cap < bytes) cap *= 2;
    void* p = nullptr;
    check(pyg_host_alloc((size_t)cap, &p), "pinned allocation");
    if (data) {
        memcpy(p, data, (size_t)ntuples * tuple_bytes);
        pyg_host_free(data);
    }
    data = (uint8_t*)p;
    cap_bytes = cap;
}

void HostRel::append(const uint8_t* src, int64_t n)
{
    reserve((ntuples + n) * tuple_bytes);
    memcpy(data + ntuples * tuple_bytes, src, (size_t)n * tuple_bytes);
    ntuples += n;
}

void drain(Operator* op, unsigned short tid, HostRel& out)
{
    out.tuple_bytes = op->getOutSchema().tuple_bytes;
    out.ntuples = 0;
    for (;;) {
        Operator::GetNextResultT r = op->getNext(tid);
        if (r.first == Operator::Error) throw EngineError("child '" + op->name + "' returned Error");
        if (r.second && r.second->ntuples) out.append(r.second->data, r.second->ntuples);
        if (r.first == Operator::Finished) break;
    }
}

// -------------------------------------------------------------- Operator

void Operator::init(const Setting& root, const Setting& node)
{
    buffsize = root.getInt("buffsize", 1 << 20);
    if (buffsize < 1) throw EngineError("buffsize must be positive");
}

pyg_rel input_rel(Operator* op, unsigned short tid, HostRel& host)
{
    const void* d = nullptr;
    int64_t n = 0;
    if (op->device_result(&d, &n)) return op->getOutSchema().rel(d, n, true);
    drain(op, tid, host);
    return op->getOutSchema().rel(host.data, host.ntuples, false);
}

int64_t ResultBuffer::d2h_bytes = 0;

ResultBuffer::~ResultBuffer()
{
    if (dev && Operator::ctx) pyg_free(Operator::ctx, dev);
}

void ResultBuffer::keep_device(void* d, int64_t cnt, int32_t tuple_bytes)
{
    if (dev) pyg_free(Operator::ctx, dev);
    dev = d;
    n = cnt;
    host.tuple_bytes = tuple_bytes;
    host.ntuples = 0;
    host_valid = false;
    served = 0;
}

void ResultBuffer::keep_host()
{
    if (dev) pyg_free(Operator::ctx, dev);
    dev = nullptr;
    n = host.ntuples;
    host_valid = true;
    served = 0;
}

bool ResultBuffer::device(const void** d, int64_t* cnt) const
{
    if (!dev) return false;
    *d = dev;
    *cnt = n;
    return true;
}

Operator::GetNextResultT ResultBuffer::next(int64_t buffsize, int32_t tuple_bytes)
{
    if (!host_valid) {
        // First page pulled by a host consumer: one copy of the result.
        host.tuple_bytes = tuple_bytes;
        host.ntuples = 0;
        host.reserve(n * tuple_bytes);
        if (n) check(pyg_memcpy_d2h(Operator::ctx, host.data, dev, (size_t)n * tuple_bytes), "copy result");
        host.ntuples = n;
        d2h_bytes += n * tuple_bytes;
        host_valid = true;
    }
    int64_t per = buffsize / (tuple_bytes ? tuple_bytes : 1);
    if (per < 1) per = 1;
    const int64_t left = host.ntuples - served;
    const int64_t k = left < per ? left : per;
    page.data = host.data ? host.data + served * tuple_bytes : nullptr;
    page.ntuples = k;
    page.tuple_bytes = tuple_bytes;
    served += k;
    return std::make_pair(served >= host.ntuples ? Operator::Finished : Operator::Ready, &page);
}

Operator::GetNextResultT MaterializedOp::getNext(unsigned short tid) { return out.next(buffsize, schema.tuple_bytes); }

Operator::ResultCode MaterializedOp::scanStop(unsigned short tid)
{
    out.rewind();
    return Ready;
}

// ------------------------------------------------------------------ scans

int64_t ScanIngest::bytes = 0;
double ScanIngest::seconds = 0;

static double now_seconds()
{
    timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec + t.tv_nsec * 1e-9;
}

// `scan` / `parallelscan` / `partitionedscan` (operators/scan.cpp,
// parallelscan.cpp:41-190): all listed files, binary (raw packed tuples,
// operators/loaders/table.cpp:198-348) or '|'-separated text.  Loading is
// lazy: a GPU parent (device_result) streams the files straight into HBM
// through the overlapped upload ring (pyg_upload_*: the next chunk is read
// or parsed while the previous one crosses PCIe); a host consumer
// (getNext) loads them into pinned host pages.
class ScanOp : public MaterializedOp {
public:
    void init(const Setting& root, const Setting& node) override
    {
        Operator::init(root, node);
        const Setting& sch = node["schema"];
        for (size_t i = 0; i < sch.size(); ++i) schema.add(Schema::type_of(sch[i].asString()));
        std::string path = root.getString("path", "./");
        if (!path.empty() && path.back() != '/') path += '/';
        const Setting& f = node["files"];
        if (f.isAggregate())
            for (size_t i = 0; i < f.size(); ++i) files.push_back(path + f[i].asString());
        else
            files.push_back(path + f.asString());
        binary = node.getString("filetype", "text") == "binary";
        sep = node.getString("separators", "|");
    }

    ResultCode scanStart(unsigned short tid) override
    {
        out.rewind();
        return Ready;
    }

    GetNextResultT getNext(unsigned short tid) override
    {
        if (!host_loaded && !dev_loaded) load_host();
        return out.next(buffsize, schema.tuple_bytes);
    }

    bool device_result(const void** dev, int64_t* n) override
    {
        if (!dev_loaded) load_device();
        return out.device(dev, n);
    }

private:
    static int64_t file_bytes(const std::string& fn)
    {
        struct stat st;
        if (stat(fn.c_str(), &st) != 0) throw EngineError("cannot open input file " + fn);
        return (int64_t)st.st_size;
    }

    // Parses one '|'-separated text line into a packed tuple.
    void parse_line(const std::string& line, uint8_t* tup) const
    {
        size_t pos = 0;
        for (size_t c = 0; c < schema.columns(); ++c) {
            size_t e = line.find_first_of(sep, pos);
            std::string field = line.substr(pos, e == std::string::npos ? std::string::npos : e - pos);
            int64_t v = strtoll(field.c_str(), nullptr, 10);
            if (schema.types[c] == PYG_INT32) {
                int32_t w = (int32_t)v;
                memcpy(tup + schema.offs[c], &w, 4);
            } else {
                memcpy(tup + schema.offs[c], &v, 8);
            }
            pos = e == std::string::npos ? line.size() : e + 1;
        }
    }

    // Calls sink(ptr, bytes) with runs of packed tuples read from every
    // file; `want` asks the sink for its next buffer of at most `cap` bytes.
    template <class Want, class Sink>
    void read_files(Want want, Sink sink)
    {
        const int32_t tb = schema.tuple_bytes;
        for (auto& fn : files) {
            if (binary) {
                int64_t left = file_bytes(fn);
                if (left % tb) throw EngineError(fn + ": size is not a multiple of the tuple size");
                FILE* f = fopen(fn.c_str(), "rb");
                if (!f) throw EngineError("cannot open input file " + fn);
                while (left > 0) {
                    size_t cap = 0;
                    uint8_t* buf = want(&cap);
                    int64_t k = std::min<int64_t>(left, (int64_t)(cap / tb) * tb);
                    if (k <= 0 || fread(buf, 1, (size_t)k, f) != (size_t)k) {
                        fclose(f);
                        throw EngineError(fn + ": short read");
                    }
                    sink(buf, k);
                    left -= k;
                }
                fclose(f);
            } else {
                std::ifstream in(fn, std::ios::binary);
                if (!in) throw EngineError("cannot open input file " + fn);
                std::string line;
                size_t cap = 0, used = 0;
                uint8_t* buf = nullptr;
                while (std::getline(in, line)) {
                    if (line.empty()) continue;
                    if (!buf || used + tb > cap) {
                        if (buf && used) sink(buf, (int64_t)used);
                        buf = want(&cap);
                        used = 0;
                        if (cap < (size_t)tb) throw EngineError("staging buffer smaller than a tuple");
                    }
                    parse_line(line, buf + used);
                    used += tb;
                }
                if (buf && used) sink(buf, (int64_t)used);
            }
        }
    }

    void load_host()
    {
        HostRel& result = out.host;
        result.tuple_bytes = schema.tuple_bytes;
        result.ntuples = 0;
        std::vector<uint8_t> text(1 << 20);
        read_files(
            [&](size_t* cap) -> uint8_t* {
                if (binary) {
                    // Binary files are read straight into the pinned pages.
                    result.reserve(result.ntuples * schema.tuple_bytes + (1 << 24));
                    *cap = (size_t)(result.cap_bytes - result.ntuples * schema.tuple_bytes);
                    return result.data + result.ntuples * schema.tuple_bytes;
                }
                *cap = text.size();
                return text.data();
            },
            [&](uint8_t* buf, int64_t bytes) {
                if (binary)
                    result.ntuples += bytes / schema.tuple_bytes;
                else
                    result.append(buf, bytes / schema.tuple_bytes);
            });
        out.keep_host();
        host_loaded = true;
        dev_loaded = false;
    }

    void load_device()
    {
        int64_t total = 0;
        for (auto& fn : files) total += file_bytes(fn);
        const double t0 = now_seconds();
        pyg_upload* up = nullptr;
        check(pyg_upload_open(ctx, (size_t)std::max<int64_t>(total, schema.tuple_bytes), kSlotBytes, kSlots, &up),
              "ingest open");
        try {
            read_files(
                [&](size_t* cap) -> uint8_t* {
                    void* b = nullptr;
                    check(pyg_upload_slot(ctx, up, &b, cap), "ingest slot");
                    return (uint8_t*)b;
                },
                [&](uint8_t* buf, int64_t bytes) { check(pyg_upload_commit(ctx, up, (size_t)bytes), "ingest copy"); });
        } catch (...) {
            pyg_upload_abort(ctx, up);
            throw;
        }
        void* d = nullptr;
        size_t bytes = 0;
        check(pyg_upload_finish(ctx, up, &d, &bytes), "ingest finish");
        out.keep_device(d, (int64_t)bytes / schema.tuple_bytes, schema.tuple_bytes);
        ScanIngest::bytes += (int64_t)bytes;
        ScanIngest::seconds += now_seconds() - t0;
        dev_loaded = true;
        host_loaded = false;
    }

    static constexpr size_t kSlotBytes = size_t(32) << 20;
    static constexpr int kSlots = 3;
    std::vector<std::string> files;
    bool binary = false, host_loaded = false, dev_loaded = false;
    std::string sep;
};

// `merge` (operators/merge.cpp): the GPU replaces the worker threads; the
// input passes through.
class MergeOp : public SingleInputOp {
public:
    void init(const Setting& root, const Setting& node) override
    {
        Operator::init(root, node);
        schema = nextOp->getOutSchema();
    }
    ResultCode scanStart(unsigned short tid) override { return nextOp->scanStart(tid); }
    GetNextResultT getNext(unsigned short tid) override { return nextOp->getNext(tid); }
    ResultCode scanStop(unsigned short tid) override { return nextOp->scanStop(tid); }
    bool device_result(const void** dev, int64_t* n) override { return nextOp->device_result(dev, n); }
};

// `printer_tuplecount` (operators/printer_tuplecount.cpp): counts tuples.
class TupleCountPrinter : public SingleInputOp {
public:
    void init(const Setting& root, const Setting& node) override
    {
        Operator::init(root, node);
        schema = nextOp->getOutSchema();
    }
    ResultCode scanStart(unsigned short tid) override { return nextOp->scanStart(tid); }
    GetNextResultT getNext(unsigned short tid) override
    {
        GetNextResultT r = nextOp->getNext(tid);
        if (r.second) total += r.second->ntuples;
        return r;
    }
    ResultCode scanStop(unsigned short tid) override { return nextOp->scanStop(tid); }
    // A GPU parent reading the child's device buffer passes every tuple.
    bool device_result(const void** dev, int64_t* n) override
    {
        if (!nextOp->device_result(dev, n)) return false;
        total += *n;
        return true;
    }
    int64_t total = 0;
};

// ------------------------------------------------------------- hash join

static std::vector<pyg_proj> parse_projection(const Setting& line)
{
    // "B$i" / "P$i" (operators/join.cpp:142-183).
    std::vector<pyg_proj> out;
    for (size_t i = 0; i < line.size(); ++i) {
        const std::string& s = line[i].asString();
        size_t d = s.find('$');
        if (d == std::string::npos || d == 0) throw EngineError("bad projection '" + s + "'");
        char side = s[d - 1];
        if (side != 'B' && side != 'P') throw EngineError("bad projection '" + s + "'");
        pyg_proj p;
        p.side = side == 'P' ? 1 : 0;
        p.col = (int32_t)strtol(s.c_str() + d + 1, nullptr, 10);
        out.push_back(p);
    }
    return out;
}

static std::vector<int32_t> parse_attrs(const Setting& s)
{
    std::vector<int32_t> v;
    if (s.isAggregate())
        for (size_t i = 0; i < s.size(); ++i) v.push_back((int32_t)s[i].asInt());
    else
        v.push_back((int32_t)s.asInt());
    return v;
}

// `hashjoin` (HashJoinOp, operators/join.cpp:367-903).
class HashJoinOp : public DualInputOp {
public:
    void init(const Setting& root, const Setting& node) override
    {
        Operator::init(root, node);
        proj = parse_projection(node["projection"]);
        bkeys = parse_attrs(node["buildjattr"]);
        pkeys = parse_attrs(node["probejattr"]);
        if (bkeys.size() != pkeys.size()) throw EngineError("hashjoin: key arity differs");
        for (auto& p : proj) {
            Schema& s = p.side ? probeOp->getOutSchema() : buildOp->getOutSchema();
            if (p.col < 0 || (size_t)p.col >= s.columns()) throw EngineError("hashjoin: projection out of range");
            schema.add(s.types[p.col]);
        }
        if (node.exists("gpu") && node["gpu"].exists("loadfactor"))
            load_factor = (float)node["gpu"]["loadfactor"].asFloat();
    }

    // An aggregate above asks for count + column sums instead of rows.
    bool fuse = false;
    pyg_join_result fused;

    ResultCode scanStart(unsigned short tid) override
    {
        if (buildOp->scanStart(tid) == Error || probeOp->scanStart(tid) == Error) return Error;
        HostRel R, S;
        pyg_rel r = input_rel(buildOp, tid, R);
        pyg_rel s = input_rel(probeOp, tid, S);
        buildOp->scanStop(tid);
        if (fuse) {
            pyg_join_opts o = {PYG_JOIN_AUTO, 0, load_factor, 0};
            check(pyg_hashjoin_agg(ctx, &r, bkeys.data(), &s, pkeys.data(), (int32_t)bkeys.size(), proj.data(),
                                   (int32_t)proj.size(), &o, &fused, nullptr),
                  "hashjoin (fused aggregate)");
            out.host.ntuples = 0;
            out.keep_host();
            return Ready;
        }
        std::vector<int32_t> pay;
        for (auto& p : proj)
            if (!p.side) pay.push_back(p.col);
        pyg_hashtable* ht = nullptr;
        check(pyg_hashjoin_build(ctx, &r, bkeys.data(), (int32_t)bkeys.size(), pay.data(), (int32_t)pay.size(),
                                 PYG_HT_MATERIALIZE, load_factor, &ht),
              "hashjoin build");
        int64_t n = 0;
        int rc = pyg_hashjoin_probe_materialize(ctx, ht, &s, pkeys.data(), proj.data(), (int32_t)proj.size(), nullptr,
                                                0, &n);
        if (rc != PYG_OK && rc != PYG_ERR_CAPACITY) check(rc, "hashjoin probe");
        void* dev = nullptr;
        check(pyg_alloc(ctx, (size_t)(n > 0 ? n : 1) * schema.tuple_bytes, &dev), "hashjoin output");
        rc = pyg_hashjoin_probe_materialize(ctx, ht, &s, pkeys.data(), proj.data(), (int32_t)proj.size(), dev, n, &n);
        pyg_hashtable_free(ctx, ht);
        if (rc != PYG_OK) pyg_free(ctx, dev);
        check(rc, "hashjoin probe");
        out.keep_device(dev, n, schema.tuple_bytes);
        return Ready;
    }

    GetNextResultT getNext(unsigned short tid) override { return out.next(buffsize, schema.tuple_bytes); }
    bool device_result(const void** dev, int64_t* n) override { return out.device(dev, n); }

    ResultCode scanStop(unsigned short tid) override
    {
        out.rewind();
        return probeOp->scanStop(tid);
    }

    std::vector<pyg_proj> proj;
    std::vector<int32_t> bkeys, pkeys;

private:
    float load_factor = 0.5f;
    ResultBuffer out;
};

// ------------------------------------------------------------ aggregates

// `aggregate_sum` / `aggregate_count` (GenericAggregate + AggregateSum /
// AggregateCount, operators/genericaggregate.cpp:51-494).  Groups come out
// ordered by key (the reference emits hash order; any order is valid).
class AggregateOp : public MaterializedOp {
public:
    explicit AggregateOp(bool sum) : is_sum(sum) {}
    Operator* nextOp = nullptr;
    std::vector<Operator*> children() override { return {nextOp}; }

    void init(const Setting& root, const Setting& node) override
    {
        Operator::init(root, node);
        if (node.exists("fields")) {
            const Setting& f = node["fields"];
            for (size_t i = 0; i < f.size(); ++i) keys.push_back((int32_t)f[i].asInt());
        } else {
            keys.push_back((int32_t)node["field"].asInt());
        }
        Schema& in = nextOp->getOutSchema();
        for (int32_t k : keys) {
            if (k < 0 || (size_t)k >= in.columns()) throw EngineError(name + ": group field out of range");
            schema.add(in.types[k]);
        }
        if (is_sum) {
            sumfield = (int32_t)node["sumfield"].asInt();
            if (sumfield < 0 || (size_t)sumfield >= in.columns()) throw EngineError(name + ": sumfield out of range");
            schema.add(in.types[sumfield]);
        } else {
            schema.add(PYG_INT64);
        }
        if (node.exists("hash") && node["hash"].exists("buckets")) expected = node["hash"]["buckets"].asInt();
        if (keys.size() > 2) throw EngineError(name + ": at most two group-by columns on the GPU path");
    }

    ResultCode scanStart(unsigned short tid) override
    {
        out.rewind();
        // No GROUP BY straight over a hash join (possibly through
        // printer_tuplecount / merge): fuse the aggregate into the probe.
        if (keys.empty()) {
            std::vector<TupleCountPrinter*> counters;
            Operator* op = nextOp;
            while (op) {
                if (auto* c = dynamic_cast<TupleCountPrinter*>(op)) {
                    counters.push_back(c);
                    op = c->nextOp;
                } else if (auto* m = dynamic_cast<MergeOp*>(op)) {
                    op = m->nextOp;
                } else {
                    break;
                }
            }
            auto* hj = dynamic_cast<HashJoinOp*>(op);
            if (hj) {
                hj->fuse = true;
                if (nextOp->scanStart(tid) == Error) return Error;
                nextOp->scanStop(tid);
                for (auto* c : counters) c->total += hj->fused.count;
                uint64_t v = is_sum ? (uint64_t)hj->fused.sums[sumfield] : (uint64_t)hj->fused.count;
                HostRel& result = out.host;
                result.tuple_bytes = schema.tuple_bytes;
                result.ntuples = 0;
                if (hj->fused.count > 0) {
                    uint8_t row[8];
                    if (schema.types[0] == PYG_INT32) {
                        uint32_t w = (uint32_t)v;
                        memcpy(row, &w, 4);
                    } else {
                        memcpy(row, &v, 8);
                    }
                    result.append(row, 1);
                }
                out.keep_host();
                return Ready;
            }
        }
        if (nextOp->scanStart(tid) == Error) return Error;
        HostRel in;
        pyg_rel r = input_rel(nextOp, tid, in);
        int64_t cap = r.ntuples > 0 ? r.ntuples : 1;
        void* dev = nullptr;
        check(pyg_alloc(ctx, (size_t)cap * schema.tuple_bytes, &dev), name.c_str());
        int64_t g = 0;
        int rc = pyg_groupby(ctx, &r, keys.data(), (int32_t)keys.size(), is_sum ? PYG_AGG_SUM : PYG_AGG_COUNT,
                             is_sum ? sumfield : 0, 1, expected, dev, cap, &g);
        nextOp->scanStop(tid);
        if (rc != PYG_OK) pyg_free(ctx, dev);
        check(rc, name.c_str());
        out.keep_device(dev, g, schema.tuple_bytes);
        return Ready;
    }

private:
    bool is_sum;
    std::vector<int32_t> keys;
    int32_t sumfield = 0;
    int64_t expected = 0;
};

// ------------------------------------------------------ partition / sort

// `partition` (PartitionOp, operators/partition.cpp:44-404): exact range
// partition on `attr` over `range` into `buckets`; the partitions come out
// one after another (partition b is what reference thread b serves).
class PartitionOp : public MaterializedOp {
public:
    Operator* nextOp = nullptr;
    std::vector<Operator*> children() override { return {nextOp}; }
    void init(const Setting& root, const Setting& node) override
    {
        Operator::init(root, node);
        schema = nextOp->getOutSchema();
        attr = (int32_t)node["attr"].asInt();
        mn = node["range"][0].asInt();
        mx = node["range"][1].asInt();
        buckets = (int32_t)node["buckets"].asInt();
        sortout = node.getString("sort", "no") == "yes";
        sortattr = (int32_t)node.getInt("sortattr", attr);
    }
    ResultCode scanStart(unsigned short tid) override
    {
        if (nextOp->scanStart(tid) == Error) return Error;
        HostRel in;
        pyg_rel r = input_rel(nextOp, tid, in);
        const int64_t n_in = r.ntuples;
        void* dev = nullptr;
        check(pyg_alloc(ctx, (size_t)(n_in > 0 ? n_in : 1) * schema.tuple_bytes, &dev), "partition");
        pyg_splitter s = {PYG_SPLIT_EXACTRANGE, buckets, mn, mx, nullptr};
        offsets.assign(buckets + 1, 0);
        int rc = pyg_partition(ctx, &r, attr, &s, dev, offsets.data());
        if (rc == PYG_OK && sortout) {
            // Sort each partition on sortattr (PartitionOp with sort = yes).
            void* tmp = nullptr;
            rc = pyg_alloc(ctx, (size_t)(n_in > 0 ? n_in : 1) * schema.tuple_bytes, &tmp);
            for (int b = 0; rc == PYG_OK && b < buckets; ++b) {
                int64_t n = offsets[b + 1] - offsets[b];
                if (n < 2) continue;
                pyg_rel pr = schema.rel((uint8_t*)dev + offsets[b] * schema.tuple_bytes, n, true);
                rc = pyg_sort(ctx, &pr, sortattr, (uint8_t*)tmp + offsets[b] * schema.tuple_bytes);
                if (rc == PYG_OK)
                    rc = pyg_memcpy_d2d(ctx, (uint8_t*)dev + offsets[b] * schema.tuple_bytes,
                                        (uint8_t*)tmp + offsets[b] * schema.tuple_bytes, (size_t)n * schema.tuple_bytes);
            }
            pyg_free(ctx, tmp);
        }
        nextOp->scanStop(tid);
        if (rc != PYG_OK) pyg_free(ctx, dev);
        check(rc, "partition");
        out.keep_device(dev, n_in, schema.tuple_bytes);
        return Ready;
    }
    std::vector<int64_t> offsets;

private:
    int32_t attr = 0, buckets = 1, sortattr = 0;
    int64_t mn = 0, mx = 0;
    bool sortout = false;
};

// `sort` (SortOp, operators/sort.cpp:87-311) on `attr`.
class SortOp : public MaterializedOp {
public:
    Operator* nextOp = nullptr;
    std::vector<Operator*> children() override { return {nextOp}; }
    void init(const Setting& root, const Setting& node) override
    {
        Operator::init(root, node);
        schema = nextOp->getOutSchema();
        attr = (int32_t)node["attr"].asInt();
    }
    ResultCode scanStart(unsigned short tid) override
    {
        if (nextOp->scanStart(tid) == Error) return Error;
        HostRel in;
        pyg_rel r = input_rel(nextOp, tid, in);
        void* dev = nullptr;
        check(pyg_alloc(ctx, (size_t)(r.ntuples > 0 ? r.ntuples : 1) * schema.tuple_bytes, &dev), "sort");
        int rc = pyg_sort(ctx, &r, attr, dev);
        nextOp->scanStop(tid);
        if (rc != PYG_OK) pyg_free(ctx, dev);
        check(rc, "sort");
        out.keep_device(dev, r.ntuples, schema.tuple_bytes);
        return Ready;
    }

private:
    int32_t attr = 0;
};

// `sortlimit` (SortLimit, operators/sortlimit.cpp:32-262): the first
// limit[0] tuples in the order of the `by` columns ("$i" strings, as
// parseSortInput reads them, :18-30), ascending when asc[0] == 1 else
// descending, ties in input order; pyg_sortlimit on the GPU.
class SortLimitOp : public MaterializedOp {
public:
    Operator* nextOp = nullptr;
    std::vector<Operator*> children() override { return {nextOp}; }
    void init(const Setting& root, const Setting& node) override
    {
        Operator::init(root, node);
        schema = nextOp->getOutSchema();
        const Setting& by = node["by"];
        for (size_t i = 0; i < by.size(); ++i) {
            const std::string& s = by[i].asString();
            const size_t d = s.find('$');
            if (d == std::string::npos || d + 1 >= s.size())
                throw EngineError("sortlimit: `by` entries name columns as \"$i\"");
            const int c = std::stoi(s.substr(d + 1));
            if (c < 0 || (size_t)c >= schema.columns()) throw EngineError("sortlimit: column out of range");
            keys.push_back(c);
        }
        asc = node["asc"][0].asInt() == 1;
        limit = node["limit"][0].asInt();
    }
    ResultCode scanStart(unsigned short tid) override
    {
        if (nextOp->scanStart(tid) == Error) return Error;
        HostRel in;
        pyg_rel r = input_rel(nextOp, tid, in);
        const int64_t k = limit < r.ntuples ? limit : r.ntuples;
        void* dev = nullptr;
        check(pyg_alloc(ctx, (size_t)(k > 0 ? k : 1) * schema.tuple_bytes, &dev), "sortlimit");
        int64_t n = 0;
        int rc = pyg_sortlimit(ctx, &r, keys.data(), (int32_t)keys.size(), asc ? 1 : 0, limit, dev, k, &n);
        nextOp->scanStop(tid);
        if (rc != PYG_OK) pyg_free(ctx, dev);
        check(rc, "sortlimit");
        out.keep_device(dev, n, schema.tuple_bytes);
        return Ready;
    }

private:
    std::vector<int32_t> keys;
    bool asc = true;
    int64_t limit = 0;
};

// `shmwriter` (MemSegmentWriter, operators/memsegmentwriter.cpp): writes
// its input's tuples into memory segments instead of returning them.  A
// segment is the file paths[i] + counter (a "/dev/shm/..." path is opened
// with shm_open, anything else as a file), created exclusively and mapped,
// of at most `size` bytes of whole tuples; when one is full the next path
// takes over round-robin, the seven-digit counter advancing after each
// cycle (:239-265, :380-452).  The last segment is truncated to the bytes
// it holds, and deleted when it holds none.  getNext returns Finished with
// an empty page.  The NUMA `policy` / `numanodes` settings are accepted
// and, as in a reference build without NUMA, only warned about.
class ShmWriterOp : public Operator {
public:
    Operator* nextOp = nullptr;
    std::vector<Operator*> children() override { return {nextOp}; }
    void init(const Setting& root, const Setting& node) override
    {
        Operator::init(root, node);
        schema = nextOp->getOutSchema();
        seg_bytes = node["size"].asInt();
        if (node.exists("policy"))
            std::cerr << " ** NUMA POLICY WARNING: Memory policy is ignored by the GPU engine." << std::endl;
        const Setting& p = node["paths"];
        if (p.isAggregate())
            for (size_t i = 0; i < p.size(); ++i) paths.push_back(p[i].asString());
        else
            paths.push_back(p.asString());
        if (paths.empty()) throw EngineError("shmwriter: no paths");
        if (seg_bytes < schema.tuple_bytes) throw EngineError("shmwriter: size below one tuple");
    }
    ResultCode scanStart(unsigned short tid) override { return nextOp->scanStart(tid); }
    ResultCode scanStop(unsigned short tid) override { return nextOp->scanStop(tid); }
    GetNextResultT getNext(unsigned short tid) override
    {
        const int64_t tb = schema.tuple_bytes;
        const int64_t per = seg_bytes / tb;  // tuples per segment
        std::string counter = "0000000";
        size_t node = 0;
        Segment seg;
        seg.open(paths[node] + counter, (size_t)seg_bytes);
        GetNextResultT r;
        do {
            r = nextOp->getNext(tid);
            if (r.first == Error) {
                seg.close(0);
                return r;
            }
            const Page* in = r.second;
            int64_t at = 0;
            while (in && at < in->ntuples) {
                const int64_t room = per - seg.used / tb;
                const int64_t take = std::min(room, in->ntuples - at);
                memcpy(seg.mem + seg.used, in->data + at * tb, (size_t)(take * tb));
                seg.used += (size_t)(take * tb);
                at += take;
                if (at < in->ntuples) {  // full: the next path, the counter after a cycle
                    seg.close(seg.used);
                    node = (node + 1) % paths.size();
                    if (node == 0) advance(counter);
                    seg.open(paths[node] + counter, (size_t)seg_bytes);
                }
            }
        } while (r.first == Ready);
        seg.close(seg.used);
        empty.ntuples = 0;
        empty.tuple_bytes = schema.tuple_bytes;
        return std::make_pair(Finished, &empty);
    }

private:
    struct Segment {
        std::string name;
        uint8_t* mem = nullptr;
        size_t cap = 0, used = 0;
        void open(const std::string& path, size_t bytes)
        {
            name = path;
            const bool shm = path.compare(0, 8, "/dev/shm") == 0;
            const int fd = shm ? shm_open(path.c_str() + 8, O_RDWR | O_EXCL | O_CREAT, S_IRUSR | S_IWUSR)
                               : ::open(path.c_str(), O_RDWR | O_EXCL | O_CREAT, S_IRUSR | S_IWUSR);
            if (fd == -1) throw EngineError("shmwriter: cannot create segment " + path);
            if (ftruncate(fd, (off_t)bytes) != 0) {
                ::close(fd);
                throw EngineError("shmwriter: cannot size segment " + path);
            }
            void* m = mmap(nullptr, bytes, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_NORESERVE, fd, 0);
            ::close(fd);
            if (m == MAP_FAILED) throw EngineError("shmwriter: cannot map segment " + path);
            mem = (uint8_t*)m;
            cap = bytes;
            used = 0;
        }
        // Unmaps, then truncates to the bytes written (unlinks when none).
        void close(size_t bytes)
        {
            if (!mem) return;
            munmap(mem, cap);
            mem = nullptr;
            const bool shm = name.compare(0, 8, "/dev/shm") == 0;
            if (bytes == 0) {
                if (shm) shm_unlink(name.c_str() + 8);
                else unlink(name.c_str());
                return;
            }
            if (truncate(name.c_str(), (off_t)bytes) != 0) throw EngineError("shmwriter: cannot truncate " + name);
        }
    };
    static void advance(std::string& c)
    {
        for (int pos = (int)c.size() - 1; pos >= 0; --pos) {
            if (c[pos] != '9') {
                ++c[pos];
                return;
            }
            c[pos] = '0';
        }
        throw EngineError("shmwriter: segment counter overflowed");
    }
    int64_t seg_bytes = 0;
    std::vector<std::string> paths;
    Page empty;
};

// Largest number of tuples of `in` that share one value of column `key`:
// a GPU count per key (pyg_groupby), then the maximum on the host.
static int64_t max_key_multiplicity(pyg_ctx* ctx, const pyg_rel& in, int32_t key)
{
    if (in.ntuples == 0) return 0;
    const int kb = in.col_type[key] == PYG_INT32 ? 4 : 8;
    const size_t tb = (size_t)kb + 8;  // key, count
    void* out = nullptr;
    check(pyg_alloc(ctx, (size_t)in.ntuples * tb, &out), "key multiplicity");
    int64_t groups = 0;
    int rc = pyg_groupby(ctx, &in, &key, 1, PYG_AGG_COUNT, 0, 0, 0, out, in.ntuples, &groups);
    std::vector<uint8_t> h;
    if (rc == PYG_OK) {
        h.resize((size_t)groups * tb);
        if (groups) rc = pyg_memcpy_d2h(ctx, h.data(), out, h.size());
    }
    pyg_free(ctx, out);
    check(rc, "key multiplicity");
    int64_t most = 0;
    for (int64_t g = 0; g < groups; ++g) {
        int64_t c;
        memcpy(&c, h.data() + (size_t)g * tb + kb, 8);
        most = c > most ? c : most;
    }
    return most;
}

// `sortmergejoin` / `mpsmjoin` / `newmpsmjoin` / `preprejoin`
// (operators/join.cpp:905-2212): MPSM join on single keys.  The
// buildprepartitioned range (if any) gives equal-width splitters as the
// reference; an optional gpu { splitter = "sampled" | "learned" |
// "exactrange"; fanout = N; } group picks the splitters.
// `newmpsmjoin` and `preprejoin` merge through a buffer that holds at most
// `mostfreqbuildkeyoccurances` build tuples of one key (newmpsmjoin adds
// the setting as 1 when it is missing, operators/join.cpp:1628-1631;
// preprejoin requires it, :1821, and sizes its buffer by it, :1857-1859).
// The reference overruns that buffer when a build key repeats more often;
// here such a build side is refused with an error naming both numbers.
class MpsmJoinOp : public DualInputOp {
public:
    void init(const Setting& root, const Setting& node) override
    {
        Operator::init(root, node);
        proj = parse_projection(node["projection"]);
        bkey = parse_attrs(node["buildjattr"]).at(0);
        pkey = parse_attrs(node["probejattr"]).at(0);
        for (auto& p : proj) {
            Schema& s = p.side ? probeOp->getOutSchema() : buildOp->getOutSchema();
            if (p.col < 0 || (size_t)p.col >= s.columns()) throw EngineError("mpsm: projection out of range");
            schema.add(s.types[p.col]);
        }
        memset(&opts, 0, sizeof(opts));
        opts.splitter_kind = PYG_MPSM_SPLIT_SAMPLED;
        opts.fanout = 1024;
        opts.sample_rate = 0.01;
        opts.cdf_leaves = 1024;
        opts.page_tuples = 256;
        opts.seed = 1;
        if (node.exists("buildprepartitioned")) {
            opts.splitter_kind = PYG_MPSM_SPLIT_EXACTRANGE;
            opts.fanout = (int32_t)node["buildprepartitioned"]["buckets"].asInt();
        }
        if (node.exists("gpu")) {
            const Setting& g = node["gpu"];
            std::string k = g.getString("splitter", "sampled");
            opts.splitter_kind = k == "learned" ? PYG_MPSM_SPLIT_LEARNED
                                 : k == "exactrange" ? PYG_MPSM_SPLIT_EXACTRANGE : PYG_MPSM_SPLIT_SAMPLED;
            opts.fanout = (int32_t)g.getInt("fanout", opts.fanout);
        }
        if (type == "preprejoin" && !node.exists("mostfreqbuildkeyoccurances"))
            throw EngineError("preprejoin: mostfreqbuildkeyoccurances is required");
        if (type == "newmpsmjoin" || type == "preprejoin") {
            mfbko = node.getInt("mostfreqbuildkeyoccurances", 1);
            if (mfbko < 1) throw EngineError(type + ": mostfreqbuildkeyoccurances must be at least 1");
        }
    }
    ResultCode scanStart(unsigned short tid) override
    {
        if (buildOp->scanStart(tid) == Error || probeOp->scanStart(tid) == Error) return Error;
        HostRel R, S;
        pyg_rel r = input_rel(buildOp, tid, R);
        pyg_rel s = input_rel(probeOp, tid, S);
        if (mfbko > 0) {
            const int64_t most = max_key_multiplicity(ctx, r, bkey);
            if (most > mfbko)
                throw EngineError(type + ": a build key occurs " + std::to_string(most) +
                                  " times, more than mostfreqbuildkeyoccurances = " + std::to_string(mfbko));
        }
        int64_t n = 0;
        int rc = pyg_mpsm_join_materialize(ctx, &r, bkey, &s, pkey, proj.data(), (int32_t)proj.size(), &opts, nullptr,
                                           0, &n);
        if (rc != PYG_OK && rc != PYG_ERR_CAPACITY) check(rc, "mpsm join");
        void* dev = nullptr;
        check(pyg_alloc(ctx, (size_t)(n > 0 ? n : 1) * schema.tuple_bytes, &dev), "mpsm output");
        rc = pyg_mpsm_join_materialize(ctx, &r, bkey, &s, pkey, proj.data(), (int32_t)proj.size(), &opts, dev, n, &n);
        buildOp->scanStop(tid);
        probeOp->scanStop(tid);
        if (rc != PYG_OK) pyg_free(ctx, dev);
        check(rc, "mpsm join");
        out.keep_device(dev, n, schema.tuple_bytes);
        return Ready;
    }
    GetNextResultT getNext(unsigned short tid) override { return out.next(buffsize, schema.tuple_bytes); }
    bool device_result(const void** dev, int64_t* n) override { return out.device(dev, n); }
    ResultCode scanStop(unsigned short tid) override
    {
        out.rewind();
        return Ready;
    }

private:
    std::vector<pyg_proj> proj;
    int32_t bkey = 0, pkey = 0;
    int64_t mfbko = 0;  // 0: no bound (sortmergejoin, mpsmjoin)
    pyg_mpsm_opts opts;
    ResultBuffer out;
};

// ------------------------------------------------------------------ Query

static void set_input(Operator* op, Operator* child)
{
    if (auto* s = dynamic_cast<SingleInputOp*>(op)) s->nextOp = child;
    else if (auto* a = dynamic_cast<AggregateOp*>(op)) a->nextOp = child;
    else if (auto* p = dynamic_cast<PartitionOp*>(op)) p->nextOp = child;
    else if (auto* so = dynamic_cast<SortOp*>(op)) so->nextOp = child;
    else if (auto* sl = dynamic_cast<SortLimitOp*>(op)) sl->nextOp = child;
    else if (auto* sw = dynamic_cast<ShmWriterOp*>(op)) sw->nextOp = child;
    else throw EngineError("operator '" + op->name + "' takes no input");
}

static Operator* construct(Query& q, const Setting& root, const Setting& node)
{
    const std::string& name = node["name"].asString();
    const Setting& cfg = root[name];
    const std::string type = cfg["type"].asString();
    std::unique_ptr<Operator> op;
    if (type == "scan" || type == "parallelscan" || type == "partitionedscan") op.reset(new ScanOp());
    else if (type == "hashjoin") op.reset(new HashJoinOp());
    else if (type == "sortmergejoin" || type == "mpsmjoin" || type == "newmpsmjoin" || type == "preprejoin")
        op.reset(new MpsmJoinOp());
    else if (type == "aggregate_sum") op.reset(new AggregateOp(true));
    else if (type == "aggregate_count") op.reset(new AggregateOp(false));
    else if (type == "merge") op.reset(new MergeOp());
    else if (type == "printer_tuplecount") op.reset(new TupleCountPrinter());
    else if (type == "partition") op.reset(new PartitionOp());
    else if (type == "sort") op.reset(new SortOp());
    else if (type == "sortlimit") op.reset(new SortLimitOp());
    else if (type == "shmwriter") op.reset(new ShmWriterOp());
    else throw EngineError("plan node type '" + type + "' is not on the GPU join/aggregation path");
    op->type = type;
    op->name = name;
    Operator* raw = op.get();
    q.ops.push_back(std::move(op));
    if (auto* d = dynamic_cast<DualInputOp*>(raw)) {
        d->buildOp = construct(q, root, node["build"]);
        d->probeOp = construct(q, root, node["probe"]);
    } else if (node.exists("input")) {
        set_input(raw, construct(q, root, node["input"]));
    } else if (!dynamic_cast<ScanOp*>(raw)) {
        throw EngineError("operator '" + name + "' needs an input");
    }
    raw->init(root, cfg);  // after the children, as Query::create does
    return raw;
}

void Query::create(std::unique_ptr<Setting> plan_root)
{
    plan = std::move(plan_root);
    root = construct(*this, *plan, (*plan)["treeroot"]);
}

void Query::threadInit()
{
    for (auto& op : ops) op->threadInit(0);
}

void Query::threadClose()
{
    for (auto& op : ops) op->threadClose(0);
}

std::vector<std::string> Query::counter_report() const
{
    std::vector<std::string> out;
    for (auto& op : ops)
        if (auto* c = dynamic_cast<TupleCountPrinter*>(op.get()))
            out.push_back("TupleCountPrinter (total=" + std::to_string(c->total) + " tuples)");
    return out;
}

}  // namespace pyg_host

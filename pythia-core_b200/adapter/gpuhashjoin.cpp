// GpuHashJoinOp: the reference engine's `hashjoin` on the GPU, behind the
// reference's own Operator contract.  The class comment in gpuhashjoin.h
// lists which reference method each member replaces.
#include "gpuhashjoin.h"

#include <pthread.h>
#include <stdio.h>
#include <string.h>

#include "exceptions.h"

pyg_ctx* GpuHashJoinOp::ctx_ = 0;

// A libpyg context serves one host thread at a time, and the leaders of
// different thread groups join concurrently: they take turns on it.
static pthread_mutex_t g_ctx_mutex = PTHREAD_MUTEX_INITIALIZER;

namespace {
struct CtxLock {
    CtxLock() { pthread_mutex_lock(&g_ctx_mutex); }
    ~CtxLock() { pthread_mutex_unlock(&g_ctx_mutex); }
};
}  // namespace

pyg_ctx* GpuHashJoinOp::context() { return ctx_; }

GpuHashJoinOp::GpuHashJoinOp() : load_factor_(0.5f) {}

GpuHashJoinOp::~GpuHashJoinOp()
{
    for (size_t i = 0; i < threads_.size(); ++i) delete threads_[i];
}

// Maps a reference column to its libpyg type: keys need CT_INTEGER /
// CT_LONG; other columns only need a 4- or 8-byte width (copied as bits).
static int32_t pyg_type_of(Schema& s, unsigned int col)
{
    const unsigned int size = s.get(col).size;
    if (size == 4) return PYG_INT32;
    if (size == 8) return PYG_INT64;
    throw InvalidParameter();
}

void GpuHashJoinOp::init(libconfig::Config& root, libconfig::Setting& node)
{
    JoinOp::init(root, node);
    Schema& bs = buildOp->getOutSchema();
    Schema& ps = probeOp->getOutSchema();
    unsigned int keybytes = 0;
    for (size_t i = 0; i < joinvec1.size(); ++i) {
        ColumnType bt = bs.getColumnType(joinvec1[i]);
        ColumnType pt = ps.getColumnType(joinvec2[i]);
        if ((bt != CT_INTEGER && bt != CT_LONG) || bt != pt) throw InvalidParameter();
        keybytes += bs.get(joinvec1[i]).size;
        bkeys_.push_back(joinvec1[i]);
        pkeys_.push_back(joinvec2[i]);
    }
    if (bkeys_.empty() || bkeys_.size() > 2 || keybytes > 8) throw InvalidParameter();
    if (bs.columns() > PYG_MAX_COLS || ps.columns() > PYG_MAX_COLS) throw InvalidParameter();
    for (unsigned int c = 0; c < bs.columns(); ++c) pyg_type_of(bs, c);
    for (unsigned int c = 0; c < ps.columns(); ++c) pyg_type_of(ps, c);
    for (size_t i = 0; i < projection.size(); ++i) {
        pyg_proj p;
        p.side = projection[i].first == BuildSide ? 0 : 1;
        p.col = (int32_t)projection[i].second;
        proj_.push_back(p);
        if (p.side == 0) payload_.push_back(p.col);
    }
    if (node.exists("gpu") && node["gpu"].exists("loadfactor")) load_factor_ = (float)(double)node["gpu"]["loadfactor"];
    int device = 0;
    if (node.exists("gpu") && node["gpu"].exists("device")) device = node["gpu"]["device"];
    if (!ctx_ && pyg_ctx_create(device, &ctx_) != PYG_OK) throw QueryExecutionError();
    groups_.assign(groupleader.size(), Group());
    threads_.assign(MAX_THREADS, (ThreadState*)0);
}

void GpuHashJoinOp::threadInit(unsigned short threadid)
{
    if (!threads_[threadid]) threads_[threadid] = new ThreadState();
}

bool GpuHashJoinOp::drain(Operator* op, unsigned short threadid, std::vector<char>& out, unsigned int tuplesize)
{
    GetNextResultT r;
    r.first = Operator::Ready;
    while (r.first == Operator::Ready) {
        r = op->getNext(threadid);
        if (r.first == Operator::Error) return false;
        if (!r.second) continue;
        // A page is a run of tuples from its start to its free pointer.
        Page::Iterator it = r.second->createIterator();
        void* first = it.next();
        if (!first) continue;
        const unsigned long long used = r.second->getUsedSpace();
        const size_t at = out.size();
        out.resize(at + used);
        memcpy(&out[at], first, used);
    }
    return out.size() % tuplesize == 0;
}

pyg_rel GpuHashJoinOp::as_rel(Schema& s, const std::vector<char>& data)
{
    pyg_rel r;
    memset(&r, 0, sizeof(r));
    const unsigned int tb = s.getTupleSize();
    r.base = data.empty() ? 0 : &data[0];
    r.ntuples = (int64_t)(data.size() / tb);
    r.tuple_bytes = (int32_t)tb;
    r.ncols = (int32_t)s.columns();
    char probe[64];
    for (unsigned int c = 0; c < s.columns(); ++c) {
        r.col_offset[c] = (int32_t)((char*)s.calcOffset(probe, c) - probe);
        r.col_type[c] = pyg_type_of(s, c);
    }
    r.on_device = 0;
    return r;
}

// The group leader's GPU join over every thread's drained tuples.
void GpuHashJoinOp::join_group(unsigned short groupno)
{
    Group& g = groups_[groupno];
    std::vector<char> R, S;
    for (unsigned short t = 0; t < MAX_THREADS; ++t) {
        if (threadgroups[t] != groupno || !threads_[t]) continue;
        ThreadState& ts = *threads_[t];
        if (ts.failed) g.failed = true;
        R.insert(R.end(), ts.build.begin(), ts.build.end());
        S.insert(S.end(), ts.probe.begin(), ts.probe.end());
        std::vector<char>().swap(ts.build);
        std::vector<char>().swap(ts.probe);
    }
    if (g.out) pyg_host_free(g.out);
    g.out = 0;
    g.nout = 0;
    if (g.failed) return;
    pyg_rel r = as_rel(buildOp->getOutSchema(), R);
    pyg_rel s = as_rel(probeOp->getOutSchema(), S);
    const unsigned int tb = schema.getTupleSize();
    CtxLock lock;
    pyg_hashtable* ht = 0;
    void* dev = 0;
    int64_t n = 0;
    int rc = pyg_hashjoin_build(ctx_, &r, &bkeys_[0], (int32_t)bkeys_.size(), payload_.empty() ? 0 : &payload_[0],
                                (int32_t)payload_.size(), PYG_HT_MATERIALIZE, load_factor_, &ht);
    if (rc == PYG_OK) {
        // First pass counts the pairs, second writes them.
        rc = pyg_hashjoin_probe_materialize(ctx_, ht, &s, &pkeys_[0], &proj_[0], (int32_t)proj_.size(), 0, 0, &n);
        if (rc == PYG_ERR_CAPACITY) rc = PYG_OK;
    }
    if (rc == PYG_OK) rc = pyg_alloc(ctx_, (size_t)(n > 0 ? n : 1) * tb, &dev);
    if (rc == PYG_OK)
        rc = pyg_hashjoin_probe_materialize(ctx_, ht, &s, &pkeys_[0], &proj_[0], (int32_t)proj_.size(), dev, n, &n);
    void* host = 0;
    if (rc == PYG_OK) rc = pyg_host_alloc((size_t)(n > 0 ? n : 1) * tb, &host);
    if (rc == PYG_OK && n > 0) rc = pyg_memcpy_d2h(ctx_, host, dev, (size_t)n * tb);
    if (dev) pyg_free(ctx_, dev);
    if (ht) pyg_hashtable_free(ctx_, ht);
    if (rc != PYG_OK) {
        fprintf(stderr, "GpuHashJoinOp: group %u: %s\n", (unsigned)groupno, pyg_last_error());
        if (host) pyg_host_free(host);
        g.failed = true;
        return;
    }
    g.out = (char*)host;
    g.nout = n;
}

Operator::ResultCode GpuHashJoinOp::scanStart(unsigned short threadid, Page* indexdatapage, Schema& indexdataschema)
{
    const unsigned short groupno = threadgroups.at(threadid);
    ThreadState& ts = *threads_.at(threadid);
    ts.failed = false;
    ts.build.clear();
    ts.probe.clear();
    if (isLeftThread(threadid)) {
        if (buildOp->scanStart(threadid, indexdatapage, indexdataschema) == Error ||
            !drain(buildOp, threadid, ts.build, buildOp->getOutSchema().getTupleSize()) ||
            buildOp->scanStop(threadid) == Error)
            ts.failed = true;
    }
    if (probeOp->scanStart(threadid, indexdatapage, indexdataschema) == Error ||
        !drain(probeOp, threadid, ts.probe, probeOp->getOutSchema().getTupleSize()))
        ts.failed = true;
    groups_[groupno].failed = false;

    barriers[groupno].Arrive();
    if (groupleader[groupno] == threadid) join_group(groupno);
    barriers[groupno].Arrive();

    Group& g = groups_[groupno];
    if (g.failed) return Error;
    const long long size = groupsize[groupno], at = threadposingrp[threadid];
    ts.pos = g.nout * at / size;
    ts.end = g.nout * (at + 1) / size;
    return Ready;
}

Operator::GetNextResultT GpuHashJoinOp::getNext(unsigned short threadid)
{
    ThreadState& ts = *threads_.at(threadid);
    const Group& g = groups_[threadgroups.at(threadid)];
    const unsigned int tb = schema.getTupleSize();
    long long per = buffsize / tb;
    if (per < 1) per = 1;
    const long long k = ts.end - ts.pos < per ? ts.end - ts.pos : per;
    // The page wraps the group output in place; it stays valid until the
    // thread's next getNext or threadClose.
    delete ts.page;
    char* at = g.out ? g.out + ts.pos * tb : 0;
    static char empty[64];
    if (!at) at = empty;
    ts.page = new Page(at, (unsigned long long)(k > 0 ? k : 1) * tb, at + k * tb, tb);
    ts.pos += k;
    return GetNextResultT(ts.pos >= ts.end ? Finished : Ready, ts.page);
}

Operator::ResultCode GpuHashJoinOp::scanStop(unsigned short threadid) { return probeOp->scanStop(threadid); }

void GpuHashJoinOp::threadClose(unsigned short threadid)
{
    const unsigned short groupno = threadgroups.at(threadid);
    ThreadState* ts = threads_.at(threadid);
    if (ts) {
        delete ts->page;
        ts->page = 0;
    }
    barriers[groupno].Arrive();
    if (groupleader[groupno] == threadid) {
        Group& g = groups_[groupno];
        CtxLock lock;
        if (g.out) pyg_host_free(g.out);
        g.out = 0;
        g.nout = 0;
    }
}

void GpuHashJoinOp::destroy() {}

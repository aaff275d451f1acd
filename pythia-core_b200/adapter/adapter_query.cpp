// adapter_query: runs a reference plan file in the reference engine
// (Query::create, query.cpp:321-326, linked from the reference's own
// objects) with every `hashjoin` node replaced by GpuHashJoinOp, and prints
// the rows and the response time in the reference driver's output format
// (drivers/executequery.cpp:67-154).  With --cpu the plan runs unchanged,
// on the reference's own HashJoinOp, for comparison.
//
// The substitution is what one line in the reference's constructsubtree
// (query.cpp:178-199) would do for a node of type "gpuhashjoin"; the
// reference's user-defined operator map only takes single-input operators,
// so this driver swaps the operator after Query::create instead: it walks
// the plan's tree of settings and the operator tree together, builds a
// GpuHashJoinOp over the hashjoin's two children and initialises it with
// the hashjoin's own setting.
#include <stdio.h>
#include <string.h>
#include <time.h>

#include <iostream>
#include <string>

#include "gpuhashjoin.h"
#include "libconfig.h++"
#include "query.h"
#include "visitors/allvisitors.h"

static int replaced = 0;

static void substitute(libconfig::Config& cfg, libconfig::Setting& cfgnode, Operator** slot)
{
    std::string name = (const char*)cfgnode["name"];
    std::string type = (const char*)cfg.getRoot()[name]["type"];
    Operator* op = *slot;
    DualInputOp* dual = dynamic_cast<DualInputOp*>(op);
    SingleInputOp* single = dynamic_cast<SingleInputOp*>(op);
    if (dual) {
        substitute(cfg, cfgnode["build"], &dual->buildOp);
        substitute(cfg, cfgnode["probe"], &dual->probeOp);
    } else if (single) {
        substitute(cfg, cfgnode["input"], &single->nextOp);
    }
    if (type == "hashjoin") {
        GpuHashJoinOp* g = new GpuHashJoinOp();
        g->buildOp = dual->buildOp;
        g->probeOp = dual->probeOp;
        g->init(cfg, cfg.getRoot()[name]);
        *slot = g;  // the CPU operator is left unlinked
        ++replaced;
    }
}

int main(int argc, char** argv)
{
    bool cpu = false;
    const char* plan = 0;
    for (int i = 1; i < argc; ++i) {
        if (!strcmp(argv[i], "--cpu"))
            cpu = true;
        else
            plan = argv[i];
    }
    if (!plan) {
        std::cerr << "usage: adapter_query [--cpu] plan.conf" << std::endl;
        return 2;
    }
    try {
        libconfig::Config cfg;
        cfg.readFile(plan);
        Query q;
        q.create(cfg);
        if (!cpu) substitute(cfg, cfg.lookup("treeroot"), &q.tree);
        std::cout << "GpuHashJoinOps: " << replaced << std::endl;
        std::cout << "BUFFSIZE: " << (int)cfg.getRoot()["buffsize"] << std::endl;
        q.threadInit();
        timespec t0, t1;
        clock_gettime(CLOCK_MONOTONIC, &t0);
        if (q.scanStart() == Operator::Error) throw QueryExecutionError();
        Operator::GetNextResultT r;
        r.first = Operator::Ready;
        while (r.first == Operator::Ready) {
            r = q.getNext();
            if (r.first == Operator::Error) throw QueryExecutionError();
            if (!r.second) continue;
            Operator::Page::Iterator it = r.second->createIterator();
            void* tup;
            while ((tup = it.next())) std::cout << q.getOutSchema().prettyprint(tup, '|') << "\n";
        }
        if (q.scanStop() == Operator::Error) throw QueryExecutionError();
        clock_gettime(CLOCK_MONOTONIC, &t1);
        q.threadClose();
        const double sec = (t1.tv_sec - t0.tv_sec) + (t1.tv_nsec - t0.tv_nsec) * 1e-9;
        std::cout << "ResponseTimeInCycles: 0" << std::endl;
        std::cout << "ResponseTimeInSec: " << sec << std::endl;
        if (GpuHashJoinOp::context())
            std::cout << "GpuKernelLaunches: " << pyg_ctx_kernel_launches(GpuHashJoinOp::context()) << std::endl;
        std::cout.flush();
    } catch (libconfig::ParseException& e) {
        std::cerr << "plan parse error at line " << e.getLine() << std::endl;
        return 1;
    } catch (...) {
        std::cerr << "query failed" << std::endl;
        return 1;
    }
    return 0;
}

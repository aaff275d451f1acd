// pyg_executequery: runs a reference plan file on the GPU and prints the
// result rows and timing in the reference driver's format
// (drivers/executequery.cpp:67-154): rows '|'-separated, then
// ResponseTimeInCycles / ResponseTimeInSec, then the tuple counters.
//
//   pyg_executequery plan.conf [device]
#include <time.h>

#include <cstdio>
#include <cstdlib>
#include <iostream>

#include "engine.h"

using namespace pyg_host;

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::cout << "ERROR: Configuration file not specified." << std::endl;
        std::cout << "Usage: " << argv[0] << " conf-file [device]" << std::endl;
        return 2;
    }
    int device = argc > 2 ? atoi(argv[2]) : 0;
    try {
        Query q;
        q.create(parse_plan_file(argv[1]));
        int rc = pyg_ctx_create(device, &Operator::ctx);
        if (rc != PYG_OK) {
            std::cerr << "ERROR: " << pyg_last_error() << std::endl;
            return 3;
        }
        std::cout << "CFLGS: " << pyg_version() << std::endl;
        std::cout << "BUFFSIZE: " << q.plan->getInt("buffsize", 1 << 20) << std::endl;
        q.threadInit();
        timespec t0, t1;
        clock_gettime(CLOCK_MONOTONIC, &t0);
        if (q.scanStart() == Operator::Error) throw EngineError("Scan initialization failed.");
        Operator::GetNextResultT r;
        r.first = Operator::Ready;
        std::string out;
        while (r.first == Operator::Ready) {
            r = q.getNext();
            if (r.first == Operator::Error) throw EngineError("GetNext returned error.");
            const Schema& s = q.root->getOutSchema();
            for (int64_t i = 0; r.second && i < r.second->ntuples; ++i) {
                out += s.prettyprint(r.second->data + i * s.tuple_bytes, '|');
                out += '\n';
            }
            if (out.size() > (1 << 20)) {
                std::cout << out;
                out.clear();
            }
        }
        if (q.scanStop() == Operator::Error) throw EngineError("Scan stop failed.");
        clock_gettime(CLOCK_MONOTONIC, &t1);
        std::cout << out;
        double sec = (t1.tv_sec - t0.tv_sec) + (t1.tv_nsec - t0.tv_nsec) / 1e9;
        std::cout << "ResponseTimeInCycles: 0" << std::endl;
        std::cout << "ResponseTimeInSec: " << sec << std::endl;
        for (auto& line : q.counter_report()) std::cout << line << std::endl;
        std::cout << "GpuKernelLaunches: " << pyg_ctx_kernel_launches(Operator::ctx) << std::endl;
        std::cout << "DeviceToHostResultBytes: " << ResultBuffer::d2h_bytes << std::endl;
        std::cout << "IngestToDeviceBytes: " << ScanIngest::bytes << std::endl;
        std::cout << "IngestSeconds: " << ScanIngest::seconds << std::endl;
        q.threadClose();
        pyg_ctx_destroy(Operator::ctx);
    } catch (const std::exception& e) {
        std::cerr << "ERROR: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}

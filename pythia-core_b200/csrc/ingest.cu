// Overlapped ingest: a host byte stream uploaded into one device buffer
// through a ring of pinned staging slots (the file -> device pipeline of a
// scan).  The reference loads a scan's files whole into memory before any
// operator reads them (ParallelScanOp::scanStart / MemMappedTable::load,
// operators/parallelscan.cpp:176-190, operators/loaders/table.cpp:198-348);
// here the caller fills slot i+1 on the host while slot i's copy runs on the
// context's copy stream, so reading / parsing overlaps the PCIe transfer and
// the relation lands in HBM without a whole-relation host copy.
#include "pyg_internal.cuh"

using namespace pyg;

struct pyg_upload {
    void* dev = nullptr;        // destination, stream-ordered allocation
    size_t cap = 0;             // bytes allocated at dev
    size_t used = 0;            // bytes queued so far
    size_t slot_bytes = 0;
    int nslots = 0;
    int next = 0;               // slot handed out by the next pyg_upload_slot
    bool handed = false;        // a slot is out and not yet committed
    void* slot[8] = {};
    cudaEvent_t done[8] = {};   // recorded after each slot's copy
    bool pending[8] = {};
    cudaEvent_t ready = nullptr;  // dev allocated (ctx stream) -> copy stream
};

static void upload_release(pyg_ctx* ctx, pyg_upload* up, bool free_dev)
{
    cudaStreamSynchronize(ctx->copy_stream);
    for (int i = 0; i < up->nslots; ++i) {
        if (up->slot[i]) cudaFreeHost(up->slot[i]);
        if (up->done[i]) cudaEventDestroy(up->done[i]);
    }
    if (up->ready) cudaEventDestroy(up->ready);
    if (free_dev && up->dev) dfree(ctx, up->dev);
    delete up;
}

// Orders the copy stream after the destination's allocation / growth on the
// context's stream.
static int upload_order(pyg_ctx* ctx, pyg_upload* up)
{
    PYG_CUDA(cudaEventRecord(up->ready, ctx->stream));
    PYG_CUDA(cudaStreamWaitEvent(ctx->copy_stream, up->ready, 0));
    return PYG_OK;
}

int pyg_upload_open(pyg_ctx* ctx, size_t capacity, size_t slot_bytes, int32_t slots, pyg_upload** out)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out || slot_bytes == 0 || slots < 2 || slots > 8) {
        set_error("pyg_upload_open: need out, slot_bytes > 0 and 2..8 slots");
        return PYG_ERR_ARG;
    }
    *out = nullptr;
    pyg_upload* up = new pyg_upload();
    up->slot_bytes = slot_bytes;
    up->nslots = slots;
    cudaError_t e = cudaEventCreateWithFlags(&up->ready, cudaEventDisableTiming);
    for (int i = 0; i < slots && e == cudaSuccess; ++i) {
        e = cudaMallocHost(&up->slot[i], slot_bytes);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&up->done[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        upload_release(ctx, up, true);
        return cuda_status(e, "pyg_upload_open staging");
    }
    up->cap = capacity ? capacity : slot_bytes;
    rc = dalloc(ctx, &up->dev, up->cap);
    if (!rc) rc = upload_order(ctx, up);
    if (rc) {
        upload_release(ctx, up, true);
        return rc;
    }
    *out = up;
    return PYG_OK;
}

int pyg_upload_slot(pyg_ctx* ctx, pyg_upload* up, void** buf, size_t* bytes)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!up || !buf) {
        set_error("pyg_upload_slot: null argument");
        return PYG_ERR_ARG;
    }
    const int s = up->next;
    if (up->pending[s]) {
        // The slot's previous copy must finish before the host refills it.
        PYG_CUDA(cudaEventSynchronize(up->done[s]));
        up->pending[s] = false;
    }
    up->handed = true;
    *buf = up->slot[s];
    if (bytes) *bytes = up->slot_bytes;
    return PYG_OK;
}

int pyg_upload_commit(pyg_ctx* ctx, pyg_upload* up, size_t bytes)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!up || !up->handed || bytes > up->slot_bytes) {
        set_error("pyg_upload_commit: no slot handed out, or %zu bytes exceed the slot", bytes);
        return PYG_ERR_ARG;
    }
    const int s = up->next;
    up->handed = false;
    up->next = (s + 1) % up->nslots;
    if (bytes == 0) return PYG_OK;
    if (up->used + bytes > up->cap) {
        // Grow the destination (2x): copies queued so far must land first.
        size_t cap = up->cap;
        while (cap < up->used + bytes) cap *= 2;
        void* nd = nullptr;
        PYG_CUDA(cudaStreamSynchronize(ctx->copy_stream));
        for (int i = 0; i < up->nslots; ++i) up->pending[i] = false;
        rc = dalloc(ctx, &nd, cap);
        if (rc) return rc;
        if (up->used) PYG_CUDA(cudaMemcpyAsync(nd, up->dev, up->used, cudaMemcpyDeviceToDevice, ctx->stream));
        dfree(ctx, up->dev);
        up->dev = nd;
        up->cap = cap;
        rc = upload_order(ctx, up);
        if (rc) return rc;
    }
    PYG_CUDA(cudaMemcpyAsync((char*)up->dev + up->used, up->slot[s], bytes, cudaMemcpyHostToDevice,
                             ctx->copy_stream));
    PYG_CUDA(cudaEventRecord(up->done[s], ctx->copy_stream));
    up->pending[s] = true;
    up->used += bytes;
    return PYG_OK;
}

int pyg_upload_finish(pyg_ctx* ctx, pyg_upload* up, void** device_buffer, size_t* total_bytes)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!up || !device_buffer) {
        set_error("pyg_upload_finish: null argument");
        return PYG_ERR_ARG;
    }
    cudaError_t e = cudaStreamSynchronize(ctx->copy_stream);
    if (e != cudaSuccess) {
        upload_release(ctx, up, true);
        return cuda_status(e, "pyg_upload_finish");
    }
    *device_buffer = up->dev;
    if (total_bytes) *total_bytes = up->used;
    up->dev = nullptr;
    upload_release(ctx, up, false);
    return PYG_OK;
}

int pyg_upload_abort(pyg_ctx* ctx, pyg_upload* up)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (up) upload_release(ctx, up, true);
    return PYG_OK;
}

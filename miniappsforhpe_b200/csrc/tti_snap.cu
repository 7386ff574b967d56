// Device-resident snapshot store with the rtm_snap call sequence.
//
// The reference (snap_helpers/rtm_snap.h:19-41, rtm_snap_gpu.cu:31-280)
// hands every snapshot to a helper thread that copies it to pinned host
// memory and on to RAM or O_DIRECT files, and reads them back LIFO during the
// adjoint pass.  On B200 the snapshots of one shot fit in HBM, so this store
// keeps them there: a write is a stream-ordered device-to-device copy on the
// store's own copy stream, a read is the reverse copy, and events carry the
// ordering the reference's helper-thread token provided
// (helper_thread_synchronizer.h:22-47).  Waits on the host are bounded.
//
// A store may also have a host tier (the reference's host-RAM buffers,
// file_snap_orig.cpp:221-352): slots beyond the device capacity live in
// pinned host memory and are written and read by the same copy stream.
// Being LIFO, the slots written last (host) are read first, so their
// host-to-device copies overlap the first adjoint steps.

#include <cuda_runtime.h>

#include <chrono>
#include <new>
#include <thread>
#include <vector>

#include "tti_common.cuh"

struct tti_snap_store {
    int nvol = 0;
    std::vector<int64_t> nelem;
    int64_t slot_elems = 0;
    int capacity = 0;       // device slots
    int host_capacity = 0;  // pinned host slots after them
    int count = 0;
    float* data = nullptr;
    float* host = nullptr;
    cudaStream_t copy = nullptr;
    cudaEvent_t write_done = nullptr, read_done = nullptr, ready = nullptr;
    bool write_pending = false, read_pending = false;
};

namespace {

int rc_of(cudaError_t e)
{
    if (e == cudaSuccess) return TTI_OK;
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? TTI_ENOMEM : TTI_ELAUNCH;
}

// Slot k: device slots first, then the host tier.
float* slot_ptr(tti_snap_store* s, int k)
{
    if (k < s->capacity) return s->data + (size_t)k * s->slot_elems;
    return s->host + (size_t)(k - s->capacity) * s->slot_elems;
}

// Poll an event for at most ~10 s.
int bounded_event_wait(cudaEvent_t ev)
{
    auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess) return TTI_OK;
        if (e != cudaErrorNotReady) return rc_of(e);
        if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(10)) return TTI_ETIMEOUT;
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

} // namespace

extern "C" {

int tti_snap_create(int nvol, const int64_t* nelem, int capacity, tti_snap_store** out)
{
    return tti_snap_create_tiered(nvol, nelem, capacity, 0, out);
}

int tti_snap_create_tiered(int nvol, const int64_t* nelem, int device_capacity, int host_capacity,
                           tti_snap_store** out)
{
    const int capacity = device_capacity;
    if (!out || nvol <= 0 || !nelem || capacity < 0 || host_capacity < 0 || capacity + host_capacity <= 0)
        return TTI_EINVAL;
    *out = nullptr;
    tti_snap_store* s = new (std::nothrow) tti_snap_store();
    if (!s) return TTI_ENOMEM;
    s->nvol = nvol;
    for (int k = 0; k < nvol; ++k) {
        if (nelem[k] <= 0) {
            delete s;
            return TTI_EINVAL;
        }
        s->nelem.push_back(nelem[k]);
        s->slot_elems += nelem[k];
    }
    s->capacity = capacity;
    s->host_capacity = host_capacity;
    int rc = TTI_OK;
    if (capacity) rc = rc_of(cudaMalloc(&s->data, (size_t)s->slot_elems * capacity * sizeof(float)));
    if (!rc && host_capacity)
        rc = rc_of(cudaMallocHost(&s->host, (size_t)s->slot_elems * host_capacity * sizeof(float)));
    if (!rc) rc = rc_of(cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking));
    if (!rc) rc = rc_of(cudaEventCreateWithFlags(&s->write_done, cudaEventDisableTiming));
    if (!rc) rc = rc_of(cudaEventCreateWithFlags(&s->read_done, cudaEventDisableTiming));
    if (!rc) rc = rc_of(cudaEventCreateWithFlags(&s->ready, cudaEventDisableTiming));
    if (rc) {
        tti_snap_destroy(s);
        return rc;
    }
    *out = s;
    return TTI_OK;
}

int tti_snap_destroy(tti_snap_store* s)
{
    if (!s) return TTI_EINVAL;
    if (s->copy) cudaStreamSynchronize(s->copy);
    if (s->data) cudaFree(s->data);
    if (s->host) cudaFreeHost(s->host);
    if (s->write_done) cudaEventDestroy(s->write_done);
    if (s->read_done) cudaEventDestroy(s->read_done);
    if (s->ready) cudaEventDestroy(s->ready);
    if (s->copy) cudaStreamDestroy(s->copy);
    cudaGetLastError();
    delete s;
    return TTI_OK;
}

int tti_snap_lock_for_write(tti_snap_store* s)
{
    if (!s) return TTI_EINVAL;
    if (!s->write_pending) return TTI_OK;
    int rc = bounded_event_wait(s->write_done);
    if (!rc) s->write_pending = false;
    return rc;
}

int tti_snap_start_write(tti_snap_store* s, float* const* vols, tti_stream_t stream)
{
    if (!s || !vols) return TTI_EINVAL;
    if (s->count >= s->capacity + s->host_capacity) return TTI_ENOMEM;
    for (int k = 0; k < s->nvol; ++k)
        if (!vols[k]) return TTI_EINVAL;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    int rc = rc_of(cudaEventRecord(s->ready, st));
    if (!rc) rc = rc_of(cudaStreamWaitEvent(s->copy, s->ready, 0));
    float* dst = slot_ptr(s, s->count);
    const cudaMemcpyKind kind = s->count < s->capacity ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    for (int k = 0; k < s->nvol && !rc; ++k) {
        rc = rc_of(cudaMemcpyAsync(dst, vols[k], s->nelem[k] * sizeof(float), kind, s->copy));
        dst += s->nelem[k];
    }
    if (!rc) rc = rc_of(cudaEventRecord(s->write_done, s->copy));
    if (!rc) {
        s->write_pending = true;
        s->count++;
    }
    return rc;
}

int tti_snap_start_read(tti_snap_store* s, float* const* vols, tti_stream_t stream)
{
    if (!s || !vols) return TTI_EINVAL;
    if (s->count <= 0) return TTI_ESTATE;
    for (int k = 0; k < s->nvol; ++k)
        if (!vols[k]) return TTI_EINVAL;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    int rc = rc_of(cudaEventRecord(s->ready, st));
    if (!rc) rc = rc_of(cudaStreamWaitEvent(s->copy, s->ready, 0));
    const float* src = slot_ptr(s, s->count - 1);
    const cudaMemcpyKind kind = s->count - 1 < s->capacity ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    for (int k = 0; k < s->nvol && !rc; ++k) {
        rc = rc_of(cudaMemcpyAsync(vols[k], src, s->nelem[k] * sizeof(float), kind, s->copy));
        src += s->nelem[k];
    }
    if (!rc) rc = rc_of(cudaEventRecord(s->read_done, s->copy));
    if (!rc) {
        s->read_pending = true;
        s->count--;
    }
    return rc;
}

int tti_snap_finish_read(tti_snap_store* s, tti_stream_t stream)
{
    if (!s) return TTI_EINVAL;
    if (!s->read_pending) return TTI_ESTATE;
    int rc = rc_of(cudaStreamWaitEvent(reinterpret_cast<cudaStream_t>(stream), s->read_done, 0));
    if (!rc) s->read_pending = false;
    return rc;
}

int tti_snap_count(tti_snap_store* s) { return s ? s->count : -1; }

} // extern "C"

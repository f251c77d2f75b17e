// Several devices behind one projection call: the B200 form of
// RayCasterProjector::Settings::deviceIDs (modules/src/projectors/raycasterprojector.h:30).
//
// The reference replicates the volume on every listed OpenCL device
// (raycasterprojector.cpp:239-251) and deals the views out round-robin, one
// kernel launch and one read-back per view (:321-357), over
// min(#deviceIDs, #views) devices (:188); an empty list means every device
// (:449-454).  Here each device takes one contiguous block of views
// (ctlcu_split_views) and projects it with one ctlcu_project_volume call on
// its own context, in its own host thread: the volume is uploaded to each
// device by a plain host-to-device copy, and each block lands in its own
// disjoint slice of the caller's host output, so there is no exchange between
// the devices at all.  A view's result does not depend on the device or the
// block it is computed in, so the output equals a single-device call bit for
// bit.
#include "ctlcu.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include <nvtx3/nvToolsExt.h>

struct ctlcu_group {
    std::vector<ctlcu_ctx*> ctxs;  // one per listed device (a device may be listed twice)
    std::vector<int> devices;
    std::mutex mu;                 // serialises calls on the group
    std::string err;
};

namespace {

int group_fail(ctlcu_group* g, int code, const char* fmt, ...)
{
    char buf[768];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g->err = buf;
    return code;
}

bool host_memory(const void* p)
{
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return attr.type == cudaMemoryTypeUnregistered || attr.type == cudaMemoryTypeHost;
}

}  // namespace

extern "C" {

int ctlcu_device_count(int* n)
{
    if (!n)
        return CTLCU_ERR_INVALID_ARGUMENT;
    *n = 0;
    if (cudaGetDeviceCount(n) != cudaSuccess) {
        cudaGetLastError();
        *n = 0;
    }
    return CTLCU_OK;
}

int ctlcu_split_views(uint32_t n_views, uint32_t n_parts, uint32_t* first)
{
    if (!first || n_parts == 0)
        return CTLCU_ERR_INVALID_ARGUMENT;
    // contiguous blocks whose sizes differ by at most one, the larger ones first
    const uint32_t base = n_views / n_parts, extra = n_views % n_parts;
    first[0] = 0;
    for (uint32_t i = 0; i < n_parts; ++i)
        first[i + 1] = first[i] + base + (i < extra ? 1u : 0u);
    return CTLCU_OK;
}

int ctlcu_group_create(const int* devices, uint32_t n_devices, ctlcu_group** out)
{
    if (!out || (n_devices > 0 && !devices))
        return CTLCU_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    std::vector<int> list(devices, devices + n_devices);
    if (list.empty()) {
        // raycasterprojector.cpp:449-454: no device IDs means every device
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess) {
            cudaGetLastError();
            return CTLCU_ERR_NO_DEVICE;
        }
        for (int d = 0; d < count; ++d)
            list.push_back(d);
    }
    if (list.empty())
        return CTLCU_ERR_NO_DEVICE;
    ctlcu_group* g = new (std::nothrow) ctlcu_group;
    if (!g)
        return CTLCU_ERR_OUT_OF_MEMORY;
    for (int d : list) {
        ctlcu_ctx* ctx = nullptr;
        const int r = ctlcu_create(d, &ctx);
        if (r != CTLCU_OK) {
            // raycasterprojector.cpp:442-447: an unavailable device ID is an error
            for (ctlcu_ctx* c : g->ctxs)
                ctlcu_destroy(c);
            delete g;
            return r;
        }
        g->ctxs.push_back(ctx);
        g->devices.push_back(d);
    }
    *out = g;
    return CTLCU_OK;
}

int ctlcu_group_destroy(ctlcu_group* g)
{
    if (!g)
        return CTLCU_ERR_INVALID_ARGUMENT;
    for (ctlcu_ctx* c : g->ctxs)
        ctlcu_destroy(c);
    delete g;
    return CTLCU_OK;
}

const char* ctlcu_group_last_error(const ctlcu_group* g) { return g ? g->err.c_str() : "no group"; }

int ctlcu_group_size(const ctlcu_group* g, uint32_t* n_devices)
{
    if (!g || !n_devices)
        return CTLCU_ERR_INVALID_ARGUMENT;
    *n_devices = (uint32_t)g->ctxs.size();
    return CTLCU_OK;
}

int ctlcu_group_context(ctlcu_group* g, uint32_t index, ctlcu_ctx** ctx)
{
    if (!g || !ctx || index >= g->ctxs.size())
        return CTLCU_ERR_INVALID_ARGUMENT;
    *ctx = g->ctxs[index];
    return CTLCU_OK;
}

int ctlcu_group_project_volume(ctlcu_group* g, const ctlcu_volume_desc* desc, const float* volume,
                               const ctlcu_settings* settings, const double* pmats, uint32_t n_views,
                               uint32_t n_modules, uint32_t channels, uint32_t rows, float* out)
{
    if (!g)
        return CTLCU_ERR_INVALID_ARGUMENT;
    nvtxRangePushA("ctlcu_group_project_volume");
    struct Pop {
        ~Pop() { nvtxRangePop(); }
    } pop_;
    std::lock_guard<std::mutex> lk(g->mu);
    if (!desc || !volume || !settings || !pmats || !out)
        return group_fail(g, CTLCU_ERR_INVALID_ARGUMENT, "desc, volume, settings, pmats or out is NULL");
    if (!host_memory(volume) || !host_memory(pmats) || !host_memory(out))
        return group_fail(g, CTLCU_ERR_INVALID_ARGUMENT,
                          "a projection over several devices takes host volume, pmats and out");
    if (n_views == 0 || n_modules == 0 || channels == 0 || rows == 0)
        return group_fail(g, CTLCU_ERR_INVALID_ARGUMENT, "empty projection job (%u views, %u modules, %ux%u)",
                          n_views, n_modules, channels, rows);
    // raycasterprojector.cpp:188: min(#devices, #views) devices take part
    const uint32_t used = (uint32_t)std::min<size_t>(g->ctxs.size(), n_views);
    std::vector<uint32_t> first(used + 1);
    ctlcu_split_views(n_views, used, first.data());
    const size_t pm_per_view = (size_t)n_modules * 12;
    const size_t out_per_view = (size_t)n_modules * rows * channels;
    std::vector<int> status(used, CTLCU_OK);
    auto run = [&](uint32_t i) {
        const uint32_t v0 = first[i], n = first[i + 1] - first[i];
        status[i] = ctlcu_project_volume(g->ctxs[i], desc, volume, settings, pmats + v0 * pm_per_view, n, n_modules,
                                         channels, rows, out + v0 * out_per_view);
    };
    if (used == 1) {
        run(0);
    } else {
        std::vector<std::thread> threads;
        threads.reserve(used);
        for (uint32_t i = 0; i < used; ++i)
            threads.emplace_back(run, i);
        for (auto& t : threads)
            t.join();
    }
    // the first hard error wins; a singular matrix on any device is reported
    // like a single call reports it (its pixels are 0, the rest is valid)
    int singular = -1;
    for (uint32_t i = 0; i < used; ++i) {
        if (status[i] == CTLCU_OK)
            continue;
        if (status[i] == CTLCU_ERR_SINGULAR_GEOMETRY) {
            if (singular < 0)
                singular = (int)i;
            continue;
        }
        return group_fail(g, status[i], "device %u of the group (cuda:%d), views %u..%u: %s", i, g->devices[i],
                          first[i], first[i + 1] - 1, ctlcu_last_error(g->ctxs[i]));
    }
    if (singular >= 0)
        return group_fail(g, CTLCU_ERR_SINGULAR_GEOMETRY, "device %d of the group (cuda:%d): %s", singular,
                          g->devices[singular], ctlcu_last_error(g->ctxs[singular]));
    g->err.clear();
    return CTLCU_OK;
}

}  // extern "C"

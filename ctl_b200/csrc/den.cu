// DEN files straight from and into device memory.
//
// Reference (modules/src/io/den/): a DEN file is a 6-byte header of three
// uint16 (rows, cols, count) and count rows x cols matrices, row-major, with
// the element type implied by the file size (den_header.tpp:51-80,
// den_utils.tpp:8-24); DFileFormat::gen_save (dfileformat.tpp:148-187) writes
// it from host memory and rejects empty data, mismatched sizes and any
// dimension above 65535.  CTL writes ProjectionData with cols = channels,
// rows = detector rows, count = modules x views (denfileio.h:53-68) after
// copying every view to the host (projectors/raycasterprojector.cpp:300-314).
//
// Here device data goes to the file through two pinned staging buffers: the
// copy of chunk i+1 runs while chunk i is written, and reading mirrors it.
#include "ctlcu.h"
#include "internal.cuh"

#include <cstdio>
#include <cstring>
#include <string>

namespace ctlcu {

cudaError_t DenStaging::ensure()
{
    for (int i = 0; i < 2; ++i) {
        if (!buf[i]) {
            cudaError_t e = cudaMallocHost(&buf[i], kBytes);
            if (e != cudaSuccess) {
                buf[i] = nullptr;
                return e;
            }
        }
        if (!ev[i]) {
            cudaError_t e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
            if (e != cudaSuccess) {
                ev[i] = nullptr;
                return e;
            }
        }
    }
    return cudaSuccess;
}

void DenStaging::release()
{
    for (int i = 0; i < 2; ++i) {
        if (buf[i])
            cudaFreeHost(buf[i]);
        if (ev[i])
            cudaEventDestroy(ev[i]);
        buf[i] = nullptr;
        ev[i] = nullptr;
    }
}

namespace {

constexpr size_t kStage = DenStaging::kBytes;

bool is_device(const void* p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

// 0 on success, else a ctlcu_status; msg receives the reason.
int den_write(const char* path, const void* data, uint32_t elem, uint32_t rows, uint32_t cols, uint32_t count,
              cudaStream_t st, DenStaging* stage, std::string& msg)
{
    if (!(elem == 1 || elem == 2 || elem == 4 || elem == 8)) {
        msg = "element size must be 1, 2, 4 or 8 bytes";
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    if (rows == 0 || cols == 0 || count == 0) {
        msg = "empty data";
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    if (rows > 0xFFFFu || cols > 0xFFFFu || count > 0xFFFFu) {
        msg = "at least one header dimension exceeds 16 bit (65535)";
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) {
        msg = std::string("cannot open ") + path + " for writing";
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    const uint16_t head[3] = { (uint16_t)rows, (uint16_t)cols, (uint16_t)count };
    const size_t total = (size_t)rows * cols * count * elem;
    int r = std::fwrite(head, 1, 6, f) == 6 ? file_write_data(f, data, total, st, stage, msg)
                                            : CTLCU_ERR_INVALID_ARGUMENT;
    const bool closed = std::fclose(f) == 0;
    if (r == CTLCU_OK && !closed)
        r = CTLCU_ERR_INVALID_ARGUMENT;
    if (r == CTLCU_ERR_INVALID_ARGUMENT && msg.empty())
        msg = std::string("writing ") + path + " failed";
    return r;
}

int file_write_data(FILE* f, const void* data, size_t total, cudaStream_t st, DenStaging* stage, std::string& msg)
{
    if (!stage || !is_device(data))
        return std::fwrite(data, 1, total, f) == total ? CTLCU_OK : CTLCU_ERR_INVALID_ARGUMENT;
    DenStaging& s = *stage;
    cudaError_t e = s.ensure();
    const char* src = static_cast<const char*>(data);
    const size_t n = (total + kStage - 1) / kStage;
    auto issue = [&](size_t i) {
        const size_t off = i * kStage, len = std::min(kStage, total - off);
        cudaError_t r = cudaMemcpyAsync(s.buf[i & 1], src + off, len, cudaMemcpyDeviceToHost, st);
        return r == cudaSuccess ? cudaEventRecord(s.ev[i & 1], st) : r;
    };
    bool ok = true;
    if (e == cudaSuccess && n > 0)
        e = issue(0);
    for (size_t i = 0; e == cudaSuccess && ok && i < n; ++i) {
        if (i + 1 < n)
            e = issue(i + 1);  // its buffer was written out in iteration i - 1
        if (e == cudaSuccess)
            e = cudaEventSynchronize(s.ev[i & 1]);
        const size_t len = std::min(kStage, total - i * kStage);
        if (e == cudaSuccess)
            ok = std::fwrite(s.buf[i & 1], 1, len, f) == len;
    }
    if (e != cudaSuccess) {
        cudaStreamSynchronize(st);
        msg = std::string("device copy: ") + cudaGetErrorString(e);
        return CTLCU_ERR_CUDA;
    }
    return ok ? CTLCU_OK : CTLCU_ERR_INVALID_ARGUMENT;
}

int file_read_data(FILE* f, void* data, size_t total, cudaStream_t st, DenStaging* stage, std::string& msg)
{
    if (!stage || !is_device(data))
        return std::fread(data, 1, total, f) == total ? CTLCU_OK : CTLCU_ERR_INVALID_ARGUMENT;
    DenStaging& s = *stage;
    cudaError_t e = s.ensure();
    char* dst = static_cast<char*>(data);
    const size_t n = (total + kStage - 1) / kStage;
    bool ok = true;
    for (size_t i = 0; e == cudaSuccess && ok && i < n; ++i) {
        const size_t off = i * kStage, len = std::min<uint64_t>(kStage, total - off);
        if (i >= 2)
            e = cudaEventSynchronize(s.ev[i & 1]);  // the copy out of this buffer is done
        if (e != cudaSuccess)
            break;
        ok = std::fread(s.buf[i & 1], 1, len, f) == len;
        if (ok)
            e = cudaMemcpyAsync(dst + off, s.buf[i & 1], len, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaEventRecord(s.ev[i & 1], st);
    }
    // the data is in place, and the staging buffers free for the next call, once
    // the copies out of them are done
    const cudaError_t w = cudaStreamSynchronize(st);
    if (e == cudaSuccess)
        e = w;
    if (e != cudaSuccess) {
        msg = std::string("device copy: ") + cudaGetErrorString(e);
        return CTLCU_ERR_CUDA;
    }
    return ok ? CTLCU_OK : CTLCU_ERR_INVALID_ARGUMENT;
}

int den_header(const char* path, uint32_t dims[3], uint32_t* elem, std::string& msg)
{
    FILE* f = std::fopen(path, "rb");
    if (!f) {
        msg = std::string("cannot open ") + path;
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    uint16_t head[3] = { 0, 0, 0 };
    const size_t got = std::fread(head, 1, 6, f);
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fclose(f);
    if (got != 6 || size < 6) {
        msg = "incomplete DEN header";
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    dims[0] = head[0];
    dims[1] = head[1];
    dims[2] = head[2];
    // den_utils.tpp:8-24: the element size is data bytes / elements
    const uint64_t n = (uint64_t)head[0] * head[1] * head[2];
    const uint64_t bytes = (uint64_t)(size - 6);
    if (n == 0 || bytes == 0 || bytes % n) {
        msg = "DEN header does not match the data size";
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    const uint64_t e = bytes / n;
    if (!(e == 1 || e == 2 || e == 4 || e == 8)) {
        msg = "DEN data of an unknown element size";
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    *elem = (uint32_t)e;
    return CTLCU_OK;
}

int den_read(const char* path, void* data, uint64_t capacity, uint32_t first, uint32_t n_mats, cudaStream_t st,
             DenStaging* stage, std::string& msg)
{
    uint32_t dims[3], elem = 0;
    int r = den_header(path, dims, &elem, msg);
    if (r)
        return r;
    const uint64_t mat = (uint64_t)dims[0] * dims[1] * elem;
    if (n_mats == 0)
        n_mats = first < dims[2] ? dims[2] - first : 0;
    if ((uint64_t)first + n_mats > dims[2] || n_mats == 0) {
        msg = "matrix range outside the file";
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    const uint64_t total = mat * n_mats;
    if (total > capacity) {
        msg = "destination smaller than the data";
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    FILE* f = std::fopen(path, "rb");
    if (!f || std::fseek(f, (long)(6 + mat * first), SEEK_SET) != 0) {
        if (f)
            std::fclose(f);
        msg = std::string("cannot read ") + path;
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    const int rd = file_read_data(f, data, total, st, stage, msg);
    std::fclose(f);
    if (rd == CTLCU_ERR_INVALID_ARGUMENT && msg.empty())
        msg = std::string("reading ") + path + " failed";
    return rd;
}

}  // namespace ctlcu

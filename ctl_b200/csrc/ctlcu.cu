// C ABI of the B200 forward projector: contexts, resident volumes, projection.
//
// Replaces the host side of CTL::OCL::RayCasterProjector
// (modules/src/projectors/raycasterprojector.cpp) and its OpenCL runtime glue
// (modules/src/ocl/openclconfig.cpp, pinnedmem.h): one context per device with
// a stream and a stream-ordered memory pool; volumes uploaded once and kept
// resident; all views of a call in one kernel launch instead of one launch,
// one upload and one read-back per view (raycasterprojector.cpp:321-357).
#include "ctlcu.h"
#include "internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>
#include <initializer_list>

using namespace ctlcu;

namespace {

struct TexEntry {
    cudaArray_t array = nullptr;
    cudaTextureObject_t object = 0;
    size_t bytes = 0;
};

struct VolumeEntry {
    ctlcu_volume_desc desc{};
    void* data = nullptr;       // padded storage (cudaMalloc, or pool memory when `pooled`)
    size_t bytes = 0;
    bool pooled = false;
    float* mean = nullptr;      // padded 1x1x1 mean volume (f = 0), float
    void* cells = nullptr;      // coefficient cells (CTLCU_KERNEL_CELLS), built on first use
    size_t cell_bytes = 0;
    uint32_t plan_refs = 0;     // plans that reference this volume (release is refused meanwhile)
    void* pairs = nullptr;      // x-pair array (CTLCU_KERNEL_PAIRS), built on first use
    size_t pair_bytes = 0;
    uint64_t handle = 0;        // 0 for the temporary volume of ctlcu_project_volume
    std::map<int, TexEntry> tex;  // hardware-filter copies keyed by up-sampling factor
};

}  // namespace

struct ctlcu_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    std::string err;
    std::unordered_map<uint64_t, VolumeEntry> vols;
    uint64_t next_handle = 1;
    uint64_t budget = 0;  // 0 = unlimited
    uint64_t used = 0;
    int* d_flags = nullptr;
    unsigned long long* d_counter = nullptr;
    uint64_t launches = 0;
    cudaEvent_t order = nullptr;  // orders caller streams after volume staging on `stream`
    // autotuned sample loop and launch shape per (volume, channels, rows, modules)
    struct Tuned {
        int kernel;
        LaunchShape shape;
    };
    std::map<std::tuple<uint64_t, uint32_t, uint32_t, uint32_t>, Tuned> tuned;
    DenStaging den;  // pinned buffers for DEN file streaming, allocated on first use
    cudaStream_t copy_stream = nullptr;  // device-to-host copies that overlap projection
    cudaStream_t aux_stream = nullptr;   // every other chunk of a projection into host memory
    // ctlcu_project_volume's resident copies of host volumes (ctlcu_set_volume_cache):
    // the volume's description and a hash of its whole content identify it
    struct Cached {
        ctlcu_volume_desc desc;
        uint64_t hash;
        uint64_t handle;  // in `vols`, never handed to the caller
        uint64_t last;    // use clock, for least-recently-used eviction
    };
    std::vector<Cached> cache;
    uint32_t cache_max = 0;  // 0: every call uploads its volume (the reference's behaviour)
    uint64_t cache_clock = 0, cache_hits = 0, cache_misses = 0;
};

namespace {

int fail(ctlcu_ctx* ctx, int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (ctx)
        ctx->err = buf;
    return code;
}

#define CU_TRY(ctx, call)                                                                         \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            return fail((ctx), e_ == cudaErrorMemoryAllocation ? CTLCU_ERR_OUT_OF_MEMORY          \
                                                               : CTLCU_ERR_CUDA,                  \
                        "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
        }                                                                                         \
    } while (0)

// Where `p` lives, seen from the current device (every entry point makes its
// context's device current before it looks): host memory, device memory the
// current device's kernels may dereference (its own, or managed), or device
// memory of another GPU.
enum class Mem { Host, Local, Foreign };

Mem mem_kind(const void* p)
{
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return Mem::Host;
    }
    if (attr.type == cudaMemoryTypeManaged)
        return Mem::Local;
    if (attr.type != cudaMemoryTypeDevice)
        return Mem::Host;
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) {
        cudaGetLastError();
        return Mem::Foreign;
    }
    return attr.device == cur ? Mem::Local : Mem::Foreign;
}

// Device memory of the current device (see mem_kind).  Memory of another GPU
// is not: entry points refuse it first with check_local.
bool is_device_ptr(const void* p) { return mem_kind(p) == Mem::Local; }

// CTLCU_ERR_INVALID_ARGUMENT if any of the pointers is device memory of a GPU
// other than the context's (current) one: its kernels would dereference it
// without peer access.  Null pointers pass (the callers check them).
int check_local(ctlcu_ctx* ctx, std::initializer_list<const void*> ptrs)
{
    for (const void* p : ptrs)
        if (p && mem_kind(p) == Mem::Foreign)
            return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT,
                        "a buffer is device memory of another GPU than the context's (cuda:%d)", ctx->device);
    return CTLCU_OK;
}

size_t dtype_size(int dtype) { return dtype == CTLCU_F32 ? 4 : 2; }

int check_settings(ctlcu_ctx* ctx, const ctlcu_settings* s)
{
    if (!s)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "settings is NULL");
    if (s->rays_per_pixel[0] < 1 || s->rays_per_pixel[0] > 64 || s->rays_per_pixel[1] < 1 ||
        s->rays_per_pixel[1] > 64)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "raysPerPixel must be in 1..64 (got %u, %u)",
                    s->rays_per_pixel[0], s->rays_per_pixel[1]);
    if (!std::isfinite(s->ray_sampling) || s->ray_sampling < 1e-3f || s->ray_sampling > 1e3f)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "raySampling must be in [1e-3, 1e3] (got %g)",
                    (double)s->ray_sampling);
    if (s->volume_upsampling > 64)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "volumeUpSampling must be <= 64 (got %u)",
                    s->volume_upsampling);
    if (s->interpolate != 0 && s->interpolate != 1)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "interpolate must be 0 or 1");
    if (s->interp_mode != CTLCU_INTERP_SOFTWARE && s->interp_mode != CTLCU_INTERP_TEXTURE)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "unknown interp_mode %d", s->interp_mode);
    if (s->accum < CTLCU_ACCUM_FP64 || s->accum > CTLCU_ACCUM_FP32)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "unknown accum %d", s->accum);
    if (s->kernel < CTLCU_KERNEL_AUTO || s->kernel > CTLCU_KERNEL_PAIRS)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "unknown kernel %d", s->kernel);
    if ((s->kernel == CTLCU_KERNEL_CELLS || s->kernel == CTLCU_KERNEL_PAIRS) &&
        (!s->interpolate || s->interp_mode != CTLCU_INTERP_SOFTWARE || s->volume_upsampling != 1))
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT,
                    "the cell kernel needs software trilinear interpolation and volumeUpSampling 1");
    // launch shape: each field 0 (tuned or default) or one of its values
    if (s->block_rays != 0 && s->block_rays != 128 && s->block_rays != 256 && s->block_rays != 512)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "block_rays must be 0, 128, 256 or 512 (got %d)", s->block_rays);
    if (s->views_per_block != 0 && s->views_per_block != 1 && s->views_per_block != 2 && s->views_per_block != 4)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "views_per_block must be 0, 1, 2 or 4 (got %d)",
                    s->views_per_block);
    if (s->lanes_x != 0 && s->lanes_x != 4 && s->lanes_x != 8)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "lanes_x must be 0, 4 or 8 (got %d)", s->lanes_x);
    if (s->unroll != 0 && s->unroll != 2 && s->unroll != 4 && s->unroll != 8)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "unroll must be 0, 2, 4 or 8 (got %d)", s->unroll);
    // with any of the three left 0, shape_of completes them to a valid shape
    if (s->block_rays && s->views_per_block && s->lanes_x) {
        LaunchShape sh;
        sh.block = (uint32_t)s->block_rays;
        sh.views = (uint32_t)s->views_per_block;
        sh.lanes_x = (uint32_t)s->lanes_x;
        if (const char* why = shape_error(sh))
            return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "launch shape %d rays / %d views / lanes_x %d: %s",
                        s->block_rays, s->views_per_block, s->lanes_x, why);
    }
    return CTLCU_OK;
}

// The launch shape of resolved settings: zero fields take the defaults (a
// warp patch of 8x4 where 4x8 does not fit the tile).
LaunchShape shape_of(const ctlcu_settings* s)
{
    LaunchShape sh;
    if (s->block_rays)
        sh.block = (uint32_t)s->block_rays;
    if (s->views_per_block)
        sh.views = (uint32_t)s->views_per_block;
    if (s->unroll)
        sh.unroll = (uint32_t)s->unroll;
    if (s->lanes_x)
        sh.lanes_x = (uint32_t)s->lanes_x;
    else if (shape_error(sh))
        sh.lanes_x = 8;
    return sh;
}

// The shape fields of `s` filled in from `sh` where they are 0.
void fill_shape(ctlcu_settings& s, const LaunchShape& sh)
{
    if (!s.block_rays)
        s.block_rays = (int32_t)sh.block;
    if (!s.views_per_block)
        s.views_per_block = (int32_t)sh.views;
    if (!s.lanes_x)
        s.lanes_x = (int32_t)sh.lanes_x;
    if (!s.unroll)
        s.unroll = (int32_t)sh.unroll;
}

uint32_t log2u(uint32_t v)
{
    uint32_t r = 0;
    while ((1u << r) < v)
        ++r;
    return r;
}

int check_desc(ctlcu_ctx* ctx, const ctlcu_volume_desc* d)
{
    if (!d)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "volume desc is NULL");
    for (int k = 0; k < 3; ++k) {
        if (d->n[k] == 0)
            return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "volume has no voxels (%u x %u x %u)", d->n[0],
                        d->n[1], d->n[2]);
        if (!(d->voxel_mm[k] > 0.0f) || !std::isfinite(d->voxel_mm[k]))
            return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "voxel size must be positive (axis %d: %g)", k,
                        (double)d->voxel_mm[k]);
        if (!std::isfinite(d->offset_mm[k]))
            return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "volume offset is not finite");
    }
    if (d->dtype < CTLCU_F32 || d->dtype > CTLCU_F16)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "unknown dtype %d", d->dtype);
    const uint64_t padded = (uint64_t)(d->n[0] + 2 * kPad) * (d->n[1] + 2 * kPad) * (d->n[2] + 2 * kPad);
    if (padded >= (1ull << 31))
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "volume too large (%llu padded voxels, limit 2^31)",
                    (unsigned long long)padded);
    return CTLCU_OK;
}

int check_job(ctlcu_ctx* ctx, uint32_t V, uint32_t M, uint32_t C, uint32_t R)
{
    if (V == 0 || M == 0 || C == 0 || R == 0)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "empty projection job (%u views, %u modules, %ux%u)",
                    V, M, C, R);
    if ((uint64_t)V * M > 0x7fffffffull / 1024)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "too many view-modules");
    return CTLCU_OK;
}

// Upload (or device-copy) `data` into a new zero-padded volume in the storage dtype.
int make_volume(ctlcu_ctx* ctx, const ctlcu_volume_desc* d, const float* data, bool on_device,
                bool pooled, VolumeEntry& v)
{
    const int n[3] = { (int)d->n[0], (int)d->n[1], (int)d->n[2] };
    const size_t padded = (size_t)(n[0] + 2 * kPad) * (n[1] + 2 * kPad) * (n[2] + 2 * kPad);
    const size_t bytes = padded * dtype_size(d->dtype);
    if (ctx->budget && ctx->used + bytes > ctx->budget)
        return fail(ctx, CTLCU_ERR_OUT_OF_MEMORY,
                    "volume of %zu bytes exceeds the memory budget (%llu of %llu bytes used)", bytes,
                    (unsigned long long)ctx->used, (unsigned long long)ctx->budget);
    v.desc = *d;
    v.bytes = bytes;
    v.pooled = pooled;
    if (pooled)
        CU_TRY(ctx, cudaMallocAsync(&v.data, bytes, ctx->stream));
    else
        CU_TRY(ctx, cudaMalloc(&v.data, bytes));
    CU_TRY(ctx, cudaMemsetAsync(v.data, 0, bytes, ctx->stream));
    const size_t nbytes = (size_t)n[0] * n[1] * n[2] * sizeof(float);
    const float* src = data;
    float* staging = nullptr;
    if (!on_device) {
        CU_TRY(ctx, cudaMallocAsync((void**)&staging, nbytes, ctx->stream));
        CU_TRY(ctx, cudaMemcpyAsync(staging, data, nbytes, cudaMemcpyHostToDevice, ctx->stream));
        src = staging;
    }
    CU_TRY(ctx, launch_pad_convert(src, v.data, n, d->dtype, ctx->stream));
    ++ctx->launches;
    if (staging)
        CU_TRY(ctx, cudaFreeAsync(staging, ctx->stream));
    ctx->used += bytes;
    return CTLCU_OK;
}

void free_volume(ctlcu_ctx* ctx, VolumeEntry& v)
{
    for (auto& t : v.tex) {
        if (t.second.object)
            cudaDestroyTextureObject(t.second.object);
        if (t.second.array)
            cudaFreeArray(t.second.array);
        ctx->used -= std::min<uint64_t>(ctx->used, t.second.bytes);
    }
    v.tex.clear();
    if (v.mean)
        cudaFreeAsync(v.mean, ctx->stream);
    v.mean = nullptr;
    if (v.cells) {
        if (v.pooled)
            cudaFreeAsync(v.cells, ctx->stream);
        else
            cudaFree(v.cells);
        ctx->used -= std::min<uint64_t>(ctx->used, v.cell_bytes);
    }
    v.cells = nullptr;
    v.cell_bytes = 0;
    if (v.pairs) {
        if (v.pooled)
            cudaFreeAsync(v.pairs, ctx->stream);
        else
            cudaFree(v.pairs);
        ctx->used -= std::min<uint64_t>(ctx->used, v.pair_bytes);
    }
    v.pairs = nullptr;
    v.pair_bytes = 0;
    if (v.data) {
        if (v.pooled)
            cudaFreeAsync(v.data, ctx->stream);
        else
            cudaFree(v.data);
        ctx->used -= std::min<uint64_t>(ctx->used, v.bytes);
    }
    v.data = nullptr;
}

// Mean-voxel volume for volumeUpSampling = 0, computed once per volume.
int ensure_mean(ctlcu_ctx* ctx, VolumeEntry& v)
{
    if (v.mean)
        return CTLCU_OK;
    const int n[3] = { (int)v.desc.n[0], (int)v.desc.n[1], (int)v.desc.n[2] };
    const size_t e = 1 + 2 * kPad;
    double* sum = nullptr;
    CU_TRY(ctx, cudaMallocAsync((void**)&sum, sizeof(double), ctx->stream));
    CU_TRY(ctx, cudaMemsetAsync(sum, 0, sizeof(double), ctx->stream));
    CU_TRY(ctx, cudaMallocAsync((void**)&v.mean, e * e * e * sizeof(float), ctx->stream));
    CU_TRY(ctx, cudaMemsetAsync(v.mean, 0, e * e * e * sizeof(float), ctx->stream));
    CU_TRY(ctx, launch_mean(v.data, n, v.desc.dtype, sum, ctx->stream));
    CU_TRY(ctx, launch_mean_volume(sum, (double)n[0] * n[1] * n[2], v.mean, ctx->stream));
    ctx->launches += 2;
    CU_TRY(ctx, cudaFreeAsync(sum, ctx->stream));
    return CTLCU_OK;
}

// Coefficient cells of the padded volume, built once per volume on its first
// cell-kernel projection.
int ensure_cells(ctlcu_ctx* ctx, VolumeEntry& v)
{
    if (v.cells)
        return CTLCU_OK;
    const int n[3] = { (int)v.desc.n[0], (int)v.desc.n[1], (int)v.desc.n[2] };
    const CellLayout L = cell_layout(n);
    const size_t bytes = (size_t)L.count * kCellBytes;
    if (ctx->budget && ctx->used + bytes > ctx->budget)
        return fail(ctx, CTLCU_ERR_OUT_OF_MEMORY,
                    "cell array of %zu bytes exceeds the memory budget (%llu of %llu bytes used)", bytes,
                    (unsigned long long)ctx->used, (unsigned long long)ctx->budget);
    if (v.pooled)
        CU_TRY(ctx, cudaMallocAsync(&v.cells, bytes, ctx->stream));
    else
        CU_TRY(ctx, cudaMalloc(&v.cells, bytes));
    v.cell_bytes = bytes;
    ctx->used += bytes;
    CU_TRY(ctx, launch_build_cells(v.data, n, v.desc.dtype, L, v.cells, ctx->stream));
    ++ctx->launches;
    return CTLCU_OK;
}

// x-pair array of the padded volume, built once per volume on first use.
int ensure_pairs(ctlcu_ctx* ctx, VolumeEntry& v)
{
    if (v.pairs)
        return CTLCU_OK;
    const int n[3] = { (int)v.desc.n[0], (int)v.desc.n[1], (int)v.desc.n[2] };
    const PairLayout L = pair_layout(n);
    const size_t bytes = (size_t)L.count * sizeof(float2);
    if (ctx->budget && ctx->used + bytes > ctx->budget)
        return fail(ctx, CTLCU_ERR_OUT_OF_MEMORY,
                    "pair array of %zu bytes exceeds the memory budget (%llu of %llu bytes used)", bytes,
                    (unsigned long long)ctx->used, (unsigned long long)ctx->budget);
    if (v.pooled)
        CU_TRY(ctx, cudaMallocAsync(&v.pairs, bytes, ctx->stream));
    else
        CU_TRY(ctx, cudaMalloc(&v.pairs, bytes));
    v.pair_bytes = bytes;
    ctx->used += bytes;
    CU_TRY(ctx, launch_build_pairs(v.data, n, v.desc.dtype, L, v.pairs, ctx->stream));
    ++ctx->launches;
    return CTLCU_OK;
}

// Hardware-filter texture of the volume as the rays see it (f >= 1: replicated
// f^3; f = 0: the mean voxel).  Border colour 0, unnormalised coordinates.
int ensure_texture(ctlcu_ctx* ctx, VolumeEntry& v, int f, cudaTextureObject_t* out)
{
    auto it = v.tex.find(f);
    if (it != v.tex.end()) {
        *out = it->second.object;
        return CTLCU_OK;
    }
    if (v.desc.dtype == CTLCU_BF16)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT,
                    "hardware texture interpolation supports F32 and F16 storage, not BF16");
    int n[3] = { (int)v.desc.n[0], (int)v.desc.n[1], (int)v.desc.n[2] };
    const void* src = v.data;
    int dtype = v.desc.dtype;
    int g[3];
    if (f == 0) {
        int r = ensure_mean(ctx, v);
        if (r)
            return r;
        n[0] = n[1] = n[2] = 1;
        src = v.mean;
        dtype = CTLCU_F32;
        g[0] = g[1] = g[2] = 1;
    } else {
        for (int k = 0; k < 3; ++k)
            g[k] = n[k] * f;
    }
    const size_t esz = dtype_size(dtype);
    const size_t bytes = (size_t)g[0] * g[1] * g[2] * esz;
    if (ctx->budget && ctx->used + bytes > ctx->budget)
        return fail(ctx, CTLCU_ERR_OUT_OF_MEMORY, "texture copy of %zu bytes exceeds the memory budget",
                    bytes);
    void* dense = nullptr;
    CU_TRY(ctx, cudaMallocAsync(&dense, bytes, ctx->stream));
    CU_TRY(ctx, launch_unpad_upsample(src, n, dtype, f == 0 ? 1 : f, dense, ctx->stream));
    ++ctx->launches;
    TexEntry t;
    const cudaChannelFormatDesc ch = dtype == CTLCU_F32 ? cudaCreateChannelDesc<float>()
                                                        : cudaCreateChannelDescHalf();
    CU_TRY(ctx, cudaMalloc3DArray(&t.array, &ch, make_cudaExtent(g[0], g[1], g[2])));
    cudaMemcpy3DParms p = {};
    p.srcPtr = make_cudaPitchedPtr(dense, g[0] * esz, g[0], g[1]);
    p.dstArray = t.array;
    p.extent = make_cudaExtent(g[0], g[1], g[2]);
    p.kind = cudaMemcpyDeviceToDevice;
    CU_TRY(ctx, cudaMemcpy3DAsync(&p, ctx->stream));
    CU_TRY(ctx, cudaFreeAsync(dense, ctx->stream));
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = t.array;
    cudaTextureDesc td = {};
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
    td.borderColor[0] = td.borderColor[1] = td.borderColor[2] = td.borderColor[3] = 0.0f;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    CU_TRY(ctx, cudaCreateTextureObject(&t.object, &rd, &td, nullptr));
    t.bytes = bytes;
    ctx->used += bytes;
    v.tex[f] = t;
    *out = t.object;
    return CTLCU_OK;
}

// Fill the volume-dependent part of ProjectArgs (up-sampling, step, corner).
// Mirrors raycasterprojector.cpp:145-179 and :552-558.
int volume_args(ctlcu_ctx* ctx, VolumeEntry& v, const ctlcu_settings* s, ProjectArgs& a, Mode& mode,
                int& dtype)
{
    const bool interp = s->interpolate != 0;
    const int f = interp ? (int)s->volume_upsampling : 1;  // no interpolation forces f = 1
    mode = !interp ? Mode::Nearest : (s->interp_mode == CTLCU_INTERP_TEXTURE ? Mode::Texture : Mode::Trilinear);
    const ctlcu_volume_desc& d = v.desc;
    float voxel[3];
    a.tex = 0;
    if (f == 0) {
        int r = ensure_mean(ctx, v);
        if (r)
            return r;
        for (int k = 0; k < 3; ++k) {
            voxel[k] = d.voxel_mm[k] * (float)d.n[k];
            a.grid[k] = 1;
            a.ext[k] = 1 + 2 * kPad;
        }
        a.vol = v.mean;
        a.up = 1;
        dtype = CTLCU_F32;
    } else {
        for (int k = 0; k < 3; ++k) {
            voxel[k] = f == 1 ? d.voxel_mm[k] : d.voxel_mm[k] / (float)f;
            a.grid[k] = (int)d.n[k] * f;
            a.ext[k] = (int)d.n[k] + 2 * kPad;
        }
        a.vol = v.data;
        a.up = f;
        dtype = d.dtype;
    }
    if (mode == Mode::Texture) {
        int r = ensure_texture(ctx, v, f, &a.tex);
        if (r)
            return r;
    }
    if (mode == Mode::Trilinear && f == 1 && s->kernel == CTLCU_KERNEL_PAIRS) {
        int r = ensure_pairs(ctx, v);
        if (r)
            return r;
        mode = Mode::Pairs;
        a.cells = v.pairs;
        const int n[3] = { (int)d.n[0], (int)d.n[1], (int)d.n[2] };
        const PairLayout L = pair_layout(n);
        a.csy = L.sy;
        a.csz = L.sz;
        a.cmax = L.max_base;
    } else if (mode == Mode::Trilinear && f == 1 && s->kernel != CTLCU_KERNEL_GATHER) {
        int r = ensure_cells(ctx, v);
        if (r)
            return r;
        mode = Mode::Cells;
        a.cells = v.cells;
        const int n[3] = { (int)d.n[0], (int)d.n[1], (int)d.n[2] };
        const CellLayout L = cell_layout(n);
        a.csy = L.sy;
        a.csz = L.sz;
        a.cmax = L.max_index;
    }
    a.sy = a.ext[0];
    a.sz = a.ext[0] * a.ext[1];
    const float smallest = std::min(std::min(voxel[0], voxel[1]), voxel[2]);
    a.increment = (double)smallest * (double)s->ray_sampling;
    for (int k = 0; k < 3; ++k) {
        a.voxel[k] = (double)voxel[k];
        a.corner[k] = (double)d.offset_mm[k] - 0.5 * (double)a.grid[k] * a.voxel[k];
    }
    return CTLCU_OK;
}

void job_args(ProjectArgs& a, const ctlcu_settings* s, uint32_t V, uint32_t M, uint32_t C, uint32_t R)
{
    const LaunchShape sh = shape_of(s);
    const uint32_t tx = shape_tile_x(sh.block, sh.views), ty = shape_tile_y(sh.block, sh.views);
    a.channels = C;
    a.rows = R;
    a.n_vm = V * M;
    a.n_modules = M;
    a.tiles_x = (C + tx - 1) / tx;
    a.tiles_per_vm = a.tiles_x * ((R + ty - 1) / ty);
    a.rays_x = s->rays_per_pixel[0];
    a.rays_y = s->rays_per_pixel[1];
    a.vm_group = CTLCU_VM_GROUP;
    a.n_views = V;
    a.view_groups = (V + sh.views - 1) / sh.views;
    a.block = sh.block;
    a.unroll = sh.unroll;
    a.vpb_shift = log2u(sh.views);
    a.wpv_shift = log2u(sh.block / 32 / sh.views);
    a.lx_shift = log2u(sh.lanes_x);
    a.wx_shift = log2u(tx / sh.lanes_x);
    a.tx_shift = log2u(tx);
    a.ty_shift = log2u(ty);
}

VolumeEntry* find_volume(ctlcu_ctx* ctx, uint64_t h)
{
    auto it = ctx->vols.find(h);
    return it == ctx->vols.end() ? nullptr : &it->second;
}

// Cell arrays, textures and mean voxels are built on the context's stream;
// work on another stream `st` must start after them.
int order_after_staging(ctlcu_ctx* ctx, cudaStream_t st)
{
    if (st == ctx->stream)
        return CTLCU_OK;
    CU_TRY(ctx, cudaEventRecord(ctx->order, ctx->stream));
    CU_TRY(ctx, cudaStreamWaitEvent(st, ctx->order, 0));
    return CTLCU_OK;
}

// Setup + projection on `s` with device pmats/out.  Scratch comes from the
// stream-ordered pool, so concurrent calls on different streams do not share it.
// CTLCU_KERNEL_AUTO resolved: the autotuned loop for this volume and detector
// if there is one, else the cell loop where it applies.  Launch-shape fields
// left 0 take the tuned shape when the loop is the tuned one, else the
// defaults, so every shape field of the result is set.
ctlcu_settings resolve_kernel(ctlcu_ctx* ctx, const VolumeEntry& v, const ctlcu_settings* s, uint32_t C, uint32_t R,
                              uint32_t M)
{
    ctlcu_settings e = *s;
    const bool fast = e.interpolate && e.interp_mode == CTLCU_INTERP_SOFTWARE && e.volume_upsampling == 1;
    auto it = ctx->tuned.find(std::make_tuple(v.handle, C, R, M));
    const bool have = it != ctx->tuned.end();
    if (e.kernel == CTLCU_KERNEL_AUTO && fast)
        e.kernel = have ? it->second.kernel : CTLCU_KERNEL_CELLS;
    const int loop = e.kernel == CTLCU_KERNEL_AUTO ? CTLCU_KERNEL_GATHER : e.kernel;
    if (have && fast && loop == it->second.kernel) {
        ctlcu_settings t = e;
        fill_shape(t, it->second.shape);
        if (!shape_error(shape_of(&t))) {
            fill_shape(e, it->second.shape);
            return e;
        }
    }
    fill_shape(e, shape_of(&e));
    return e;
}

int project_device(ctlcu_ctx* ctx, VolumeEntry& v, const ctlcu_settings* s_in, const double* d_pm,
                   uint32_t V, uint32_t M, uint32_t C, uint32_t R, float* d_out, cudaStream_t st,
                   bool st_ordered = false)
{
    const ctlcu_settings eff = resolve_kernel(ctx, v, s_in, C, R, M);
    const ctlcu_settings* s = &eff;
    ProjectArgs a = {};
    Mode mode;
    int dtype;
    int r = volume_args(ctx, v, s, a, mode, dtype);
    if (r)
        return r;
    if (!st_ordered) {
        r = order_after_staging(ctx, st);
        if (r)
            return r;
    }
    job_args(a, s, V, M, C, R);
    ViewGeom* geom = nullptr;
    CU_TRY(ctx, cudaMallocAsync((void**)&geom, sizeof(ViewGeom) * (size_t)V * M, st));
    CU_TRY(ctx, launch_setup(d_pm, V, M, geom, nullptr, nullptr, ctx->d_flags, st));
    a.geom = geom;
    a.out = d_out;
    a.flags = ctx->d_flags;
    a.counter = nullptr;
    CU_TRY(ctx, launch_project(a, mode, (Accum)s->accum, dtype, st));
    ctx->launches += 2;
    CU_TRY(ctx, cudaFreeAsync(geom, st));
    return CTLCU_OK;
}

// Views per chunk of a projection into host memory: five equal chunks, then
// chunks of 4/47, 2/47 and 1/47 of the views (8, 4, 2, 1 parts of 47), so
// that the copy that follows the last kernel is of about 2% of the output.  A
// chunk's copy to the host takes a few percent of the time its views take to
// project, so it stays hidden behind the next chunk, half as large.  Fewer
// than 64 views: two chunks (3/4, 1/4); fewer than 8: one.
std::vector<uint32_t> host_chunks(uint32_t V)
{
    if (V < 8)
        return { V };
    if (V < 64) {
        const uint32_t a = (3 * V + 3) / 4;
        return { a, V - a };
    }
    const uint32_t t4 = std::max(1u, 4 * V / 47), t2 = std::max(1u, 2 * V / 47), t1 = std::max(1u, V / 47);
    const uint32_t lead = V - t4 - t2 - t1;
    std::vector<uint32_t> n;
    for (uint32_t i = 0; i < 5; ++i)
        n.push_back(lead / 5 + (i < lead % 5 ? 1u : 0u));
    n.push_back(t4);
    n.push_back(t2);
    n.push_back(t1);
    return n;
}

int read_flags(ctlcu_ctx* ctx)
{
    int flags = 0;
    CU_TRY(ctx, cudaMemcpy(&flags, ctx->d_flags, sizeof(int), cudaMemcpyDeviceToHost));
    if (flags) {
        CU_TRY(ctx, cudaMemset(ctx->d_flags, 0, sizeof(int)));
        if (flags & kFlagSingular)
            return fail(ctx, CTLCU_ERR_SINGULAR_GEOMETRY,
                        "a projection matrix has a singular or non-finite M; its pixels were set to 0");
        return fail(ctx, CTLCU_ERR_SINGULAR_GEOMETRY, "a ray had non-finite entry/exit parameters");
    }
    return CTLCU_OK;
}

// Host/device dispatch shared by ctlcu_project and ctlcu_project_volume.
int project_any(ctlcu_ctx* ctx, VolumeEntry& v, const ctlcu_settings* s, const double* pmats,
                uint32_t V, uint32_t M, uint32_t C, uint32_t R, float* out, cudaStream_t st,
                bool force_sync)
{
    const bool pm_dev = is_device_ptr(pmats), out_dev = is_device_ptr(out);
    const size_t pm_bytes = sizeof(double) * 12 * (size_t)V * M;
    const size_t out_bytes = sizeof(float) * (size_t)V * M * R * C;
    const double* d_pm = pmats;
    double* pm_tmp = nullptr;
    float* d_out = out;
    if (!pm_dev || !out_dev)
        st = ctx->stream;
    if (!pm_dev) {
        CU_TRY(ctx, cudaMallocAsync((void**)&pm_tmp, pm_bytes, st));
        CU_TRY(ctx, cudaMemcpyAsync(pm_tmp, pmats, pm_bytes, cudaMemcpyHostToDevice, st));
        d_pm = pm_tmp;
    }
    if (!out_dev)
        CU_TRY(ctx, cudaMallocAsync((void**)&d_out, out_bytes, st));
    int r = CTLCU_OK;
    if (out_dev) {
        r = project_device(ctx, v, s, d_pm, V, M, C, R, d_out, st);
    } else {
        // Host output: the views go in chunks, and each chunk's copy to the host
        // runs on the copy stream while the next chunk is projected.  Chunks
        // alternate between two streams, so that a chunk's first blocks fill
        // the SMs that the previous chunk's last blocks leave idle, and the
        // last chunks are small, so that little copying follows the last kernel.
        if (!ctx->copy_stream)
            CU_TRY(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
        if (!ctx->aux_stream)
            CU_TRY(ctx, cudaStreamCreateWithFlags(&ctx->aux_stream, cudaStreamNonBlocking));
        // the second stream starts after the pmats upload and the volume staging on `st`
        CU_TRY(ctx, cudaEventRecord(ctx->order, st));
        CU_TRY(ctx, cudaStreamWaitEvent(ctx->aux_stream, ctx->order, 0));
        const cudaStream_t lanes[2] = { st, ctx->aux_stream };
        const std::vector<uint32_t> sizes = host_chunks(V);
        const size_t view_values = (size_t)M * R * C;
        uint32_t first = 0;
        for (size_t i = 0; r == CTLCU_OK && i < sizes.size(); first += sizes[i], ++i) {
            const uint32_t n = sizes[i];
            const cudaStream_t cs = lanes[i & 1];
            r = project_device(ctx, v, s, d_pm + (size_t)first * M * 12, n, M, C, R, d_out + first * view_values, cs,
                               true);
            cudaEvent_t done = nullptr;
            cudaError_t e = r ? cudaSuccess : cudaEventCreateWithFlags(&done, cudaEventDisableTiming);
            if (!r && e == cudaSuccess)
                e = cudaEventRecord(done, cs);
            if (!r && e == cudaSuccess)
                e = cudaStreamWaitEvent(ctx->copy_stream, done, 0);
            if (!r && e == cudaSuccess)
                e = cudaMemcpyAsync(out + first * view_values, d_out + first * view_values,
                                    sizeof(float) * n * view_values, cudaMemcpyDeviceToHost, ctx->copy_stream);
            if (done)
                cudaEventDestroy(done);
            if (!r && e != cudaSuccess)
                r = fail(ctx, CTLCU_ERR_CUDA, "copy of projections to the host failed: %s", cudaGetErrorString(e));
        }
        // the device buffers are freed on `st`: order that after the last copy
        // and after everything on the second stream
        cudaEvent_t copied = nullptr, aux_done = nullptr;
        if (cudaEventCreateWithFlags(&copied, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&aux_done, cudaEventDisableTiming) == cudaSuccess) {
            cudaEventRecord(copied, ctx->copy_stream);
            cudaEventRecord(aux_done, ctx->aux_stream);
            cudaStreamWaitEvent(st, copied, 0);
            cudaStreamWaitEvent(st, aux_done, 0);
        } else {
            cudaStreamSynchronize(ctx->copy_stream);
            cudaStreamSynchronize(ctx->aux_stream);
        }
        if (copied)
            cudaEventDestroy(copied);
        if (aux_done)
            cudaEventDestroy(aux_done);
    }
    if (pm_tmp)
        cudaFreeAsync(pm_tmp, st);
    if (!out_dev)
        cudaFreeAsync(d_out, st);
    if (r)
        return r;
    if (!pm_dev || !out_dev || force_sync) {
        CU_TRY(ctx, cudaStreamSynchronize(st));
        return read_flags(ctx);
    }
    return CTLCU_OK;
}

// ---- the volume cache of ctlcu_project_volume ---------------------------------------------------

// 64-bit hash of n floats: four interleaved multiply-rotate accumulators over
// 8-byte words (the round of the published XXH64 algorithm), merged with a
// final avalanche.  Large volumes are hashed by several host threads in
// fixed-size chunks, whose hashes are then hashed in order, so the result
// does not depend on the thread count.
uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }

constexpr uint64_t kP1 = 11400714785074694791ull, kP2 = 14029467366897019727ull, kP3 = 1609587929392839161ull;

uint64_t mix64(uint64_t h)
{
    h ^= h >> 33;
    h *= kP2;
    h ^= h >> 29;
    h *= kP3;
    h ^= h >> 32;
    return h;
}

// n 8-byte words at p (any alignment: each word is read with memcpy, one
// unaligned load on the host CPU).
uint64_t hash_words(const unsigned char* p, size_t n, uint64_t seed)
{
    auto word = [p](size_t i) {
        uint64_t x;
        std::memcpy(&x, p + 8 * i, 8);
        return x;
    };
    uint64_t a[4] = { seed + kP1 + kP2, seed + kP2, seed, seed - kP1 };
    size_t i = 0;
    for (; i + 4 <= n; i += 4)
        for (int k = 0; k < 4; ++k)
            a[k] = rotl64(a[k] + word(i + k) * kP2, 31) * kP1;
    uint64_t h = rotl64(a[0], 1) + rotl64(a[1], 7) + rotl64(a[2], 12) + rotl64(a[3], 18);
    for (; i < n; ++i)
        h = rotl64(h ^ (rotl64(word(i) * kP2, 31) * kP1), 27) * kP1 + kP3;
    return mix64(h ^ (uint64_t)n);
}

uint64_t volume_hash(const ctlcu_volume_desc* d, const float* data)
{
    const size_t n = (size_t)d->n[0] * d->n[1] * d->n[2];
    const size_t words = n / 2;
    const unsigned char* bytes = reinterpret_cast<const unsigned char*>(data);
    constexpr size_t kChunk = size_t(1) << 21;  // words per chunk (16 MiB)
    const size_t chunks = (words + kChunk - 1) / kChunk;
    std::vector<uint64_t> part(chunks + 2, 0);
    auto run = [&](size_t c0, size_t c1) {
        for (size_t c = c0; c < c1; ++c) {
            const size_t w0 = c * kChunk, nw = std::min(kChunk, words - w0);
            part[c] = hash_words(bytes + 8 * w0, nw, c);
        }
    };
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const size_t nt = std::min<size_t>(hw, chunks);
    if (nt <= 1) {
        run(0, chunks);
    } else {
        std::vector<std::thread> ts;
        for (size_t t = 0; t < nt; ++t)
            ts.emplace_back(run, chunks * t / nt, chunks * (t + 1) / nt);
        for (auto& t : ts)
            t.join();
    }
    uint32_t tail = 0;
    if (n & 1)
        std::memcpy(&tail, data + n - 1, 4);
    part[chunks] = tail;
    unsigned char desc_bytes[48];
    std::memset(desc_bytes, 0, sizeof desc_bytes);
    std::memcpy(desc_bytes, d, std::min(sizeof desc_bytes, sizeof *d));
    part[chunks + 1] = hash_words(desc_bytes, 6, 0x9e3779b97f4a7c15ull);
    return hash_words(reinterpret_cast<const unsigned char*>(part.data()), part.size(), 0);
}

bool same_desc(const ctlcu_volume_desc& a, const ctlcu_volume_desc& b)
{
    for (int k = 0; k < 3; ++k)
        if (a.n[k] != b.n[k] || a.voxel_mm[k] != b.voxel_mm[k] || a.offset_mm[k] != b.offset_mm[k])
            return false;
    return a.dtype == b.dtype;
}

void evict_cached(ctlcu_ctx* ctx, size_t i)
{
    const uint64_t h = ctx->cache[i].handle;
    if (VolumeEntry* v = find_volume(ctx, h)) {
        cudaStreamSynchronize(ctx->stream);
        free_volume(ctx, *v);
        ctx->vols.erase(h);
    }
    ctx->cache.erase(ctx->cache.begin() + (ptrdiff_t)i);
}

// The resident copy of host volume `data` in the cache, uploaded (and the least
// recently used entry evicted) on a miss.
int cached_volume(ctlcu_ctx* ctx, const ctlcu_volume_desc* d, const float* data, VolumeEntry** out)
{
    const uint64_t h = volume_hash(d, data);
    for (auto& c : ctx->cache)
        if (c.hash == h && same_desc(c.desc, *d)) {
            if (VolumeEntry* v = find_volume(ctx, c.handle)) {
                c.last = ++ctx->cache_clock;
                ++ctx->cache_hits;
                *out = v;
                return CTLCU_OK;
            }
        }
    ++ctx->cache_misses;
    while (!ctx->cache.empty() && ctx->cache.size() >= ctx->cache_max) {
        size_t lru = 0;
        for (size_t i = 1; i < ctx->cache.size(); ++i)
            if (ctx->cache[i].last < ctx->cache[lru].last)
                lru = i;
        evict_cached(ctx, lru);
    }
    VolumeEntry v;
    int r = make_volume(ctx, d, data, false, false, v);
    if (r) {
        free_volume(ctx, v);
        return r;
    }
    const uint64_t handle = ctx->next_handle++;
    v.handle = handle;
    ctx->vols.emplace(handle, v);
    ctx->cache.push_back({ *d, h, handle, ++ctx->cache_clock });
    *out = find_volume(ctx, handle);
    return CTLCU_OK;
}

// ---- batches --------------------------------------------------------------------------------

struct BatchPrep {
    bool persistent = false;        // all requests go through the persistent cell kernel
    std::vector<BatchSetup> setups; // per request
    std::vector<BatchReq> reqs;     // per request (a.geom set at upload)
    std::vector<uint32_t> first_vm; // per request
    uint32_t total_vm = 0, total_items = 0;
    Accum acc = Accum::F64;
    Mode mode = Mode::Cells;        // Cells or Pairs, the same for every request
    LaunchShape shape;              // the same for every request
};

struct BatchDevice {
    ViewGeom* geom = nullptr;
    BatchSetup* setups = nullptr;
    BatchReq* reqs = nullptr;
    unsigned int* counter = nullptr;
};

// Validate the requests and, when the settings select the cell kernel, build
// the per-request launch arguments (building cell arrays as needed).
int prepare_batch(ctlcu_ctx* ctx, const ctlcu_request* requests, uint32_t n, const ctlcu_settings* s,
                  BatchPrep& bp)
{
    for (uint32_t i = 0; i < n; ++i) {
        const ctlcu_request& q = requests[i];
        int r = check_job(ctx, q.n_views, q.n_modules, q.channels, q.rows);
        if (r)
            return r;
        if (!find_volume(ctx, q.volume))
            return fail(ctx, CTLCU_ERR_INVALID_HANDLE, "request %u: unknown volume handle %llu", i,
                        (unsigned long long)q.volume);
        if (!q.pmats || !q.out || !is_device_ptr(q.pmats) || !is_device_ptr(q.out))
            return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT,
                        "request %u: pmats/out must be device memory of the context's GPU (cuda:%d)", i, ctx->device);
    }
    bp.persistent = s->interpolate && s->interp_mode == CTLCU_INTERP_SOFTWARE && s->volume_upsampling == 1 &&
                    s->kernel != CTLCU_KERNEL_GATHER;
    if (!bp.persistent)
        return CTLCU_OK;
    bp.acc = (Accum)s->accum;
    // one sample loop and launch shape for the whole launch: the first request's
    // (autotuned) choice
    const ctlcu_settings eff = resolve_kernel(ctx, *find_volume(ctx, requests[0].volume), s, requests[0].channels,
                                              requests[0].rows, requests[0].n_modules);
    bp.shape = shape_of(&eff);
    uint64_t vm = 0, items = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const ctlcu_request& q = requests[i];
        BatchReq br = {};
        Mode mode;
        int dtype;
        int r = volume_args(ctx, *find_volume(ctx, q.volume), &eff, br.a, mode, dtype);
        if (r)
            return r;
        if (mode != Mode::Cells && mode != Mode::Pairs)
            return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "request %u does not take the cell kernel", i);
        bp.mode = mode;
        job_args(br.a, &eff, q.n_views, q.n_modules, q.channels, q.rows);
        br.a.out = q.out;
        br.a.flags = ctx->d_flags;
        br.a.counter = nullptr;
        br.first_item = (uint32_t)items;
        br.items = br.a.view_groups * br.a.n_modules * br.a.tiles_per_vm;
        bp.first_vm.push_back((uint32_t)vm);
        bp.setups.push_back(BatchSetup{ q.pmats, (uint32_t)vm, q.n_modules });
        bp.reqs.push_back(br);
        vm += (uint64_t)q.n_views * q.n_modules;
        items += br.items;
        if (vm > 0x7fffffffull || items > 0x7fffffffull)
            return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "batch too large");
    }
    bp.total_vm = (uint32_t)vm;
    bp.total_items = (uint32_t)items;
    return CTLCU_OK;
}

int upload_batch(ctlcu_ctx* ctx, BatchPrep& bp, cudaStream_t st, bool pooled, BatchDevice& bd)
{
    const size_t n = bp.reqs.size();
    auto alloc = [&](void** p, size_t bytes) {
        return pooled ? cudaMallocAsync(p, bytes, st) : cudaMalloc(p, bytes);
    };
    CU_TRY(ctx, alloc((void**)&bd.geom, sizeof(ViewGeom) * (size_t)bp.total_vm));
    CU_TRY(ctx, alloc((void**)&bd.setups, sizeof(BatchSetup) * n));
    CU_TRY(ctx, alloc((void**)&bd.reqs, sizeof(BatchReq) * n));
    CU_TRY(ctx, alloc((void**)&bd.counter, sizeof(unsigned int)));
    for (size_t i = 0; i < n; ++i)
        bp.reqs[i].a.geom = bd.geom + bp.first_vm[i];
    CU_TRY(ctx, cudaMemcpyAsync(bd.setups, bp.setups.data(), sizeof(BatchSetup) * n, cudaMemcpyHostToDevice, st));
    CU_TRY(ctx, cudaMemcpyAsync(bd.reqs, bp.reqs.data(), sizeof(BatchReq) * n, cudaMemcpyHostToDevice, st));
    return CTLCU_OK;
}

int enqueue_batch(ctlcu_ctx* ctx, const BatchPrep& bp, const BatchDevice& bd, const ctlcu_settings*,
                  cudaStream_t st)
{
    const uint32_t n = (uint32_t)bp.reqs.size();
    CU_TRY(ctx, cudaMemsetAsync(bd.counter, 0, sizeof(unsigned int), st));
    CU_TRY(ctx, launch_batch_setup(bd.setups, n, bp.total_vm, bd.geom, ctx->d_flags, st));
    int blocks = 0;
    CU_TRY(ctx, launch_batch(bd.reqs, n, bp.total_items, bp.mode, bp.acc, bp.shape, bd.counter, &blocks, st));
    ctx->launches += 2;
    return CTLCU_OK;
}

// The batch as one grid launch per request (the single-request kernel, whose
// arguments sit in the constant bank), dealt out longest first over `branch`
// streams that fork from and join back into `st`: launches of different
// requests overlap, so one fills the SMs that another's last wave leaves idle.
// With no branches, the launches go in order on `st`.
int enqueue_batch_grids(ctlcu_ctx* ctx, const BatchPrep& bp, const BatchDevice& bd, cudaStream_t st,
                        const std::vector<cudaStream_t>& branch, const std::vector<cudaEvent_t>& ev)
{
    const uint32_t n = (uint32_t)bp.reqs.size();
    CU_TRY(ctx, launch_batch_setup(bd.setups, n, bp.total_vm, bd.geom, ctx->d_flags, st));
    if (branch.empty()) {
        for (uint32_t i = 0; i < n; ++i)
            CU_TRY(ctx, launch_project(bp.reqs[i].a, bp.mode, bp.acc, 0, st));
        return CTLCU_OK;
    }
    CU_TRY(ctx, cudaEventRecord(ev[0], st));
    for (cudaStream_t b : branch)
        CU_TRY(ctx, cudaStreamWaitEvent(b, ev[0], 0));
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; ++i)
        order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t x, uint32_t y) { return bp.reqs[x].items > bp.reqs[y].items; });
    std::vector<uint64_t> load(branch.size(), 0);
    for (uint32_t i : order) {
        const size_t k = (size_t)(std::min_element(load.begin(), load.end()) - load.begin());
        load[k] += bp.reqs[i].items;
        CU_TRY(ctx, launch_project(bp.reqs[i].a, bp.mode, bp.acc, 0, branch[k]));
    }
    for (size_t k = 0; k < branch.size(); ++k) {
        CU_TRY(ctx, cudaEventRecord(ev[k + 1], branch[k]));
        CU_TRY(ctx, cudaStreamWaitEvent(st, ev[k + 1], 0));
    }
    return CTLCU_OK;
}

void free_batch(BatchDevice& bd, cudaStream_t st, bool pooled)
{
    void* ptrs[4] = { bd.geom, bd.setups, bd.reqs, bd.counter };
    for (void* p : ptrs)
        if (p) {
            if (pooled)
                cudaFreeAsync(p, st);
            else
                cudaFree(p);
        }
    bd = BatchDevice{};
}

// ---- no-allocation projection ---------------------------------------------------------------

// Geometry scratch of ctlcu_project_noalloc, in static device memory.  Host
// code must not pass `g_noalloc_geom` itself to a kernel (on the host it names
// a stand-in, not device memory): it uses the address that cudaGetSymbolAddress
// returns, looked up once per device.
constexpr int kNoAllocMaxDevices = 64;
static __device__ __align__(256) ViewGeom g_noalloc_geom[CTLCU_NOALLOC_MAX_VIEW_MODULES];
std::mutex g_noalloc_mu;
ViewGeom* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the context's device, which is current.
// Looked up once per device and kept: it belongs to the device's primary
// context, so it does not survive a cudaDeviceReset of that device (documented
// at ctlcu_project_noalloc).
int noalloc_scratch(ctlcu_ctx* ctx, ViewGeom** out)
{
    if (ctx->device < 0 || ctx->device >= kNoAllocMaxDevices)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "device ordinal %d is above the no-allocation limit %d",
                    ctx->device, kNoAllocMaxDevices);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[ctx->device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_geom);
        if (e != cudaSuccess || !p)
            return fail(ctx, CTLCU_ERR_CUDA, "address of the no-allocation scratch array: %s",
                        cudaGetErrorString(e));
        g_noalloc_ptr[ctx->device] = (ViewGeom*)p;
    }
    *out = g_noalloc_ptr[ctx->device];
    return CTLCU_OK;
}

// The derived array that volume_args would have to build for these (resolved)
// settings, or nullptr when every array they read exists already.
const char* missing_array(const VolumeEntry& v, const ctlcu_settings* s)
{
    const bool interp = s->interpolate != 0;
    const int f = interp ? (int)s->volume_upsampling : 1;
    if (f == 0 && !v.mean)
        return "mean-voxel volume (volume_upsampling 0)";
    if (interp && s->interp_mode == CTLCU_INTERP_TEXTURE)
        return v.tex.count(f) ? nullptr : "interpolation texture";
    if (interp && f == 1 && s->kernel == CTLCU_KERNEL_PAIRS)
        return v.pairs ? nullptr : "pair array";
    if (interp && f == 1 && s->kernel != CTLCU_KERNEL_GATHER)
        return v.cells ? nullptr : "cell array";
    return nullptr;
}

// Runs op(device_data, stream) over `bytes` of float data in device or host
// memory.  Host data is staged through pool memory on the context's stream,
// and the call returns when the result is back in host memory.
template <typename Op>
int on_device_data(ctlcu_ctx* ctx, float* data, size_t bytes, void* stream, const char* what, Op op)
{
    if (int r = check_local(ctx, { data }))
        return r;
    const bool dev = is_device_ptr(data);
    cudaStream_t st = dev && stream ? (cudaStream_t)stream : ctx->stream;
    float* d = data;
    if (!dev) {
        CU_TRY(ctx, cudaMallocAsync((void**)&d, bytes, st));
        CU_TRY(ctx, cudaMemcpyAsync(d, data, bytes, cudaMemcpyHostToDevice, st));
    }
    cudaError_t e = op(d, st);
    if (e == cudaSuccess && !dev)
        e = cudaMemcpyAsync(data, d, bytes, cudaMemcpyDeviceToHost, st);
    if (!dev)
        cudaFreeAsync(d, st);
    if (e != cudaSuccess)
        return fail(ctx, CTLCU_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    ++ctx->launches;
    if (!dev)
        CU_TRY(ctx, cudaStreamSynchronize(st));
    return CTLCU_OK;
}

// ctlcu_transform_to_extinction / _intensity
int transform(ctlcu_ctx* ctx, float* data, uint32_t n_views, uint64_t per_view, const double* i0, void* stream,
              bool to_extinction)
{
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!data)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "data is NULL");
    if (n_views == 0 || per_view == 0)
        return CTLCU_OK;
    if (per_view > (1ull << 40) / n_views)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "too many values");
    cudaSetDevice(ctx->device);
    const size_t bytes = sizeof(float) * per_view * n_views;
    return on_device_data(ctx, data, bytes, stream, to_extinction ? "transform to extinction" : "transform to intensity",
                          [&](float* d, cudaStream_t st) {
                              double* di0 = nullptr;
                              cudaError_t e = cudaSuccess;
                              if (i0) {
                                  e = cudaMallocAsync((void**)&di0, sizeof(double) * n_views, st);
                                  if (e == cudaSuccess)
                                      e = cudaMemcpyAsync(di0, i0, sizeof(double) * n_views, cudaMemcpyHostToDevice, st);
                              }
                              if (e == cudaSuccess)
                                  e = launch_transform(d, per_view, n_views, di0, to_extinction, st);
                              if (di0)
                                  cudaFreeAsync(di0, st);
                              return e;
                          });
}

}  // namespace

extern "C" {

int ctlcu_abi_version(void) { return CTLCU_ABI_VERSION; }

ctlcu_settings ctlcu_settings_default(void)
{
    ctlcu_settings s;
    s.rays_per_pixel[0] = s.rays_per_pixel[1] = 1;
    s.ray_sampling = 0.3f;
    s.volume_upsampling = 1;
    s.interpolate = 1;
    s.interp_mode = CTLCU_INTERP_SOFTWARE;
    s.accum = CTLCU_ACCUM_KAHAN;
    s.kernel = CTLCU_KERNEL_AUTO;
    s.views_per_block = s.lanes_x = s.block_rays = s.unroll = 0;  // tuned or default launch shape
    return s;
}

int ctlcu_create(int device, ctlcu_ctx** out)
{
    if (!out)
        return CTLCU_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        return CTLCU_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= count)
        return CTLCU_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess)
        return CTLCU_ERR_CUDA;
    ctlcu_ctx* ctx = new (std::nothrow) ctlcu_ctx;
    if (!ctx)
        return CTLCU_ERR_OUT_OF_MEMORY;
    ctx->device = device;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;  // keep freed scratch in the pool between calls
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->order, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(&ctx->d_flags, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&ctx->d_counter, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMemset(ctx->d_flags, 0, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        if (ctx->stream)
            cudaStreamDestroy(ctx->stream);
        cudaFree(ctx->d_flags);
        cudaFree(ctx->d_counter);
        delete ctx;
        return CTLCU_ERR_CUDA;
    }
    *out = ctx;
    return CTLCU_OK;
}

int ctlcu_destroy(ctlcu_ctx* ctx)
{
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        for (auto& kv : ctx->vols)
            free_volume(ctx, kv.second);
        ctx->vols.clear();
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->d_flags);
        cudaFree(ctx->d_counter);
        if (ctx->order)
            cudaEventDestroy(ctx->order);
        ctx->den.release();
        if (ctx->copy_stream) {
            cudaStreamSynchronize(ctx->copy_stream);
            cudaStreamDestroy(ctx->copy_stream);
        }
        if (ctx->aux_stream) {
            cudaStreamSynchronize(ctx->aux_stream);
            cudaStreamDestroy(ctx->aux_stream);
        }
        cudaStreamDestroy(ctx->stream);
    }
    delete ctx;
    return CTLCU_OK;
}

const char* ctlcu_last_error(const ctlcu_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int ctlcu_set_memory_budget(ctlcu_ctx* ctx, uint64_t bytes)
{
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->budget = bytes;
    return CTLCU_OK;
}

int ctlcu_memory_used(ctlcu_ctx* ctx, uint64_t* bytes)
{
    if (!ctx || !bytes)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    *bytes = ctx->used;
    return CTLCU_OK;
}

int ctlcu_stream(ctlcu_ctx* ctx, void** stream)
{
    if (!ctx || !stream)
        return CTLCU_ERR_INVALID_ARGUMENT;
    *stream = ctx->stream;
    return CTLCU_OK;
}

int ctlcu_volume_create(ctlcu_ctx* ctx, const ctlcu_volume_desc* desc, const float* data,
                        int data_on_device, uint64_t* handle)
{
    TraceRange trace_("ctlcu_volume_create");
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!data || !handle)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "volume data or handle pointer is NULL");
    int r = check_desc(ctx, desc);
    if (r)
        return r;
    cudaSetDevice(ctx->device);
    VolumeEntry v;
    r = make_volume(ctx, desc, data, data_on_device != 0, false, v);
    if (r) {
        free_volume(ctx, v);
        return r;
    }
    // the caller may free or reuse `data` once this returns
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        free_volume(ctx, v);
        return fail(ctx, CTLCU_ERR_CUDA, "volume upload failed: %s", cudaGetErrorString(e));
    }
    const uint64_t h = ctx->next_handle++;
    v.handle = h;
    ctx->vols.emplace(h, v);
    *handle = h;
    return CTLCU_OK;
}

int ctlcu_volume_release(ctlcu_ctx* ctx, uint64_t handle)
{
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    VolumeEntry* v = find_volume(ctx, handle);
    if (!v)
        return fail(ctx, CTLCU_ERR_INVALID_HANDLE, "unknown volume handle %llu", (unsigned long long)handle);
    if (v->plan_refs)
        return fail(ctx, CTLCU_ERR_BUSY, "volume %llu is used by %u plan(s); destroy them first",
                    (unsigned long long)handle, v->plan_refs);
    cudaSetDevice(ctx->device);
    // work already queued on other streams may still read it
    cudaDeviceSynchronize();
    free_volume(ctx, *v);
    ctx->vols.erase(handle);
    for (auto it = ctx->tuned.begin(); it != ctx->tuned.end();)
        it = std::get<0>(it->first) == handle ? ctx->tuned.erase(it) : std::next(it);
    return CTLCU_OK;
}

int ctlcu_volume_bytes(ctlcu_ctx* ctx, uint64_t handle, uint64_t* bytes)
{
    if (!ctx || !bytes)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    VolumeEntry* v = find_volume(ctx, handle);
    if (!v)
        return fail(ctx, CTLCU_ERR_INVALID_HANDLE, "unknown volume handle %llu", (unsigned long long)handle);
    uint64_t b = v->bytes + v->cell_bytes + v->pair_bytes;
    for (auto& t : v->tex)
        b += t.second.bytes;
    *bytes = b;
    return CTLCU_OK;
}

int ctlcu_set_volume_cache(ctlcu_ctx* ctx, uint32_t max_volumes)
{
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    ctx->cache_max = max_volumes;
    while (ctx->cache.size() > max_volumes) {
        size_t lru = 0;
        for (size_t i = 1; i < ctx->cache.size(); ++i)
            if (ctx->cache[i].last < ctx->cache[lru].last)
                lru = i;
        evict_cached(ctx, lru);
    }
    return CTLCU_OK;
}

int ctlcu_volume_cache_stats(ctlcu_ctx* ctx, uint64_t* hits, uint64_t* misses, uint32_t* resident)
{
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (hits)
        *hits = ctx->cache_hits;
    if (misses)
        *misses = ctx->cache_misses;
    if (resident)
        *resident = (uint32_t)ctx->cache.size();
    return CTLCU_OK;
}

int ctlcu_project(ctlcu_ctx* ctx, uint64_t volume, const ctlcu_settings* settings, const double* pmats,
                  uint32_t n_views, uint32_t n_modules, uint32_t channels, uint32_t rows, float* out,
                  void* stream)
{
    TraceRange trace_("ctlcu_project");
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!pmats || !out)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "pmats or out is NULL");
    int r = check_settings(ctx, settings);
    if (r)
        return r;
    r = check_job(ctx, n_views, n_modules, channels, rows);
    if (r)
        return r;
    VolumeEntry* v = find_volume(ctx, volume);
    if (!v)
        return fail(ctx, CTLCU_ERR_INVALID_HANDLE, "unknown volume handle %llu", (unsigned long long)volume);
    cudaSetDevice(ctx->device);
    r = check_local(ctx, { pmats, out });
    if (r)
        return r;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    return project_any(ctx, *v, settings, pmats, n_views, n_modules, channels, rows, out, st, false);
}

int ctlcu_project_volume(ctlcu_ctx* ctx, const ctlcu_volume_desc* desc, const float* volume,
                         const ctlcu_settings* settings, const double* pmats, uint32_t n_views,
                         uint32_t n_modules, uint32_t channels, uint32_t rows, float* out)
{
    TraceRange trace_("ctlcu_project_volume");
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!volume || !pmats || !out)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "volume, pmats or out is NULL");
    int r = check_desc(ctx, desc);
    if (r)
        return r;
    r = check_settings(ctx, settings);
    if (r)
        return r;
    r = check_job(ctx, n_views, n_modules, channels, rows);
    if (r)
        return r;
    cudaSetDevice(ctx->device);
    r = check_local(ctx, { volume, pmats, out });
    if (r)
        return r;
    if (ctx->cache_max && !is_device_ptr(volume)) {
        // a host volume seen before (same description and content) is projected
        // from its resident copy: no upload, no cell build
        VolumeEntry* cv = nullptr;
        r = cached_volume(ctx, desc, volume, &cv);
        if (r == CTLCU_OK)
            r = project_any(ctx, *cv, settings, pmats, n_views, n_modules, channels, rows, out, ctx->stream, true);
        return r;
    }
    VolumeEntry v;
    r = make_volume(ctx, desc, volume, is_device_ptr(volume), true, v);
    if (r == CTLCU_OK)
        r = project_any(ctx, v, settings, pmats, n_views, n_modules, channels, rows, out, ctx->stream, true);
    free_volume(ctx, v);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (r == CTLCU_OK && e != cudaSuccess)
        r = fail(ctx, CTLCU_ERR_CUDA, "projection failed: %s", cudaGetErrorString(e));
    return r;
}

int ctlcu_project_batch(ctlcu_ctx* ctx, const ctlcu_request* requests, uint32_t n_requests,
                        const ctlcu_settings* settings, void* stream)
{
    TraceRange trace_("ctlcu_project_batch");
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!requests || n_requests == 0)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "empty batch");
    int r = check_settings(ctx, settings);
    if (r)
        return r;
    cudaSetDevice(ctx->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    BatchPrep bp;
    r = prepare_batch(ctx, requests, n_requests, settings, bp);
    if (r == CTLCU_OK)
        r = order_after_staging(ctx, st);
    if (r)
        return r;
    if (!bp.persistent) {
        // settings outside the cell kernel: one launch per request
        for (uint32_t i = 0; i < n_requests; ++i) {
            const ctlcu_request& q = requests[i];
            r = project_device(ctx, *find_volume(ctx, q.volume), settings, q.pmats, q.n_views, q.n_modules,
                               q.channels, q.rows, q.out, st);
            if (r)
                return r;
        }
        return CTLCU_OK;
    }
    // one grid launch per request, in order on `st`: the single-request kernel
    // keeps its arguments in the constant bank, where the persistent kernel of
    // plans reads them from shared memory, and measured no slower on every batch
    // tried.  Batches on other streams (the DRR server runs two) fill the SMs
    // that one request's last wave leaves idle.
    BatchDevice bd;
    r = upload_batch(ctx, bp, st, true, bd);
    if (r == CTLCU_OK)
        r = enqueue_batch_grids(ctx, bp, bd, st, {}, {});
    if (r == CTLCU_OK)
        ctx->launches += 1 + (uint64_t)n_requests;
    free_batch(bd, st, true);
    return r;
}

// ---- plans: a batch captured once as a CUDA graph and replayed -------------------------------

struct ctlcu_plan {
    ctlcu_ctx* ctx = nullptr;
    BatchPrep bp;
    BatchDevice bd;
    std::vector<uint64_t> volumes;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ctlcu_settings settings{};
    int form = CTLCU_PLAN_PERSISTENT;   // the form the graph holds
    float ms[2] = { 0.0f, 0.0f };       // replay time of each form, measured at creation
    uint64_t launches_per_replay = 2;
};

namespace {

// Captures the plan's batch in `form` into an instantiated graph.
int capture_plan(ctlcu_plan* p, int form, cudaGraph_t* graph, cudaGraphExec_t* exec)
{
    ctlcu_ctx* ctx = p->ctx;
    *graph = nullptr;
    *exec = nullptr;
    const size_t n_branch = std::min<size_t>(4, p->bp.reqs.size());
    cudaStream_t cs = nullptr;
    std::vector<cudaStream_t> branch;
    std::vector<cudaEvent_t> ev;
    int r = CTLCU_OK;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess)
        r = fail(ctx, CTLCU_ERR_CUDA, "stream creation failed");
    for (size_t k = 0; r == CTLCU_OK && form == CTLCU_PLAN_GRIDS && k < n_branch; ++k) {
        cudaStream_t b = nullptr;
        if (cudaStreamCreateWithFlags(&b, cudaStreamNonBlocking) != cudaSuccess)
            r = fail(ctx, CTLCU_ERR_CUDA, "stream creation failed");
        else
            branch.push_back(b);
    }
    for (size_t k = 0; r == CTLCU_OK && form == CTLCU_PLAN_GRIDS && k <= n_branch; ++k) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
            r = fail(ctx, CTLCU_ERR_CUDA, "event creation failed");
        else
            ev.push_back(e);
    }
    if (r == CTLCU_OK) {
        if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            r = fail(ctx, CTLCU_ERR_CUDA, "graph capture failed to start");
        } else {
            const uint64_t before = ctx->launches;
            r = form == CTLCU_PLAN_GRIDS ? enqueue_batch_grids(ctx, p->bp, p->bd, cs, branch, ev)
                                         : enqueue_batch(ctx, p->bp, p->bd, &p->settings, cs);
            ctx->launches = before;  // counted per replay instead
            const cudaError_t e = cudaStreamEndCapture(cs, graph);
            if (r == CTLCU_OK && e != cudaSuccess)
                r = fail(ctx, CTLCU_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
            if (r == CTLCU_OK && cudaGraphInstantiate(exec, *graph, 0) != cudaSuccess)
                r = fail(ctx, CTLCU_ERR_CUDA, "graph instantiation failed");
        }
    }
    for (cudaEvent_t e : ev)
        cudaEventDestroy(e);
    for (cudaStream_t b : branch)
        cudaStreamDestroy(b);
    if (cs)
        cudaStreamDestroy(cs);
    if (r) {
        if (*exec)
            cudaGraphExecDestroy(*exec);
        if (*graph)
            cudaGraphDestroy(*graph);
        *graph = nullptr;
        *exec = nullptr;
    }
    return r;
}

// Mean replay time (ms) of `exec` on the context's stream: one untimed replay, then 3.
int time_plan(ctlcu_ctx* ctx, cudaGraphExec_t exec, float* ms)
{
    cudaEvent_t a = nullptr, b = nullptr;
    CU_TRY(ctx, cudaEventCreate(&a));
    cudaError_t e = cudaEventCreate(&b);
    if (e == cudaSuccess)
        e = cudaGraphLaunch(exec, ctx->stream);
    if (e == cudaSuccess)
        e = cudaEventRecord(a, ctx->stream);
    for (int i = 0; i < 3 && e == cudaSuccess; ++i)
        e = cudaGraphLaunch(exec, ctx->stream);
    if (e == cudaSuccess)
        e = cudaEventRecord(b, ctx->stream);
    if (e == cudaSuccess)
        e = cudaEventSynchronize(b);
    if (e == cudaSuccess)
        e = cudaEventElapsedTime(ms, a, b);
    cudaEventDestroy(a);
    if (b)
        cudaEventDestroy(b);
    if (e != cudaSuccess)
        return fail(ctx, CTLCU_ERR_CUDA, "timing the plan failed: %s", cudaGetErrorString(e));
    *ms /= 3.0f;
    return CTLCU_OK;
}

}  // namespace

int ctlcu_plan_create(ctlcu_ctx* ctx, const ctlcu_request* requests, uint32_t n_requests,
                      const ctlcu_settings* settings, ctlcu_plan** out)
{
    return ctlcu_plan_create_form(ctx, requests, n_requests, settings, CTLCU_PLAN_CHOOSE, out);
}

int ctlcu_plan_create_form(ctlcu_ctx* ctx, const ctlcu_request* requests, uint32_t n_requests,
                           const ctlcu_settings* settings, int form, ctlcu_plan** out)
{
    if (!ctx || !out)
        return CTLCU_ERR_INVALID_ARGUMENT;
    if (form != CTLCU_PLAN_CHOOSE && form != CTLCU_PLAN_PERSISTENT && form != CTLCU_PLAN_GRIDS)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "unknown plan form %d", form);
    std::lock_guard<std::mutex> lk(ctx->mu);
    *out = nullptr;
    if (!requests || n_requests == 0)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "empty batch");
    int r = check_settings(ctx, settings);
    if (r)
        return r;
    cudaSetDevice(ctx->device);
    ctlcu_plan* p = new (std::nothrow) ctlcu_plan;
    if (!p)
        return fail(ctx, CTLCU_ERR_OUT_OF_MEMORY, "plan allocation failed");
    p->ctx = ctx;
    p->settings = *settings;
    r = prepare_batch(ctx, requests, n_requests, settings, p->bp);
    if (r == CTLCU_OK && !p->bp.persistent)
        r = fail(ctx, CTLCU_ERR_INVALID_ARGUMENT,
                 "plans need the cell kernel (software trilinear, volumeUpSampling 1)");
    if (r == CTLCU_OK)
        r = upload_batch(ctx, p->bp, ctx->stream, false, p->bd);
    if (r == CTLCU_OK) {
        // descriptors must be on the device before the graph is first replayed
        cudaStreamSynchronize(ctx->stream);
        // the requested form, or both forms captured and timed once and the faster kept
        cudaGraph_t g[2] = { nullptr, nullptr };
        cudaGraphExec_t x[2] = { nullptr, nullptr };
        for (int f = 0; f < 2 && r == CTLCU_OK; ++f)
            if (form == CTLCU_PLAN_CHOOSE || form == f)
                r = capture_plan(p, f, &g[f], &x[f]);
        if (form == CTLCU_PLAN_CHOOSE) {
            for (int f = 0; f < 2 && r == CTLCU_OK; ++f)
                r = time_plan(ctx, x[f], &p->ms[f]);
            if (r == CTLCU_OK) {
                // a singular matrix raised while timing is reported again by the replays' ctlcu_sync
                r = read_flags(ctx);
                if (r == CTLCU_ERR_SINGULAR_GEOMETRY)
                    r = CTLCU_OK;
            }
        }
        const int keep = form != CTLCU_PLAN_CHOOSE ? form
                         : (r == CTLCU_OK && p->ms[CTLCU_PLAN_GRIDS] < p->ms[CTLCU_PLAN_PERSISTENT])
                             ? CTLCU_PLAN_GRIDS : CTLCU_PLAN_PERSISTENT;
        for (int f = 0; f < 2; ++f) {
            if (f == keep && r == CTLCU_OK) {
                p->graph = g[f];
                p->exec = x[f];
            } else {
                if (x[f])
                    cudaGraphExecDestroy(x[f]);
                if (g[f])
                    cudaGraphDestroy(g[f]);
            }
        }
        p->form = keep;
        p->launches_per_replay = keep == CTLCU_PLAN_GRIDS ? 1 + (uint64_t)n_requests : 2;
    }
    if (r) {
        if (p->exec)
            cudaGraphExecDestroy(p->exec);
        if (p->graph)
            cudaGraphDestroy(p->graph);
        free_batch(p->bd, ctx->stream, false);
        delete p;
        return r;
    }
    for (uint32_t i = 0; i < n_requests; ++i) {
        p->volumes.push_back(requests[i].volume);
        ++find_volume(ctx, requests[i].volume)->plan_refs;
    }
    *out = p;
    return CTLCU_OK;
}

int ctlcu_plan_info(const ctlcu_plan* plan, int* form, float* ms_persistent, float* ms_grids)
{
    if (!plan)
        return CTLCU_ERR_INVALID_ARGUMENT;
    if (form)
        *form = plan->form;
    if (ms_persistent)
        *ms_persistent = plan->ms[CTLCU_PLAN_PERSISTENT];
    if (ms_grids)
        *ms_grids = plan->ms[CTLCU_PLAN_GRIDS];
    return CTLCU_OK;
}

int ctlcu_plan_launch(ctlcu_plan* plan, void* stream)
{
    TraceRange trace_("ctlcu_plan_launch");
    if (!plan)
        return CTLCU_ERR_INVALID_ARGUMENT;
    ctlcu_ctx* ctx = plan->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    CU_TRY(ctx, cudaGraphLaunch(plan->exec, st));
    ctx->launches += plan->launches_per_replay;
    return CTLCU_OK;
}

int ctlcu_plan_destroy(ctlcu_plan* plan)
{
    if (!plan)
        return CTLCU_ERR_INVALID_ARGUMENT;
    ctlcu_ctx* ctx = plan->ctx;
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        cudaSetDevice(ctx->device);
        cudaDeviceSynchronize();
        if (plan->exec)
            cudaGraphExecDestroy(plan->exec);
        if (plan->graph)
            cudaGraphDestroy(plan->graph);
        free_batch(plan->bd, ctx->stream, false);
        for (uint64_t h : plan->volumes) {
            VolumeEntry* v = find_volume(ctx, h);
            if (v && v->plan_refs)
                --v->plan_refs;
        }
    }
    delete plan;
    return CTLCU_OK;
}

int ctlcu_sync(ctlcu_ctx* ctx)
{
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    CU_TRY(ctx, cudaDeviceSynchronize());
    return read_flags(ctx);
}

int ctlcu_count_samples(ctlcu_ctx* ctx, uint64_t volume, const ctlcu_settings* settings,
                        const double* pmats, uint32_t n_views, uint32_t n_modules, uint32_t channels,
                        uint32_t rows, uint64_t* samples)
{
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!pmats || !samples)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "pmats or samples is NULL");
    int r = check_settings(ctx, settings);
    if (r)
        return r;
    r = check_job(ctx, n_views, n_modules, channels, rows);
    if (r)
        return r;
    VolumeEntry* v = find_volume(ctx, volume);
    if (!v)
        return fail(ctx, CTLCU_ERR_INVALID_HANDLE, "unknown volume handle %llu", (unsigned long long)volume);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    ProjectArgs a = {};
    Mode mode;
    int dtype;
    r = volume_args(ctx, *v, settings, a, mode, dtype);
    if (r)
        return r;
    job_args(a, settings, n_views, n_modules, channels, rows);
    const size_t pm_bytes = sizeof(double) * 12 * (size_t)n_views * n_modules;
    double* d_pm = nullptr;
    ViewGeom* geom = nullptr;
    if (int rc = check_local(ctx, { pmats }))
        return rc;
    const bool pm_dev = is_device_ptr(pmats);
    if (!pm_dev) {
        CU_TRY(ctx, cudaMallocAsync((void**)&d_pm, pm_bytes, st));
        CU_TRY(ctx, cudaMemcpyAsync(d_pm, pmats, pm_bytes, cudaMemcpyHostToDevice, st));
    }
    CU_TRY(ctx, cudaMallocAsync((void**)&geom, sizeof(ViewGeom) * (size_t)n_views * n_modules, st));
    CU_TRY(ctx, launch_setup(pm_dev ? pmats : d_pm, n_views, n_modules, geom, nullptr, nullptr, ctx->d_flags, st));
    CU_TRY(ctx, cudaMemsetAsync(ctx->d_counter, 0, sizeof(unsigned long long), st));
    a.geom = geom;
    a.counter = ctx->d_counter;
    a.flags = ctx->d_flags;
    CU_TRY(ctx, launch_count(a, mode, st));
    ctx->launches += 2;
    unsigned long long n = 0;
    CU_TRY(ctx, cudaMemcpyAsync(&n, ctx->d_counter, sizeof n, cudaMemcpyDeviceToHost, st));
    CU_TRY(ctx, cudaFreeAsync(geom, st));
    if (d_pm)
        CU_TRY(ctx, cudaFreeAsync(d_pm, st));
    CU_TRY(ctx, cudaStreamSynchronize(st));
    *samples = n;
    return read_flags(ctx);
}

int ctlcu_autotune(ctlcu_ctx* ctx, uint64_t volume, const ctlcu_settings* settings, const double* pmats,
                   uint32_t n_views, uint32_t n_modules, uint32_t channels, uint32_t rows, uint32_t max_views,
                   int* kernel_out, float* ms_out)
{
    TraceRange trace_("ctlcu_autotune");
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!pmats || !kernel_out)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "pmats or kernel_out is NULL");
    int r = check_settings(ctx, settings);
    if (r)
        return r;
    r = check_job(ctx, n_views, n_modules, channels, rows);
    if (r)
        return r;
    VolumeEntry* v = find_volume(ctx, volume);
    if (!v)
        return fail(ctx, CTLCU_ERR_INVALID_HANDLE, "unknown volume handle %llu", (unsigned long long)volume);
    cudaSetDevice(ctx->device);
    const ctlcu_settings& s = *settings;
    if (!(s.interpolate && s.interp_mode == CTLCU_INTERP_SOFTWARE && s.volume_upsampling == 1)) {
        *kernel_out = CTLCU_KERNEL_GATHER;  // only the gather loop serves these settings
        return CTLCU_OK;
    }
    // A contiguous run of views from the middle of the job: neighbouring views
    // share cached cells as they do in the full job.  It holds at least
    // max_views views and is lengthened until its rays fill every SM about four
    // times over (2048 resident threads per SM), so the timings see the full
    // job's regime rather than a part-empty grid; the job caps it.
    const size_t per_view = (size_t)n_modules * 12;
    std::vector<double> hp((size_t)n_views * per_view);
    if (int rc = check_local(ctx, { pmats }))
        return rc;
    if (is_device_ptr(pmats))
        CU_TRY(ctx, cudaMemcpy(hp.data(), pmats, hp.size() * sizeof(double), cudaMemcpyDeviceToHost));
    else
        std::memcpy(hp.data(), pmats, hp.size() * sizeof(double));
    int sms = 0;
    CU_TRY(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    const uint64_t rays_per_view = (uint64_t)n_modules * channels * rows;
    const uint64_t want_rays = 4ull * (uint64_t)sms * 2048ull;
    const uint64_t fill = (want_rays + rays_per_view - 1) / rays_per_view;
    const uint32_t nv = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(max_views ? max_views : 8, fill), n_views);
    const uint32_t first = (n_views - nv) / 2;
    std::vector<double> sub(hp.begin() + (size_t)first * per_view, hp.begin() + (size_t)(first + nv) * per_view);
    double* d_pm = nullptr;
    float* d_out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const int cand[3] = { CTLCU_KERNEL_CELLS, CTLCU_KERNEL_PAIRS, CTLCU_KERNEL_GATHER };
    float ms[3] = { 0.f, 0.f, 0.f };
    auto cleanup = [&]() {
        cudaFree(d_pm);
        cudaFree(d_out);
        if (e0)
            cudaEventDestroy(e0);
        if (e1)
            cudaEventDestroy(e1);
    };
    if (cudaMalloc(&d_pm, sub.size() * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&d_out, (size_t)nv * n_modules * rows * channels * sizeof(float)) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
        cudaMemcpy(d_pm, sub.data(), sub.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
        cleanup();
        return fail(ctx, CTLCU_ERR_OUT_OF_MEMORY, "autotune scratch allocation failed");
    }
    // Mean time per run, after one run that builds the loop's array and warms
    // the caches: 3 runs, or as many as make about 5 ms when 3 are shorter.
    auto timed = [&](const ctlcu_settings& t, int reps, float& out_ms) {
        int rr = CTLCU_OK;
        cudaEventRecord(e0, ctx->stream);
        for (int k = 0; k < reps && rr == CTLCU_OK; ++k)
            rr = project_device(ctx, *v, &t, d_pm, nv, n_modules, channels, rows, d_out, ctx->stream);
        cudaEventRecord(e1, ctx->stream);
        if (rr)
            return rr;
        if (cudaEventSynchronize(e1) != cudaSuccess)
            return fail(ctx, CTLCU_ERR_CUDA, "autotune run failed");
        cudaEventElapsedTime(&out_ms, e0, e1);
        out_ms /= (float)reps;
        return (int)CTLCU_OK;
    };
    auto time_runs = [&](const ctlcu_settings& t, float& out_ms) {
        int rr = project_device(ctx, *v, &t, d_pm, nv, n_modules, channels, rows, d_out, ctx->stream);
        if (rr)
            return rr;
        rr = timed(t, 3, out_ms);
        if (rr == CTLCU_OK && 3.0f * out_ms < 5.0f)
            rr = timed(t, std::min(100, (int)std::ceil(5.0f / std::max(out_ms, 1e-3f))), out_ms);
        return rr;
    };
    // 1. the sample loop, with the caller's launch shape (defaults where 0)
    for (int c = 0; c < 3 && r == CTLCU_OK; ++c) {
        ctlcu_settings t = s;
        t.kernel = cand[c];
        fill_shape(t, shape_of(&t));
        r = time_runs(t, ms[c]);
    }
    int best = 0;
    for (int c = 1; c < 3; ++c)
        if (ms[c] < ms[best])
            best = c;
    // 2. the launch shape of that loop, one field at a time; a change is kept
    // when it is at least 1% faster, so timing noise does not flip a choice
    ctlcu_settings bs = s;
    bs.kernel = cand[best];
    fill_shape(bs, shape_of(&bs));
    float best_ms = ms[best];
    struct Field {
        int32_t ctlcu_settings::*f;
        int32_t caller;
        int32_t values[3];
    };
    const Field fields[4] = { { &ctlcu_settings::views_per_block, s.views_per_block, { 1, 2, 4 } },
                              { &ctlcu_settings::lanes_x, s.lanes_x, { 4, 8, 0 } },
                              { &ctlcu_settings::block_rays, s.block_rays, { 128, 256, 512 } },
                              { &ctlcu_settings::unroll, s.unroll, { 2, 4, 8 } } };
    for (const Field& fd : fields) {
        if (fd.caller != 0 || r != CTLCU_OK)
            continue;  // fixed by the caller
        if (fd.f == &ctlcu_settings::unroll && bs.kernel == CTLCU_KERNEL_GATHER)
            continue;  // the gather loop has no partial sums
        const int32_t current = bs.*(fd.f);
        for (int32_t value : fd.values) {
            if (value == 0 || value == current || r != CTLCU_OK)
                continue;
            ctlcu_settings t = bs;
            t.*(fd.f) = value;
            if (shape_error(shape_of(&t)))
                continue;
            float m = 0.f;
            r = time_runs(t, m);
            if (r == CTLCU_OK && m < 0.99f * best_ms) {
                best_ms = m;
                bs = t;
            }
        }
    }
    // 3. a shape other than the starting one must beat it again, timed afresh
    // and interleaved, before it is kept
    ctlcu_settings start = s;
    start.kernel = cand[best];
    fill_shape(start, shape_of(&start));
    const bool moved = bs.views_per_block != start.views_per_block || bs.lanes_x != start.lanes_x ||
                       bs.block_rays != start.block_rays || bs.unroll != start.unroll;
    if (r == CTLCU_OK && moved) {
        float a0 = 0.f, b0 = 0.f, a1 = 0.f, b1 = 0.f;
        r = time_runs(start, a0);
        if (r == CTLCU_OK)
            r = time_runs(bs, b0);
        if (r == CTLCU_OK)
            r = time_runs(start, a1);
        if (r == CTLCU_OK)
            r = time_runs(bs, b1);
        if (r == CTLCU_OK && !(b0 + b1 < 0.99f * (a0 + a1)))
            bs = start;
    }
    cleanup();
    if (r)
        return r;
    ctx->tuned[std::make_tuple(volume, channels, rows, n_modules)] = ctlcu_ctx::Tuned{ cand[best], shape_of(&bs) };
    // keep only the array the chosen loop reads
    cudaStreamSynchronize(ctx->stream);
    if (cand[best] != CTLCU_KERNEL_CELLS && v->cells) {
        cudaFree(v->cells);
        ctx->used -= std::min<uint64_t>(ctx->used, v->cell_bytes);
        v->cells = nullptr;
        v->cell_bytes = 0;
    }
    if (cand[best] != CTLCU_KERNEL_PAIRS && v->pairs) {
        cudaFree(v->pairs);
        ctx->used -= std::min<uint64_t>(ctx->used, v->pair_bytes);
        v->pairs = nullptr;
        v->pair_bytes = 0;
    }
    *kernel_out = cand[best];
    if (ms_out)
        for (int c = 0; c < 3; ++c)
            ms_out[c] = ms[c];
    return read_flags(ctx);
}

int ctlcu_tuned_settings(ctlcu_ctx* ctx, uint64_t volume, const ctlcu_settings* settings, uint32_t n_modules,
                         uint32_t channels, uint32_t rows, ctlcu_settings* out)
{
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!out)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "out is NULL");
    int r = check_settings(ctx, settings);
    if (r)
        return r;
    r = check_job(ctx, 1, n_modules, channels, rows);
    if (r)
        return r;
    VolumeEntry* v = find_volume(ctx, volume);
    if (!v)
        return fail(ctx, CTLCU_ERR_INVALID_HANDLE, "unknown volume handle %llu", (unsigned long long)volume);
    *out = resolve_kernel(ctx, *v, settings, channels, rows, n_modules);
    return CTLCU_OK;
}

int ctlcu_view_setup(ctlcu_ctx* ctx, const double* pmats, uint32_t n_views, uint32_t n_modules,
                     double* qr_out, double* src_out)
{
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!pmats || !qr_out || !src_out || n_views == 0 || n_modules == 0)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "bad view_setup arguments");
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const size_t nvm = (size_t)n_views * n_modules;
    double *d_pm = nullptr, *d_qr = nullptr, *d_src = nullptr;
    ViewGeom* geom = nullptr;
    CU_TRY(ctx, cudaMallocAsync((void**)&d_pm, nvm * 12 * sizeof(double), st));
    CU_TRY(ctx, cudaMallocAsync((void**)&d_qr, nvm * 15 * sizeof(double), st));
    CU_TRY(ctx, cudaMallocAsync((void**)&d_src, (size_t)n_views * 3 * sizeof(double), st));
    CU_TRY(ctx, cudaMallocAsync((void**)&geom, nvm * sizeof(ViewGeom), st));
    CU_TRY(ctx, cudaMemcpyAsync(d_pm, pmats, nvm * 12 * sizeof(double), cudaMemcpyHostToDevice, st));
    CU_TRY(ctx, launch_setup(d_pm, n_views, n_modules, geom, d_qr, d_src, nullptr, st));
    ++ctx->launches;
    CU_TRY(ctx, cudaMemcpyAsync(qr_out, d_qr, nvm * 15 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CU_TRY(ctx, cudaMemcpyAsync(src_out, d_src, (size_t)n_views * 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    cudaFreeAsync(d_pm, st);
    cudaFreeAsync(d_qr, st);
    cudaFreeAsync(d_src, st);
    cudaFreeAsync(geom, st);
    CU_TRY(ctx, cudaStreamSynchronize(st));
    return CTLCU_OK;
}

int ctlcu_launch_count(ctlcu_ctx* ctx, uint64_t* launches)
{
    if (!ctx || !launches)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    *launches = ctx->launches;
    return CTLCU_OK;
}

int ctlcu_average_samples(ctlcu_ctx* ctx, const float* in, uint32_t n_samples, uint64_t values_per_sample,
                          float* out, int low_extinction, void* stream)
{
    TraceRange trace_("ctlcu_average_samples");
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!in || !out || n_samples == 0)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "in/out is NULL or no samples");
    cudaSetDevice(ctx->device);
    if (!is_device_ptr(in) || !is_device_ptr(out))
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "in and out must be device memory");
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    CU_TRY(ctx, launch_average_samples(in, n_samples, values_per_sample, out, low_extinction != 0, st));
    ++ctx->launches;
    return CTLCU_OK;
}

int ctlcu_spectral_combine(ctlcu_ctx* ctx, const float* material_projs, uint32_t n_materials, uint32_t n_views,
                           uint64_t values_per_view, const float* mu_per_mm, const double* intensities,
                           const float* response, uint32_t n_bins, const double* total_intensity, float* out,
                           void* stream)
{
    TraceRange trace_("ctlcu_spectral_combine");
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!material_projs || !mu_per_mm || !intensities || !total_intensity || !out || !n_materials || !n_bins)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "NULL argument, no materials or no energy bins");
    if (n_views == 0 || values_per_view == 0)
        return CTLCU_OK;
    cudaSetDevice(ctx->device);
    if (!is_device_ptr(material_projs) || !is_device_ptr(out))
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "projections must be device memory");
    // spectraleffectsextension.cpp:339: a bin whose intensities sum to (fuzzy) zero is skipped
    std::vector<int> skip(n_bins, 0);
    for (uint32_t b = 0; b < n_bins; ++b) {
        double s = 0.0;
        for (uint32_t v = 0; v < n_views; ++v)
            s += intensities[(size_t)b * n_views + v];
        skip[b] = std::fabs(s) <= 1e-12;
    }
    std::vector<float> resp(n_bins, 1.0f);
    if (response)
        std::copy(response, response + n_bins, resp.begin());
    const size_t b_mu = sizeof(float) * n_bins * n_materials, b_int = sizeof(double) * n_bins * n_views,
                 b_resp = sizeof(float) * n_bins, b_skip = sizeof(int) * n_bins, b_tot = sizeof(double) * n_views;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    char* buf = nullptr;
    const size_t o_int = 0, o_tot = o_int + b_int, o_mu = o_tot + b_tot, o_resp = o_mu + b_mu, o_skip = o_resp + b_resp;
    CU_TRY(ctx, cudaMallocAsync((void**)&buf, o_skip + b_skip, st));
    cudaError_t e = cudaMemcpyAsync(buf + o_int, intensities, b_int, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(buf + o_tot, total_intensity, b_tot, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(buf + o_mu, mu_per_mm, b_mu, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(buf + o_resp, resp.data(), b_resp, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(buf + o_skip, skip.data(), b_skip, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = launch_spectral(material_projs, n_materials, values_per_view, n_views, (const float*)(buf + o_mu),
                            (const double*)(buf + o_int), (const float*)(buf + o_resp), (const int*)(buf + o_skip),
                            n_bins, (const double*)(buf + o_tot), out, st);
    // the host vectors die on return: the copies out of them must be done
    const cudaError_t w = cudaStreamSynchronize(st);
    cudaFreeAsync(buf, st);
    if (e == cudaSuccess)
        e = w;
    if (e != cudaSuccess)
        return fail(ctx, CTLCU_ERR_CUDA, "spectral combine: %s", cudaGetErrorString(e));
    ++ctx->launches;
    return CTLCU_OK;
}

int ctlcu_spectral_combine_noisy(ctlcu_ctx* ctx, const float* material_projs, uint32_t n_materials, uint32_t n_views,
                                 uint32_t n_modules, uint64_t pixels_per_module, const float* mu_per_mm,
                                 const double* intensities, const float* response, uint32_t n_bins,
                                 const double* total_intensity, const float* i0_per_bin_module, uint64_t seed,
                                 float* out, void* stream)
{
    TraceRange trace_("ctlcu_spectral_combine_noisy");
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!material_projs || !mu_per_mm || !intensities || !total_intensity || !i0_per_bin_module || !out ||
        !n_materials || !n_bins)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "NULL argument, no materials or no energy bins");
    if (n_views == 0 || n_modules == 0 || pixels_per_module == 0)
        return CTLCU_OK;
    if (pixels_per_module > 0xffffffffull / n_modules)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "too many pixels per view");
    cudaSetDevice(ctx->device);
    if (!is_device_ptr(material_projs) || !is_device_ptr(out))
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "projections must be device memory");
    // spectraleffectsextension.cpp:373: a bin without flux is skipped; poissonnoiseextension.cpp:160:
    // projections whose i0 sums to zero pass the noise step unchanged
    std::vector<int> skip(n_bins, 0), quiet(n_bins, 0);
    for (uint32_t b = 0; b < n_bins; ++b) {
        double s = 0.0, q = 0.0;
        for (uint32_t v = 0; v < n_views; ++v)
            s += intensities[(size_t)b * n_views + v];
        for (uint32_t k = 0; k < n_modules; ++k)
            q += i0_per_bin_module[(size_t)b * n_modules + k];
        skip[b] = std::fabs(s) <= 1e-12;
        quiet[b] = std::fabs(q) <= 1e-12;
    }
    std::vector<float> resp(n_bins, 1.0f);
    if (response)
        std::copy(response, response + n_bins, resp.begin());
    const size_t b_mu = sizeof(float) * n_bins * n_materials, b_int = sizeof(double) * n_bins * n_views,
                 b_resp = sizeof(float) * n_bins, b_flag = sizeof(int) * n_bins, b_tot = sizeof(double) * n_views,
                 b_i0 = sizeof(float) * n_bins * n_modules;
    const size_t o_int = 0, o_tot = o_int + b_int, o_mu = o_tot + b_tot, o_resp = o_mu + b_mu,
                 o_skip = o_resp + b_resp, o_quiet = o_skip + b_flag, o_i0 = o_quiet + b_flag;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    char* buf = nullptr;
    CU_TRY(ctx, cudaMallocAsync((void**)&buf, o_i0 + b_i0, st));
    const std::pair<size_t, std::pair<const void*, size_t>> copies[] = {
        { o_int, { intensities, b_int } }, { o_tot, { total_intensity, b_tot } },
        { o_mu, { mu_per_mm, b_mu } },     { o_resp, { resp.data(), b_resp } },
        { o_skip, { skip.data(), b_flag } }, { o_quiet, { quiet.data(), b_flag } },
        { o_i0, { i0_per_bin_module, b_i0 } } };
    cudaError_t e = cudaSuccess;
    for (const auto& c : copies)
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(buf + c.first, c.second.first, c.second.second, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = launch_spectral_noisy(material_projs, n_materials, n_views, n_modules, (uint32_t)pixels_per_module,
                                  (const float*)(buf + o_mu), (const double*)(buf + o_int),
                                  (const float*)(buf + o_resp), (const int*)(buf + o_skip),
                                  (const int*)(buf + o_quiet), n_bins, (const double*)(buf + o_tot),
                                  (const float*)(buf + o_i0), seed, out, st);
    // the host vectors die on return: the copies out of them must be done
    const cudaError_t w = cudaStreamSynchronize(st);
    cudaFreeAsync(buf, st);
    if (e == cudaSuccess)
        e = w;
    if (e != cudaSuccess)
        return fail(ctx, CTLCU_ERR_CUDA, "noisy spectral combine: %s", cudaGetErrorString(e));
    ++ctx->launches;
    return CTLCU_OK;
}

int ctlcu_combine_linear(ctlcu_ctx* ctx, const float* slope_proj, const float* offset_proj, const double* times,
                         uint32_t n_views, uint64_t values_per_view, float* out, void* stream)
{
    TraceRange trace_("ctlcu_combine_linear");
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!slope_proj || !offset_proj || !times || !out)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n_views == 0 || values_per_view == 0)
        return CTLCU_OK;
    cudaSetDevice(ctx->device);
    if (!is_device_ptr(slope_proj) || !is_device_ptr(offset_proj) || !is_device_ptr(out))
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "projections must be device memory");
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    double* d_t = nullptr;
    CU_TRY(ctx, cudaMallocAsync((void**)&d_t, sizeof(double) * n_views, st));
    cudaError_t e = cudaMemcpyAsync(d_t, times, sizeof(double) * n_views, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = launch_combine_linear(slope_proj, offset_proj, d_t, values_per_view, n_views, out, st);
    cudaFreeAsync(d_t, st);
    if (e != cudaSuccess)
        return fail(ctx, CTLCU_ERR_CUDA, "combine: %s", cudaGetErrorString(e));
    ++ctx->launches;
    return CTLCU_OK;
}

int ctlcu_den_write(ctlcu_ctx* ctx, const char* path, const void* data, uint32_t elem_bytes, uint32_t rows,
                    uint32_t cols, uint32_t count, void* stream)
{
    TraceRange trace_("ctlcu_den_write");
    if (!ctx) {
        // host data needs no context (nor a GPU)
        if (!path || !data || mem_kind(data) != Mem::Host)
            return CTLCU_ERR_INVALID_ARGUMENT;
        std::string msg;
        return den_write(path, data, elem_bytes, rows, cols, count, nullptr, nullptr, msg);
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!path || !data)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "path or data is NULL");
    cudaSetDevice(ctx->device);
    std::string msg;
    const int r = den_write(path, data, elem_bytes, rows, cols, count, stream ? (cudaStream_t)stream : ctx->stream,
                            &ctx->den, msg);
    return r ? fail(ctx, r, "DEN write: %s", msg.c_str()) : CTLCU_OK;
}

int ctlcu_nrrd_write_projections(ctlcu_ctx* ctx, const char* path, const float* data, uint32_t n_views,
                                 uint32_t n_modules, uint32_t rows, uint32_t channels, void* stream)
{
    TraceRange trace_("ctlcu_nrrd_write_projections");
    std::string msg;
    if (!ctx) {
        if (!path || !data || mem_kind(data) != Mem::Host)
            return CTLCU_ERR_INVALID_ARGUMENT;
        return nrrd_write_projections(path, data, n_views, n_modules, rows, channels, nullptr, nullptr, msg);
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!path || !data)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "path or data is NULL");
    cudaSetDevice(ctx->device);
    const int r = nrrd_write_projections(path, data, n_views, n_modules, rows, channels,
                                         stream ? (cudaStream_t)stream : ctx->stream, &ctx->den, msg);
    return r ? fail(ctx, r, "NRRD write: %s", msg.c_str()) : CTLCU_OK;
}

int ctlcu_nrrd_header(const char* path, uint32_t* version, uint32_t* n_dims, uint32_t sizes[4], uint32_t* elem_bytes,
                      uint64_t* data_offset)
{
    if (!path || !version || !n_dims || !sizes || !elem_bytes || !data_offset)
        return CTLCU_ERR_INVALID_ARGUMENT;
    NrrdHeader h;
    std::string msg;
    const int r = nrrd_header(path, h, msg);
    if (r)
        return r;
    *version = h.version;
    *n_dims = h.n_dims;
    for (int k = 0; k < 4; ++k)
        sizes[k] = h.sizes[k];
    *elem_bytes = h.elem;
    *data_offset = h.offset;
    return CTLCU_OK;
}

int ctlcu_nrrd_read(ctlcu_ctx* ctx, const char* path, void* data, uint64_t capacity_bytes, void* stream)
{
    TraceRange trace_("ctlcu_nrrd_read");
    std::string msg;
    if (!ctx) {
        if (!path || !data || mem_kind(data) != Mem::Host)
            return CTLCU_ERR_INVALID_ARGUMENT;
        return nrrd_read(path, data, capacity_bytes, nullptr, nullptr, msg);
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!path || !data)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "path or data is NULL");
    cudaSetDevice(ctx->device);
    const int r = nrrd_read(path, data, capacity_bytes, stream ? (cudaStream_t)stream : ctx->stream, &ctx->den, msg);
    return r ? fail(ctx, r, "NRRD read: %s", msg.c_str()) : CTLCU_OK;
}

int ctlcu_den_header(const char* path, uint32_t dims[3], uint32_t* elem_bytes)
{
    if (!path || !dims || !elem_bytes)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::string msg;
    return den_header(path, dims, elem_bytes, msg);
}

int ctlcu_den_read(ctlcu_ctx* ctx, const char* path, void* data, uint64_t capacity_bytes, uint32_t first, uint32_t n,
                   void* stream)
{
    TraceRange trace_("ctlcu_den_read");
    if (!ctx) {
        if (!path || !data || mem_kind(data) != Mem::Host)
            return CTLCU_ERR_INVALID_ARGUMENT;
        std::string msg;
        return den_read(path, data, capacity_bytes, first, n, nullptr, nullptr, msg);
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!path || !data)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "path or data is NULL");
    cudaSetDevice(ctx->device);
    std::string msg;
    const int r = den_read(path, data, capacity_bytes, first, n, stream ? (cudaStream_t)stream : ctx->stream,
                           &ctx->den, msg);
    return r ? fail(ctx, r, "DEN read: %s", msg.c_str()) : CTLCU_OK;
}

int ctlcu_transform_to_extinction(ctlcu_ctx* ctx, float* data, uint32_t n_views, uint64_t values_per_view,
                                  const double* i0, void* stream)
{
    TraceRange trace_("ctlcu_transform_to_extinction");
    return transform(ctx, data, n_views, values_per_view, i0, stream, true);
}

int ctlcu_transform_to_intensity(ctlcu_ctx* ctx, float* data, uint32_t n_views, uint64_t values_per_view,
                                 const double* i0, void* stream)
{
    TraceRange trace_("ctlcu_transform_to_intensity");
    return transform(ctx, data, n_views, values_per_view, i0, stream, false);
}

int ctlcu_poisson_noise(ctlcu_ctx* ctx, float* data, uint32_t n_views, uint32_t n_modules, uint32_t pixels_per_module,
                        const float* i0_per_module, uint64_t seed, void* stream)
{
    TraceRange trace_("ctlcu_poisson_noise");
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!data || !i0_per_module)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "data or i0_per_module is NULL");
    const uint64_t per_view = (uint64_t)n_modules * pixels_per_module;
    if (n_views == 0 || per_view == 0)
        return CTLCU_OK;
    if (per_view > 0xffffffffull)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "more than 2^32 pixels per view");
    // poissonnoiseextension.cpp:160: views whose i0 sum is (fuzzy) zero are skipped
    float sum = 0.0f;
    for (uint32_t m = 0; m < n_modules; ++m)
        sum += i0_per_module[m];
    if (std::fabs(sum) <= 1e-5f)
        return CTLCU_OK;
    cudaSetDevice(ctx->device);
    const size_t bytes = sizeof(float) * per_view * n_views;
    return on_device_data(ctx, data, bytes, stream, "Poisson noise", [&](float* d, cudaStream_t st) {
        float* di0 = nullptr;
        cudaError_t e = cudaMallocAsync((void**)&di0, sizeof(float) * n_modules, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(di0, i0_per_module, sizeof(float) * n_modules, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = launch_poisson_noise(d, n_views, n_modules, pixels_per_module, di0, seed, st);
        if (di0)
            cudaFreeAsync(di0, st);
        return e;
    });
}

int ctlcu_detector_saturation(ctlcu_ctx* ctx, float* data, uint32_t n_views, uint32_t n_modules,
                              uint64_t pixels_per_module, int32_t domain, const ctlcu_saturation_model* model,
                              const float* scale_per_view_module, void* stream)
{
    TraceRange trace_("ctlcu_detector_saturation");
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!data || !model)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "data or model is NULL");
    if (domain < CTLCU_SATURATION_EXTINCTION || domain > CTLCU_SATURATION_INTENSITY)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "unknown saturation domain %d", domain);
    if (model->kind != CTLCU_SATURATION_LINEAR && model->kind != CTLCU_SATURATION_SPLINE)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "unknown saturation model %d", model->kind);
    if (model->kind == CTLCU_SATURATION_SPLINE && !(model->soft_a > 0.0f && model->soft_b > 0.0f))
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "spline softening must be positive (%g, %g)",
                    (double)model->soft_a, (double)model->soft_b);
    if (domain != CTLCU_SATURATION_EXTINCTION && !scale_per_view_module)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "the photon count and intensity domains need the per-view, "
                                                     "per-module photon counts");
    if (n_views == 0 || n_modules == 0 || pixels_per_module == 0)
        return CTLCU_OK;
    if (pixels_per_module > (1ull << 40) / ((uint64_t)n_views * n_modules))
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "too many values");
    cudaSetDevice(ctx->device);
    const size_t bytes = sizeof(float) * pixels_per_module * n_modules * n_views;
    const ctlcu_saturation_model m = *model;
    return on_device_data(ctx, data, bytes, stream, "detector saturation", [&](float* d, cudaStream_t st) {
        float* ds = nullptr;
        cudaError_t e = cudaSuccess;
        if (domain != CTLCU_SATURATION_EXTINCTION) {
            const size_t sb = sizeof(float) * (size_t)n_views * n_modules;
            e = cudaMallocAsync((void**)&ds, sb, st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(ds, scale_per_view_module, sb, cudaMemcpyHostToDevice, st);
        }
        if (e == cudaSuccess)
            e = launch_saturation(d, n_views, n_modules, pixels_per_module, domain, m, ds, st);
        if (ds)
            cudaFreeAsync(ds, st);
        return e;
    });
}

int ctlcu_encode_geometry(ctlcu_ctx* ctx, const ctlcu_detector_desc* detector,
                          const ctlcu_trajectory_desc* trajectory, uint32_t n_views, double* pmats, void* stream)
{
    return ctlcu_encode_geometry_shifted(ctx, detector, trajectory, n_views, nullptr, 0, pmats, stream);
}

int ctlcu_encode_geometry_shifted(ctlcu_ctx* ctx, const ctlcu_detector_desc* detector,
                                  const ctlcu_trajectory_desc* trajectory, uint32_t n_views,
                                  const double* source_shifts_mm, uint32_t n_shifts, double* pmats, void* stream)
{
    TraceRange trace_("ctlcu_encode_geometry_shifted");
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (source_shifts_mm && n_shifts == 0)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "n_shifts is 0");
    for (uint32_t k = 0; source_shifts_mm && k < 3 * n_shifts; ++k)
        if (!std::isfinite(source_shifts_mm[k]))
            return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "source shifts must be finite");
    const uint32_t shifts = source_shifts_mm ? n_shifts : 1u;
    if (!detector || !trajectory || !pmats)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "detector, trajectory or pmats is NULL");
    const ctlcu_detector_desc& d = *detector;
    const ctlcu_trajectory_desc& t = *trajectory;
    if (n_views == 0)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "n_views is 0");
    if (d.pixels[0] == 0 || d.pixels[1] == 0 || !(d.pixel_mm[0] > 0.0) || !(d.pixel_mm[1] > 0.0))
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "detector pixel counts and sizes must be positive");
    if (d.n_modules == 0 || (d.flat_panel && d.n_modules != 1))
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "a detector has >= 1 modules, a flat panel exactly 1");
    if (!d.flat_panel && std::fabs(d.angulation_rad) <= 1e-12 && d.n_modules > 1)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT,
                    "a cylindrical detector of several modules needs a nonzero angulation");
    if (!std::isfinite(d.angulation_rad) || !std::isfinite(d.module_spacing_mm) || !std::isfinite(d.skew))
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "detector parameters must be finite");
    const bool tubular = t.kind == CTLCU_TRAJ_HELICAL || t.kind == CTLCU_TRAJ_AXIAL;
    const bool carm = t.kind == CTLCU_TRAJ_WOBBLE || t.kind == CTLCU_TRAJ_SHORT_SCAN ||
                      t.kind == CTLCU_TRAJ_CIRCLE_PLUS_LINE;
    if (!tubular && !carm)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "unknown trajectory kind %d", t.kind);
    if (tubular && !(t.sdd_mm > 0.0 && t.sid_mm > 0.0))
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "a tubular gantry needs positive SDD and SID");
    if (carm && !(t.carm_span_mm > 0.0))
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "a C-arm gantry needs a positive C-arm span");
    if (t.kind == CTLCU_TRAJ_CIRCLE_PLUS_LINE && !(t.line_fraction >= 0.0 && t.line_fraction <= 1.0))
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "line_fraction must lie in [0, 1]");
    const uint64_t n = (uint64_t)n_views * d.n_modules * shifts;
    if (n > 0x7fffffffull)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "too many matrices");
    cudaSetDevice(ctx->device);
    if (int rc = check_local(ctx, { pmats }))
        return rc;
    const bool dev = is_device_ptr(pmats);
    cudaStream_t st = dev && stream ? (cudaStream_t)stream : ctx->stream;
    double* out = pmats;
    double* d_shifts = nullptr;
    if (!dev)
        CU_TRY(ctx, cudaMallocAsync((void**)&out, n * 12 * sizeof(double), st));
    cudaError_t e = cudaSuccess;
    if (source_shifts_mm) {
        e = cudaMallocAsync((void**)&d_shifts, sizeof(double) * 3 * shifts, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_shifts, source_shifts_mm, sizeof(double) * 3 * shifts, cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess)
        e = launch_encode_geometry(d, t, n_views, d_shifts, shifts, out, st);
    if (e == cudaSuccess && !dev)
        e = cudaMemcpyAsync(pmats, out, n * 12 * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (d_shifts)
        cudaFreeAsync(d_shifts, st);
    if (!dev)
        cudaFreeAsync(out, st);
    if (e != cudaSuccess)
        return fail(ctx, CTLCU_ERR_CUDA, "geometry encoding: %s", cudaGetErrorString(e));
    ++ctx->launches;
    if (!dev)
        CU_TRY(ctx, cudaStreamSynchronize(st));
    return CTLCU_OK;
}

// ctlcu_project with device pmats/out whose setup writes the ray geometry into
// the static scratch array instead of pool memory.  Nothing has to be cleared
// first: the setup kernel writes every (view, module) entry that the
// projection then reads, and the flag word is zero between calls (read_flags
// clears it).
int ctlcu_project_noalloc(ctlcu_ctx* ctx, uint64_t volume, const ctlcu_settings* settings,
                          const double* pmats, uint32_t n_views, uint32_t n_modules, uint32_t channels,
                          uint32_t rows, float* out, void* stream)
{
    if (!ctx)
        return CTLCU_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!pmats || !out)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT, "pmats or out is NULL");
    int r = check_settings(ctx, settings);
    if (r)
        return r;
    r = check_job(ctx, n_views, n_modules, channels, rows);
    if (r)
        return r;
    const uint64_t nvm = (uint64_t)n_views * n_modules;
    if (nvm > CTLCU_NOALLOC_MAX_VIEW_MODULES)
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT,
                    "%llu view-modules exceed the no-allocation scratch limit of %d; split the call",
                    (unsigned long long)nvm, CTLCU_NOALLOC_MAX_VIEW_MODULES);
    VolumeEntry* v = find_volume(ctx, volume);
    if (!v)
        return fail(ctx, CTLCU_ERR_INVALID_HANDLE, "unknown volume handle %llu", (unsigned long long)volume);
    cudaSetDevice(ctx->device);
    if (!is_device_ptr(pmats) || !is_device_ptr(out))
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT,
                    "the no-allocation call needs device pmats and out (host buffers need staging memory)");
    const ctlcu_settings eff = resolve_kernel(ctx, *v, settings, channels, rows, n_modules);
    if (const char* what = missing_array(*v, &eff))
        return fail(ctx, CTLCU_ERR_INVALID_ARGUMENT,
                    "the %s of this volume is not built; project it once with ctlcu_project first", what);
    ViewGeom* geom = nullptr;
    r = noalloc_scratch(ctx, &geom);
    if (r)
        return r;
    ProjectArgs a = {};
    Mode mode;
    int dtype;
    r = volume_args(ctx, *v, &eff, a, mode, dtype);
    if (r)
        return r;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    r = order_after_staging(ctx, st);
    if (r)
        return r;
    job_args(a, &eff, n_views, n_modules, channels, rows);
    CU_TRY(ctx, launch_setup(pmats, n_views, n_modules, geom, nullptr, nullptr, ctx->d_flags, st));
    a.geom = geom;
    a.out = out;
    a.flags = ctx->d_flags;
    a.counter = nullptr;
    CU_TRY(ctx, launch_project(a, mode, (Accum)eff.accum, dtype, st));
    ctx->launches += 2;
    return CTLCU_OK;
}

}  // extern "C"

// Internal types shared by the ctlcu translation units.
#pragma once

#include "ctlcu.h"

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace ctlcu {

// Zero voxels stored on every side of a resident volume.  With two layers and
// per-axis index clamping, every trilinear tap of any sample position (inside
// or outside the volume) reads either a real voxel or a zero, which is the
// OpenCL CLK_ADDRESS_CLAMP border of the reference (border colour 0).
constexpr int kPad = 2;

// Register budgets of the sample loops (measured best; see the launch shapes below).
#ifndef CTLCU_CELL_MAXREG
#define CTLCU_CELL_MAXREG 48  // cell and pair loops: 5 blocks of 256 threads per SM
#endif
#ifndef CTLCU_GATHER_MAXREG
#define CTLCU_GATHER_MAXREG 80  // gather, nearest-voxel and texture loops: 3 blocks of 256 per SM
#endif
#ifndef CTLCU_VM_GROUP
#define CTLCU_VM_GROUP 8  // view groups per chunk in the block order
#endif

// Launch shape of the projection kernels, chosen per call at run time
// (ctlcu_settings views_per_block, lanes_x, block_rays, unroll; the
// autotuner picks them per volume and detector).  A thread block holds
// `block` rays: one detector tile of tile_x x tile_y pixels for each of
// `views` consecutive views of one module.  Adjacent views of a scan see a
// tile through nearly the same part of the volume, so their rays share cached
// cells.  Each warp is a lanes_x x (32 / lanes_x) pixel patch of one view, so
// its 32 rays are neighbours.  `unroll` samples of the cell and pair loops
// form one FP32 partial sum before it goes to the accumulator.
struct LaunchShape {
    uint32_t block = 256;   // rays (threads) per block: 128, 256 or 512
    uint32_t views = 2;     // views per block: 1, 2 or 4
    uint32_t lanes_x = 4;   // lanes of a warp along the channels: 4 (4x8 patch) or 8 (8x4)
    uint32_t unroll = 4;    // samples per partial sum: 2, 4 or 8
};
constexpr uint32_t kMaxBlock = 512;

// Tile of a shape: pixels per view = block / views, 16 channels wide from 128
// pixels up, else 8.
__host__ __device__ constexpr uint32_t shape_tile_x(uint32_t block, uint32_t views)
{
    return block / views >= 128 ? 16u : 8u;
}
__host__ __device__ constexpr uint32_t shape_tile_y(uint32_t block, uint32_t views)
{
    return block / views / shape_tile_x(block, views);
}

// Null if the shape is valid, else what is wrong with it.
inline const char* shape_error(const LaunchShape& s)
{
    if (s.block != 128 && s.block != 256 && s.block != 512)
        return "block_rays must be 128, 256 or 512";
    if (s.views != 1 && s.views != 2 && s.views != 4)
        return "views_per_block must be 1, 2 or 4";
    if (s.lanes_x != 4 && s.lanes_x != 8)
        return "lanes_x must be 4 or 8";
    if (s.unroll != 2 && s.unroll != 4 && s.unroll != 8)
        return "unroll must be 2, 4 or 8";
    if (shape_tile_y(s.block, s.views) % (32u / s.lanes_x) != 0)
        return "the warp patch (lanes_x x 32/lanes_x) does not tile the detector tile of this block";
    return nullptr;
}

// Error bits raised by kernels into the context's device flag word.
constexpr int kFlagSingular = 1;   // a projection matrix with singular / non-finite M
constexpr int kFlagNonFinite = 2;  // a ray with non-finite entry/exit parameters


// Per (view, module) geometry, written by the FP64 setup kernel.
struct ViewGeom {
    double A[9];    // sign(det M) * M^-1, row major: direction = A * [x, y, 1]
    double src[3];  // source position in mm (from the view's module-0 matrix)
    int valid;      // 0 when M is singular or not finite
    int pad_;
};

// Round-to-integer constant: for |v| < 2^22, the float sum v + kMagic is
// kMagic + rint(v) and its bit pattern is kMagicBits + rint(v).
constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23
constexpr uint32_t kMagicBits = 0x4B400000u;

// Bytes per cell of the coefficient cell array (8 floats).
constexpr int kCellBytes = 32;

// Layout of the cell array of a volume with n voxels per axis: cells span
// padded voxels, (n + 2 kPad - 1) per axis, x fastest, row stride sy, slice
// stride sz.  sz is padded so that 1 + sy + sz is a multiple of 1024; then
// kMagicBits * (1 + sy + sz) = 0 mod 2^32, and the index of the cell whose
// per-axis magic sums have bit patterns bx, by, bz is exactly
// bx + by sy + bz sz in 32-bit arithmetic.
struct CellLayout {
    uint32_t cx, cy, cz;  // cells per axis
    uint32_t sy, sz;      // strides (cells) of y and of the slowest axis
    uint64_t count;       // cells allocated
    uint32_t max_index;   // index of the last real cell
};

inline CellLayout cell_layout(const int n[3])
{
    CellLayout L;
    L.cx = (uint32_t)(n[0] + 2 * kPad - 1);
    L.cy = (uint32_t)(n[1] + 2 * kPad - 1);
    L.cz = (uint32_t)(n[2] + 2 * kPad - 1);
    L.sy = L.cx;
    const uint32_t base = L.cx * L.cy;
    const uint32_t e = (1024u - ((1u + L.sy + base) & 1023u)) & 1023u;
    L.sz = base + e;
    L.count = (uint64_t)L.sz * L.cz;
    L.max_index = (L.cz - 1) * L.sz + (L.cy - 1) * L.sy + (L.cx - 1);
    return L;
}

// Linear cell index from per-axis indices (or their magic-sum bit patterns).
__host__ __device__ __forceinline__ uint32_t cell_linear(uint32_t ix, uint32_t iy, uint32_t iz, uint32_t sy,
                                                         uint32_t sz)
{
    return ix + iy * sy + iz * sz;
}

// x-pair array: for every padded voxel (x < ext_x - 1, y, z) the float2
// (mid, diff) = ((v[x] + v[x+1]) / 2, v[x+1] - v[x]), computed in FP64.  A
// trilinear cell reads four entries (its two rows in y times two slices in
// z); the x interpolation of an entry at offset h from the cell centre is
// mid + h * diff.  8 bytes per voxel; strides padded like the cell array so
// the magic offsets cancel.
struct PairLayout {
    uint32_t px, ey, ez;  // entries per row, rows, slices
    uint32_t sy, sz;      // strides (entries)
    uint64_t count;       // entries allocated (sz * ez)
    uint32_t max_base;    // largest first-entry index whose 4 entries are in the array
};

inline PairLayout pair_layout(const int n[3])
{
    PairLayout L;
    L.px = (uint32_t)(n[0] + 2 * kPad - 1);
    L.ey = (uint32_t)(n[1] + 2 * kPad);
    L.ez = (uint32_t)(n[2] + 2 * kPad);
    L.sy = L.px;
    const uint32_t base = L.px * L.ey;
    const uint32_t e = (1024u - ((1u + L.sy + base) & 1023u)) & 1023u;
    L.sz = base + e;
    L.count = (uint64_t)L.sz * L.ez;
    L.max_base = (uint32_t)(L.count - 1 - L.sy - L.sz);
    return L;
}

enum class Mode : int { Trilinear = 0, Nearest = 1, Texture = 2, Cells = 3, Pairs = 4 };
enum class Accum : int { F64 = 0, Kahan = 1, F32 = 2 };

// Everything a projection launch needs, passed by value.
struct ProjectArgs {
    const void* vol;          // padded storage, x fastest
    cudaTextureObject_t tex;  // hardware-filtered texture (Mode::Texture)
    int ext[3];               // padded extents (voxels)
    int sy, sz;               // padded strides (voxels)
    int grid[3];              // voxel grid the rays see (f * n, or 1 for the mean voxel)
    int up;                   // virtual up-sampling factor (>= 1)
    double voxel[3];          // voxel size of that grid (mm)
    double corner[3];         // low corner of that grid (mm)
    double increment;         // step length (mm)
    const void* cells;        // Mode::Cells: coefficient cells, x fastest
    uint32_t csy, csz;        // cell strides (cells per row, per slice)
    uint32_t cmax;            // last valid cell index
    uint32_t vm_group;        // view groups per chunk of the block order
    uint32_t n_views;         // views (n_vm / n_modules)
    uint32_t view_groups;     // ceil(n_views / views per block)
    // launch shape (LaunchShape), as block size and log2 factors of the pixel mapping
    uint32_t block;           // threads per block
    uint32_t unroll;          // samples per partial sum (cell and pair loops)
    uint32_t vpb_shift;       // log2 views per block
    uint32_t wpv_shift;       // log2 warps per view
    uint32_t lx_shift;        // log2 lanes along the channels
    uint32_t wx_shift;        // log2 warps along the channels of a tile
    uint32_t tx_shift, ty_shift;  // log2 tile width and height
    const ViewGeom* geom;     // [n_vm]
    float* out;               // [n_vm][rows][channels]
    uint32_t channels, rows;
    uint32_t n_vm;            // views * modules
    uint32_t n_modules;
    uint32_t tiles_x, tiles_per_vm;
    uint32_t rays_x, rays_y;
    int* flags;
    unsigned long long* counter;  // sample count (count kernel only)
};

// One request of a batched setup (device array).
struct BatchSetup {
    const double* pmats;  // n_vm * 12 doubles
    uint32_t first_vm;    // first global view-module index of this request
    uint32_t n_modules;
};

// One request of a batched projection (device array): its launch arguments
// (geom pointing at its ViewGeom entries) and its range of work items (block
// tiles of the single-request launch).
struct BatchReq {
    ProjectArgs a;
    uint32_t first_item;  // first work item (block) of this request
    uint32_t items;       // work items of this request
};

// Launchers (raycast.cu / setup.cu / volume.cu).  All asynchronous on `s`.
cudaError_t launch_batch_setup(const BatchSetup* reqs, uint32_t n_reqs, uint32_t total, ViewGeom* geom,
                               int* flags, cudaStream_t s);
// Persistent launch (Mode::Cells or Mode::Pairs) over all work items of a
// batch (total_items block tiles, each block / 32 warp patches, dealt out to
// warps one patch at a time), every request with the launch shape `shape`
// (block size and unroll); `counter` must be zero at launch.  Returns the
// grid size in *blocks.
cudaError_t launch_batch(const BatchReq* reqs, uint32_t n_reqs, uint32_t total_items, Mode mode, Accum acc,
                         const LaunchShape& shape, unsigned int* counter, int* blocks, cudaStream_t s);
cudaError_t launch_setup(const double* pmats, uint32_t n_views, uint32_t n_modules, ViewGeom* geom,
                         double* qr_out, double* src_out, int* flags, cudaStream_t s);
cudaError_t launch_project(const ProjectArgs& a, Mode mode, Accum acc, int dtype, cudaStream_t s);
cudaError_t launch_count(const ProjectArgs& a, Mode mode, cudaStream_t s);
cudaError_t launch_pad_convert(const float* src, void* dst, const int n[3], int dtype, cudaStream_t s);
cudaError_t launch_mean(const void* padded, const int n[3], int dtype, double* sum_out, cudaStream_t s);
cudaError_t launch_mean_volume(const double* sum, double count, float* dst_padded, cudaStream_t s);
cudaError_t launch_build_cells(const void* padded, const int n[3], int dtype, const CellLayout& L,
                               void* cells, cudaStream_t s);
cudaError_t launch_build_pairs(const void* padded, const int n[3], int dtype, const PairLayout& L,
                               void* pairs, cudaStream_t s);
cudaError_t launch_unpad_upsample(const void* padded, const int n[3], int dtype, int f, void* dst,
                                  cudaStream_t s);
cudaError_t launch_encode_geometry(const ctlcu_detector_desc& det, const ctlcu_trajectory_desc& traj,
                                   uint32_t n_views, const double* d_shifts, uint32_t n_shifts, double* pmats,
                                   cudaStream_t s);
cudaError_t launch_average_samples(const float* in, uint32_t n_samples, uint64_t n, float* out, bool low_extinction,
                                   cudaStream_t s);
cudaError_t launch_combine_linear(const float* slope, const float* offset, const double* d_times, uint64_t per_view,
                                  uint32_t n_views, float* out, cudaStream_t s);
cudaError_t launch_spectral(const float* proj, uint32_t n_materials, uint64_t per_view, uint32_t n_views,
                            const float* mu, const double* intensity, const float* response, const int* skip,
                            uint32_t n_bins, const double* total, float* out, cudaStream_t s);
cudaError_t launch_saturation(float* data, uint32_t n_views, uint32_t n_modules, uint64_t ppm, int domain,
                              const ctlcu_saturation_model& model, const float* scale, cudaStream_t s);
cudaError_t launch_spectral_noisy(const float* proj, uint32_t n_materials, uint32_t n_views, uint32_t n_modules,
                                  uint32_t ppm, const float* mu, const double* intensity, const float* response,
                                  const int* skip, const int* quiet, uint32_t n_bins, const double* total,
                                  const float* i0, uint64_t seed, float* out, cudaStream_t s);
cudaError_t launch_poisson_noise(float* data, uint32_t n_views, uint32_t n_modules, uint32_t ppm, const float* i0,
                                 uint64_t seed, cudaStream_t s);
cudaError_t launch_transform(float* data, uint64_t per_view, uint32_t n_views, const double* i0, bool to_extinction,
                             cudaStream_t s);
}  // namespace ctlcu

#include <cstdio>
#include <string>

#include <nvtx3/nvToolsExt.h>

namespace ctlcu {
// A named NVTX range around a C-ABI call, for timeline tools (Nsight Systems,
// Nsight Compute's --nvtx filters); a no-op when no tool is attached.
struct TraceRange {
    explicit TraceRange(const char* name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange&) = delete;
    TraceRange& operator=(const TraceRange&) = delete;
};

// Two pinned host buffers and their events for streaming device data to and
// from files; a context keeps one, allocated on first use.
struct DenStaging {
    static constexpr size_t kBytes = 32u << 20;  // per buffer
    void* buf[2] = { nullptr, nullptr };
    cudaEvent_t ev[2] = { nullptr, nullptr };
    cudaError_t ensure();
    void release();
};
int den_write(const char* path, const void* data, uint32_t elem, uint32_t rows, uint32_t cols, uint32_t count,
              cudaStream_t st, DenStaging* stage, std::string& msg);
int den_header(const char* path, uint32_t dims[3], uint32_t* elem, std::string& msg);
int den_read(const char* path, void* data, uint64_t capacity, uint32_t first, uint32_t n_mats, cudaStream_t st,
             DenStaging* stage, std::string& msg);
// Write / read `total` bytes of host or device data at an open file's position
// (device data through the staging buffers, copies overlapping the file I/O).
int file_write_data(FILE* f, const void* data, size_t total, cudaStream_t st, DenStaging* stage, std::string& msg);
int file_read_data(FILE* f, void* data, size_t total, cudaStream_t st, DenStaging* stage, std::string& msg);
struct NrrdHeader {
    uint32_t version = 0, n_dims = 0, sizes[4] = { 0, 0, 0, 0 };
    uint32_t elem = 0;       // bytes per element
    bool is_float = false;   // float/double (else integer)
    uint64_t offset = 0;     // bytes before the data
};
int nrrd_header(const char* path, NrrdHeader& h, std::string& msg);
int nrrd_write_projections(const char* path, const float* data, uint32_t views, uint32_t modules, uint32_t rows,
                           uint32_t channels, cudaStream_t st, DenStaging* stage, std::string& msg);
int nrrd_read(const char* path, void* data, uint64_t capacity, cudaStream_t st, DenStaging* stage, std::string& msg);

}  // namespace ctlcu

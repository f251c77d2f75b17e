// Internal types shared by the ctlcu translation units.
#pragma once

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

// Detector tile handled by one thread block: 16 x 16 pixels, each warp an
// 8 (channels) x 4 (rows) patch so that the 32 rays of a warp are neighbours
// and their samples share cache lines.
constexpr int kTileX = 16;
constexpr int kTileY = 16;
constexpr int kBlock = kTileX * kTileY;

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

enum class Mode : int { Trilinear = 0, Nearest = 1, Texture = 2, Cells = 3 };
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
    uint32_t ckoff;           // kMagicBits * (1 + csy + csz) mod 2^32
    uint32_t vm_group;        // blocks cover `vm_group` consecutive view-modules per tile
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

// Launchers (raycast.cu / setup.cu / volume.cu).  All asynchronous on `s`.
cudaError_t launch_setup(const double* pmats, uint32_t n_views, uint32_t n_modules, ViewGeom* geom,
                         double* qr_out, double* src_out, int* flags, cudaStream_t s);
cudaError_t launch_project(const ProjectArgs& a, Mode mode, Accum acc, int dtype, cudaStream_t s);
cudaError_t launch_count(const ProjectArgs& a, Mode mode, cudaStream_t s);
cudaError_t launch_pad_convert(const float* src, void* dst, const int n[3], int dtype, cudaStream_t s);
cudaError_t launch_mean(const void* padded, const int n[3], int dtype, double* sum_out, cudaStream_t s);
cudaError_t launch_mean_volume(const double* sum, double count, float* dst_padded, cudaStream_t s);
cudaError_t launch_build_cells(const void* padded, const int n[3], int dtype, void* cells, cudaStream_t s);
cudaError_t launch_unpad_upsample(const void* padded, const int n[3], int dtype, int f, void* dst,
                                  cudaStream_t s);

}  // namespace ctlcu

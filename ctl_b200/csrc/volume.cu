// Volume staging kernels: zero-padded resident copies in the storage dtype,
// the f = 0 mean voxel, and materialised up-sampling for the texture path.
//
// Reference: VolumeSpecs::upSampleVolume (modules/src/projectors/raycasterprojector.cpp:576-672)
// builds, on the host and per project() call, either one voxel holding the
// mean (f = 0), the volume as is (f = 1), or an f^3 nearest-neighbour
// replication (f >= 2).  Here f >= 2 is virtual for the software path (index
// math in raycast.cu) and materialised only for the hardware-texture path.
#include "internal.cuh"

namespace ctlcu {

namespace {

template <typename T>
__device__ __forceinline__ T from_float(float v);
template <>
__device__ __forceinline__ float from_float<float>(float v) { return v; }
template <>
__device__ __forceinline__ __nv_bfloat16 from_float<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <>
__device__ __forceinline__ __half from_float<__half>(float v) { return __float2half_rn(v); }

template <typename T>
__device__ __forceinline__ float to_float(T v);
template <>
__device__ __forceinline__ float to_float<float>(float v) { return v; }
template <>
__device__ __forceinline__ float to_float<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <>
__device__ __forceinline__ float to_float<__half>(__half v) { return __half2float(v); }

// dst (padded, zero-initialised by the caller) <- convert(src), one thread per voxel
template <typename T>
__global__ void pad_convert_kernel(const float* __restrict__ src, T* __restrict__ dst, int nx, int ny,
                                   int nz)
{
    const int ex = nx + 2 * kPad, ey = ny + 2 * kPad;
    const size_t total = (size_t)nx * ny * nz;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx);
        const size_t r = i / nx;
        const int y = (int)(r % ny);
        const int z = (int)(r / ny);
        dst[(size_t)(x + kPad) + (size_t)ex * ((size_t)(y + kPad) + (size_t)ey * (size_t)(z + kPad))] =
            from_float<T>(src[i]);
    }
}

// FP64 sum of the (dequantised) stored voxels; one atomicAdd per block
template <typename T>
__global__ void sum_kernel(const T* __restrict__ padded, int nx, int ny, int nz, double* sum)
{
    const int ex = nx + 2 * kPad, ey = ny + 2 * kPad;
    const size_t total = (size_t)nx * ny * nz;
    double s = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx);
        const size_t r = i / nx;
        const int y = (int)(r % ny);
        const int z = (int)(r / ny);
        s += (double)to_float<T>(
            padded[(size_t)(x + kPad) + (size_t)ex * ((size_t)(y + kPad) + (size_t)ey * (size_t)(z + kPad))]);
    }
    __shared__ double part[32];
    for (int o = 16; o > 0; o >>= 1)
        s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0)
        part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = (threadIdx.x < (blockDim.x >> 5)) ? part[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1)
            s += __shfl_down_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0)
            atomicAdd(sum, s);
    }
}

// 1x1x1 volume (padded to (1+2P)^3, zero-initialised by the caller) holding the mean
__global__ void mean_volume_kernel(const double* sum, double count, float* dst)
{
    const int e = 1 + 2 * kPad;
    dst[kPad + e * (kPad + e * kPad)] = (float)(*sum / count);
}

// dst (dense, f*n per axis, storage dtype) <- nearest replication of the stored volume
template <typename T>
__global__ void upsample_kernel(const T* __restrict__ padded, int nx, int ny, int nz, int f,
                                T* __restrict__ dst)
{
    const int ex = nx + 2 * kPad, ey = ny + 2 * kPad;
    const size_t X = (size_t)nx * f, Y = (size_t)ny * f, Z = (size_t)nz * f;
    const size_t total = X * Y * Z;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t x = i % X;
        const size_t r = i / X;
        const size_t y = r % Y;
        const size_t z = r / Y;
        dst[i] = padded[(x / f + kPad) + ex * ((y / f + kPad) + (size_t)ey * (z / f + kPad))];
    }
}

// Coefficient cells.  Cell (i, j, k) spans padded voxels i..i+1, j..j+1, k..k+1.
// With h = w - 1/2 the local offsets from the cell centre, its trilinear
// interpolant is
//   f = C0 + Cx hx + Cy hy + Cz hz + Cxy hx hy + Cxz hx hz + Cyz hy hz + Cxyz hx hy hz,
//   C0 = sum v / 8, Cx = sum sx v / 4, Cxy = sum sx sy v / 2, Cxyz = sum sx sy sz v
// (s = -1 for the low corner, +1 for the high one, per axis).  The 8
// coefficients are computed in FP64 and stored as FP32 in the order
//   (C0, Cz), (Cx, Cxz), (Cy, Cyz), (Cxy, Cxyz)
// so the sampler evaluates f with three packed f32x2 FMAs and one FMA.
template <typename T>
__global__ void build_cells_kernel(const T* __restrict__ padded, int ex, int ey, int ez, uint32_t csy,
                                   uint32_t csz, float4* __restrict__ cells)
{
    const int cx = ex - 1, cy = ey - 1, cz = ez - 1;
    const size_t total = (size_t)cx * cy * cz;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % cx);
        const size_t r = i / cx;
        const int y = (int)(r % cy);
        const int z = (int)(r / cy);
        const size_t o = (size_t)x + (size_t)ex * ((size_t)y + (size_t)ey * z);
        const size_t sy = ex, sz = (size_t)ex * ey;
        double v[2][2][2];  // [z][y][x]
        for (int c = 0; c < 2; ++c)
            for (int b = 0; b < 2; ++b)
                for (int a = 0; a < 2; ++a)
                    v[c][b][a] = (double)to_float<T>(padded[o + a + b * sy + c * sz]);
        double C0 = 0, Cx = 0, Cy = 0, Cz = 0, Cxy = 0, Cxz = 0, Cyz = 0, Cxyz = 0;
        for (int c = 0; c < 2; ++c)
            for (int b = 0; b < 2; ++b)
                for (int a = 0; a < 2; ++a) {
                    const double sx = a ? 1.0 : -1.0, sy_ = b ? 1.0 : -1.0, sz_ = c ? 1.0 : -1.0;
                    const double t = v[c][b][a];
                    C0 += t;
                    Cx += sx * t;
                    Cy += sy_ * t;
                    Cz += sz_ * t;
                    Cxy += sx * sy_ * t;
                    Cxz += sx * sz_ * t;
                    Cyz += sy_ * sz_ * t;
                    Cxyz += sx * sy_ * sz_ * t;
                }
        const size_t c = cell_linear((uint32_t)x, (uint32_t)y, (uint32_t)z, csy, csz);
        cells[2 * c] = make_float4((float)(C0 * 0.125), (float)(Cz * 0.25), (float)(Cx * 0.25), (float)(Cxz * 0.5));
        cells[2 * c + 1] = make_float4((float)(Cy * 0.25), (float)(Cyz * 0.5), (float)(Cxy * 0.5), (float)Cxyz);
    }
}

// x-pair entries (mid, diff) of the padded volume, see PairLayout.
template <typename T>
__global__ void build_pairs_kernel(const T* __restrict__ padded, int ex, int ey, int ez, uint32_t psy,
                                   uint32_t psz, float2* __restrict__ pairs)
{
    const int px = ex - 1;
    const size_t total = (size_t)px * ey * ez;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % px);
        const size_t r = i / px;
        const int y = (int)(r % ey);
        const int z = (int)(r / ey);
        const size_t o = (size_t)x + (size_t)ex * ((size_t)y + (size_t)ey * z);
        const double a = (double)to_float<T>(padded[o]), b = (double)to_float<T>(padded[o + 1]);
        pairs[(size_t)x + (size_t)psy * y + (size_t)psz * z] = make_float2((float)(0.5 * (a + b)), (float)(b - a));
    }
}

unsigned grid_for(size_t n)
{
    size_t b = (n + 255) / 256;
    if (b > 148 * 64)
        b = 148 * 64;
    return (unsigned)(b ? b : 1);
}

}  // namespace

cudaError_t launch_pad_convert(const float* src, void* dst, const int n[3], int dtype, cudaStream_t s)
{
    const unsigned g = grid_for((size_t)n[0] * n[1] * n[2]);
    switch (dtype) {
    case 0: pad_convert_kernel<float><<<g, 256, 0, s>>>(src, (float*)dst, n[0], n[1], n[2]); break;
    case 1: pad_convert_kernel<__nv_bfloat16><<<g, 256, 0, s>>>(src, (__nv_bfloat16*)dst, n[0], n[1], n[2]); break;
    case 2: pad_convert_kernel<__half><<<g, 256, 0, s>>>(src, (__half*)dst, n[0], n[1], n[2]); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_mean(const void* padded, const int n[3], int dtype, double* sum_out, cudaStream_t s)
{
    const unsigned g = grid_for((size_t)n[0] * n[1] * n[2]);
    switch (dtype) {
    case 0: sum_kernel<float><<<g, 256, 0, s>>>((const float*)padded, n[0], n[1], n[2], sum_out); break;
    case 1: sum_kernel<__nv_bfloat16><<<g, 256, 0, s>>>((const __nv_bfloat16*)padded, n[0], n[1], n[2], sum_out); break;
    case 2: sum_kernel<__half><<<g, 256, 0, s>>>((const __half*)padded, n[0], n[1], n[2], sum_out); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_mean_volume(const double* sum, double count, float* dst_padded, cudaStream_t s)
{
    mean_volume_kernel<<<1, 1, 0, s>>>(sum, count, dst_padded);
    return cudaGetLastError();
}

cudaError_t launch_build_cells(const void* padded, const int n[3], int dtype, const CellLayout& L,
                               void* cells, cudaStream_t s)
{
    const int ex = n[0] + 2 * kPad, ey = n[1] + 2 * kPad, ez = n[2] + 2 * kPad;
    const unsigned g = grid_for((size_t)(ex - 1) * (ey - 1) * (ez - 1));
    // the stride padding between slices is never sampled; keep it zero
    cudaError_t e = cudaMemsetAsync(cells, 0, L.count * kCellBytes, s);
    if (e != cudaSuccess)
        return e;
    switch (dtype) {
    case 0: build_cells_kernel<float><<<g, 256, 0, s>>>((const float*)padded, ex, ey, ez, L.sy, L.sz, (float4*)cells); break;
    case 1: build_cells_kernel<__nv_bfloat16><<<g, 256, 0, s>>>((const __nv_bfloat16*)padded, ex, ey, ez, L.sy, L.sz, (float4*)cells); break;
    case 2: build_cells_kernel<__half><<<g, 256, 0, s>>>((const __half*)padded, ex, ey, ez, L.sy, L.sz, (float4*)cells); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_build_pairs(const void* padded, const int n[3], int dtype, const PairLayout& L,
                               void* pairs, cudaStream_t s)
{
    const int ex = n[0] + 2 * kPad, ey = n[1] + 2 * kPad, ez = n[2] + 2 * kPad;
    const unsigned g = grid_for((size_t)(ex - 1) * ey * ez);
    cudaError_t e = cudaMemsetAsync(pairs, 0, L.count * sizeof(float2), s);
    if (e != cudaSuccess)
        return e;
    switch (dtype) {
    case 0: build_pairs_kernel<float><<<g, 256, 0, s>>>((const float*)padded, ex, ey, ez, L.sy, L.sz, (float2*)pairs); break;
    case 1: build_pairs_kernel<__nv_bfloat16><<<g, 256, 0, s>>>((const __nv_bfloat16*)padded, ex, ey, ez, L.sy, L.sz, (float2*)pairs); break;
    case 2: build_pairs_kernel<__half><<<g, 256, 0, s>>>((const __half*)padded, ex, ey, ez, L.sy, L.sz, (float2*)pairs); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_unpad_upsample(const void* padded, const int n[3], int dtype, int f, void* dst,
                                  cudaStream_t s)
{
    const unsigned g = grid_for((size_t)n[0] * n[1] * n[2] * f * f * f);
    switch (dtype) {
    case 0: upsample_kernel<float><<<g, 256, 0, s>>>((const float*)padded, n[0], n[1], n[2], f, (float*)dst); break;
    case 1: upsample_kernel<__nv_bfloat16><<<g, 256, 0, s>>>((const __nv_bfloat16*)padded, n[0], n[1], n[2], f, (__nv_bfloat16*)dst); break;
    case 2: upsample_kernel<__half><<<g, 256, 0, s>>>((const __half*)padded, n[0], n[1], n[2], f, (__half*)dst); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace ctlcu

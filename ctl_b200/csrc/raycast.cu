// Cone-beam ray casting kernels (sm_100a).
//
// One thread per detector pixel; a block covers one detector tile of a few
// neighbouring views of one module, each warp a small pixel patch of one view
// (LaunchShape, chosen per call).  Per ray, in FP64: direction
// A*[x,y,1] normalised and scaled to one step in voxel units, entry/exit
// parameters against the (half-voxel padded) volume box with the 0.01-voxel
// face tolerance, first/last sample index.  The sample loop then runs in FP32
// on positions rebased at the first sample, so their magnitude is bounded by
// the volume extent rather than the source distance.
//
// Reference: modules/src/ocl/cl_src/projectors/raycasterprojector_interp.cl:18-148
// (trilinear, image3d_t + CLK_FILTER_LINEAR + CLK_ADDRESS_CLAMP) and
// raycasterprojector_no_interp.cl:16-154 (nearest voxel), launched per view
// over (channels, rows, modules) by raycasterprojector.cpp:339-343.  Here all
// views of a call go in one launch.
//
// Sampling scheme (identical to the reference): sample i sits at
// source + i*step for i = floor(tmin) .. floor(tmax)+1, tmin/tmax clamped at
// 0; a ray that hits no face takes no samples; the result is
// increment * sum / raysPerPixel.  Samples outside the padded box read zeros.
#include "internal.cuh"

#include <algorithm>
#include <cfloat>

namespace ctlcu {

namespace {

template <typename T>
__device__ __forceinline__ float load_voxel(const T* p);

template <>
__device__ __forceinline__ float load_voxel<float>(const float* p)
{
    return __ldg(p);
}
template <>
__device__ __forceinline__ float load_voxel<__nv_bfloat16>(const __nv_bfloat16* p)
{
    const unsigned short u = __ldg(reinterpret_cast<const unsigned short*>(p));
    return __uint_as_float(static_cast<unsigned int>(u) << 16);
}
template <>
__device__ __forceinline__ float load_voxel<__half>(const __half* p)
{
    const unsigned short u = __ldg(reinterpret_cast<const unsigned short*>(p));
    return __half2float(__ushort_as_half(u));
}

template <Accum A>
struct Accumulator;

template <>
struct Accumulator<Accum::F64> {
    double s = 0.0;
    __device__ __forceinline__ void add(float v) { s += static_cast<double>(v); }
    __device__ __forceinline__ double value() const { return s; }
};

template <>
struct Accumulator<Accum::Kahan> {
    float s = 0.0f, c = 0.0f;
    __device__ __forceinline__ void add(float v)
    {
        const float y = v - c;
        const float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ double value() const { return static_cast<double>(s); }
};

template <>
struct Accumulator<Accum::F32> {
    float s = 0.0f;
    __device__ __forceinline__ void add(float v) { s += v; }
    __device__ __forceinline__ double value() const { return static_cast<double>(s); }
};

// One ray ready for the sample loop.  The cell, pair and trilinear loops run in
// FP32 relative to the ray's integer origin (CellFrame); the texture loop runs
// from the rounded absolute base, its 8-bit filter weights being far coarser;
// the nearest-voxel loop keeps FP64, because a position error there moves a
// sample into the neighbouring voxel.
struct Ray {
    double base[3];  // coordinate of the first sample in the loop's index space
    double step[3];  // one step in voxel units
    int n;           // number of samples (0: the ray misses)
};

// Face test of raycasterprojector_interp.cl:136-148.
__device__ __forceinline__ void check_face(double h0, double h1, double lo0, double lo1, double hi0,
                                           double hi1, double lambda, double& tmin, double& tmax)
{
    const bool inside = (h0 >= lo0) && (h1 >= lo1) && (h0 <= hi0) && (h1 <= hi1);
    if (inside && lambda < tmin)
        tmin = lambda;
    if (inside && lambda > tmax)
        tmax = lambda;
}

// FP64 ray setup for detector coordinate (px, py).  `shift` is added to the
// rebased first-sample position to map it into the loop's index space.
template <Mode M>
__device__ __forceinline__ Ray setup_ray(const ProjectArgs& a, const ViewGeom& g, double px, double py,
                                         int* flags)
{
    Ray r;
    double d0 = g.A[0] * px + g.A[1] * py + g.A[2];
    double d1 = g.A[3] * px + g.A[4] * py + g.A[5];
    double d2 = g.A[6] * px + g.A[7] * py + g.A[8];
    const double nrm = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    d0 = d0 / nrm * (a.increment / a.voxel[0]);
    d1 = d1 / nrm * (a.increment / a.voxel[1]);
    d2 = d2 / nrm * (a.increment / a.voxel[2]);
    const double s0 = g.src[0] / a.voxel[0], s1 = g.src[1] / a.voxel[1], s2 = g.src[2] / a.voxel[2];
    const double k0 = a.corner[0] / a.voxel[0], k1 = a.corner[1] / a.voxel[1],
                 k2 = a.corner[2] / a.voxel[2];
    const double pad = (M == Mode::Nearest) ? 0.0 : 0.5;
    const double c10 = k0 - pad, c11 = k1 - pad, c12 = k2 - pad;
    const double c20 = k0 + a.grid[0] + pad, c21 = k1 + a.grid[1] + pad, c22 = k2 + a.grid[2] + pad;
    const double l10 = (c10 - s0) / d0, l11 = (c11 - s1) / d1, l12 = (c12 - s2) / d2;
    const double l20 = (c20 - s0) / d0, l21 = (c21 - s1) / d1, l22 = (c22 - s2) / d2;
    const double e = 0.01;
    double tmin = DBL_MAX, tmax = 0.0;
    check_face(s1 + l10 * d1, s2 + l10 * d2, c11 - e, c12 - e, c21 + e, c22 + e, l10, tmin, tmax);
    check_face(s0 + l11 * d0, s2 + l11 * d2, c10 - e, c12 - e, c20 + e, c22 + e, l11, tmin, tmax);
    check_face(s0 + l12 * d0, s1 + l12 * d1, c10 - e, c11 - e, c20 + e, c21 + e, l12, tmin, tmax);
    check_face(s1 + l20 * d1, s2 + l20 * d2, c11 - e, c12 - e, c21 + e, c22 + e, l20, tmin, tmax);
    check_face(s0 + l21 * d0, s2 + l21 * d2, c10 - e, c12 - e, c20 + e, c22 + e, l21, tmin, tmax);
    check_face(s0 + l22 * d0, s1 + l22 * d1, c10 - e, c11 - e, c20 + e, c21 + e, l22, tmin, tmax);
    r.n = 0;
    if (tmin == DBL_MAX) {
        r.base[0] = r.base[1] = r.base[2] = 0.0;
        r.step[0] = r.step[1] = r.step[2] = 0.0;
        return r;
    }
    const double t0 = fmax(tmin, 0.0), t1 = fmax(tmax, 0.0);
    // the box diagonal bounds any honest ray; beyond it the inputs are broken
    if (!(t1 - t0 < 1.0e7) || !isfinite(t0)) {
        if (flags)
            atomicOr(flags, kFlagNonFinite);
        r.n = 0;
        r.base[0] = r.base[1] = r.base[2] = 0.0;
        r.step[0] = r.step[1] = r.step[2] = 0.0;
        return r;
    }
    if (M == Mode::Cells || M == Mode::Pairs) {
        // Only samples inside the box contribute (the reference's first and last
        // samples, floor(tmin) and floor(tmax)+1, lie outside it and read zeros),
        // so the loop runs over ceil(t0) .. floor(t1).  Coordinates are
        // v = p - 1 + pad: the cell index is rint(v), the offset from the
        // cell centre v - rint(v).
        const double i0 = ceil(t0), i1 = floor(t1);
        r.n = i1 >= i0 ? static_cast<int>(i1 - i0) + 1 : 0;
        r.base[0] = (s0 - k0) + i0 * d0 + (kPad - 1.0);
        r.base[1] = (s1 - k1) + i0 * d1 + (kPad - 1.0);
        r.base[2] = (s2 - k2) + i0 * d2 + (kPad - 1.0);
        r.step[0] = d0;
        r.step[1] = d1;
        r.step[2] = d2;
        return r;
    }
    const double i0 = floor(t0), i1 = floor(t1) + 1.0;
    r.n = static_cast<int>(i1 - i0) + 1;
    // position relative to the corner: (source - corner) + i * step
    double shift;
    if (M == Mode::Trilinear)
        shift = (a.up == 1) ? (kPad - 0.5) : -0.5;  // taps at floor(p - 0.5) (+ pad)
    else if (M == Mode::Nearest)
        shift = kPad;                                // voxel floor(p) (+ pad)
    else
        shift = 0.0;                                 // texture: hardware subtracts 0.5
    r.base[0] = (s0 - k0) + i0 * d0 + shift;
    r.base[1] = (s1 - k1) + i0 * d1 + shift;
    r.base[2] = (s2 - k2) + i0 * d2 + shift;
    r.step[0] = d0;
    r.step[1] = d1;
    r.step[2] = d2;
    return r;
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return min(max(v, lo), hi); }

__device__ __forceinline__ int floor_div(int i, int f) { return i >= 0 ? i / f : -((f - 1 - i) / f); }

// Sample loop, trilinear with zero border, volume stored as T (padded).
// Positions are formed relative to the integer part (ox, oy, oz) of the first
// sample, for the reason given at CellFrame; the offset is folded into the
// ray's base pointer and its clamp bounds, so a sample costs what it did with
// absolute coordinates.
template <typename T, Accum ACC, bool UP>
__device__ __forceinline__ void march_trilinear(const ProjectArgs& a, const Ray& r, Accumulator<ACC>& acc)
{
    const T* __restrict__ vol = static_cast<const T*>(a.vol);
    const int sy = a.sy, sz = a.sz;
    const int mx = a.ext[0] - 2, my = a.ext[1] - 2, mz = a.ext[2] - 2;
    const int ox = (int)rint(r.base[0]), oy = (int)rint(r.base[1]), oz = (int)rint(r.base[2]);
    const float bx = (float)(r.base[0] - ox), by = (float)(r.base[1] - oy), bz = (float)(r.base[2] - oz);
    const float dx = (float)r.step[0], dy = (float)r.step[1], dz = (float)r.step[2];
    // the ray's origin tap; indexes relative to it are clamped so that the
    // absolute tap stays in [0, m] on each axis
    const T* __restrict__ vray = vol + ((ptrdiff_t)ox + (ptrdiff_t)oy * sy + (ptrdiff_t)oz * sz);
    for (int k = 0; k < r.n; ++k) {
        const float kf = static_cast<float>(k);
        const float ux = fmaf(kf, dx, bx);
        const float uy = fmaf(kf, dy, by);
        const float uz = fmaf(kf, dz, bz);
        const float fx = floorf(ux), fy = floorf(uy), fz = floorf(uz);
        const float wx = ux - fx, wy = uy - fy, wz = uz - fz;
        float v000, v100, v010, v110, v001, v101, v011, v111;
        if (!UP) {
            const int ix = clampi(__float2int_rz(fx), -ox, mx - ox);
            const int iy = clampi(__float2int_rz(fy), -oy, my - oy);
            const int iz = clampi(__float2int_rz(fz), -oz, mz - oz);
            const T* p = vray + (ix + iy * sy + iz * sz);
            v000 = load_voxel(p);
            v100 = load_voxel(p + 1);
            v010 = load_voxel(p + sy);
            v110 = load_voxel(p + sy + 1);
            v001 = load_voxel(p + sz);
            v101 = load_voxel(p + sz + 1);
            v011 = load_voxel(p + sz + sy);
            v111 = load_voxel(p + sz + sy + 1);
        } else {
            // virtual replication: grid index g maps to stored voxel floor(g / f)
            const int f = a.up;
            const int gx = __float2int_rz(fmaxf(fminf(fx, 1.0e8f), -1.0e8f)) + ox;
            const int gy = __float2int_rz(fmaxf(fminf(fy, 1.0e8f), -1.0e8f)) + oy;
            const int gz = __float2int_rz(fmaxf(fminf(fz, 1.0e8f), -1.0e8f)) + oz;
            const int x0 = clampi(floor_div(gx, f) + kPad, 0, mx + 1);
            const int x1 = clampi(floor_div(gx + 1, f) + kPad, 0, mx + 1);
            const int y0 = clampi(floor_div(gy, f) + kPad, 0, my + 1) * sy;
            const int y1 = clampi(floor_div(gy + 1, f) + kPad, 0, my + 1) * sy;
            const int z0 = clampi(floor_div(gz, f) + kPad, 0, mz + 1) * sz;
            const int z1 = clampi(floor_div(gz + 1, f) + kPad, 0, mz + 1) * sz;
            v000 = load_voxel(vol + (x0 + y0 + z0));
            v100 = load_voxel(vol + (x1 + y0 + z0));
            v010 = load_voxel(vol + (x0 + y1 + z0));
            v110 = load_voxel(vol + (x1 + y1 + z0));
            v001 = load_voxel(vol + (x0 + y0 + z1));
            v101 = load_voxel(vol + (x1 + y0 + z1));
            v011 = load_voxel(vol + (x0 + y1 + z1));
            v111 = load_voxel(vol + (x1 + y1 + z1));
        }
        const float c00 = fmaf(wx, v100 - v000, v000);
        const float c10 = fmaf(wx, v110 - v010, v010);
        const float c01 = fmaf(wx, v101 - v001, v001);
        const float c11 = fmaf(wx, v111 - v011, v011);
        const float c0 = fmaf(wy, c10 - c00, c00);
        const float c1 = fmaf(wy, c11 - c01, c01);
        acc.add(fmaf(wz, c1 - c0, c0));
    }
}

// Sample loop, nearest voxel floor(p) with bounds test (zeros outside).
template <typename T, Accum ACC>
__device__ __forceinline__ void march_nearest(const ProjectArgs& a, const Ray& r, Accumulator<ACC>& acc)
{
    const T* __restrict__ vol = static_cast<const T*>(a.vol);
    const int mx = a.ext[0] - 1, my = a.ext[1] - 1, mz = a.ext[2] - 1;
    for (int k = 0; k < r.n; ++k) {
        const double kd = static_cast<double>(k);
        const double px = fmin(fmax(fma(kd, r.step[0], r.base[0]), -1.0), 1.0e9);
        const double py = fmin(fmax(fma(kd, r.step[1], r.base[1]), -1.0), 1.0e9);
        const double pz = fmin(fmax(fma(kd, r.step[2], r.base[2]), -1.0), 1.0e9);
        const int ix = clampi(__double2int_rd(px), 0, mx);
        const int iy = clampi(__double2int_rd(py), 0, my);
        const int iz = clampi(__double2int_rd(pz), 0, mz);
        acc.add(load_voxel(vol + (ix + iy * a.sy + iz * a.sz)));
    }
}

// Per-ray frame of the cell and pair loops.  Each axis of the first-sample
// position is split into an integer I = rint(base) and an FP32 remainder, and
// positions are formed as v' = (base - I) + k step.  Along an axis on which the
// ray moves little (a ray grazing a face of the volume) v' stays near zero,
// where FP32 is fine-grained; an absolute coordinate of a few hundred voxels
// would carry a rounding offset of up to 3e-5 voxel into every sample, and on
// a grazing ray that offset changes the line integral by up to 1e-3.  I is
// folded into the rounding constant m = kMagic + I (exact in FP32, |I| < 2^22),
// so t = v' + m has the bits kMagicBits + I + rint(v') of the absolute cell.
struct CellFrame {
    float2 bxy;  // base - I, x and y
    float bz;
    float2 mxy;  // kMagic + I, x and y
    float mz;
};

__device__ __forceinline__ CellFrame cell_frame(const Ray& r)
{
    CellFrame f;
    const double ix = rint(r.base[0]), iy = rint(r.base[1]), iz = rint(r.base[2]);
    f.bxy = make_float2((float)(r.base[0] - ix), (float)(r.base[1] - iy));
    f.bz = (float)(r.base[2] - iz);
    f.mxy = make_float2(__fadd_rn(kMagic, (float)ix), __fadd_rn(kMagic, (float)iy));
    f.mz = __fadd_rn(kMagic, (float)iz);
    return f;
}

// The coefficients of the cell a ray is in, reloaded only when its cell
// changes (consecutive samples of a ray often share a cell).
struct CellCache {
    uint32_t idx = 0xffffffffu;  // cell whose coefficients c0..c7 hold
    float c0 = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f, c4 = 0.f, c5 = 0.f, c6 = 0.f, c7 = 0.f;
};

// The interpolant of the cached cell at offsets (hx, hy, hz) from its centre,
// loading the cell first if `idx` differs from the cached one: a predicated
// 32-byte load, so the registers keep the cached cell when it does not.
__device__ __forceinline__ float cell_eval(const char* __restrict__ cells, uint32_t idx, float hx, float hy,
                                           float hz, CellCache& cc)
{
    {
        const char* p = cells + (size_t)idx * kCellBytes;
        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %8, %9;\n\t"
                     "@p ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%10];\n\t}"
                     : "+f"(cc.c0), "+f"(cc.c1), "+f"(cc.c2), "+f"(cc.c3), "+f"(cc.c4), "+f"(cc.c5),
                       "+f"(cc.c6), "+f"(cc.c7)
                     : "r"(idx), "r"(cc.idx), "l"(p));
        cc.idx = idx;
    }
    const float2 hx2 = make_float2(hx, hx);
    const float2 ea = __ffma2_rn(hx2, make_float2(cc.c2, cc.c3), make_float2(cc.c0, cc.c1));
    const float2 eb = __ffma2_rn(hx2, make_float2(cc.c6, cc.c7), make_float2(cc.c4, cc.c5));
    const float2 g = __ffma2_rn(make_float2(hy, hy), eb, ea);
    return fmaf(hz, g.y, g.x);
}

// Two consecutive samples of a ray (steps k and k + 1, the lanes of kk) from
// the coefficient cells.  Per axis: v' = (base - I) + k step; t = v' + m rounds
// to the cell index (its bits minus kMagicBits, see CellFrame); h = v' - (t - m)
// is the offset from the cell centre in [-1/2, 1/2].  Each packed f32x2
// operation holds one axis of both samples.  A sample that lands exactly
// between two cells may take either of them; both give the same interpolated
// value.  The cell index is clamped to the array as a guard; the loop bounds
// already keep every sample inside it.
__device__ __forceinline__ float2 cell_sample_pair(const char* __restrict__ cells, float2 kk, const CellFrame& fr,
                                                   float2 dx2, float2 dy2, float2 dz2, uint32_t sy, uint32_t sz,
                                                   uint32_t cmax, CellCache& cc)
{
    const float2 none2 = make_float2(-1.0f, -1.0f);
    const float2 mx2 = make_float2(fr.mxy.x, fr.mxy.x), my2 = make_float2(fr.mxy.y, fr.mxy.y);
    const float2 mz2 = make_float2(fr.mz, fr.mz);
    const float2 vx = __ffma2_rn(kk, dx2, make_float2(fr.bxy.x, fr.bxy.x));
    const float2 vy = __ffma2_rn(kk, dy2, make_float2(fr.bxy.y, fr.bxy.y));
    const float2 vz = __ffma2_rn(kk, dz2, make_float2(fr.bz, fr.bz));
    const float2 tx = __fadd2_rn(vx, mx2), ty = __fadd2_rn(vy, my2), tz = __fadd2_rn(vz, mz2);
    const float2 hx = __ffma2_rn(__ffma2_rn(mx2, none2, tx), none2, vx);  // v - (t - m)
    const float2 hy = __ffma2_rn(__ffma2_rn(my2, none2, ty), none2, vy);
    const float2 hz = __ffma2_rn(__ffma2_rn(mz2, none2, tz), none2, vz);
    const uint32_t i0 = min(cell_linear(__float_as_uint(tx.x), __float_as_uint(ty.x), __float_as_uint(tz.x), sy, sz),
                            cmax);
    const uint32_t i1 = min(cell_linear(__float_as_uint(tx.y), __float_as_uint(ty.y), __float_as_uint(tz.y), sy, sz),
                            cmax);
    const float f0 = cell_eval(cells, i0, hx.x, hy.x, hz.x, cc);
    const float f1 = cell_eval(cells, i1, hx.y, hy.y, hz.y, cc);
    return make_float2(f0, f1);
}

// Sample loop over the coefficient cells, U samples per partial sum (FP32)
// handed to the accumulator.
template <Accum ACC, int U>
__device__ __forceinline__ void march_cells(const ProjectArgs& a, const Ray& r, Accumulator<ACC>& acc)
{
    const char* __restrict__ cells = static_cast<const char*>(a.cells);
    const CellFrame fr = cell_frame(r);
    const float2 dx2 = make_float2((float)r.step[0], (float)r.step[0]);
    const float2 dy2 = make_float2((float)r.step[1], (float)r.step[1]);
    const float2 dz2 = make_float2((float)r.step[2], (float)r.step[2]);
    const uint32_t sy = a.csy, sz = a.csz, cmax = a.cmax;
    const float2 two2 = make_float2(2.0f, 2.0f);
    float2 kk = make_float2(0.0f, 1.0f);  // steps k and k + 1
    CellCache cc;
    int k = 0;
    for (; k + U <= r.n; k += U) {
        float part = 0.0f;
#pragma unroll
        for (int j = 0; j < U; j += 2) {
            const float2 f = cell_sample_pair(cells, kk, fr, dx2, dy2, dz2, sy, sz, cmax, cc);
            part += f.x;
            part += f.y;
            kk = __fadd2_rn(kk, two2);
        }
        acc.add(part);
    }
    if (k < r.n) {
        // the last r.n - k < U samples, pairwise; a lone last sample takes the
        // first value of a pair whose second step lies beyond the ray (its cell
        // index is clamped like any other, its value unused)
        for (; k + 1 < r.n; k += 2) {
            const float2 f = cell_sample_pair(cells, kk, fr, dx2, dy2, dz2, sy, sz, cmax, cc);
            acc.add(f.x);
            acc.add(f.y);
            kk = __fadd2_rn(kk, two2);
        }
        if (k < r.n)
            acc.add(cell_sample_pair(cells, kk, fr, dx2, dy2, dz2, sy, sz, cmax, cc).x);
    }
}

// x-pair entries of the current cell: rows (y, z), (y+1, z), (y, z+1), (y+1, z+1).
struct PairCache {
    uint32_t idx = 0xffffffffu;
    float m00 = 0.f, d00 = 0.f, m10 = 0.f, d10 = 0.f, m01 = 0.f, d01 = 0.f, m11 = 0.f, d11 = 0.f;
};

// One sample from the x-pair array: the same cell index and centre offsets as
// cell_sample_pair, four 8-byte entries loaded only when the cell changes, x by
// mid + hx diff, then y and z linearly.
__device__ __forceinline__ float pair_sample(const char* __restrict__ pairs, float2 kk, const CellFrame& fr,
                                             float2 dxy, float dz, uint32_t sy, uint32_t sz, uint32_t pmax,
                                             PairCache& pc)
{
    const float2 none2 = make_float2(-1.0f, -1.0f);
    const float2 vxy = __ffma2_rn(kk, dxy, fr.bxy);
    const float vz = fmaf(kk.x, dz, fr.bz);
    const float2 txy = __fadd2_rn(vxy, fr.mxy);
    const float tz = __fadd_rn(vz, fr.mz);
    const float2 fxy = __ffma2_rn(fr.mxy, none2, txy);  // t - m, exact
    const float fz = __fsub_rn(tz, fr.mz);
    const float2 hxy = __ffma2_rn(fxy, none2, vxy);
    const float hz = fmaf(fz, -1.0f, vz);
    uint32_t idx = __float_as_uint(txy.x) + __float_as_uint(txy.y) * sy + __float_as_uint(tz) * sz;
    idx = min(idx, pmax);
    {
        const char* p0 = pairs + (size_t)idx * 8;
        const char* p1 = p0 + (size_t)sy * 8;
        const char* p2 = p0 + (size_t)sz * 8;
        const char* p3 = p2 + (size_t)sy * 8;
        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %8, %9;\n\t"
                     "@p ld.global.nc.v2.f32 {%0, %1}, [%10];\n\t"
                     "@p ld.global.nc.v2.f32 {%2, %3}, [%11];\n\t"
                     "@p ld.global.nc.v2.f32 {%4, %5}, [%12];\n\t"
                     "@p ld.global.nc.v2.f32 {%6, %7}, [%13];\n\t}"
                     : "+f"(pc.m00), "+f"(pc.d00), "+f"(pc.m10), "+f"(pc.d10), "+f"(pc.m01), "+f"(pc.d01),
                       "+f"(pc.m11), "+f"(pc.d11)
                     : "r"(idx), "r"(pc.idx), "l"(p0), "l"(p1), "l"(p2), "l"(p3));
        pc.idx = idx;
    }
    const float hx = hxy.x;
    const float2 lo = make_float2(fmaf(hx, pc.d00, pc.m00), fmaf(hx, pc.d01, pc.m01));  // (y, z), (y, z+1)
    const float2 hi = make_float2(fmaf(hx, pc.d10, pc.m10), fmaf(hx, pc.d11, pc.m11));  // (y+1, z), (y+1, z+1)
    const float wy = hxy.y + 0.5f, wz = hz + 0.5f;
    const float2 e = __ffma2_rn(make_float2(wy, wy), __ffma2_rn(lo, none2, hi), lo);     // z, z+1
    return fmaf(wz, e.y - e.x, e.x);
}

// Sample loop over the x-pair array (same structure as march_cells).
template <Accum ACC, int U>
__device__ __forceinline__ void march_pairs(const ProjectArgs& a, const Ray& r, Accumulator<ACC>& acc)
{
    const char* __restrict__ pairs = static_cast<const char*>(a.cells);
    const CellFrame fr = cell_frame(r);
    const float2 dxy = make_float2((float)r.step[0], (float)r.step[1]);
    const float dz = (float)r.step[2];
    const uint32_t sy = a.csy, sz = a.csz, pmax = a.cmax;
    const float2 one2 = make_float2(1.0f, 1.0f);
    float2 kk = make_float2(0.0f, 0.0f);
    PairCache pc;
    int k = 0;
    for (; k + U <= r.n; k += U) {
        float part = 0.0f;
#pragma unroll
        for (int j = 0; j < U; ++j) {
            part += pair_sample(pairs, kk, fr, dxy, dz, sy, sz, pmax, pc);
            kk = __fadd2_rn(kk, one2);
        }
        acc.add(part);
    }
    for (; k < r.n; ++k) {
        acc.add(pair_sample(pairs, kk, fr, dxy, dz, sy, sz, pmax, pc));
        kk = __fadd2_rn(kk, one2);
    }
}

// Sample loop, hardware texture filter (border colour 0, unnormalised coords).
template <Accum ACC>
__device__ __forceinline__ void march_texture(const ProjectArgs& a, const Ray& r, Accumulator<ACC>& acc)
{
    const float bx = (float)r.base[0], by = (float)r.base[1], bz = (float)r.base[2];
    const float dx = (float)r.step[0], dy = (float)r.step[1], dz = (float)r.step[2];
    for (int k = 0; k < r.n; ++k) {
        const float kf = static_cast<float>(k);
        acc.add(tex3D<float>(a.tex, fmaf(kf, dx, bx), fmaf(kf, dy, by), fmaf(kf, dz, bz)));
    }
}

// Pixel of thread `tid` of work item (block) `b` of a.block threads, for the
// launch shape in `a` (every factor of the mapping is a power of two).
__device__ __forceinline__ bool pixel_of_item(const ProjectArgs& a, uint32_t b, uint32_t tid, uint32_t& vm,
                                              uint32_t& x, uint32_t& y)
{
    // Block order: chunks of vm_group view groups; within a chunk (module,
    // tile, view group).  Blocks resident at the same time then cover the same
    // tiles of neighbouring views, whose rays cross nearly the same part of
    // the volume.
    const uint32_t G = a.vm_group;
    const uint32_t T = a.tiles_per_vm;
    const uint32_t per_chunk = G * a.n_modules * T;
    const uint32_t c = b / per_chunk;
    const uint32_t first = c * G;
    const uint32_t gsize = min(G, a.view_groups - first);
    const uint32_t r = b - c * per_chunk;
    const uint32_t q = r / gsize;
    const uint32_t vg = first + (r - q * gsize);
    const uint32_t m = q / T;
    const uint32_t t = q - m * T;
    const uint32_t lane = tid & 31u, warp = tid >> 5;
    const uint32_t slot = warp >> a.wpv_shift, w = warp & ((1u << a.wpv_shift) - 1u);
    const uint32_t view = (vg << a.vpb_shift) + slot;
    vm = view * a.n_modules + m;
    const uint32_t ty = t / a.tiles_x, tx = t - ty * a.tiles_x;
    const uint32_t ly_shift = 5u - a.lx_shift;
    x = (tx << a.tx_shift) + ((w & ((1u << a.wx_shift) - 1u)) << a.lx_shift) + (lane & ((1u << a.lx_shift) - 1u));
    y = (ty << a.ty_shift) + ((w >> a.wx_shift) << ly_shift) + (lane >> a.lx_shift);
    return view < a.n_views && x < a.channels && y < a.rows;
}

__device__ __forceinline__ bool pixel_of_thread(const ProjectArgs& a, uint32_t tid, uint32_t& vm, uint32_t& x,
                                                uint32_t& y)
{
    return pixel_of_item(a, blockIdx.x, tid, vm, x, y);
}

__device__ __forceinline__ bool pixel_of(const ProjectArgs& a, uint32_t& vm, uint32_t& x, uint32_t& y)
{
    return pixel_of_thread(a, threadIdx.x, vm, x, y);
}

// Writes the warp's pixel values (called by all 32 lanes): each lane holds
// `val` for pixel (vm, x, y), or ok = false for no pixel.  Four consecutive
// lanes are four consecutive channels of one detector row (a warp patch is 4
// or 8 channels wide), so where all four pixels exist and their row segment
// starts on a 16-byte boundary, the quad's first lane gathers the other three
// values and writes the segment as one 16-byte store; otherwise each lane
// stores its own value.
__device__ __forceinline__ void store_patch(const ProjectArgs& a, uint32_t vm, uint32_t x, uint32_t y, float val,
                                            bool ok)
{
    const uint32_t full = 0xffffffffu, lane = threadIdx.x & 31u, lead = lane & ~3u;
    const float v1 = __shfl_down_sync(full, val, 1);
    const float v2 = __shfl_down_sync(full, val, 2);
    const float v3 = __shfl_down_sync(full, val, 3);
    const uint32_t okmask = __ballot_sync(full, ok);
    float* dst = a.out + ((size_t)vm * a.rows + y) * a.channels + x;
    const bool whole = ((okmask >> lead) & 0xfu) == 0xfu && (reinterpret_cast<uintptr_t>(dst) & 15u) == 0;
    // the quad's choice is its first lane's
    const bool vec = __shfl_sync(full, whole ? 1 : 0, lead) != 0;
    if (vec) {
        if (lane == lead)
            *reinterpret_cast<float4*>(dst) = make_float4(val, v1, v2, v3);
    } else if (ok) {
        *dst = val;
    }
}

// The rays of work item `b` for thread `tid`, cell or pair loop (FP32 entries).
// Called by every lane of a warp (the store is warp-cooperative).
template <Mode M, Accum ACC, int U>
__device__ __forceinline__ void cells_item(const ProjectArgs& a, uint32_t b, uint32_t tid)
{
    uint32_t vm, x, y;
    const bool ok = pixel_of_item(a, b, tid, vm, x, y);
    float val = 0.0f;
    if (ok) {
        const ViewGeom& g = a.geom[vm];
        if (g.valid) {
            Accumulator<ACC> acc;
            if (a.rays_x == 1 && a.rays_y == 1) {
                // one ray through the pixel centre (x - 0.5 + 0.5 is x exactly): the
                // pixel and its geometry are dead once the ray is set up, so the
                // sample loop carries only the ray
                const Ray r = setup_ray<M>(a, g, (double)x, (double)y, a.flags);
                if (M == Mode::Pairs)
                    march_pairs<ACC, U>(a, r, acc);
                else
                    march_cells<ACC, U>(a, r, acc);
            } else {
                const double ix = 1.0 / a.rays_x, iy = 1.0 / a.rays_y;
                for (uint32_t rx = 0; rx < a.rays_x; ++rx)
                    for (uint32_t ry = 0; ry < a.rays_y; ++ry) {
                        const double px = (double)x - 0.5 + 0.5 * ix + rx * ix;
                        const double py = (double)y - 0.5 + 0.5 * iy + ry * iy;
                        const Ray r = setup_ray<M>(a, g, px, py, a.flags);
                        if (M == Mode::Pairs)
                            march_pairs<ACC, U>(a, r, acc);
                        else
                            march_cells<ACC, U>(a, r, acc);
                    }
            }
            val = static_cast<float>(a.increment * acc.value() / (double)(a.rays_x * a.rays_y));
        }
    }
    // the pixel again for the store, rather than holding it through the loop
    pixel_of_item(a, b, tid, vm, x, y);
    store_patch(a, vm, x, y, val, ok);
}

// Cell or pair loop over one block of the regular grid.
template <Mode M, Accum ACC, int U>
__global__ void __maxnreg__(CTLCU_CELL_MAXREG) cells_kernel(const ProjectArgs a)
{
    cells_item<M, ACC, U>(a, blockIdx.x, threadIdx.x);
}

// Persistent batch kernel with warp-granular work: every warp takes one warp
// patch (32 rays: patch w of block tile b of a request) at a time from
// `counter` and runs it, with no barrier between the warps of a block.  A warp
// whose rays are short (a tile edge, rays that miss the volume) takes the next
// patch at once instead of waiting for the longest ray of its tile, so the SMs
// stay busy to the end of the batch.  Warp items run in the order of the
// single-request launch's blocks and, within a block tile, its warps: warps that
// run at the same time work on neighbouring patches and views of one volume.
//
// Per warp, the request of its item is found by scanning forward from the
// previous one (a warp's items only grow), and the request's launch arguments
// are copied into the warp's own slot of shared memory only when the request
// changes.

template <Mode M, Accum ACC, int U>
__global__ void __maxnreg__(CTLCU_CELL_MAXREG)
    batch_cells_kernel(const BatchReq* __restrict__ reqs, uint32_t n_reqs, uint32_t total_warp_items,
                       uint32_t wpb_shift, unsigned int* counter)
{
    extern __shared__ __align__(16) unsigned char s_raw[];  // one ProjectArgs per warp
    static_assert(sizeof(ProjectArgs) % 4 == 0, "word copy");
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    ProjectArgs& sa = reinterpret_cast<ProjectArgs*>(s_raw)[warp];
    uint32_t req = 0, loaded = 0xffffffffu;  // the same in every lane of the warp
    for (;;) {
        uint32_t it = 0;
        if (lane == 0)
            it = atomicAdd(counter, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= total_warp_items)
            return;
        const uint32_t item = it >> wpb_shift, w = it & ((1u << wpb_shift) - 1u);
        while (req + 1 < n_reqs && reqs[req + 1].first_item <= item)
            ++req;  // the last request with first_item <= item
        if (req != loaded) {
            __syncwarp();  // every lane is done with the previous request's arguments
            const uint32_t* src = reinterpret_cast<const uint32_t*>(&reqs[req].a);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&sa);
            for (uint32_t i = lane; i < sizeof(ProjectArgs) / 4; i += 32)
                dst[i] = src[i];
            __syncwarp();
            loaded = req;
        }
        cells_item<M, ACC, U>(sa, item - reqs[req].first_item, (w << 5) + lane);
    }
}

// Gather, nearest-voxel and texture loops over one block of the regular grid.
template <typename T, Mode M, Accum ACC, bool UP>
__global__ void __maxnreg__(CTLCU_GATHER_MAXREG) project_kernel(const ProjectArgs a)
{
    static_assert(M == Mode::Trilinear || M == Mode::Nearest || M == Mode::Texture, "cells_kernel runs these");
    uint32_t vm, x, y;
    const bool ok = pixel_of(a, vm, x, y);
    float val = 0.0f;
    if (ok) {
        const ViewGeom& g = a.geom[vm];
        if (g.valid) {
            Accumulator<ACC> acc;
            const double ix = 1.0 / a.rays_x, iy = 1.0 / a.rays_y;
            for (uint32_t rx = 0; rx < a.rays_x; ++rx)
                for (uint32_t ry = 0; ry < a.rays_y; ++ry) {
                    const double px = (double)x - 0.5 + 0.5 * ix + rx * ix;
                    const double py = (double)y - 0.5 + 0.5 * iy + ry * iy;
                    const Ray r = setup_ray<M>(a, g, px, py, a.flags);
                    if (M == Mode::Trilinear)
                        march_trilinear<T, ACC, UP>(a, r, acc);
                    else if (M == Mode::Nearest)
                        march_nearest<T, ACC>(a, r, acc);
                    else
                        march_texture<ACC>(a, r, acc);
                }
            val = static_cast<float>(a.increment * acc.value() / (double)(a.rays_x * a.rays_y));
        }
    }
    store_patch(a, vm, x, y, val, ok);
}

template <Mode M>
__global__ void __launch_bounds__(kMaxBlock) count_kernel(const ProjectArgs a)
{
    uint32_t vm, x, y;
    unsigned long long n = 0;
    if (pixel_of(a, vm, x, y)) {
        const ViewGeom& g = a.geom[vm];
        if (g.valid) {
            const double ix = 1.0 / a.rays_x, iy = 1.0 / a.rays_y;
            for (uint32_t rx = 0; rx < a.rays_x; ++rx)
                for (uint32_t ry = 0; ry < a.rays_y; ++ry) {
                    const double px = (double)x - 0.5 + 0.5 * ix + rx * ix;
                    const double py = (double)y - 0.5 + 0.5 * iy + ry * iy;
                    n += (unsigned long long)setup_ray<M>(a, g, px, py, nullptr).n;
                }
        }
    }
    for (int o = 16; o > 0; o >>= 1)
        n += __shfl_down_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31u) == 0 && n)
        atomicAdd(a.counter, n);
}

// log2 of the warps in a block of 128, 256 or 512 threads.
uint32_t log2_block_warps(uint32_t block) { return block == 128 ? 2u : (block == 256 ? 3u : 4u); }

// The launch's block size must be one the pixel mapping was built for.
bool block_ok(const ProjectArgs& a)
{
    return a.block == 128 || a.block == 256 || a.block == kMaxBlock;
}

template <Mode M, Accum ACC, bool UP>
cudaError_t launch_typed(const ProjectArgs& a, int dtype, dim3 grid, cudaStream_t s)
{
    switch (dtype) {
    case 0: project_kernel<float, M, ACC, UP><<<grid, a.block, 0, s>>>(a); break;
    case 1: project_kernel<__nv_bfloat16, M, ACC, UP><<<grid, a.block, 0, s>>>(a); break;
    case 2: project_kernel<__half, M, ACC, UP><<<grid, a.block, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <Mode M, Accum ACC>
cudaError_t launch_cells(const ProjectArgs& a, dim3 grid, cudaStream_t s)
{
    switch (a.unroll) {
    case 2: cells_kernel<M, ACC, 2><<<grid, a.block, 0, s>>>(a); break;
    case 4: cells_kernel<M, ACC, 4><<<grid, a.block, 0, s>>>(a); break;
    case 8: cells_kernel<M, ACC, 8><<<grid, a.block, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <Accum ACC>
cudaError_t launch_acc(const ProjectArgs& a, Mode mode, int dtype, dim3 grid, cudaStream_t s)
{
    switch (mode) {
    case Mode::Trilinear:
        return a.up != 1 ? launch_typed<Mode::Trilinear, ACC, true>(a, dtype, grid, s)
                         : launch_typed<Mode::Trilinear, ACC, false>(a, dtype, grid, s);
    case Mode::Nearest: return launch_typed<Mode::Nearest, ACC, false>(a, dtype, grid, s);
    case Mode::Texture:
        project_kernel<float, Mode::Texture, ACC, false><<<grid, a.block, 0, s>>>(a);
        return cudaGetLastError();
    case Mode::Cells: return launch_cells<Mode::Cells, ACC>(a, grid, s);
    case Mode::Pairs: return launch_cells<Mode::Pairs, ACC>(a, grid, s);
    }
    return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t launch_project(const ProjectArgs& a, Mode mode, Accum acc, int dtype, cudaStream_t s)
{
    const uint64_t blocks = (uint64_t)a.view_groups * a.n_modules * a.tiles_per_vm;
    if (blocks == 0)
        return cudaSuccess;
    if (blocks > 0x7fffffffull || !block_ok(a))
        return cudaErrorInvalidConfiguration;
    const dim3 grid((unsigned)blocks);
    switch (acc) {
    case Accum::F64: return launch_acc<Accum::F64>(a, mode, dtype, grid, s);
    case Accum::Kahan: return launch_acc<Accum::Kahan>(a, mode, dtype, grid, s);
    case Accum::F32: return launch_acc<Accum::F32>(a, mode, dtype, grid, s);
    }
    return cudaErrorInvalidValue;
}

namespace {
template <Mode M, Accum ACC, int U>
cudaError_t launch_batch_typed(const BatchReq* reqs, uint32_t n_reqs, uint32_t total, uint32_t block,
                               unsigned int* counter, int* blocks, cudaStream_t s)
{
    // warp items: each block tile of `block` rays is block / 32 warp patches
    const uint32_t wpb = block / 32u, wpb_shift = log2_block_warps(block);
    const uint64_t warp_items = (uint64_t)total * wpb;
    // the counter runs past the end by one per warp of the grid: keep it clear of wrapping
    if (warp_items > 0xffffffffull - (1ull << 20))
        return cudaErrorInvalidValue;
    const size_t smem = sizeof(ProjectArgs) * wpb;
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_cells_kernel<M, ACC, U>, (int)block, smem);
    if (e != cudaSuccess)
        return e;
    uint64_t grid = (uint64_t)sms * (uint64_t)(per_sm > 0 ? per_sm : 1);
    if (grid > total)
        grid = total;
    *blocks = (int)grid;
    batch_cells_kernel<M, ACC, U><<<(unsigned)grid, block, smem, s>>>(reqs, n_reqs, (uint32_t)warp_items, wpb_shift,
                                                                      counter);
    return cudaGetLastError();
}

template <Mode M, Accum ACC>
cudaError_t launch_batch_unroll(const BatchReq* reqs, uint32_t n_reqs, uint32_t total, const LaunchShape& sh,
                                unsigned int* counter, int* blocks, cudaStream_t s)
{
    switch (sh.unroll) {
    case 2: return launch_batch_typed<M, ACC, 2>(reqs, n_reqs, total, sh.block, counter, blocks, s);
    case 4: return launch_batch_typed<M, ACC, 4>(reqs, n_reqs, total, sh.block, counter, blocks, s);
    case 8: return launch_batch_typed<M, ACC, 8>(reqs, n_reqs, total, sh.block, counter, blocks, s);
    }
    return cudaErrorInvalidValue;
}

template <Mode M>
cudaError_t launch_batch_mode(const BatchReq* reqs, uint32_t n_reqs, uint32_t total, Accum acc,
                              const LaunchShape& sh, unsigned int* counter, int* blocks, cudaStream_t s)
{
    switch (acc) {
    case Accum::F64: return launch_batch_unroll<M, Accum::F64>(reqs, n_reqs, total, sh, counter, blocks, s);
    case Accum::Kahan: return launch_batch_unroll<M, Accum::Kahan>(reqs, n_reqs, total, sh, counter, blocks, s);
    case Accum::F32: return launch_batch_unroll<M, Accum::F32>(reqs, n_reqs, total, sh, counter, blocks, s);
    }
    return cudaErrorInvalidValue;
}
}  // namespace

cudaError_t launch_batch(const BatchReq* reqs, uint32_t n_reqs, uint32_t total_items, Mode mode, Accum acc,
                         const LaunchShape& shape, unsigned int* counter, int* blocks, cudaStream_t s)
{
    if (total_items == 0 || n_reqs == 0)
        return cudaSuccess;
    if (shape_error(shape))
        return cudaErrorInvalidConfiguration;
    if (mode == Mode::Pairs)
        return launch_batch_mode<Mode::Pairs>(reqs, n_reqs, total_items, acc, shape, counter, blocks, s);
    if (mode == Mode::Cells)
        return launch_batch_mode<Mode::Cells>(reqs, n_reqs, total_items, acc, shape, counter, blocks, s);
    return cudaErrorInvalidValue;
}

cudaError_t launch_count(const ProjectArgs& a, Mode mode, cudaStream_t s)
{
    const uint64_t blocks = (uint64_t)a.view_groups * a.n_modules * a.tiles_per_vm;
    if (blocks == 0)
        return cudaSuccess;
    if (blocks > 0x7fffffffull || !block_ok(a))
        return cudaErrorInvalidConfiguration;
    const dim3 grid((unsigned)blocks);
    if (mode == Mode::Nearest)
        count_kernel<Mode::Nearest><<<grid, a.block, 0, s>>>(a);
    else
        count_kernel<Mode::Trilinear><<<grid, a.block, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace ctlcu

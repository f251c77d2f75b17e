/*
 * OpenCL C 1.2 stand-ins for compiling CTL's projector kernels
 * (modules/src/ocl/cl_src/projectors/raycasterprojector_interp.cl and
 *  raycasterprojector_no_interp.cl) as C++ on the host, so the reference's own
 * kernel code can be run on identical inputs.  Test infrastructure only.
 *
 * Provides: the vector types the kernels use with their swizzles and
 * component-wise operators, the built-ins they call (convert_*, normalize,
 * mad, fmax, select, all, isgreaterequal, islessequal), a work-item model
 * (get_global_id / get_global_size from thread-local state), and image3d_t
 * with read_imagef implementing the OpenCL 1.2 linear filter (section 8.3):
 *     i0 = floor(u - 0.5), a = frac(u - 0.5), 8-tap weighted sum,
 * CLK_ADDRESS_CLAMP with border colour 0 for CL_INTENSITY, in float.
 *
 * Vector literals "(floatN)(a, b, c)" are not valid C++ (comma operator); the
 * build recipe rewrites them to constructor calls "floatN(a, b, c)" on a copy
 * of the kernel source inside oracle/_ref/.  Scalar casts "(float2)x" stay and
 * use the broadcasting constructors below.
 *
 * Relational built-ins return -1 (all bits set) for true in vector form, and
 * select/all test the most significant bit, as the OpenCL spec states.
 */
#ifndef CTLB200_CL_SHIM_HPP
#define CTLB200_CL_SHIM_HPP

#include <cfloat>
#include <cmath>
#include <cstddef>
#include <cstdint>

#undef isgreaterequal
#undef islessequal

typedef unsigned int uint;
typedef int sampler_t;

#define __kernel
#define __constant const
#define __global
#define __local
#define __private
#define __read_only
#define __write_only

enum {
    CLK_NORMALIZED_COORDS_FALSE = 0,
    CLK_ADDRESS_CLAMP = 4,
    CLK_FILTER_LINEAR = 32,
};

namespace clshim {

/* ---- work-item model --------------------------------------------------- */
struct WorkItem {
    size_t id[3];
    size_t size[3];
};
extern thread_local WorkItem wi;

} // namespace clshim

inline size_t get_global_id(uint d) { return clshim::wi.id[d]; }
inline size_t get_global_size(uint d) { return clshim::wi.size[d]; }

/* ---- vector types ------------------------------------------------------- */
template <typename V, typename S, int I, int J>
struct Swz2 {
    S v[4];
    operator V() const { return V(v[I], v[J]); }
};
template <typename V, typename S, int I, int J, int K>
struct Swz3 {
    S v[4];
    operator V() const { return V(v[I], v[J], v[K]); }
};

struct float2 {
    float x, y;
    float2() : x(0), y(0) {}
    float2(float a, float b) : x(a), y(b) {}
    explicit float2(float s) : x(s), y(s) {}
};

struct float3 {
    union {
        struct { float x, y, z; };
        Swz2<float2, float, 1, 2> yz;
        Swz2<float2, float, 0, 2> xz;
        Swz2<float2, float, 0, 1> xy;
        float s[4];
    };
    float3() : x(0), y(0), z(0) { s[3] = 0; }
    float3(float a, float b, float c) : x(a), y(b), z(c) { s[3] = 0; }
    explicit float3(float a) : x(a), y(a), z(a) { s[3] = 0; }
};

struct float4 {
    union {
        struct { float x, y, z, w; };
        Swz3<float3, float, 0, 1, 2> xyz;
    };
    float4() : x(0), y(0), z(0), w(0) {}
    float4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    float4(const float3& p, float d) : x(p.x), y(p.y), z(p.z), w(d) {}
    explicit float4(float a) : x(a), y(a), z(a), w(a) {}
};

struct double3 {
    double x, y, z;
    double3(double a, double b, double c) : x(a), y(b), z(c) {}
};

struct double16 {
    double s0, s1, s2, s3, s4, s5, s6, s7, s8, s9, sa, sb, sc, sd, se, sf;
};

struct int2 {
    int x, y;
    int2() : x(0), y(0) {}
    int2(int a, int b) : x(a), y(b) {}
    explicit int2(int a) : x(a), y(a) {}
};
struct int3 {
    int x, y, z;
    int3() : x(0), y(0), z(0) {}
    int3(int a, int b, int c) : x(a), y(b), z(c) {}
};
struct int4 {
    int x, y, z, w;
    int4(int a, int b, int c, int d) : x(a), y(b), z(c), w(d) {}
    int4(const int2& a, const int2& b) : x(a.x), y(a.y), z(b.x), w(b.y) {}
};
struct uint2 {
    uint x, y;
};
struct uint3 {
    uint x, y, z;
};

/* ---- float2 arithmetic -------------------------------------------------- */
inline float2 operator+(float2 a, float2 b) { return float2(a.x + b.x, a.y + b.y); }
inline float2 operator-(float2 a, float2 b) { return float2(a.x - b.x, a.y - b.y); }
inline float2 operator*(float2 a, float2 b) { return float2(a.x * b.x, a.y * b.y); }
inline float2 operator/(float2 a, float2 b) { return float2(a.x / b.x, a.y / b.y); }
inline float2 operator*(float s, float2 b) { return float2(s * b.x, s * b.y); }
inline float2 operator*(float2 a, float s) { return float2(a.x * s, a.y * s); }

/* ---- float3 arithmetic -------------------------------------------------- */
inline float3 operator+(float3 a, float3 b) { return float3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline float3 operator-(float3 a, float3 b) { return float3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float3 operator*(float3 a, float3 b) { return float3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float3 operator/(float3 a, float3 b) { return float3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline float3 operator*(float s, float3 b) { return float3(s * b.x, s * b.y, s * b.z); }
inline float3& operator/=(float3& a, float3 b) { a = a / b; return a; }
inline float3& operator+=(float3& a, float3 b) { a = a + b; return a; }
inline float3& operator-=(float3& a, float3 b) { a = a - b; return a; }

/* ---- relational / logical (vector results: -1 true, 0 false) ----------- */
inline int2 isgreaterequal(float2 a, float2 b) { return int2(a.x >= b.x ? -1 : 0, a.y >= b.y ? -1 : 0); }
inline int2 islessequal(float2 a, float2 b) { return int2(a.x <= b.x ? -1 : 0, a.y <= b.y ? -1 : 0); }
inline int2 operator&&(int2 a, int2 b) { return int2((a.x && b.x) ? -1 : 0, (a.y && b.y) ? -1 : 0); }
inline int3 operator>=(int3 a, int3 b) { return int3(a.x >= b.x ? -1 : 0, a.y >= b.y ? -1 : 0, a.z >= b.z ? -1 : 0); }
inline int3 operator<(uint3 a, uint3 b) { return int3(a.x < b.x ? -1 : 0, a.y < b.y ? -1 : 0, a.z < b.z ? -1 : 0); }
inline int all(int4 v) { return (v.x < 0) && (v.y < 0) && (v.z < 0) && (v.w < 0); }
inline int all(int3 v) { return (v.x < 0) && (v.y < 0) && (v.z < 0); }
inline float2 select(float2 a, float2 b, int2 c) { return float2(c.x < 0 ? b.x : a.x, c.y < 0 ? b.y : a.y); }

/* ---- math built-ins ----------------------------------------------------- */
inline float2 fmax(float2 a, float2 b) { return float2(std::fmax(a.x, b.x), std::fmax(a.y, b.y)); }
inline float3 mad(float3 a, float3 b, float3 c)
{
    return float3(std::fma(a.x, b.x, c.x), std::fma(a.y, b.y, c.y), std::fma(a.z, b.z, c.z));
}
inline float3 normalize(float3 v)
{
    const float n = std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
    return float3(v.x / n, v.y / n, v.z / n);
}

/* ---- conversions -------------------------------------------------------- */
inline float2 convert_float2(uint2 v) { return float2((float)v.x, (float)v.y); }
inline float3 convert_float3(uint3 v) { return float3((float)v.x, (float)v.y, (float)v.z); }
inline float4 convert_float4(int4 v) { return float4((float)v.x, (float)v.y, (float)v.z, (float)v.w); }
inline int3 convert_int3_rtn(float3 v)
{
    return int3((int)std::floor(v.x), (int)std::floor(v.y), (int)std::floor(v.z));
}
inline uint3 convert_uint3(int3 v) { return uint3{ (uint)v.x, (uint)v.y, (uint)v.z }; }

/* ---- images -------------------------------------------------------------- */
struct image3d_t {
    const float* data; /* CL_INTENSITY / CL_FLOAT, x fastest */
    int w, h, d;
};

inline int4 get_image_dim(const image3d_t& img) { return int4(img.w, img.h, img.d, 0); }

inline float clshim_texel(const image3d_t& img, int i, int j, int k)
{
    if (i < 0 || j < 0 || k < 0 || i >= img.w || j >= img.h || k >= img.d)
        return 0.0f; /* CLK_ADDRESS_CLAMP: border colour */
    return img.data[(size_t)i + (size_t)img.w * ((size_t)j + (size_t)img.h * (size_t)k)];
}

inline float4 read_imagef(const image3d_t& img, sampler_t, float4 coord)
{
    const float u = coord.x - 0.5f, v = coord.y - 0.5f, w = coord.z - 0.5f;
    const float fu = std::floor(u), fv = std::floor(v), fw = std::floor(w);
    const int i0 = (int)fu, j0 = (int)fv, k0 = (int)fw;
    const float a = u - fu, b = v - fv, c = w - fw;
    const float T = (1 - a) * (1 - b) * (1 - c) * clshim_texel(img, i0, j0, k0)
                  + a * (1 - b) * (1 - c) * clshim_texel(img, i0 + 1, j0, k0)
                  + (1 - a) * b * (1 - c) * clshim_texel(img, i0, j0 + 1, k0)
                  + a * b * (1 - c) * clshim_texel(img, i0 + 1, j0 + 1, k0)
                  + (1 - a) * (1 - b) * c * clshim_texel(img, i0, j0, k0 + 1)
                  + a * (1 - b) * c * clshim_texel(img, i0 + 1, j0, k0 + 1)
                  + (1 - a) * b * c * clshim_texel(img, i0, j0 + 1, k0 + 1)
                  + a * b * c * clshim_texel(img, i0 + 1, j0 + 1, k0 + 1);
    return float4(T, T, T, T);
}

#endif

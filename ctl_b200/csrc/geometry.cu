// Projection-matrix generation on the device: CTL's GeometryEncoder for the
// simple systems it ships, one FP64 thread per (view, module).
//
// Reference (modules/src/...):
//   GeometryEncoder::encodeFullGeometry / encodeSingleViewGeometry
//       acquisition/geometryencoder.cpp:67-117; finalSourcePosition :227-231;
//       intrinsicParameterMatrix :262-290
//   ProjectionMatrix::compose / normalize  mat/projectionmatrix.cpp:31-48, :125-131
//   TubularGantry components/tubulargantry.cpp:53-90; CarmGantry components/carmgantry.cpp:34-71
//   gantry composition without displacements components/abstractgantry.h:159-244
//   CylindricalDetector components/cylindricaldetector.cpp:84-140, :270-283;
//   FlatPanelDetector components/flatpaneldetector.cpp:47-50, :84-88
//   trajectory protocols acquisition/trajectories.cpp:30-273
// The reference walks the views on the host, re-preparing the system object
// for each (prepareView) and composing Qt-side matrices; here every view's
// gantry state is a closed-form function of its index, so all
// views x modules matrices come out of one launch.
#include "ctlcu.h"
#include "internal.cuh"

#include <cfloat>

namespace ctlcu {

namespace {

struct M3 {
    double a[9];
};
struct V3 {
    double x, y, z;
};

__host__ __device__ inline M3 rot(double angle, int axis)
{
    const double s = sin(angle), c = cos(angle);
    if (axis == 0)
        return M3{ { 1, 0, 0, 0, c, -s, 0, s, c } };
    if (axis == 1)
        return M3{ { c, 0, s, 0, 1, 0, -s, 0, c } };
    return M3{ { c, -s, 0, s, c, 0, 0, 0, 1 } };
}

__host__ __device__ inline M3 mul(const M3& A, const M3& B)
{
    M3 C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            C.a[3 * i + j] = A.a[3 * i] * B.a[j] + A.a[3 * i + 1] * B.a[3 + j] + A.a[3 * i + 2] * B.a[6 + j];
    return C;
}

__host__ __device__ inline V3 mul(const M3& A, const V3& v)
{
    return V3{ A.a[0] * v.x + A.a[1] * v.y + A.a[2] * v.z, A.a[3] * v.x + A.a[4] * v.y + A.a[5] * v.z,
               A.a[6] * v.x + A.a[7] * v.y + A.a[8] * v.z };
}

__host__ __device__ inline M3 tr(const M3& A)
{
    return M3{ { A.a[0], A.a[3], A.a[6], A.a[1], A.a[4], A.a[7], A.a[2], A.a[5], A.a[8] } };
}

__host__ __device__ inline double det3(const M3& A)
{
    return A.a[0] * (A.a[4] * A.a[8] - A.a[5] * A.a[7]) - A.a[1] * (A.a[3] * A.a[8] - A.a[5] * A.a[6]) +
           A.a[2] * (A.a[3] * A.a[7] - A.a[4] * A.a[6]);
}

constexpr double kPi = 3.14159265358979323846;
constexpr double kPi2 = 1.57079632679489661923;

struct GeoArgs {
    ctlcu_detector_desc det;
    ctlcu_trajectory_desc traj;
    uint32_t n_views;
    double radius;      // cylinder radius (flat: unused)
    double short_span;  // angle span of a short scan (after the fan-angle default)
    uint32_t n_line;    // circle-plus-line: views on the line
    float axial_inc;    // axial scan: the reference's float increment
    const double* shifts;  // n_shifts source displacements (x, y, z) in the source frame, or null
    uint32_t n_shifts;     // >= 1; output [shift][view][module]
};

struct Gantry {
    V3 src;      // source position (world)
    M3 src_rot;  // source frame -> world (active): a source displacement moves along it
    V3 det;      // detector centre (world)
    M3 det_rot;  // world -> detector CT coordinates (passive)
};

// tubulargantry.cpp:53-90
__device__ inline Gantry tubular(double angle, double pitch, const ctlcu_trajectory_desc& t)
{
    const M3 G = mul(rot(t.tilt_rad, 0), rot(angle, 2));
    const M3 S = mul(mul(G, rot(kPi2, 2)), rot(-kPi2, 0));
    Gantry g;
    g.src = mul(G, V3{ t.sid_mm, 0.0, -pitch });
    g.det = mul(G, V3{ -(t.sdd_mm - t.sid_mm), 0.0, -pitch });
    g.src_rot = S;
    g.det_rot = tr(S);
    return g;
}

// carmgantry.cpp:34-71: source at the C-arm location, detector cArmSpan along its z axis
__device__ inline Gantry carm(const V3& pos, const M3& R, double span)
{
    Gantry g;
    g.src = pos;
    const V3 off = mul(R, V3{ 0.0, 0.0, -span });
    g.det = V3{ pos.x - off.x, pos.y - off.y, pos.z - off.z };
    g.src_rot = R;
    g.det_rot = tr(R);
    return g;
}

// The gantry after the protocol's prepare step for view v (trajectories.cpp)
__device__ inline Gantry gantry_state(const GeoArgs& a, uint32_t v)
{
    const ctlcu_trajectory_desc& t = a.traj;
    switch (t.kind) {
    case CTLCU_TRAJ_HELICAL:  // :30-44
        return tubular(v * t.angle_increment_rad + t.start_angle_rad, v * t.pitch_increment_mm + t.start_pitch_mm, t);
    case CTLCU_TRAJ_AXIAL: {  // :251-265 (a float increment, a float product)
        const float p = (float)v * a.axial_inc;
        return tubular((double)p + t.start_angle_rad, t.pitch_mm, t);
    }
    default:
        break;
    }
    const V3 src0{ 0.0, 0.0, -t.source_to_iso_mm };
    const M3 fixed = mul(rot(kPi2 + t.start_angle_rad, 2), rot(-kPi2, 0));  // :80-81
    const uint32_t n = a.n_views;
    if (t.kind == CTLCU_TRAJ_WOBBLE) {  // :66-88
        const double inc = n > 1 ? t.angle_span_rad / double(n - 1) : 0.0;
        const double phase = sin(double(v) / double(n) * 2.0 * kPi * t.wobble_freq);
        const M3 R = mul(mul(rot(v * inc, 2), fixed), rot(phase * t.wobble_angle_rad, 0));
        return carm(mul(R, src0), R, t.carm_span_mm);
    }
    if (t.kind == CTLCU_TRAJ_SHORT_SCAN) {  // :170-196
        const double inc = n > 1 ? a.short_span / double(n - 1) : 0.0;
        const M3 R = mul(rot(v * inc, 2), fixed);
        return carm(mul(R, src0), R, t.carm_span_mm);
    }
    // CTLCU_TRAJ_CIRCLE_PLUS_LINE, :114-153
    const uint32_t n_line = a.n_line, n_circle = n - n_line;
    if (v < n_circle) {
        const double inc = n_circle > 1 ? t.angle_span_rad / double(n_circle - 1) : 0.0;
        const M3 R = mul(rot(v * inc, 2), fixed);
        return carm(mul(R, src0), R, t.carm_span_mm);
    }
    const uint32_t lv = v - n_circle;
    const double linc = n_line > 1 ? t.line_length_mm / double(n_line - 1) : 0.0;
    const M3 R = mul(rot(t.angle_span_rad / 2.0, 2), fixed);
    V3 pos = mul(R, src0);
    pos.z += (lv - n_line / 2.0) * linc;
    return carm(pos, R, t.carm_span_mm);
}

__global__ void encode_kernel(const GeoArgs a, double* __restrict__ pmats)
{
    const uint32_t M = a.det.n_modules;
    const uint64_t per_shift = (uint64_t)a.n_views * M;
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= per_shift * a.n_shifts)
        return;
    const uint32_t sh = (uint32_t)(i / per_shift);
    const uint64_t j = i - (uint64_t)sh * per_shift;
    const uint32_t v = (uint32_t)(j / M), m = (uint32_t)(j - (uint64_t)v * M);
    Gantry g = gantry_state(a, v);
    if (a.shifts) {
        // a source displacement (position only) added to the prepared gantry: the
        // source moves by sourceRotation * shift (abstractgantry.h:159-164,
        // preparesteps.cpp:202-210)
        const V3 d = mul(g.src_rot, V3{ a.shifts[3 * sh], a.shifts[3 * sh + 1], a.shifts[3 * sh + 2] });
        g.src = V3{ g.src.x + d.x, g.src.y + d.y, g.src.z + d.z };
    }

    // module location (cylindricaldetector.cpp:104-140; flat panel: origin, identity)
    V3 p{ 0.0, 0.0, 0.0 };
    M3 Rm{ { 1, 0, 0, 0, 1, 0, 0, 0, 1 } };
    if (!a.det.flat_panel) {
        const double ang = (double(m) - double(M) * 0.5 + 0.5) * a.det.angulation_rad;
        const M3 R = rot(ang, 1);
        p = mul(R, V3{ 0.0, 0.0, a.radius });
        p.z -= a.radius;
        Rm = tr(R);
    }
    // geometryencoder.cpp:100-113
    const V3 q = mul(tr(g.det_rot), p);
    const V3 mod_pos{ g.det.x + q.x, g.det.y + q.y, g.det.z + q.z };
    const M3 tot = mul(Rm, g.det_rot);
    const V3 dev = mul(tot, V3{ mod_pos.x - g.src.x, mod_pos.y - g.src.y, mod_pos.z - g.src.z });
    // intrinsicParameterMatrix (:262-290)
    const double pw = a.det.pixel_mm[0], ph = a.det.pixel_mm[1], skew = a.det.skew;
    const double focal = fabs(dev.z);
    const double fx = focal / pw, fy = focal / ph;
    double dx = dev.x / pw;
    const double dy = dev.y / ph;
    dx += dy * skew / fy;
    const double px = 0.5 * double(a.det.pixels[0] - 1) - dx;
    const double py = 0.5 * double(a.det.pixels[1] - 1) - dy;
    const M3 K{ { fx, skew, px, 0.0, fy, py, 0.0, 0.0, 1.0 } };
    // P = [K R | -K R src], normalised by copysign(|M row 3|, det M) (projectionmatrix.cpp)
    const M3 Mx = mul(K, tot);
    const V3 t4 = mul(Mx, g.src);
    const double nrm = sqrt(Mx.a[6] * Mx.a[6] + Mx.a[7] * Mx.a[7] + Mx.a[8] * Mx.a[8]);
    const double den = copysign(nrm, det3(Mx));
    double* P = pmats + i * 12;
    for (int r = 0; r < 3; ++r) {
        P[4 * r + 0] = Mx.a[3 * r + 0] / den;
        P[4 * r + 1] = Mx.a[3 * r + 1] / den;
        P[4 * r + 2] = Mx.a[3 * r + 2] / den;
        P[4 * r + 3] = -(r == 0 ? t4.x : r == 1 ? t4.y : t4.z) / den;
    }
}

}  // namespace

// Host-side constants of the system (radius, short-scan span, line views,
// axial float increment), then one launch over views x modules.
cudaError_t launch_encode_geometry(const ctlcu_detector_desc& det, const ctlcu_trajectory_desc& traj,
                                   uint32_t n_views, const double* d_shifts, uint32_t n_shifts, double* pmats,
                                   cudaStream_t s)
{
    GeoArgs a = {};
    a.shifts = d_shifts;
    a.n_shifts = d_shifts ? n_shifts : 1u;
    a.det = det;
    a.traj = traj;
    a.n_views = n_views;
    // cylindricaldetector.cpp:84-93, :270-283
    const double width = double(det.pixels[0]) * det.pixel_mm[0];
    const bool flat_cyl = fabs(det.angulation_rad) <= 1e-12;
    a.radius = flat_cyl ? DBL_MAX
                        : (det.module_spacing_mm + width * cos(det.angulation_rad / 2.0)) /
                              sqrt(2.0 * (1.0 - cos(det.angulation_rad)));
    a.short_span = traj.angle_span_rad;
    if (traj.kind == CTLCU_TRAJ_SHORT_SCAN && traj.angle_span_rad < 0.0) {
        // 180 deg + the protocol's fan angle, which it takes as 2 tan (not atan)
        // of half the relevant width over the C-arm span (trajectories.cpp:183-186, :205-230)
        double relevant;
        if (det.flat_panel) {
            relevant = width;
        } else {
            const double fan = double(det.n_modules - 1) * det.angulation_rad + 2.0 * atan(0.5 * width / a.radius);
            relevant = 2.0 * a.radius * sin(fan / 2.0);
        }
        a.short_span = kPi + 2.0 * tan(0.5 * relevant / traj.carm_span_mm);
    }
    a.n_line = (uint32_t)floor(n_views * traj.line_fraction);
    a.axial_inc = n_views > 0 ? (float)(2.0 * kPi / double(n_views)) : 0.0f;
    const uint64_t total = (uint64_t)n_views * det.n_modules * a.n_shifts;
    if (total == 0)
        return cudaSuccess;
    const unsigned threads = 128;
    const uint64_t blocks = (total + threads - 1) / threads;
    if (blocks > 0x7fffffffull)
        return cudaErrorInvalidConfiguration;
    encode_kernel<<<(unsigned)blocks, threads, 0, s>>>(a, pmats);
    return cudaGetLastError();
}

}  // namespace ctlcu

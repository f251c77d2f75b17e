/*
 * Host harness that runs CTL's own projector kernel code on the CPU.
 * TEST INFRASTRUCTURE: builds oracle/_ref/libctlref.so, used by tests/ to pin
 * the FP64 oracle and by bench.py as the timed reference CPU implementation.
 *
 * The kernel bodies are the reference's files
 *   modules/src/ocl/cl_src/projectors/raycasterprojector_interp.cl
 *   modules/src/ocl/cl_src/projectors/raycasterprojector_no_interp.cl
 * included unchanged apart from the mechanical vector-literal rewrite done by
 * oracle/Makefile (see ref_shim/cl_shim.hpp).  The QR decomposition and the
 * source position come from the reference's compiled
 * modules/src/mat/matrix_algorithm.cpp and projectionmatrix.cpp.
 *
 * What this file adds is the host side of RayCasterProjector::project
 * (modules/src/projectors/raycasterprojector.cpp:139-375) without OpenCL:
 * up-sampling (:576-672), step length (:178-179), corner (:552-558),
 * decomposeM (:527-541), determineSource (:544-549), and the NDRange
 * (channels, rows, modules) per view (:340-343) executed by all host threads,
 * one detector row of work-items per task.
 */
#include "cl_shim.hpp"

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "raycast_oracle.h"

namespace clshim {
thread_local WorkItem wi;
}

namespace ref_interp {
#include "interp.cl.inc"
}
namespace ref_nointerp {
#include "no_interp.cl.inc"
}

#include "mat/matrix_algorithm.h"

namespace {

using CTL::mat::Matrix;
using CTL::mat::ProjectionMatrix;

/* raycasterprojector.cpp:527-541 */
double16 decompose_m(const Matrix<3, 3>& M)
{
    auto QR = CTL::mat::QRdecomposition(M);
    auto& Q = QR.Q;
    auto& R = QR.R;
    if (std::signbit(R(0, 0) * R(1, 1) * R(2, 2)))
        R = -R;
    double16 ret = { Q(0, 0), Q(0, 1), Q(0, 2), Q(1, 0), Q(1, 1), Q(1, 2), Q(2, 0), Q(2, 1),
                     Q(2, 2), R(0, 0), R(0, 1), R(0, 2), R(1, 1), R(1, 2), R(2, 2), 0.0 };
    return ret;
}

ProjectionMatrix pmat_from(const double* p)
{
    ProjectionMatrix P;
    for (uint r = 0; r < 3; ++r)
        for (uint c = 0; c < 4; ++c)
            P(r, c) = p[4 * r + c];
    return P;
}

} // namespace

extern "C" int ctlref_view_setup(const double* pmats, unsigned n_views, unsigned n_modules,
                                 double* qr_out, double* src_out)
{
    for (unsigned v = 0; v < n_views; ++v) {
        const double* Pv = pmats + (size_t)v * n_modules * 12;
        const auto src = pmat_from(Pv).sourcePosition();
        for (int k = 0; k < 3; ++k)
            src_out[3 * (size_t)v + k] = src(k);
        for (unsigned m = 0; m < n_modules; ++m) {
            const auto qr = decompose_m(pmat_from(Pv + (size_t)m * 12).M());
            const double* q = &qr.s0;
            for (int k = 0; k < 15; ++k)
                qr_out[((size_t)v * n_modules + m) * 15 + k] = q[k];
        }
    }
    return 0;
}

extern "C" int ctlref_project(const float* volume, const oracle_volume* vd,
                              const oracle_settings* s, const double* pmats, unsigned n_views,
                              unsigned n_modules, unsigned channels, unsigned rows, float* out,
                              int n_threads)
{
    if (!volume || !vd || !s || !pmats || !out || vd->n[0] <= 0 || vd->n[1] <= 0 || vd->n[2] <= 0)
        return 1;
    const bool interpolate = s->interpolate != 0;
    const unsigned f = interpolate ? s->volume_upsampling : 1u; /* :145-151 */

    /* VolumeSpecs::upSampleVolume (:576-672) */
    size_t X = (size_t)vd->n[0], Y = (size_t)vd->n[1], Z = (size_t)vd->n[2];
    size_t dim[3];
    float voxel[3];
    float mean = 0.0f;
    std::vector<float> up;
    const float* data = volume;
    if (f == 0) {
        dim[0] = dim[1] = dim[2] = 1;
        voxel[0] = vd->voxel_mm[0] * X;
        voxel[1] = vd->voxel_mm[1] * Y;
        voxel[2] = vd->voxel_mm[2] * Z;
        for (size_t i = 0; i < X * Y * Z; ++i)
            mean += volume[i];
        mean /= float(X * Y * Z);
        data = &mean;
    } else if (f == 1) {
        dim[0] = X;
        dim[1] = Y;
        dim[2] = Z;
        for (int k = 0; k < 3; ++k)
            voxel[k] = vd->voxel_mm[k];
    } else {
        dim[0] = X * f;
        dim[1] = Y * f;
        dim[2] = Z * f;
        for (int k = 0; k < 3; ++k)
            voxel[k] = vd->voxel_mm[k] / float(f);
        up.assign(dim[0] * dim[1] * dim[2], 0.0f);
        for (size_t z = 0; z < Z; ++z)
            for (size_t y = 0; y < Y; ++y)
                for (size_t x = 0; x < X; ++x) {
                    const float val = volume[x + X * (y + Y * z)];
                    for (size_t iz = 0; iz < f; ++iz)
                        for (size_t iy = 0; iy < f; ++iy)
                            for (size_t ix = 0; ix < f; ++ix)
                                up[x * f + ix + (y * f + iy) * dim[0] + (z * f + iz) * dim[0] * dim[1]] = val;
                }
        data = up.data();
    }

    /* :178-179 */
    const float smallest = std::min(std::min(voxel[0], voxel[1]), voxel[2]);
    const float increment_mm = smallest * s->ray_sampling;
    /* volumeCorner (:552-558) */
    const float3 corner(vd->offset_mm[0] - 0.5f * dim[0] * voxel[0],
                        vd->offset_mm[1] - 0.5f * dim[1] * voxel[1],
                        vd->offset_mm[2] - 0.5f * dim[2] * voxel[2]);
    const float3 voxel3(voxel[0], voxel[1], voxel[2]);
    const uint2 rays = { s->rays_per_pixel[0], s->rays_per_pixel[1] };
    const image3d_t img = { data, (int)dim[0], (int)dim[1], (int)dim[2] };
    const uint3 dim3 = { (uint)dim[0], (uint)dim[1], (uint)dim[2] };

    /* host setup per view (:321-328), then the NDRange (channels, rows, modules)
     * of every view spread over the host threads one detector row at a time,
     * the way an OpenCL CPU device runs work-items on all cores */
    std::vector<double16> QRs((size_t)n_views * n_modules);
    std::vector<float3> srcs(n_views);
    for (unsigned view = 0; view < n_views; ++view) {
        const double* Pv = pmats + (size_t)view * n_modules * 12;
        /* determineSource (:544-549), module 0's matrix (:324-325) */
        const auto src = pmat_from(Pv).sourcePosition();
        srcs[view] = float3((float)src(0), (float)src(1), (float)src(2));
        for (unsigned m = 0; m < n_modules; ++m)
            QRs[(size_t)view * n_modules + m] = decompose_m(pmat_from(Pv + (size_t)m * 12).M());
    }
    const uint64_t n_rows_total = (uint64_t)n_views * n_modules * rows;
    std::atomic<uint64_t> next(0);
    auto task = [&]() {
        clshim::wi.size[0] = channels;
        clshim::wi.size[1] = rows;
        clshim::wi.size[2] = n_modules;
        for (;;) {
            const uint64_t item = next.fetch_add(1);
            if (item >= n_rows_total)
                break;
            const unsigned y = (unsigned)(item % rows);
            const unsigned m = (unsigned)((item / rows) % n_modules);
            const unsigned view = (unsigned)(item / ((uint64_t)rows * n_modules));
            float* proj = out + (size_t)view * n_modules * rows * channels;
            const double16* qr = &QRs[(size_t)view * n_modules];
            for (unsigned x = 0; x < channels; ++x) {
                clshim::wi.id[0] = x;
                clshim::wi.id[1] = y;
                clshim::wi.id[2] = m;
                if (interpolate)
                    ref_interp::ray_caster(increment_mm, &rays, &srcs[view], &corner, &voxel3, qr, proj, img);
                else
                    ref_nointerp::ray_caster(increment_mm, &rays, &srcs[view], &corner, &voxel3, qr, proj,
                                             data, &dim3);
            }
        }
    };
    if (n_threads < 1)
        n_threads = 1;
    std::vector<std::thread> pool;
    for (int t = 1; t < n_threads; ++t)
        pool.emplace_back(task);
    task();
    for (auto& t : pool)
        t.join();
    return 0;
}

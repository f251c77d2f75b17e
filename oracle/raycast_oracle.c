/*
 * FP64 CPU oracle for the cone-beam ray-casting forward projector.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the correctness checker for the CUDA
 * projector in ctl_b200/csrc.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it.  The product path never calls it.
 *
 * It restates, in plain C and in double precision throughout, the sampling
 * scheme of CTL's OpenCL ray caster:
 *
 *   - per view: source position from module 0's projection matrix
 *       (modules/src/projectors/raycasterprojector.cpp:324-325,544-549,
 *        modules/src/mat/projectionmatrix.cpp:264-275)
 *   - per module: Householder QR of M with sign fix
 *       (raycasterprojector.cpp:527-541, modules/src/mat/matrix_algorithm.cpp:14-36,125-172)
 *   - volume corner  offset - dim*voxel/2
 *       (raycasterprojector.cpp:552-558)
 *   - step length  min(voxel size) * raySampling
 *       (raycasterprojector.cpp:178-179)
 *   - volume up-sampling (f=0 one mean voxel, f=1 unchanged, f>=2 replication)
 *       (raycasterprojector.cpp:576-672); no-interpolation forces f=1 (:145-151)
 *   - sub-ray grid  x - 0.5 + 0.5/n + k/n
 *       (modules/src/ocl/cl_src/projectors/raycasterprojector_interp.cl:40-41,52)
 *   - ray direction  normalize(R^-1 Q^T [x,y,1]) * increment / voxel size
 *       (raycasterprojector_interp.cl:53-57,74-86)
 *   - entry/exit parameters by face tests with a 0.01-voxel tolerance, box padded
 *     by half a voxel when interpolating, clamped at 0, miss -> no samples
 *       (raycasterprojector_interp.cl:88-148, raycasterprojector_no_interp.cl:95-154)
 *   - samples at  i*dir + (source - corner),  i = floor(tmin) .. floor(tmax)+1
 *       (raycasterprojector_interp.cl:61-67)
 *   - trilinear read with zero border per the OpenCL 1.2 linear-filter formula
 *       (image3d_t, CLK_ADDRESS_CLAMP, CLK_FILTER_LINEAR; raycasterprojector_interp.cl:13,64;
 *        same arithmetic as RayCasterProjectorCPU::interpolatedRead,
 *        modules/src/projectors/raycasterprojectorcpu.cpp:239-285)
 *     or nearest voxel floor(position) with bounds test
 *       (raycasterprojector_no_interp.cl:63-73)
 *   - output  increment * sum / nRays  at [view][module][row][channel]
 *       (raycasterprojector_interp.cl:70-71, raycasterprojector.cpp:308-313)
 *
 * Differences from the reference, all in the direction of more precision:
 * positions, directions, entry/exit parameters and interpolation weights are
 * FP64 here (FP32 in the OpenCL kernel); the f=0 mean is summed in FP64 (the
 * reference sums in FP32).  Samples outside the padded box contribute exactly
 * zero in both, so the one-sample differences FP32 entry/exit rounding can make
 * at a face do not change the result.
 *
 * Parity of this restatement is pinned against the reference's own kernel
 * source and matrix code compiled for the CPU (oracle/ref_harness.cpp ->
 * oracle/_ref/libctlref.so) and against closed-form known answers.
 */
#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "raycast_oracle.h"

/* ---------------------------------------------------------------------------
 * 3x3 / 3x4 matrix helpers (row major)
 * ------------------------------------------------------------------------- */

/* Determinant by first-row expansion, as modules/src/mat/matrix_algorithm.cpp:102-108. */
static double det3(const double m[9])
{
    return m[0] * (m[4] * m[8] - m[7] * m[5])
         - m[1] * (m[3] * m[8] - m[6] * m[5])
         + m[2] * (m[3] * m[7] - m[6] * m[4]);
}

/* 3x3 matrix made of three columns of the 3x4 matrix P. */
static void cols3(const double P[12], int a, int b, int c, double out[9])
{
    for (int r = 0; r < 3; ++r) {
        out[3 * r + 0] = P[4 * r + a];
        out[3 * r + 1] = P[4 * r + b];
        out[3 * r + 2] = P[4 * r + c];
    }
}

/* Source position C with P*[C;1] = 0 (modules/src/mat/projectionmatrix.cpp:264-275). */
void oracle_source_position(const double P[12], double src[3])
{
    double m[9];
    cols3(P, 0, 1, 2, m);
    const double hom2cart = -det3(m);
    cols3(P, 1, 2, 3, m);
    src[0] = det3(m) / hom2cart;
    cols3(P, 0, 2, 3, m);
    src[1] = -det3(m) / hom2cart;
    cols3(P, 0, 1, 3, m);
    src[2] = det3(m) / hom2cart;
}

/* Qt's qFuzzyIsNull(double): |d| <= 1e-12. */
static int fuzzy_null(double d) { return fabs(d) <= 0.000000000001; }

/*
 * Householder QR of a 3x3 matrix, packed like the reference's cl_double16:
 * qr[0..8] = Q row major, qr[9..14] = R00 R01 R02 R11 R12 R22.
 * Follows matrix_algorithm.cpp:125-172 (qrdcmp) and :14-36 (QRdecomposition),
 * then the sign rule of raycasterprojector.cpp:532-533 (R = -R when
 * R00*R11*R22 has its sign bit set).  Returns 1 if the matrix is close to
 * singular (the reference only warns in that case).
 */
int oracle_decompose_m(const double Min[9], double qr[15])
{
    double a[3][3];
    double c[2], d[3];
    int sing = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            a[i][j] = Min[3 * i + j];

    for (int k = 0; k < 2; ++k) {
        double scale = 0.0;
        for (int i = k; i < 3; ++i)
            if (scale < fabs(a[i][k]))
                scale = fabs(a[i][k]);
        if (fuzzy_null(scale)) {
            sing = 1;
            c[k] = 0.0;
            d[k] = 0.0;
        } else {
            double sum = 0.0;
            for (int i = k; i < 3; ++i)
                a[i][k] /= scale;
            for (int i = k; i < 3; ++i)
                sum += a[i][k] * a[i][k];
            const double sigma = copysign(sqrt(sum), a[k][k]);
            a[k][k] += sigma;
            c[k] = sigma * a[k][k];
            d[k] = -scale * sigma;
            for (int j = k + 1; j < 3; ++j) {
                sum = 0.0;
                for (int i = k; i < 3; ++i)
                    sum += a[i][k] * a[i][j];
                const double tau = sum / c[k];
                for (int i = k; i < 3; ++i)
                    a[i][j] -= tau * a[i][k];
            }
        }
    }
    d[2] = a[2][2];
    if (fuzzy_null(d[2]))
        sing = 1;

    /* R from the diagonal d and the upper triangle of a */
    double R[9] = { d[0], a[0][1], a[0][2],
                    0.0,  d[1],    a[1][2],
                    0.0,  0.0,     d[2] };
    /* Householder vectors: column 0 of a, and (0, a11, a21) */
    double u1[3] = { a[0][0], a[1][0], a[2][0] };
    double u2[3] = { 0.0, a[1][1], a[2][1] };
    double n1 = sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
    double n2 = sqrt(u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2]);
    for (int i = 0; i < 3; ++i) {
        u1[i] /= n1;
        u2[i] /= n2;
    }
    double Q1[9], Q2[9], Q[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            Q1[3 * i + j] = (i == j ? 1.0 : 0.0) - 2.0 * u1[i] * u1[j];
            Q2[3 * i + j] = (i == j ? 1.0 : 0.0) - 2.0 * u2[i] * u2[j];
        }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k)
                s += Q1[3 * i + k] * Q2[3 * k + j];
            Q[3 * i + j] = s;
        }
    if (signbit(R[0] * R[4] * R[8]))
        for (int i = 0; i < 9; ++i)
            R[i] = -R[i];

    for (int i = 0; i < 9; ++i)
        qr[i] = Q[i];
    qr[9] = R[0];
    qr[10] = R[1];
    qr[11] = R[2];
    qr[12] = R[4];
    qr[13] = R[5];
    qr[14] = R[8];
    return sing;
}

/* Direction R^-1 Q^T [x,y,1], normalised (raycasterprojector_interp.cl:74-86). */
static void ray_direction(double x, double y, const double qr[15], double dir[3])
{
    const double t0 = qr[0] * x + qr[3] * y + qr[6];
    const double t1 = qr[1] * x + qr[4] * y + qr[7];
    const double t2 = qr[2] * x + qr[5] * y + qr[8];
    const double dz = t2 / qr[14];
    const double dy = (t1 - dz * qr[13]) / qr[12];
    const double dx = (t0 - dy * qr[10] - dz * qr[11]) / qr[9];
    const double n = sqrt(dx * dx + dy * dy + dz * dz);
    dir[0] = dx / n;
    dir[1] = dy / n;
    dir[2] = dz / n;
}

/*
 * Face test (raycasterprojector_interp.cl:136-148): accept lambda as a new
 * minimum / maximum when the hit lies inside the (relaxed) face rectangle.
 */
static void check_face(double h0, double h1, double lo0, double lo1, double hi0, double hi1,
                       double lambda, double* tmin, double* tmax)
{
    const int inside = (h0 >= lo0) && (h1 >= lo1) && (h0 <= hi0) && (h1 <= hi1);
    if (inside && lambda < *tmin)
        *tmin = lambda;
    if (inside && lambda > *tmax)
        *tmax = lambda;
}

/*
 * Entry/exit parameters in units of steps (raycasterprojector_interp.cl:88-134).
 * Returns 0 for a ray that hits no face (the reference's (FLT_MAX, 0) result).
 */
static int intersections(const double src[3], const double dir[3], const double size[3],
                         const double corner[3], int interpolate, double* t0, double* t1)
{
    const double pad = interpolate ? 0.5 : 0.0;
    double c1[3], c2[3], l1[3], l2[3];
    for (int k = 0; k < 3; ++k) {
        c1[k] = corner[k] - pad;
        c2[k] = corner[k] + size[k] + pad;
        l1[k] = (c1[k] - src[k]) / dir[k];
        l2[k] = (c2[k] - src[k]) / dir[k];
        c1[k] -= 0.01;
        c2[k] += 0.01;
    }
    double tmin = DBL_MAX, tmax = 0.0;
    /* faces around corner1: yz, xz, xy */
    check_face(src[1] + l1[0] * dir[1], src[2] + l1[0] * dir[2], c1[1], c1[2], c2[1], c2[2], l1[0], &tmin, &tmax);
    check_face(src[0] + l1[1] * dir[0], src[2] + l1[1] * dir[2], c1[0], c1[2], c2[0], c2[2], l1[1], &tmin, &tmax);
    check_face(src[0] + l1[2] * dir[0], src[1] + l1[2] * dir[1], c1[0], c1[1], c2[0], c2[1], l1[2], &tmin, &tmax);
    /* faces around corner2 */
    check_face(src[1] + l2[0] * dir[1], src[2] + l2[0] * dir[2], c1[1], c1[2], c2[1], c2[2], l2[0], &tmin, &tmax);
    check_face(src[0] + l2[1] * dir[0], src[2] + l2[1] * dir[2], c1[0], c1[2], c2[0], c2[2], l2[1], &tmin, &tmax);
    check_face(src[0] + l2[2] * dir[0], src[1] + l2[2] * dir[1], c1[0], c1[1], c2[0], c2[1], l2[2], &tmin, &tmax);
    if (tmin == DBL_MAX)
        return 0;
    *t0 = tmin > 0.0 ? tmin : 0.0;
    *t1 = tmax > 0.0 ? tmax : 0.0;
    return 1;
}

/* Volume as the kernel sees it after up-sampling. */
typedef struct {
    const float* data;
    int64_t n[3];
} vol_view;

static double voxel_or_zero(const vol_view* v, int64_t i, int64_t j, int64_t k)
{
    if (i < 0 || j < 0 || k < 0 || i >= v->n[0] || j >= v->n[1] || k >= v->n[2])
        return 0.0;
    return (double)v->data[i + v->n[0] * (j + v->n[1] * k)];
}

/* OpenCL 1.2 linear filter, unnormalised coordinates, zero border, in FP64. */
static double read_linear(const vol_view* v, const double p[3])
{
    const double u = p[0] - 0.5, w = p[1] - 0.5, s = p[2] - 0.5;
    const double fu = floor(u), fw = floor(w), fs = floor(s);
    const int64_t i0 = (int64_t)fu, j0 = (int64_t)fw, k0 = (int64_t)fs;
    const double a = u - fu, b = w - fw, c = s - fs;
    return (1 - a) * (1 - b) * (1 - c) * voxel_or_zero(v, i0, j0, k0)
         + a * (1 - b) * (1 - c) * voxel_or_zero(v, i0 + 1, j0, k0)
         + (1 - a) * b * (1 - c) * voxel_or_zero(v, i0, j0 + 1, k0)
         + a * b * (1 - c) * voxel_or_zero(v, i0 + 1, j0 + 1, k0)
         + (1 - a) * (1 - b) * c * voxel_or_zero(v, i0, j0, k0 + 1)
         + a * (1 - b) * c * voxel_or_zero(v, i0 + 1, j0, k0 + 1)
         + (1 - a) * b * c * voxel_or_zero(v, i0, j0 + 1, k0 + 1)
         + a * b * c * voxel_or_zero(v, i0 + 1, j0 + 1, k0 + 1);
}

/* Nearest voxel floor(position) with bounds test (raycasterprojector_no_interp.cl:63-73). */
static double read_nearest(const vol_view* v, const double p[3])
{
    const double f0 = floor(p[0]), f1 = floor(p[1]), f2 = floor(p[2]);
    if (f0 < 0 || f1 < 0 || f2 < 0 || f0 >= (double)v->n[0] || f1 >= (double)v->n[1] || f2 >= (double)v->n[2])
        return 0.0;
    return (double)v->data[(int64_t)f0 + v->n[0] * ((int64_t)f1 + v->n[1] * (int64_t)f2)];
}

typedef struct {
    vol_view vol;
    double voxel[3];   /* voxel size after up-sampling (mm) */
    double corner[3];  /* low corner (mm) */
    double increment;  /* step length (mm) */
    const double* pmats;
    unsigned n_views, n_modules, channels, rows;
    unsigned rays[2];
    int interpolate;
    float* out;
    pthread_mutex_t lock;
    uint64_t samples;
    int status;
} job;

/* Per-(view, module) setup, done once before the parallel sample loops. */
typedef struct {
    double src[3];   /* source / voxel */
    double c2s[3];   /* source - corner, voxel units */
} view_setup_t;

static void project_row(job* J, const view_setup_t* vs, const double* qr, unsigned view, unsigned m,
                        unsigned y, uint64_t* samples)
{
    const unsigned M = J->n_modules, C = J->channels, R = J->rows;
    double corner[3], size[3];
    for (int k = 0; k < 3; ++k) {
        corner[k] = J->corner[k] / J->voxel[k];
        size[k] = (double)J->vol.n[k];
    }
    const double nrays = (double)J->rays[0] * (double)J->rays[1];
    for (unsigned x = 0; x < C; ++x) {
        double acc = 0.0;
        for (unsigned rx = 0; rx < J->rays[0]; ++rx)
            for (unsigned ry = 0; ry < J->rays[1]; ++ry) {
                const double px = (double)x - 0.5 + 0.5 / J->rays[0] + (double)rx / J->rays[0];
                const double py = (double)y - 0.5 + 0.5 / J->rays[1] + (double)ry / J->rays[1];
                double dir[3], t0, t1;
                ray_direction(px, py, qr, dir);
                for (int k = 0; k < 3; ++k)
                    dir[k] *= J->increment / J->voxel[k];
                if (!intersections(vs->src, dir, size, corner, J->interpolate, &t0, &t1))
                    continue;
                const int64_t i0 = (int64_t)floor(t0), i1 = (int64_t)floor(t1) + 1;
                *samples += (uint64_t)(i1 - i0 + 1);
                for (int64_t i = i0; i <= i1; ++i) {
                    const double p[3] = { (double)i * dir[0] + vs->c2s[0],
                                          (double)i * dir[1] + vs->c2s[1],
                                          (double)i * dir[2] + vs->c2s[2] };
                    acc += J->interpolate ? read_linear(&J->vol, p) : read_nearest(&J->vol, p);
                }
            }
        J->out[(((size_t)view * M + m) * R + y) * C + x] = (float)(J->increment * acc / nrays);
    }
}

typedef struct {
    job* J;
    const view_setup_t* vs;  /* [view] */
    const double* qr;        /* [view][module][15] */
    uint64_t next;           /* next (view, module, row) item */
} pool_t;

static void* worker(void* arg)
{
    pool_t* T = (pool_t*)arg;
    job* J = T->J;
    const uint64_t total = (uint64_t)J->n_views * J->n_modules * J->rows;
    uint64_t samples = 0;
    for (;;) {
        const uint64_t item = __atomic_fetch_add(&T->next, 1, __ATOMIC_RELAXED);
        if (item >= total)
            break;
        const unsigned y = (unsigned)(item % J->rows);
        const unsigned m = (unsigned)((item / J->rows) % J->n_modules);
        const unsigned v = (unsigned)(item / ((uint64_t)J->rows * J->n_modules));
        project_row(J, &T->vs[v], T->qr + ((size_t)v * J->n_modules + m) * 15, v, m, y, &samples);
    }
    pthread_mutex_lock(&J->lock);
    J->samples += samples;
    pthread_mutex_unlock(&J->lock);
    return NULL;
}

int oracle_project(const float* volume, const oracle_volume* vd, const oracle_settings* s,
                   const double* pmats, unsigned n_views, unsigned n_modules,
                   unsigned channels, unsigned rows, float* out,
                   unsigned long long* sample_count, int n_threads)
{
    if (!volume || !vd || !s || !pmats || !out)
        return ORACLE_ERR_ARG;
    if (vd->n[0] <= 0 || vd->n[1] <= 0 || vd->n[2] <= 0)
        return ORACLE_ERR_ARG;
    if (s->rays_per_pixel[0] == 0 || s->rays_per_pixel[1] == 0)
        return ORACLE_ERR_ARG;

    job J;
    memset(&J, 0, sizeof J);
    const unsigned f = s->interpolate ? s->volume_upsampling : 1u;
    float* owned = NULL;
    float mean = 0.0f;
    const int64_t X = vd->n[0], Y = vd->n[1], Z = vd->n[2];
    /* up-sampling (raycasterprojector.cpp:576-672) */
    if (f == 0) {
        double sum = 0.0;
        for (int64_t i = 0; i < X * Y * Z; ++i)
            sum += volume[i];
        mean = (float)(sum / (double)(X * Y * Z));
        J.vol.data = &mean;
        J.vol.n[0] = J.vol.n[1] = J.vol.n[2] = 1;
        for (int k = 0; k < 3; ++k)
            J.voxel[k] = (double)(vd->voxel_mm[k] * (float)vd->n[k]);
    } else if (f == 1) {
        J.vol.data = volume;
        for (int k = 0; k < 3; ++k) {
            J.vol.n[k] = vd->n[k];
            J.voxel[k] = vd->voxel_mm[k];
        }
    } else {
        const int64_t nX = X * f, nY = Y * f, nZ = Z * f;
        owned = (float*)malloc((size_t)(nX * nY * nZ) * sizeof(float));
        if (!owned)
            return ORACLE_ERR_ALLOC;
        for (int64_t z = 0; z < nZ; ++z)
            for (int64_t y = 0; y < nY; ++y)
                for (int64_t x = 0; x < nX; ++x)
                    owned[x + nX * (y + nY * z)] = volume[x / f + X * (y / f + Y * (z / f))];
        J.vol.data = owned;
        J.vol.n[0] = nX;
        J.vol.n[1] = nY;
        J.vol.n[2] = nZ;
        for (int k = 0; k < 3; ++k)
            J.voxel[k] = (double)(vd->voxel_mm[k] / (float)f);
    }
    /* corner and step (raycasterprojector.cpp:178-179,552-558) */
    for (int k = 0; k < 3; ++k)
        J.corner[k] = (double)vd->offset_mm[k] - 0.5 * (double)J.vol.n[k] * J.voxel[k];
    double vmin = J.voxel[0];
    if (J.voxel[1] < vmin) vmin = J.voxel[1];
    if (J.voxel[2] < vmin) vmin = J.voxel[2];
    J.increment = vmin * (double)s->ray_sampling;
    J.pmats = pmats;
    J.n_views = n_views;
    J.n_modules = n_modules;
    J.channels = channels;
    J.rows = rows;
    J.rays[0] = s->rays_per_pixel[0];
    J.rays[1] = s->rays_per_pixel[1];
    J.interpolate = s->interpolate;
    J.out = out;
    pthread_mutex_init(&J.lock, NULL);

    /* per-view setup (raycasterprojector.cpp:321-328) */
    view_setup_t* vs = (view_setup_t*)malloc(sizeof(view_setup_t) * (size_t)n_views);
    double* qr = (double*)malloc(sizeof(double) * 15 * (size_t)n_views * n_modules);
    if (!vs || !qr) {
        free(vs);
        free(qr);
        free(owned);
        return ORACLE_ERR_ALLOC;
    }
    for (unsigned v = 0; v < n_views; ++v) {
        const double* Pv = pmats + (size_t)v * n_modules * 12;
        double src_mm[3];
        oracle_source_position(Pv, src_mm);
        for (int k = 0; k < 3; ++k) {
            vs[v].src[k] = src_mm[k] / J.voxel[k];
            vs[v].c2s[k] = vs[v].src[k] - J.corner[k] / J.voxel[k];
        }
        for (unsigned m = 0; m < n_modules; ++m) {
            double Mm[9];
            const double* P = Pv + (size_t)m * 12;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c)
                    Mm[3 * r + c] = P[4 * r + c];
            oracle_decompose_m(Mm, qr + ((size_t)v * n_modules + m) * 15);
        }
    }
    pool_t T = { &J, vs, qr, 0 };
    if (n_threads < 1)
        n_threads = 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)n_threads);
    if (!th) {
        free(vs);
        free(qr);
        free(owned);
        return ORACLE_ERR_ALLOC;
    }
    int started = 0;
    for (int t = 1; t < n_threads; ++t)
        if (pthread_create(&th[t], NULL, worker, &T) == 0)
            ++started;
        else
            break;
    worker(&T);
    for (int t = 1; t <= started; ++t)
        pthread_join(th[t], NULL);
    free(th);
    free(vs);
    free(qr);
    pthread_mutex_destroy(&J.lock);
    free(owned);
    if (sample_count)
        *sample_count = J.samples;
    return ORACLE_OK;
}

/* Per-(view, module) setup as the reference host code computes it. */
int oracle_view_setup(const double* pmats, unsigned n_views, unsigned n_modules,
                      double* qr_out /* V*M*15 */, double* src_out /* V*3 */)
{
    for (unsigned v = 0; v < n_views; ++v) {
        const double* Pv = pmats + (size_t)v * n_modules * 12;
        oracle_source_position(Pv, src_out + 3 * (size_t)v);
        for (unsigned m = 0; m < n_modules; ++m) {
            double Mm[9];
            const double* P = Pv + (size_t)m * 12;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c)
                    Mm[3 * r + c] = P[4 * r + c];
            oracle_decompose_m(Mm, qr_out + ((size_t)v * n_modules + m) * 15);
        }
    }
    return ORACLE_OK;
}

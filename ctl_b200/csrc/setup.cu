// FP64 per-(view, module) ray setup on the device.
//
// Replaces the host loop of RayCasterProjector::project that, per view,
// determines the source position from module 0's matrix and the QR
// decomposition of every module's M (modules/src/projectors/raycasterprojector.cpp:321-328,
// decomposeM :527-541, determineSource :544-549).
//
// QR: Householder reflections H1 (column 0) and H2 (column 1), Q = H1 H2,
// R = H2 H1 M, diag(R)_k = -sign(x_k0) |x_k|.  This is the decomposition of
// mat::QRdecomposition (modules/src/mat/matrix_algorithm.cpp:14-36,125-172);
// as there, R is negated when R00 R11 R22 < 0 so that R^-1 Q^T [x,y,1]
// points from the source towards the detector.  The ray kernel needs only
// A = R^-1 Q^T (= sign(det M) M^-1), so that is what is stored per module;
// the packed QR is written out only for the parity test entry point.
#include "internal.cuh"

namespace ctlcu {

namespace {

__device__ double det3(double a, double b, double c, double d, double e, double f, double g,
                       double h, double i)
{
    return a * (e * i - h * f) - b * (d * i - g * f) + c * (d * h - g * e);
}

// Geometry of one (view, module): P its matrix, P0 the view's module-0 matrix.
// Writes *out; the packed QR to qr (if not null) and the source to src (if not null).
__device__ void view_setup_one(const double* __restrict__ P, const double* __restrict__ P0,
                               ViewGeom* __restrict__ out, double* __restrict__ qr, double* __restrict__ src_out,
                               int* flags)
{
    // source position from module 0: null vector of P by cofactors
    // (projectionmatrix.cpp:264-275)
    const double hom = -det3(P0[0], P0[1], P0[2], P0[4], P0[5], P0[6], P0[8], P0[9], P0[10]);
    double src[3];
    src[0] = det3(P0[1], P0[2], P0[3], P0[5], P0[6], P0[7], P0[9], P0[10], P0[11]) / hom;
    src[1] = -det3(P0[0], P0[2], P0[3], P0[4], P0[6], P0[7], P0[8], P0[10], P0[11]) / hom;
    src[2] = det3(P0[0], P0[1], P0[3], P0[4], P0[5], P0[7], P0[8], P0[9], P0[11]) / hom;

    // Householder QR of M
    double a[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            a[r][c] = P[4 * r + c];
    double Q[3][3] = { { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } };
    bool singular = false;
    for (int k = 0; k < 2; ++k) {
        double nrm2 = 0.0;
        for (int i = k; i < 3; ++i)
            nrm2 += a[i][k] * a[i][k];
        const double nrm = sqrt(nrm2);
        if (!(nrm > 1e-300)) {
            singular = true;
            continue;
        }
        const double alpha = -copysign(nrm, a[k][k]);
        double v[3] = { 0, 0, 0 };
        for (int i = k; i < 3; ++i)
            v[i] = a[i][k];
        v[k] -= alpha;
        double vv = 0.0;
        for (int i = k; i < 3; ++i)
            vv += v[i] * v[i];
        const double beta = 2.0 / vv;
        // a <- H a  (columns k..2)
        for (int j = k; j < 3; ++j) {
            double s = 0.0;
            for (int i = k; i < 3; ++i)
                s += v[i] * a[i][j];
            s *= beta;
            for (int i = k; i < 3; ++i)
                a[i][j] -= s * v[i];
        }
        // Q <- Q H
        for (int i = 0; i < 3; ++i) {
            double s = 0.0;
            for (int j = k; j < 3; ++j)
                s += Q[i][j] * v[j];
            s *= beta;
            for (int j = k; j < 3; ++j)
                Q[i][j] -= s * v[j];
        }
    }
    double R[3][3] = { { a[0][0], a[0][1], a[0][2] }, { 0.0, a[1][1], a[1][2] }, { 0.0, 0.0, a[2][2] } };
    if (signbit(R[0][0] * R[1][1] * R[2][2]))
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                R[i][j] = -R[i][j];
    const double detR = R[0][0] * R[1][1] * R[2][2];
    if (!(fabs(R[2][2]) > 0.0) || !isfinite(detR) || !isfinite(src[0] + src[1] + src[2]))
        singular = true;

    // A = R^-1 Q^T by back substitution, column by column
    double A[3][3];
    for (int c = 0; c < 3; ++c) {
        const double t0 = Q[c][0], t1 = Q[c][1], t2 = Q[c][2];  // column c of Q^T
        const double z = t2 / R[2][2];
        const double y = (t1 - z * R[1][2]) / R[1][1];
        const double x = (t0 - y * R[0][1] - z * R[0][2]) / R[0][0];
        A[0][c] = x;
        A[1][c] = y;
        A[2][c] = z;
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (!isfinite(A[i][j]))
                singular = true;

    ViewGeom g;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            g.A[3 * i + j] = singular ? 0.0 : A[i][j];
    for (int k = 0; k < 3; ++k)
        g.src[k] = singular ? 0.0 : src[k];
    g.valid = singular ? 0 : 1;
    g.pad_ = 0;
    *out = g;
    if (singular && flags)
        atomicOr(flags, kFlagSingular);

    if (qr) {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                qr[3 * i + j] = Q[i][j];
        qr[9] = R[0][0];
        qr[10] = R[0][1];
        qr[11] = R[0][2];
        qr[12] = R[1][1];
        qr[13] = R[1][2];
        qr[14] = R[2][2];
    }
    if (src_out)
        for (int k = 0; k < 3; ++k)
            src_out[k] = src[k];
}

__global__ void setup_kernel(const double* __restrict__ pmats, uint32_t n_views, uint32_t n_modules,
                             ViewGeom* __restrict__ geom, double* __restrict__ qr_out,
                             double* __restrict__ src_out, int* flags)
{
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n_views * n_modules)
        return;
    const uint32_t view = idx / n_modules;
    view_setup_one(pmats + (size_t)idx * 12, pmats + (size_t)view * n_modules * 12, geom + idx,
                   qr_out ? qr_out + (size_t)idx * 15 : nullptr,
                   (src_out && idx == view * n_modules) ? src_out + 3 * (size_t)view : nullptr, flags);
}

// All view-modules of a batch: entry i of requests j covers global indices
// first_vm[j] .. first_vm[j] + n_vm[j] - 1.
__global__ void batch_setup_kernel(const BatchSetup* __restrict__ reqs, uint32_t n_reqs, uint32_t total,
                                   ViewGeom* __restrict__ geom, int* flags)
{
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total)
        return;
    uint32_t lo = 0, hi = n_reqs - 1;  // last request with first_vm <= idx
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) / 2;
        if (reqs[mid].first_vm <= idx)
            lo = mid;
        else
            hi = mid - 1;
    }
    const BatchSetup& q = reqs[lo];
    const uint32_t local = idx - q.first_vm;
    const uint32_t view = local / q.n_modules;
    view_setup_one(q.pmats + (size_t)local * 12, q.pmats + (size_t)view * q.n_modules * 12, geom + idx,
                   nullptr, nullptr, flags);
}

}  // namespace

cudaError_t launch_batch_setup(const BatchSetup* reqs, uint32_t n_reqs, uint32_t total, ViewGeom* geom,
                               int* flags, cudaStream_t s)
{
    if (total == 0)
        return cudaSuccess;
    const uint32_t threads = 128;
    batch_setup_kernel<<<(total + threads - 1) / threads, threads, 0, s>>>(reqs, n_reqs, total, geom, flags);
    return cudaGetLastError();
}

cudaError_t launch_setup(const double* pmats, uint32_t n_views, uint32_t n_modules, ViewGeom* geom,
                         double* qr_out, double* src_out, int* flags, cudaStream_t s)
{
    const uint32_t n = n_views * n_modules;
    if (n == 0)
        return cudaSuccess;
    const uint32_t threads = 128;
    setup_kernel<<<(n + threads - 1) / threads, threads, 0, s>>>(pmats, n_views, n_modules, geom,
                                                                 qr_out, src_out, flags);
    return cudaGetLastError();
}

}  // namespace ctlcu

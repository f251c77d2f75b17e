// Post-projection operations on the device: extinction <-> intensity, Poisson
// (quantum) noise, detector saturation, and the per-pixel combines of the
// projector extensions (focal-spot average, linear dynamic volumes, spectral
// effects with and without nested noise).
//
// Reference (modules/src/...):
//   SingleViewData::transformToExtinction / transformToCounts (img/singleviewdata.cpp:135-172):
//     p = log(float(i0) / p),  p = float(i0) * exp(-p); transformToIntensity is
//     transformToCounts (img/projectiondata.cpp), with one i0 per view
//   PoissonNoiseExtension::extendedProject / processViewCompact
//     (projectors/poissonnoiseextension.cpp:35-68, :156-198):
//     count = i0[module] exp(-p); noisy ~ Poisson(count) for count < 1e4, else
//     Normal(count, sqrt(count)); p = log(i0[module] / noisy); views whose i0
//     sum is zero are left as they are.
//
// The reference draws each view's noise from one sequential mt19937_64 stream
// on the host (seed + view).  A sequential stream does not map onto a GPU, so
// every pixel here draws from its own counter-based stream instead:
// Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC 2011), key = the 64-bit seed, counter = (pixel of the
// view, view, draw index, 0).  The variates are exact for the same
// distributions: inversion by sequential search for count < 10, Hormann's
// transformed rejection with squeeze (PTRS; "The transformed rejection method
// for generating Poisson random variables", Insurance: Mathematics and
// Economics 12, 1993) for 10 <= count < 1e4, and Box-Muller above.  The mean
// count is formed in FP64 (the reference: FP32), so it does not depend on the
// last bit of an FP32 exp.
#include "ctlcu.h"
#include "internal.cuh"

namespace ctlcu {

namespace {

struct Philox4 {
    uint32_t x, y, z, w;
};

// Philox4x32 with 10 rounds; multipliers and Weyl key increments of the SC'11 paper
__device__ __forceinline__ Philox4 philox4x32_10(Philox4 c, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
        c = Philox4{ (uint32_t)(p1 >> 32) ^ c.y ^ k0, (uint32_t)p1, (uint32_t)(p0 >> 32) ^ c.w ^ k1, (uint32_t)p0 };
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// A double in (0, 1) from 53 random bits of two words
__device__ __forceinline__ double uniform53(uint32_t a, uint32_t b)
{
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6) + 0.5) * (1.0 / 9007199254740992.0);
}

struct Stream {
    uint32_t pixel, view, draw, k0, k1;
    __device__ __forceinline__ void next(double& u, double& v)
    {
        const Philox4 r = philox4x32_10(Philox4{ pixel, view, draw++, 0u }, k0, k1);
        u = uniform53(r.x, r.y);
        v = uniform53(r.z, r.w);
    }
};

constexpr int kMaxRejections = 64;  // PTRS accepts > 85% of candidates; 64 rejections never occur

// log(k!) for an integer k >= 0: the log of the exact product below 16 (15! < 2^53),
// Stirling's series of log Gamma(x), x = k + 1, above:
//   (x - 1/2) log x - x + log(2 pi)/2 + 1/(12x) - 1/(360x^3) + 1/(1260x^5) - 1/(1680x^7),
// whose next term is below 1e-14 from x = 17 on.  It is cheap and branch-light: the
// PTRS candidates that reach it are a few lanes of most warps.
__device__ __forceinline__ double log_factorial(double k)
{
    if (k < 16.0) {
        double p = 1.0;
        for (int i = 2; i <= (int)k; ++i)
            p *= (double)i;
        return log(p);
    }
    const double x = k + 1.0;
    const double r = 1.0 / x, r2 = r * r;
    const double series = r * (1.0 / 12.0 - r2 * (1.0 / 360.0 - r2 * (1.0 / 1260.0 - r2 * (1.0 / 1680.0))));
    return (x - 0.5) * log(x) - x + 0.91893853320467274178 + series;
}

// Poisson(lam) for 0 <= lam < 1e4, or Normal(lam, sqrt(lam)) for lam >= 1e4,
// as the FP32 count the reference then takes the log of
__device__ float noisy_count(double lam, Stream& s)
{
    double u, v;
    if (!((float)lam < 1.0e4f)) {
        s.next(u, v);
        const double z = sqrt(-2.0 * log(u)) * cos(6.283185307179586 * v);
        return (float)(lam + sqrt(lam) * z);
    }
    if (lam < 10.0) {
        // inversion: the smallest k with F(k) >= u
        s.next(u, v);
        double p = exp(-lam), F = p;
        int k = 0;
        while (u > F && k < 1000) {
            ++k;
            p *= lam / k;
            F += p;
        }
        return (float)k;
    }
    const double slam = sqrt(lam), loglam = log(lam);
    const double b = 0.931 + 2.53 * slam;
    const double a = -0.059 + 0.02483 * b;
    const double inv_alpha = 1.1239 + 1.1328 / (b - 3.4);
    const double vr = 0.9277 - 3.6224 / (b - 2.0);
    const double log_inv_alpha = log(inv_alpha);
    for (int it = 0; it < kMaxRejections; ++it) {
        s.next(u, v);
        const double U = u - 0.5;
        const double us = 0.5 - fabs(U);
        const double k = floor((2.0 * a / us + b) * U + lam + 0.43);
        if (us >= 0.07 && v <= vr)
            return (float)k;
        if (k < 0.0 || (us < 0.013 && v > us))
            continue;
        if (log(v) + log_inv_alpha - log(a / (us * us) + b) <= -lam + k * loglam - log_factorial(k))
            return (float)k;
    }
    return (float)floor(lam + 0.5);  // unreachable in practice (probability < 1e-50)
}

__global__ void poisson_kernel(float* __restrict__ data, uint32_t n_views, uint32_t n_modules, uint32_t ppm,
                               const float* __restrict__ i0, uint32_t k0, uint32_t k1)
{
    const uint64_t per_view = (uint64_t)n_modules * ppm;
    const uint64_t total = per_view * n_views;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t view = (uint32_t)(i / per_view);
        const uint32_t pix = (uint32_t)(i - (uint64_t)view * per_view);
        const float i0m = i0[pix / ppm];
        const double lam = (double)i0m * exp(-(double)data[i]);
        Stream s{ pix, view, 0u, k0, k1 };
        const float noisy = noisy_count(lam, s);
        data[i] = logf(i0m / noisy);
    }
}

__global__ void intensity_kernel(float* __restrict__ data, uint64_t per_view, uint32_t n_views,
                                 const double* __restrict__ i0, int to_extinction)
{
    const uint64_t total = per_view * n_views;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float i0f = i0 ? (float)i0[i / per_view] : 1.0f;
        const float p = data[i];
        data[i] = to_extinction ? logf(i0f / p) : i0f * expf(-p);
    }
}

// ArealFocalSpotExtension::extendedProject (projectors/arealfocalspotextension.cpp:82-160):
// the projections of the focal-spot samples averaged in intensity domain
// (exp(-p) summed in sample order, divided by the count, log(1 / x)), or in
// extinction domain with the low-extinction approximation.  in: [sample][n].
__global__ void average_kernel(const float* __restrict__ in, uint32_t n_samples, uint64_t n, float* __restrict__ out,
                               int low_extinction)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        float acc = 0.0f;
        for (uint32_t s = 0; s < n_samples; ++s) {
            const float p = in[(uint64_t)s * n + i];
            acc += low_extinction ? p : expf(-p);
        }
        acc /= (float)n_samples;
        out[i] = low_extinction ? acc : logf(1.0f / acc);
    }
}

// DynamicProjectorExtension::project over a LinearDynamicVolume
// (projectors/dynamicprojectorextension.cpp:37-60, img/lineardynamicvolume.cpp:194-198):
// the reference sets each view's voxels to slope * float(t_view) + offset and
// projects that view.  The projection is linear in the voxel values, so
// out[view] = float(t_view) * P(slope)[view] + P(offset)[view].
__global__ void combine_kernel(const float* __restrict__ slope, const float* __restrict__ offset,
                               const double* __restrict__ times, uint64_t per_view, uint32_t n_views,
                               float* __restrict__ out)
{
    const uint64_t total = per_view * n_views;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float t = (float)times[i / per_view];
        out[i] = fmaf(t, slope[i], offset[i]);
    }
}

// SpectralEffectsExtension::projectLinear / singleBinIntensityLinear
// (projectors/spectraleffectsextension.cpp:215-278, :333-353), per pixel of view v,
// in FP32 like the reference:
//   sum = sum over bins b with non-zero intensity of
//         float(intensity[b][v]) * exp(-(sum over materials m of proj[m] * mu[b][m])) * response[b]
//   out = log(float(total[v]) / sum)
// proj: [material][n], n = views x values per view; mu: [bin][material] (1/mm);
// intensity: [bin][view]; response: [bin] (1 without a detector response model).
__global__ void spectral_kernel(const float* __restrict__ proj, uint32_t n_materials, uint64_t per_view,
                                uint32_t n_views, const float* __restrict__ mu, const double* __restrict__ intensity,
                                const float* __restrict__ response, const int* __restrict__ skip, uint32_t n_bins,
                                const double* __restrict__ total, float* __restrict__ out)
{
    const uint64_t n = per_view * n_views;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)(i / per_view);
        float sum = 0.0f;
        for (uint32_t b = 0; b < n_bins; ++b) {
            if (skip[b])
                continue;
            float e = 0.0f;
            for (uint32_t m = 0; m < n_materials; ++m)
                e += proj[(uint64_t)m * n + i] * mu[(uint64_t)b * n_materials + m];
            sum += (float)intensity[(uint64_t)b * n_views + v] * expf(-e) * response[b];
        }
        out[i] = logf((float)total[v] / sum);
    }
}

// DetectorSaturationLinearModel::valueAt / DetectorSaturationSplineModel::valueAt
// (models/detectorsaturationmodels.cpp), in the reference's FP32 operation order,
// written with round-to-nearest intrinsics so that no multiply-add is contracted.
__device__ __forceinline__ float saturation_value(float x, const ctlcu_saturation_model& m)
{
    if (m.kind == CTLCU_SATURATION_LINEAR)
        return x < m.a ? m.a : (x > m.b ? m.b : x);
    const float s1s = __fsub_rn(m.a, m.soft_a), s1e = __fadd_rn(m.a, m.soft_a);
    const float s2s = __fsub_rn(m.b, m.soft_b), s2e = __fadd_rn(m.b, m.soft_b);
    if (x < s1s)
        return m.a;
    if (x < s1e) {
        // 1/(4 sa) x^2 - (a - sa)/(2 sa) x + (a + sa)^2/(4 sa)
        const float t1 = __fmul_rn(__fdiv_rn(1.0f, __fmul_rn(4.0f, m.soft_a)), __fmul_rn(x, x));
        const float t2 = __fmul_rn(__fdiv_rn(s1s, __fmul_rn(2.0f, m.soft_a)), x);
        const float t3 = __fdiv_rn(__fmul_rn(s1e, s1e), __fmul_rn(4.0f, m.soft_a));
        return __fadd_rn(__fsub_rn(t1, t2), t3);
    }
    if (x < s2s)
        return x;
    if (x < s2e) {
        // -1/(4 sb) x^2 + (b + sb)/(2 sb) x - (b - sb)^2/(4 sb)
        const float t1 = __fmul_rn(__fdiv_rn(-1.0f, __fmul_rn(4.0f, m.soft_b)), __fmul_rn(x, x));
        const float t2 = __fmul_rn(__fdiv_rn(s2e, __fmul_rn(2.0f, m.soft_b)), x);
        const float t3 = __fdiv_rn(__fmul_rn(s2s, s2s), __fmul_rn(4.0f, m.soft_b));
        return __fsub_rn(__fadd_rn(t1, t2), t3);
    }
    return m.b;
}

// DetectorSaturationExtension::processExtinctions / processCounts / processIntensities
// (projectors/detectorsaturationextension.cpp:96-226); `scale` [view][module] is the
// photon count (or count x mean energy) the extinctions refer to, unused in the
// extinction domain.
__global__ void saturation_kernel(float* __restrict__ data, uint32_t n_views, uint32_t n_modules, uint64_t ppm,
                                  int domain, ctlcu_saturation_model m, const float* __restrict__ scale)
{
    const uint64_t per_view = (uint64_t)n_modules * ppm;
    const uint64_t n = per_view * n_views;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (domain == CTLCU_SATURATION_EXTINCTION) {
            data[i] = saturation_value(data[i], m);
            continue;
        }
        const uint32_t v = (uint32_t)(i / per_view);
        const uint32_t k = (uint32_t)((i - (uint64_t)v * per_view) / ppm);
        const float s = scale[(uint64_t)v * n_modules + k];
        const float x = saturation_value(__fmul_rn(s, expf(-data[i])), m);
        data[i] = logf(__fdiv_rn(s, x));
    }
}

// SpectralEffectsExtension over a nested projector + PoissonNoiseExtension
// (spectraleffectsextension.cpp:285-314, :368-391): per energy bin, every
// material's projection mu[b][m] * proj_m gets its own noise draw with the
// bin's photon count i0[b][module], exactly as poisson_kernel would draw it
// with seed + c, where c counts the (bin, material) projections of the bins not
// skipped in loop order (one nested project() call each).  The noisy
// extinctions of a bin are summed over the materials, and the bins combined in
// the intensity domain as spectral_kernel does.  `quiet[b]`: the bin's i0 sums
// to zero, and the nested noise step leaves its projections as they are
// (poissonnoiseextension.cpp:160).
// Register budget of the (bin, material) noise kernel: sized for 3 resident 256-thread
// blocks per SM (75 registers, no spills).  Unbounded it took 90 registers and 2 blocks,
// and ran 12% slower (286 vs 252 ms at 360 x 512^2, 30 bins, 2 materials); 4 blocks
// (64 registers, a small spill) were no faster than 3.
#ifndef CTLCU_NOISE_MINB
#define CTLCU_NOISE_MINB 3
#endif
__global__ void __launch_bounds__(256, CTLCU_NOISE_MINB)
    spectral_noisy_kernel(const float* __restrict__ proj, uint32_t n_materials, uint32_t n_views,
                                      uint32_t n_modules, uint32_t ppm, const float* __restrict__ mu,
                                      const double* __restrict__ intensity, const float* __restrict__ response,
                                      const int* __restrict__ skip, const int* __restrict__ quiet, uint32_t n_bins,
                                      const double* __restrict__ total, const float* __restrict__ i0, uint64_t seed,
                                      float* __restrict__ out)
{
    const uint64_t per_view = (uint64_t)n_modules * ppm;
    const uint64_t n = per_view * n_views;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)(i / per_view);
        const uint32_t pix = (uint32_t)(i - (uint64_t)v * per_view);
        const uint32_t module = pix / ppm;
        float sum = 0.0f;
        uint64_t call = 0;
        for (uint32_t b = 0; b < n_bins; ++b) {
            if (skip[b])
                continue;
            const float i0m = i0[(uint64_t)b * n_modules + module];
            float e = 0.0f;
            for (uint32_t m = 0; m < n_materials; ++m, ++call) {
                const float em = proj[(uint64_t)m * n + i] * mu[(uint64_t)b * n_materials + m];
                if (quiet[b]) {
                    e += em;
                    continue;
                }
                const uint64_t sc = seed + call;
                const double lam = (double)i0m * exp(-(double)em);
                Stream s{ pix, v, 0u, (uint32_t)sc, (uint32_t)(sc >> 32) };
                e += logf(i0m / noisy_count(lam, s));
            }
            sum += (float)intensity[(uint64_t)b * n_views + v] * expf(-e) * response[b];
        }
        out[i] = logf((float)total[v] / sum);
    }
}

unsigned grid_for_elements(uint64_t n)
{
    uint64_t b = (n + 255) / 256;
    const uint64_t cap = 148ull * 16;  // a few waves; the loops stride over the rest
    return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

cudaError_t launch_poisson_noise(float* data, uint32_t n_views, uint32_t n_modules, uint32_t ppm, const float* i0,
                                 uint64_t seed, cudaStream_t s)
{
    const uint64_t total = (uint64_t)n_views * n_modules * ppm;
    if (total == 0)
        return cudaSuccess;
    poisson_kernel<<<grid_for_elements(total), 256, 0, s>>>(data, n_views, n_modules, ppm, i0, (uint32_t)seed,
                                                             (uint32_t)(seed >> 32));
    return cudaGetLastError();
}

cudaError_t launch_spectral(const float* proj, uint32_t n_materials, uint64_t per_view, uint32_t n_views,
                            const float* mu, const double* intensity, const float* response, const int* skip,
                            uint32_t n_bins, const double* total, float* out, cudaStream_t s)
{
    const uint64_t n = per_view * n_views;
    if (n == 0)
        return cudaSuccess;
    spectral_kernel<<<grid_for_elements(n), 256, 0, s>>>(proj, n_materials, per_view, n_views, mu, intensity, response,
                                                          skip, n_bins, total, out);
    return cudaGetLastError();
}

cudaError_t launch_saturation(float* data, uint32_t n_views, uint32_t n_modules, uint64_t ppm, int domain,
                              const ctlcu_saturation_model& model, const float* scale, cudaStream_t s)
{
    const uint64_t n = (uint64_t)n_modules * ppm * n_views;
    if (n == 0)
        return cudaSuccess;
    saturation_kernel<<<grid_for_elements(n), 256, 0, s>>>(data, n_views, n_modules, ppm, domain, model, scale);
    return cudaGetLastError();
}

cudaError_t launch_spectral_noisy(const float* proj, uint32_t n_materials, uint32_t n_views, uint32_t n_modules,
                                  uint32_t ppm, const float* mu, const double* intensity, const float* response,
                                  const int* skip, const int* quiet, uint32_t n_bins, const double* total,
                                  const float* i0, uint64_t seed, float* out, cudaStream_t s)
{
    const uint64_t n = (uint64_t)n_modules * ppm * n_views;
    if (n == 0)
        return cudaSuccess;
    spectral_noisy_kernel<<<grid_for_elements(n), 256, 0, s>>>(proj, n_materials, n_views, n_modules, ppm, mu,
                                                                intensity, response, skip, quiet, n_bins, total, i0,
                                                                seed, out);
    return cudaGetLastError();
}

cudaError_t launch_combine_linear(const float* slope, const float* offset, const double* d_times, uint64_t per_view,
                                  uint32_t n_views, float* out, cudaStream_t s)
{
    const uint64_t total = per_view * n_views;
    if (total == 0)
        return cudaSuccess;
    combine_kernel<<<grid_for_elements(total), 256, 0, s>>>(slope, offset, d_times, per_view, n_views, out);
    return cudaGetLastError();
}

cudaError_t launch_average_samples(const float* in, uint32_t n_samples, uint64_t n, float* out, bool low_extinction,
                                   cudaStream_t s)
{
    if (n == 0 || n_samples == 0)
        return cudaSuccess;
    average_kernel<<<grid_for_elements(n), 256, 0, s>>>(in, n_samples, n, out, low_extinction ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_transform(float* data, uint64_t per_view, uint32_t n_views, const double* i0, bool to_extinction,
                             cudaStream_t s)
{
    const uint64_t total = per_view * n_views;
    if (total == 0)
        return cudaSuccess;
    intensity_kernel<<<grid_for_elements(total), 256, 0, s>>>(data, per_view, n_views, i0, to_extinction ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace ctlcu

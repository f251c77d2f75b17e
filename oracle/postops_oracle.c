/*
 * Test-only CPU restatement of the device post-operations (ctl_b200/csrc/postops.cu),
 * written independently from the same published algorithms, to check the
 * device kernels draw for draw:
 *
 *   Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 *   easy as 1, 2, 3", SC 2011): key = 64-bit seed, counter = (pixel, view,
 *   draw, 0), two 53-bit uniforms in (0, 1) per block.
 *   Poisson(lam), lam < 10: inversion by sequential search.
 *   Poisson(lam), 10 <= lam < 1e4: PTRS (W. Hormann, "The transformed
 *   rejection method for generating Poisson random variables", Insurance:
 *   Mathematics and Economics 12, 1993).
 *   lam >= 1e4: Normal(lam, sqrt(lam)) by Box-Muller.
 *
 * What the noise is applied to follows PoissonNoiseExtension::processViewCompact
 * (modules/src/projectors/poissonnoiseextension.cpp:156-198): count =
 * i0[module] exp(-p) (here in FP64), p' = log(i0[module] / noisy) in FP32.
 * Nothing in the product links this file.
 */
#include <math.h>
#include <stdint.h>

typedef struct {
    uint32_t v[4];
} philox4;

static philox4 philox4x32_10(philox4 c, uint32_t k0, uint32_t k1)
{
    for (int r = 0; r < 10; ++r) {
        uint64_t a = (uint64_t)0xD2511F53u * c.v[0];
        uint64_t b = (uint64_t)0xCD9E8D57u * c.v[2];
        philox4 n;
        n.v[0] = (uint32_t)(b >> 32) ^ c.v[1] ^ k0;
        n.v[1] = (uint32_t)b;
        n.v[2] = (uint32_t)(a >> 32) ^ c.v[3] ^ k1;
        n.v[3] = (uint32_t)a;
        c = n;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

static double u53(uint32_t a, uint32_t b)
{
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6) + 0.5) / 9007199254740992.0;
}

typedef struct {
    uint32_t pixel, view, draw, k0, k1;
} stream_t;

static void next2(stream_t* s, double* u, double* v)
{
    philox4 c = { { s->pixel, s->view, s->draw++, 0u } };
    philox4 r = philox4x32_10(c, s->k0, s->k1);
    *u = u53(r.v[0], r.v[1]);
    *v = u53(r.v[2], r.v[3]);
}

/* log(k!) as the device computes it: the exact product's log below 16, Stirling's
 * series of log Gamma(k + 1) to the 1/(1680 x^7) term above. */
static double log_factorial(double k)
{
    if (k < 16.0) {
        double p = 1.0;
        for (int i = 2; i <= (int)k; ++i)
            p *= (double)i;
        return log(p);
    }
    double x = k + 1.0;
    double r = 1.0 / x, r2 = r * r;
    double series = r * (1.0 / 12.0 - r2 * (1.0 / 360.0 - r2 * (1.0 / 1260.0 - r2 * (1.0 / 1680.0))));
    return (x - 0.5) * log(x) - x + 0.91893853320467274178 + series;
}

static float noisy(double lam, stream_t* s)
{
    double u, v;
    if (!((float)lam < 1.0e4f)) {
        next2(s, &u, &v);
        return (float)(lam + sqrt(lam) * (sqrt(-2.0 * log(u)) * cos(6.283185307179586 * v)));
    }
    if (lam < 10.0) {
        next2(s, &u, &v);
        double p = exp(-lam), F = p;
        int k = 0;
        while (u > F && k < 1000) {
            ++k;
            p *= lam / k;
            F += p;
        }
        return (float)k;
    }
    double slam = sqrt(lam), loglam = log(lam);
    double b = 0.931 + 2.53 * slam;
    double a = -0.059 + 0.02483 * b;
    double ia = 1.1239 + 1.1328 / (b - 3.4);
    double vr = 0.9277 - 3.6224 / (b - 2.0);
    double lia = log(ia);
    for (int it = 0; it < 64; ++it) {
        next2(s, &u, &v);
        double U = u - 0.5;
        double us = 0.5 - fabs(U);
        double k = floor((2.0 * a / us + b) * U + lam + 0.43);
        if (us >= 0.07 && v <= vr)
            return (float)k;
        if (k < 0.0 || (us < 0.013 && v > us))
            continue;
        if (log(v) + lia - log(a / (us * us) + b) <= -lam + k * loglam - log_factorial(k))
            return (float)k;
    }
    return (float)floor(lam + 0.5);
}

/* In place over [view][module][pixel] extinction data; counts_out (optional)
 * receives the noisy counts. */
void oracle_poisson_noise(float* data, uint32_t n_views, uint32_t n_modules, uint32_t ppm, const float* i0,
                          uint64_t seed, float* counts_out)
{
    uint64_t per_view = (uint64_t)n_modules * ppm;
    for (uint32_t view = 0; view < n_views; ++view)
        for (uint64_t pix = 0; pix < per_view; ++pix) {
            uint64_t i = view * per_view + pix;
            float i0m = i0[pix / ppm];
            double lam = (double)i0m * exp(-(double)data[i]);
            stream_t s = { (uint32_t)pix, view, 0u, (uint32_t)seed, (uint32_t)(seed >> 32) };
            float n = noisy(lam, &s);
            if (counts_out)
                counts_out[i] = n;
            data[i] = logf(i0m / n);
        }
}

/* Draws of the device Poisson sampler for given means (one stream per entry):
 * for the statistical tests. */
void oracle_poisson_draws(const double* lam, uint64_t n, uint64_t seed, uint32_t view, float* out)
{
    for (uint64_t i = 0; i < n; ++i) {
        stream_t s = { (uint32_t)i, view, 0u, (uint32_t)seed, (uint32_t)(seed >> 32) };
        out[i] = noisy(lam[i], &s);
    }
}

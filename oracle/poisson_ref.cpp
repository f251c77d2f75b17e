// Test-only restatement of the reference's noise step, with the reference's own
// random machinery: PoissonNoiseExtension::processViewCompact
// (modules/src/projectors/poissonnoiseextension.cpp:156-198) draws each view's
// counts from one std::mt19937_64 seeded with seed + view
// (:35-68), std::poisson_distribution<unsigned long>(count) below 1e4 counts and
// std::normal_distribution<float>(count, sqrt(count)) above, in pixel order
// over the view's modules.  The distributions are libstdc++'s, as in a GCC
// build of the reference.  The device kernel uses different (counter-based)
// draws, so tests compare the two by distribution, not draw for draw.
// Nothing in the product links this file.
#include <cmath>
#include <cstdint>
#include <random>

extern "C" void ref_poisson_noise(float* data, uint32_t n_views, uint32_t n_modules, uint32_t ppm, const float* i0,
                                  uint32_t seed)
{
    constexpr float gaussianThreshold = 1.0e4f;
    const uint64_t perView = uint64_t(n_modules) * ppm;
    for(uint32_t view = 0; view < n_views; ++view)
    {
        float sum = 0.0f;
        for(uint32_t m = 0; m < n_modules; ++m)
            sum += i0[m];
        if(std::fabs(sum) <= 1e-5f)
            continue;
        std::mt19937_64 gen(seed + view);
        float* pix = data + view * perView;
        for(uint32_t mod = 0; mod < n_modules; ++mod)
            for(uint32_t p = 0; p < ppm; ++p, ++pix)
            {
                const float origCount = i0[mod] * std::exp(-*pix);
                float noisyCount;
                if(origCount < gaussianThreshold)
                {
                    std::poisson_distribution<unsigned long> d(origCount);
                    noisyCount = float(d(gen));
                }
                else
                {
                    std::normal_distribution<float> d(origCount, std::sqrt(origCount));
                    noisyCount = d(gen);
                }
                *pix = std::log(i0[mod] / noisyCount);
            }
    }
}

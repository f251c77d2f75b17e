"""Post-projection operations on the device: extinction <-> intensity and Poisson noise.

Parity has three legs:
  * the device kernels against a CPU restatement of the same algorithms
    (oracle/postops_oracle.c): the same counts draw for draw;
  * the device noise algorithm against the reference's own random machinery
    (oracle/poisson_ref.cpp: per-view std::mt19937_64 with libstdc++'s Poisson
    and normal distributions, as in poissonnoiseextension.cpp:156-198): the
    same distribution, checked with two-sample tests;
  * moments and goodness of fit against the Poisson law itself.
"""
import math

import numpy as np
import pytest

import oracle

SEED = 20240611


# ---- the sampler (CPU restatement of the device algorithm) --------------------------------

@pytest.mark.parametrize("lam", [0.3, 4.0, 9.999, 10.0, 37.5, 512.0, 9999.0])
def test_sampler_moments_and_fit_match_the_poisson_law(lam):
    from scipy import stats
    n = 200_000
    x = oracle.poisson_draws(np.full(n, lam), SEED, view=3).astype(np.float64)
    assert (x == np.round(x)).all() and (x >= 0).all()
    # mean and variance within 5 standard errors
    assert abs(x.mean() - lam) < 5 * math.sqrt(lam / n)
    var_se = math.sqrt((lam + 2 * lam * lam) / n)  # sd of the sample variance of a Poisson(lam)
    assert abs(x.var() - lam) < 5 * var_se
    # chi-square goodness of fit on the central bins (expected count >= 50 each)
    lo, hi = int(stats.poisson.ppf(1e-4, lam)), int(stats.poisson.ppf(1 - 1e-4, lam))
    edges = np.arange(lo, hi + 2) - 0.5
    obs, _ = np.histogram(x, bins=edges)
    exp = n * np.diff(stats.poisson.cdf(edges + 0.5 - 1e-9, lam))
    keep = exp >= 50
    chi2 = (((obs - exp) ** 2) / exp)[keep].sum()
    assert stats.chi2.sf(chi2, keep.sum() - 1) > 1e-4, (lam, chi2, keep.sum())


@pytest.mark.parametrize("lam", [1.0e4, 3.0e5])
def test_sampler_is_normal_above_the_threshold(lam):
    from scipy import stats
    n = 200_000
    x = oracle.poisson_draws(np.full(n, lam), SEED).astype(np.float64)
    z = (x - lam) / math.sqrt(lam)
    assert abs(z.mean()) < 5 / math.sqrt(n) and abs(z.std() - 1.0) < 0.02
    assert stats.kstest(z, "norm").pvalue > 1e-4


def test_sampler_streams_are_independent_of_each_other():
    a = oracle.poisson_draws(np.full(100_000, 20.0), SEED, view=0)
    b = oracle.poisson_draws(np.full(100_000, 20.0), SEED, view=1)
    c = oracle.poisson_draws(np.full(100_000, 20.0), SEED + 1, view=0)
    assert abs(np.corrcoef(a, b)[0, 1]) < 0.02 and abs(np.corrcoef(a, c)[0, 1]) < 0.02
    assert (a != b).mean() > 0.8


def _extinction_field(V=4, M=3, R=64, C=96, seed=1):
    """Extinctions from 0 to ~9 (counts from i0 down to ~1e-4 i0) in smooth ramps."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:R, 0:C]
    base = 9.0 * (x / (C - 1)) * (0.3 + 0.7 * y / (R - 1))
    out = np.empty((V, M, R, C), np.float32)
    for v in range(V):
        for m in range(M):
            out[v, m] = base * (0.8 + 0.4 * rng.random()) + 0.01
    return out


def test_noise_distribution_matches_the_reference_engine():
    """Two-sample comparison against the reference's mt19937_64 + std::
    distributions on the same clean projections: per extinction band, the
    noisy counts of the two have the same mean and variance."""
    p = np.repeat(np.linspace(0.05, 7.0, 60, dtype=np.float32), 4000).reshape(1, 1, 60, 4000)
    i0 = np.array([5.0e3], np.float32)   # counts from 4.8e3 down to 4.6
    ours, _ = oracle.poisson_noise(p, i0, SEED)
    ref = oracle.poisson_noise_reference(p, i0, SEED & 0xffffffff)
    c_ours = i0[0] / np.exp(ours[0, 0].astype(np.float64))
    c_ref = i0[0] / np.exp(ref[0, 0].astype(np.float64))
    lam = i0[0] * np.exp(-p[0, 0, :, 0].astype(np.float64))
    for r in range(60):
        n = 4000
        se_mean = math.sqrt(2 * lam[r] / n)
        assert abs(c_ours[r].mean() - c_ref[r].mean()) < 5 * se_mean, r
        se_var = math.sqrt(2 * (lam[r] + 2 * lam[r] ** 2) / n)
        assert abs(c_ours[r].var() - c_ref[r].var()) < 5 * se_var, r


def test_zero_i0_leaves_the_reference_data_unchanged():
    """The reference skips views whose i0 sums to zero (poissonnoiseextension.cpp:160);
    the device call does the same (test_device_noise_is_a_function_of_the_seed)."""
    p = _extinction_field(V=2, M=2, R=8, C=8)
    ref = oracle.poisson_noise_reference(p, np.zeros(2, np.float32), SEED)
    np.testing.assert_array_equal(ref, p)


# ---- device kernels -----------------------------------------------------------------------

@pytest.fixture(scope="module")
def ctx():
    from ctl_b200.projector import Context
    c = Context(0)
    yield c
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("on_device", [False, True], ids=["host", "device"])
def test_device_noise_matches_the_oracle_draw_for_draw(ctx, on_device):
    import torch
    p = _extinction_field()
    i0 = np.array([2.0e4, 7.5e3, 40.0], np.float32)   # all three sampler branches
    want, counts = oracle.poisson_noise(p, i0, SEED)
    if on_device:
        d = torch.from_numpy(p.copy()).cuda()
        ctx.poisson_noise(d, i0, SEED)
        got = d.cpu().numpy()
    else:
        got = ctx.poisson_noise(p.copy(), i0, SEED)
    got_counts = i0[None, :, None, None] / np.exp(got.astype(np.float64))
    same = np.isclose(got_counts, counts, rtol=1e-5, atol=1e-6) | ((counts == 0) & np.isinf(got))
    assert same.mean() >= 1 - 1e-5, (1 - same.mean())
    finite = np.isfinite(want) & same
    np.testing.assert_allclose(got[finite], want[finite], rtol=1e-6, atol=2e-7)
    # a zero count gives +inf extinction, as log(i0 / 0) does in the reference
    assert (np.isinf(got) == np.isinf(want)).mean() >= 1 - 1e-5


@pytest.mark.gpu
def test_device_noise_is_a_function_of_the_seed(ctx):
    p = _extinction_field(V=2)
    i0 = np.array([1e3, 1e3, 1e3], np.float32)
    a = ctx.poisson_noise(p.copy(), i0, 7)
    b = ctx.poisson_noise(p.copy(), i0, 7)
    c = ctx.poisson_noise(p.copy(), i0, 8)
    np.testing.assert_array_equal(a, b)
    assert (a != c).mean() > 0.5
    z = ctx.poisson_noise(p.copy(), np.zeros(3, np.float32), 7)
    np.testing.assert_array_equal(z, p)


@pytest.mark.gpu
@pytest.mark.parametrize("on_device", [False, True], ids=["host", "device"])
def test_device_transforms_match_the_fp32_formulas(ctx, on_device):
    import torch
    p = _extinction_field(V=5)
    i0 = np.array([1.0, 3.5e4, 0.25, 1e3, 7.0])
    want_int = (i0[:, None, None, None].astype(np.float32) * np.exp(-p)).astype(np.float32)
    data = torch.from_numpy(p.copy()).cuda() if on_device else p.copy()
    ctx.transform_to_intensity(data, i0)
    got = data.cpu().numpy() if on_device else data
    np.testing.assert_allclose(got, want_int, rtol=1e-6)
    ctx.transform_to_extinction(data, i0)
    back = data.cpu().numpy() if on_device else data
    np.testing.assert_allclose(back, p, rtol=1e-5, atol=2e-6)
    one = p.copy()
    ctx.transform_to_intensity(one)          # i0 = 1
    np.testing.assert_allclose(one, np.exp(-p), rtol=1e-6)

"""Parity of the CUDA projector (through the C ABI) with the FP64 oracle and
with the reference's own kernel output.

Tolerance (every case): max over pixels of
    |gpu - oracle| / max(|oracle|, 1e-3 * max|oracle|)  <=  1e-4
for FP32 storage with software trilinear interpolation or nearest voxel;
for BF16/FP16 storage the oracle runs on the dequantised volume.
"""
import numpy as np
import pytest

import oracle
from ctl_b200 import _lib as L
from ctl_b200 import geometry as G
from ctl_b200 import phantom as Ph
from ctl_b200.projector import Context, Settings, VoxelVolume
from tests._common import dequant_bf16, dequant_f16, golden_cases, golden_geometry, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-4


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def _settings(m, **kw):
    s = Settings(rays_per_pixel=list(m["rays"]), ray_sampling=m["ray_sampling"],
                 volume_upsampling=m["upsampling"], interpolate=m["interpolate"])
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def _oracle(m, vol, P):
    out, S = oracle.project_fp64(vol, m["voxel"], P, m["channels"], m["rows"], offset_mm=m["offset"],
                                 rays=m["rays"], ray_sampling=m["ray_sampling"],
                                 upsampling=m["upsampling"], interpolate=m["interpolate"])
    return out, S


@pytest.mark.parametrize("kernel", [L.KERNEL_AUTO, L.KERNEL_GATHER, L.KERNEL_PAIRS], ids=["auto", "gather", "pairs"])
@pytest.mark.parametrize("case", golden_cases(), ids=lambda c: c[0]["name"])
def test_golden_cases_match_oracle_and_reference(ctx, case, kernel):
    m, vol, P, ref = case
    if kernel == L.KERNEL_PAIRS and (not m["interpolate"] or m["upsampling"] != 1):
        pytest.skip("the pair kernel serves software trilinear interpolation without up-sampling")
    gpu = ctx.project_volume(VoxelVolume(vol, m["voxel"], m["offset"]), P, m["channels"], m["rows"],
                             _settings(m, kernel=kernel))
    want, _ = _oracle(m, vol, P)
    e = rel_err(gpu, want)
    assert e.max() <= TOL, f"max rel err vs FP64 oracle {e.max():.3e}"
    # against the reference kernel's own output: the FP32-vs-FP64 gap of the reference
    er = rel_err(gpu, ref)
    if m["upsampling"] == 0 and m["interpolate"]:
        assert er.max() < 3e-4
    elif m["interpolate"]:
        assert er.max() < 5e-4 and er.mean() < 1e-5
    else:
        assert np.quantile(er, 0.999) < 1e-3 and er.mean() < 1e-4


@pytest.mark.parametrize("kernel", [L.KERNEL_CELLS, L.KERNEL_GATHER, L.KERNEL_PAIRS], ids=["cells", "gather", "pairs"])
@pytest.mark.parametrize("accum,tol", [(L.ACCUM_FP64, TOL), (L.ACCUM_KAHAN, TOL), (L.ACCUM_FP32, 2e-3)])
def test_accumulation_modes(ctx, accum, tol, kernel):
    m, vol, P, _ = golden_cases()[0]
    gpu = ctx.project_volume(VoxelVolume(vol, m["voxel"], m["offset"]), P, m["channels"], m["rows"],
                             _settings(m, accum=accum, kernel=kernel))
    want, _ = _oracle(m, vol, P)
    assert rel_err(gpu, want).max() <= tol


@pytest.mark.parametrize("kernel", [L.KERNEL_CELLS, L.KERNEL_GATHER, L.KERNEL_PAIRS], ids=["cells", "gather", "pairs"])
@pytest.mark.parametrize("storage,deq", [(L.BF16, dequant_bf16), (L.F16, dequant_f16)])
def test_reduced_precision_storage_vs_dequantised_oracle(ctx, storage, deq, kernel):
    m, vol, P, _ = golden_cases()[0]
    for accum in (L.ACCUM_FP64, L.ACCUM_KAHAN):
        gpu = ctx.project_volume(VoxelVolume(vol, m["voxel"], m["offset"]), P, m["channels"], m["rows"],
                                 _settings(m, storage=storage, accum=accum, kernel=kernel))
        want, _ = _oracle(m, deq(vol), P)
        assert rel_err(gpu, want).max() <= TOL


def test_texture_filter_is_close_but_coarser(ctx):
    """Hardware filtering uses 8-bit fractional weights: close, not 1e-4."""
    m, vol, P, _ = golden_cases()[0]
    gpu = ctx.project_volume(VoxelVolume(vol, m["voxel"], m["offset"]), P, m["channels"], m["rows"],
                             _settings(m, interp_mode=L.INTERP_TEXTURE))
    want, _ = _oracle(m, vol, P)
    e = rel_err(gpu, want)
    assert e.max() < 2e-2 and e.mean() < 2e-3


def test_view_setup_matches_reference_mat_code(ctx):
    g = golden_geometry()
    for key in ("tube", "carm"):
        qr, src = ctx.view_setup(g[f"{key}_pmats"])
        np.testing.assert_allclose(qr, g[f"{key}_qr"], rtol=0, atol=1e-9 * np.abs(g[f"{key}_qr"]).max())
        np.testing.assert_allclose(src, g[f"{key}_src"], rtol=0, atol=1e-9)


def test_sample_count_matches_oracle(ctx):
    for m, vol, P, _ in golden_cases():
        v = ctx.volume(VoxelVolume(vol, m["voxel"], m["offset"]))
        n = ctx.count_samples(v, P, m["channels"], m["rows"], _settings(m))
        _, S = _oracle(m, vol, P)
        assert abs(n - S) <= max(2, 1e-5 * S), (m["name"], n, S)
        v.release()


def test_resident_device_and_host_paths_agree_bitwise(ctx):
    import torch
    m, vol, P, _ = golden_cases()[5]
    s = _settings(m)
    host = ctx.project_volume(VoxelVolume(vol, m["voxel"], m["offset"]), P, m["channels"], m["rows"], s)
    v = ctx.volume(VoxelVolume(vol, m["voxel"], m["offset"]))
    res = ctx.project(v, P, m["channels"], m["rows"], s)
    dP = torch.from_numpy(np.ascontiguousarray(P)).cuda()
    dev = ctx.project(v, dP, m["channels"], m["rows"], s)
    ctx.sync()
    np.testing.assert_array_equal(host, res)
    np.testing.assert_array_equal(host, dev.cpu().numpy())
    v.release()


@pytest.mark.parametrize("n_views", [1, 7, 8, 9, 63, 64, 65, 90, 181])
def test_host_output_chunks_cover_every_view_once(ctx, n_views):
    """A projection into host memory goes in chunks over two streams (five equal
    chunks and three smaller ones from 64 views up, two below, one below 8); every
    view lands once, with the bits of the device-output call."""
    import torch
    from ctl_b200 import workloads as W
    job = W.c1()
    P = np.ascontiguousarray(np.concatenate([job.pmats, job.pmats, job.pmats])[:n_views])
    v = ctx.volume(VoxelVolume(job.volume, job.voxel))
    dev = ctx.project(v, torch.from_numpy(P).cuda(), job.channels, job.rows, Settings())
    host = np.full((n_views, 1, job.rows, job.channels), np.nan, np.float32)
    ctx.project(v, P, job.channels, job.rows, Settings(), out=host)
    once = ctx.project_volume(VoxelVolume(job.volume, job.voxel), P, job.channels, job.rows, Settings())
    want = dev.cpu().numpy()
    np.testing.assert_array_equal(host, want)
    np.testing.assert_array_equal(once, want)
    v.release()


def test_device_call_is_ordered_on_torchs_current_stream(ctx):
    """Without an explicit stream, a device-tensor call runs on torch's current
    stream (the default stream included), so a torch read-back that follows it
    sees the finished projections without any ctlcu_sync."""
    import torch
    vol = Ph.ellipsoid_phantom((256, 256, 256), (1, 1, 1), 40, seed=2)
    P = _c2_geometry()[:32]
    v = ctx.volume(VoxelVolume(vol, (1, 1, 1)))
    want = ctx.project(v, P, 512, 512, Settings(kernel=L.KERNEL_GATHER))  # host pmats: synchronous
    dP = torch.from_numpy(np.ascontiguousarray(P)).cuda()
    torch.cuda.synchronize()
    for stream in (torch.cuda.default_stream(), torch.cuda.Stream()):
        with torch.cuda.stream(stream):
            got = ctx.project(v, dP, 512, 512, Settings(kernel=L.KERNEL_GATHER)).cpu().numpy()
        np.testing.assert_array_equal(got, want)
    v.release()


def test_batch_equals_individual_calls(ctx):
    import torch
    cases = golden_cases()
    reqs, singles = [], []
    vols = []
    for m, vol, P, _ in (cases[0], cases[5], cases[7]):
        v = ctx.volume(VoxelVolume(vol, m["voxel"], m["offset"]))
        vols.append(v)
        dP = torch.from_numpy(np.ascontiguousarray(P)).cuda()
        out = torch.zeros((P.shape[0], P.shape[1], m["rows"], m["channels"]), device="cuda")
        reqs.append((v, dP, out))
        singles.append(ctx.project(v, P, m["channels"], m["rows"], Settings()))
    ctx.project_batch(reqs, Settings())
    ctx.sync()
    for (v, dP, out), want in zip(reqs, singles):
        np.testing.assert_array_equal(out.cpu().numpy(), want)
    for v in vols:
        v.release()


def test_errors_are_status_codes(ctx):
    m, vol, P, _ = golden_cases()[0]
    with pytest.raises(L.CtlcuError) as e:
        ctx.project(type("V", (), {"handle": 987654})(), P, 8, 8)
    assert e.value.status == L.ERR_INVALID_HANDLE
    with pytest.raises(L.CtlcuError) as e:
        ctx.project_volume(VoxelVolume(vol, m["voxel"]), P, 8, 8, Settings(ray_sampling=0.0))
    assert e.value.status == L.ERR_INVALID_ARGUMENT
    with pytest.raises(L.CtlcuError) as e:
        ctx.project_volume(VoxelVolume(vol, (0.0, 1.0, 1.0)), P, 8, 8)
    assert e.value.status == L.ERR_INVALID_ARGUMENT
    # a singular matrix: status code, its pixels are zero, the others are projected
    Pbad = P[:2].copy()
    Pbad[1, 0, :, :3] = 0.0
    with pytest.raises(L.CtlcuError) as e:
        ctx.project_volume(VoxelVolume(vol, m["voxel"]), Pbad, 16, 16)
    assert e.value.status == L.ERR_SINGULAR_GEOMETRY
    ctx.sync()
    # memory budget: admission refused, nothing leaked
    used = ctx.memory_used()
    ctx.set_memory_budget(used + 1024)
    with pytest.raises(L.CtlcuError) as e:
        ctx.volume(VoxelVolume(vol, m["voxel"]))
    assert e.value.status == L.ERR_OUT_OF_MEMORY
    ctx.set_memory_budget(0)
    assert ctx.memory_used() == used


# ---- full-size configurations, checked with the oracle on a few views -------------------------

def _c2_geometry(n_views=360):
    det = G.FlatDetector(512, 512, 0.6, 0.6)
    fan = G.fan_angle(det, 1200.0)
    return G.circular_flat(n_views, 750.0, 1200.0, det, angle_range=np.pi * 200 / 180 + fan,
                           rng=np.random.default_rng(2024), jitter_mm=0.5, tilt_deg=0.2)


def test_c2_full_size_views_match_oracle(ctx):
    """256^3 -> 512^2: two full views of the short-scan configuration against the oracle."""
    vol = Ph.ellipsoid_phantom((256, 256, 256), (1, 1, 1), 40, seed=2)
    P = _c2_geometry()[[0, 181]]
    v = ctx.volume(VoxelVolume(vol, (1, 1, 1)))
    want, _ = oracle.project_fp64(vol, (1, 1, 1), P, 512, 512)
    for kernel in (L.KERNEL_CELLS, L.KERNEL_GATHER, L.KERNEL_PAIRS):
        for accum in (L.ACCUM_FP64, L.ACCUM_KAHAN):
            gpu = ctx.project(v, P, 512, 512, Settings(accum=accum, kernel=kernel))
            e = rel_err(gpu, want)
            assert e.max() <= TOL, (kernel, accum, e.max())
    v.release()


@pytest.mark.parametrize("storage,deq", [(L.BF16, dequant_bf16), (L.F16, dequant_f16)], ids=["bf16", "f16"])
def test_c2_full_size_16bit_storage_matches_dequantised_oracle(ctx, storage, deq):
    """256^3 -> 512^2 with the volume stored in 16 bits: the cell, pair and
    gather loops against the oracle on the dequantised volume."""
    vol = Ph.ellipsoid_phantom((256, 256, 256), (1, 1, 1), 40, seed=2)
    P = _c2_geometry()[[0, 181]]
    v = ctx.volume(VoxelVolume(vol, (1, 1, 1)), storage)
    want, _ = oracle.project_fp64(deq(vol), (1, 1, 1), P, 512, 512)
    for kernel in (L.KERNEL_CELLS, L.KERNEL_PAIRS, L.KERNEL_GATHER):
        gpu = ctx.project(v, P, 512, 512, Settings(kernel=kernel))
        e = rel_err(gpu, want)
        assert e.max() <= TOL, (kernel, e.max())
    v.release()


def test_batch_mixing_storage_types_matches_single_calls(ctx):
    """One persistent launch over volumes stored as FP32 and BF16 gives each
    request the result of its own single call."""
    import torch
    m, vol, P, _ = golden_cases()[0]
    vf = ctx.volume(VoxelVolume(vol, m["voxel"], m["offset"]), L.F32)
    vb = ctx.volume(VoxelVolume(vol, m["voxel"], m["offset"]), L.BF16)
    for kernel in (L.KERNEL_CELLS, L.KERNEL_PAIRS):
        s = _settings(m, kernel=kernel)
        dP = torch.from_numpy(np.ascontiguousarray(P)).cuda()
        outs = [torch.empty((P.shape[0], P.shape[1], m["rows"], m["channels"]), device="cuda") for _ in range(2)]
        ctx.project_batch([(vf, dP, outs[0]), (vb, dP, outs[1])], s)
        torch.cuda.synchronize()
        ctx.sync()
        for v, o in ((vf, outs[0]), (vb, outs[1])):
            np.testing.assert_array_equal(o.cpu().numpy(), ctx.project(v, P, m["channels"], m["rows"], s))
    vf.release()
    vb.release()


@pytest.mark.parametrize("kernel", [L.KERNEL_CELLS, L.KERNEL_PAIRS, L.KERNEL_GATHER], ids=["cells", "pairs", "gather"])
def test_sub_rays_in_every_loop_match_oracle(ctx, kernel):
    """raysPerPixel (3, 2) through the cell, pair and gather loops (the golden sub-ray
    cases use up-sampling or nearest voxel, so they take other loops)."""
    m, vol, P, _ = golden_cases()[5]   # anisotropic, off-centre, non-cubic; 40 x 36 detector
    s = _settings(m, kernel=kernel)
    s.rays_per_pixel = [3, 2]
    gpu = ctx.project_volume(VoxelVolume(vol, m["voxel"], m["offset"]), P, m["channels"], m["rows"], s)
    want, _ = oracle.project_fp64(vol, m["voxel"], P, m["channels"], m["rows"], offset_mm=m["offset"], rays=(3, 2))
    assert rel_err(gpu, want).max() <= TOL


def test_c3_full_size_512_cubed_helical_matches_oracle(ctx):
    """512^3 (0.5 mm, a 4.4 GB cell array) -> two helical views of 64 curved modules of
    16 x 16: the largest configuration, against the oracle."""
    from ctl_b200 import workloads as W
    P = W.c3_geometry()[[0, 719]]
    vol = W.phantom_device((512, 512, 512), (0.5, 0.5, 0.5), 40, seed=3, texture=0.01, device="cuda")
    v = ctx.volume(VoxelVolume(vol, (0.5, 0.5, 0.5)))
    host = vol.cpu().numpy()
    del vol
    want, _ = oracle.project_fp64(host, (0.5, 0.5, 0.5), P, 16, 16)
    for kernel in (L.KERNEL_CELLS, L.KERNEL_GATHER):
        gpu = ctx.project(v, P, 16, 16, Settings(kernel=kernel))
        assert rel_err(gpu, want).max() <= TOL, kernel
    v.release()


def test_cells_kernel_rejects_unsupported_settings(ctx):
    m, vol, P, _ = golden_cases()[0]
    for bad in (dict(interpolate=False), dict(volume_upsampling=2), dict(interp_mode=L.INTERP_TEXTURE)):
        with pytest.raises(L.CtlcuError) as e:
            ctx.project_volume(VoxelVolume(vol, m["voxel"]), P, 8, 8, Settings(kernel=L.KERNEL_CELLS, **bad))
        assert e.value.status == L.ERR_INVALID_ARGUMENT


def test_c2_linearity_at_full_size(ctx):
    """project(2 a + b) = 2 project(a) + project(b) over all 360 views (size-independent check)."""
    a = Ph.ellipsoid_phantom((256, 256, 256), (1, 1, 1), 40, seed=2)
    b = Ph.ellipsoid_phantom((256, 256, 256), (1, 1, 1), 40, seed=3)
    P = _c2_geometry()
    pa = ctx.project_volume(VoxelVolume(a, (1, 1, 1)), P, 512, 512)
    pb = ctx.project_volume(VoxelVolume(b, (1, 1, 1)), P, 512, 512)
    pc = ctx.project_volume(VoxelVolume(2 * a + b, (1, 1, 1)), P, 512, 512)
    e = rel_err(pc, 2 * pa + pb)
    assert e.max() < 1e-5


def test_uniform_cube_chord_full_detector(ctx):
    """A uniform 128^3 cube: every central-row pixel's value is mu times its chord (+- one step)."""
    n, mu = 128, 0.02
    vol = np.full((n, n, n), mu, np.float32)
    det = G.FlatDetector(257, 257, 1.0, 1.0)
    P = G.circular_flat(1, 750.0, 1000.0, det)
    out = ctx.project_volume(VoxelVolume(vol, (1, 1, 1)), P, 257, 257)
    assert abs(out[0, 0, 128, 128] - mu * n) <= 2 * mu * 0.3
    assert out[0, 0, 0, 0] == 0.0


# ---- batches and plans ------------------------------------------------------------------------

def _uneven_requests(ctx, rng_seed=5):
    """Small batch of uneven volumes / views / detectors (the batched configuration in miniature)."""
    import torch
    rng = np.random.default_rng(rng_seed)
    reqs, meta = [], []
    for i in range(5):
        shape = tuple(int(s) for s in rng.choice([24, 32, 40], 3))
        vox = float(rng.choice([2.0, 3.0]))
        vol = Ph.ellipsoid_phantom(shape, (vox, vox, vox), 4, seed=100 + i)
        V = int(rng.integers(2, 7))
        C, R = int(rng.choice([24, 40])), int(rng.choice([16, 32]))
        P = G.circular_flat(V, 750.0, 1000.0, G.FlatDetector(C, R, 2.0, 2.0), start=float(rng.uniform(0, 6)))
        v = ctx.volume(VoxelVolume(vol, (vox,) * 3))
        dP = torch.from_numpy(np.ascontiguousarray(P)).cuda()
        out = torch.zeros((V, 1, R, C), device="cuda")
        reqs.append((v, dP, out))
        meta.append((vol, vox, P, C, R))
    return reqs, meta


@pytest.mark.parametrize("kernel", [L.KERNEL_CELLS, L.KERNEL_PAIRS], ids=["cells", "pairs"])
def test_plan_forms_agree_with_single_calls(ctx, kernel):
    """A plan's two forms -- one persistent launch over every request's warp patches,
    and one grid launch per request on parallel graph branches -- give the same bits,
    and those of single calls, within the oracle's bar."""
    import torch
    reqs, meta = _uneven_requests(ctx, rng_seed=21)
    got = {}
    for form in (L.PLAN_PERSISTENT, L.PLAN_GRIDS):
        for _, _, out in reqs:
            out.zero_()
        plan = ctx.plan(reqs, Settings(kernel=kernel), form=form)
        assert plan.info()["form"] == ("persistent" if form == L.PLAN_PERSISTENT else "grids")
        plan.launch()
        ctx.sync()
        got[form] = [out.clone() for _, _, out in reqs]
        plan.close()
    for a, b in zip(got[L.PLAN_PERSISTENT], got[L.PLAN_GRIDS]):
        assert torch.equal(a, b)
    for out, (v, dP, _), (vol, vox, P, C, R) in zip(got[L.PLAN_GRIDS], reqs, meta):
        single = ctx.project(v, P, C, R, Settings(kernel=kernel))
        np.testing.assert_array_equal(out.cpu().numpy(), single)
        want, _ = oracle.project_fp64(vol, (vox,) * 3, P, C, R)
        assert rel_err(out.cpu().numpy(), want).max() <= TOL
    with pytest.raises(L.CtlcuError):
        ctx.plan(reqs, Settings(), form=7)
    for v, _, _ in reqs:
        v.release()


@pytest.mark.parametrize("kernel", [L.KERNEL_CELLS, L.KERNEL_PAIRS], ids=["cells", "pairs"])
def test_batch_matches_oracle_and_single_calls(ctx, kernel):
    reqs, meta = _uneven_requests(ctx)
    ctx.project_batch(reqs, Settings(kernel=kernel))
    ctx.sync()
    for (v, dP, out), (vol, vox, P, C, R) in zip(reqs, meta):
        single = ctx.project(v, P, C, R, Settings(kernel=kernel))
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, single, rtol=1e-6, atol=1e-7)
        want, _ = oracle.project_fp64(vol, (vox,) * 3, P, C, R)
        assert rel_err(got, want).max() <= TOL
    for v, _, _ in reqs:
        v.release()


def test_plan_replay_and_in_place_update(ctx):
    import torch
    reqs, meta = _uneven_requests(ctx, rng_seed=9)
    plan = ctx.plan(reqs, Settings())
    plan.launch()
    ctx.sync()
    first = [out.clone() for _, _, out in reqs]
    for _, _, out in reqs:
        out.zero_()
    plan.launch()
    ctx.sync()
    for (_, _, out), f in zip(reqs, first):
        assert torch.equal(out, f)
    # new geometry written in place is picked up by the next replay
    v0, dP0, out0 = reqs[0]
    vol, vox, P, C, R = meta[0]
    P2 = G.circular_flat(P.shape[0], 750.0, 1000.0, G.FlatDetector(C, R, 2.0, 2.0), start=1.234)
    dP0.copy_(torch.from_numpy(P2))
    plan.launch()
    ctx.sync()
    want, _ = oracle.project_fp64(vol, (vox,) * 3, P2, C, R)
    assert rel_err(out0.cpu().numpy(), want).max() <= TOL
    # a volume in a plan cannot be released until the plan is gone
    with pytest.raises(L.CtlcuError) as e:
        v0.release()
    assert e.value.status == L.ERR_BUSY
    plan.close()
    for v, _, _ in reqs:
        v.release()


def test_batch_outside_cell_kernel_falls_back_per_request(ctx):
    reqs, meta = _uneven_requests(ctx, rng_seed=3)
    s = Settings(interpolate=False)
    ctx.project_batch(reqs, s)
    ctx.sync()
    for (v, dP, out), (vol, vox, P, C, R) in zip(reqs, meta):
        want, _ = oracle.project_fp64(vol, (vox,) * 3, P, C, R, interpolate=False)
        assert rel_err(out.cpu().numpy(), want).max() <= TOL
        v.release()


def test_autotune_chooses_and_auto_follows(ctx):
    m, vol, P, _ = golden_cases()[0]
    v = ctx.volume(VoxelVolume(vol, m["voxel"], m["offset"]))
    kernel, ms = ctx.autotune(v, P, m["channels"], m["rows"], Settings())
    assert kernel in (L.KERNEL_CELLS, L.KERNEL_PAIRS, L.KERNEL_GATHER)
    assert all(t > 0 for t in ms.values())
    got = ctx.project(v, P, m["channels"], m["rows"], Settings())
    want, _ = _oracle(m, vol, P)
    assert rel_err(got, want).max() <= TOL
    # settings outside the fast loops: only the gather loop applies
    k2, _ = ctx.autotune(v, P, m["channels"], m["rows"], Settings(interpolate=False))
    assert k2 == L.KERNEL_GATHER
    v.release()

"""GPU checks of the learned surrogate: the tcgen05 BF16 GEMM against FP64
products of the same BF16 values, the network's forward pass and gradient
against the CPU oracle (oracle/mlp_oracle.py, itself pinned to finite
differences), the training samples against oracle/surrogate_oracle.py, the
model map's fallback path, and what the trained network gains over the centre
value alone.

Tolerances:
  * GEMM: relative 1e-5 of the output scale (FP32 accumulation of BF16 products);
  * forward output: relative L2 5e-4; gradient blocks: relative L2 2e-3 -- the
    kernels use tanh.approx where the oracle uses tanh, which flips some BF16
    roundings of activations (measured 7e-5 and at most 1.8e-4);
  * samples: features 1e-5, targets 1e-4 relative (FP64 math, FP32 storage);
  * the model map with every map redone by the rule: 1e-5 relative against the
    plain FP32 map (the FP64 12-point rule against the FP32 window path).
"""
import numpy as np
import pytest

from helpers import max_rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from xtsrcmaps_b200 import api as A
    from xtsrcmaps_b200 import build

    build.build()
    A.init(0)
    return A


def _psf_tables(A, name, seed, n=None):
    """Device uPsf / partial / exposure of a synthetic job."""
    import torch

    from xtsrcmaps_b200.synth import make_job

    job = make_job(name, seed=seed, n_sources=n)
    ltf = A.livetime_efficiency_factors(job.logEs, job.effic_front)
    nf = A.normalize_rpsf(job.rpsf_front, job.scale_front)
    nb = A.normalize_rpsf(job.rpsf_back, job.scale_back)
    ex = A.compute_exposure(job.exp_cube, job.wexp_cube, job.logEs, job.src_sph, job.aeff_front,
                            job.aeff_back, ltf)
    ps = A.compute_psf_data(nf, nb, ex, job.logEs, ltf)
    d = torch.device("cuda")
    t = lambda x: torch.as_tensor(np.ascontiguousarray(x), device=d)
    return job, t(ps.uPsf), t(ps.partial_psf_integral), t(ex.exposure)


def _bf16(rng, shape):
    import torch

    return torch.as_tensor(rng.normal(0.0, 1.0, shape).astype(np.float32)).to(torch.bfloat16)


@pytest.mark.parametrize("M,K,at,bt,ct,acc", [(256, 128, 0, 0, 0, 0), (384, 128, 1, 1, 1, 0),
                                             (128, 4096, 0, 0, 0, 1), (256, 192, 1, 0, 1, 0),
                                             (128, 1024, 1, 1, 0, 1)])
def test_gemm_bf16_layouts(api, M, K, at, bt, ct, acc):
    import torch

    from xtsrcmaps_b200.surrogate import gemm_bf16

    rng = np.random.default_rng(M + K)
    A = _bf16(rng, (K, M) if at else (M, K))
    B = _bf16(rng, (K, 128) if bt else (128, K))
    Amk = (A.T if at else A).double().numpy()
    Bnk = (B.T if bt else B).double().numpy()
    ref = Amk @ Bnk.T
    d = torch.device("cuda")
    out = gemm_bf16(A.to(d), B.to(d), M, K, bool(at), bool(bt), bool(ct), accumulate=bool(acc))
    got = out.cpu().double().numpy()
    got = got.T if ct else got
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()


def _rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def test_forward_and_gradient_match_oracle(api):
    import torch

    from oracle import mlp_oracle as MO
    from xtsrcmaps_b200.surrogate import Surrogate

    d = torch.device("cuda")
    net = Surrogate(device=d, seed=1)
    rng = np.random.default_rng(2)
    n = 1024
    X = rng.normal(0.5, 2.0, (n, 5)).astype(np.float32)
    Y = rng.normal(0.0, 1.5, n).astype(np.float32)
    net.in_mu = np.full(5, 0.5, np.float32)
    net.in_sd = np.full(5, 2.0, np.float32)
    net.out_mu, net.out_sd = 0.25, 1.5
    p = net.params.cpu().numpy()
    y = net.predict(torch.as_tensor(X, device=d)).cpu().numpy()
    y_ref = MO.predict(p, X, net.in_mu, net.in_sd, net.out_mu, net.out_sd)
    # the GPU's tanh.approx against the oracle's exact tanh (rel-L2 measured 7e-5)
    assert _rel_l2(y, y_ref) < 5e-4
    g, loss = net.gradient(torch.as_tensor(X, device=d), torch.as_tensor(Y, device=d))
    loss_ref, g_ref = MO.loss_and_grads(p, X, Y, net.in_mu, net.in_sd, net.out_mu, net.out_sd)
    assert abs(loss - loss_ref) <= 1e-3 * loss_ref
    g = g.cpu().numpy()
    for name, lo, hi in (("W1", MO.W1, MO.B1), ("b1", MO.B1, MO.W2), ("W2", MO.W2, MO.B2), ("b2", MO.B2, MO.W3),
                         ("W3", MO.W3, MO.B3), ("b3", MO.B3, MO.W4), ("W4", MO.W4, MO.B4), ("b4", MO.B4, MO.NPARAM)):
        assert _rel_l2(g[lo:hi], g_ref[lo:hi]) < 2e-3, name  # measured at most 1.8e-4


def test_inference_kernels_agree(api):
    """The four-tile inference kernel (the default) and the two-warpgroup kernel at
    one or two blocks per SM compute the same arithmetic: identical outputs, also
    for a row count that leaves the last tile and slots partly empty."""
    import torch

    from xtsrcmaps_b200.surrogate import Surrogate

    d = torch.device("cuda")
    net = Surrogate(device=d, seed=3)
    rng = np.random.default_rng(5)
    X = torch.as_tensor(rng.normal(0.0, 1.5, (128 * 700 + 77, 5)).astype(np.float32), device=d)
    before = api.get_tuning()
    try:
        ys = []
        for mb in (0, 1, 2):
            api.set_tuning(mlp_blocks_per_sm=mb)
            ys.append(net.predict(X).cpu().numpy())
    finally:
        api.set_tuning(**before)
    assert np.isfinite(ys[0]).all()
    np.testing.assert_array_equal(ys[0], ys[1])
    np.testing.assert_array_equal(ys[0], ys[2])


def test_samples_match_oracle(api):
    import torch

    from oracle import surrogate_oracle as SO
    from xtsrcmaps_b200.surrogate import samples

    job, upsf, _, _ = _psf_tables(api, "c1", seed=4, n=5)
    X, Y = samples(upsf, job.logEs, 300, seed=12345, rho_min=20.0)
    X, Y = X.cpu().numpy(), Y.cpu().numpy()
    U = upsf.cpu().numpy()
    for i in range(300):
        x, y = SO.sample(U, job.logEs, i, 12345, 20.0)
        np.testing.assert_allclose(X[i], x, rtol=1e-5, atol=1e-5)
        assert abs(Y[i] - y) <= 1e-4 * abs(y) + 1e-5, (i, Y[i], y)


def test_map_fallback_equals_rule(api):
    """With a check tolerance no network meets, every map is redone by the FP64
    12-point rule: the plain path's values."""
    import torch

    from xtsrcmaps_b200.surrogate import Surrogate, model_map, samples

    job, upsf, partial, expo = _psf_tables(api, "c1", seed=6, n=4)
    net = Surrogate(device=torch.device("cuda"), seed=0)
    X, Y = samples(upsf, job.logEs, 128 * 64, seed=3)
    net.fit_standardisation(X, Y)
    src = torch.as_tensor(job.src_sph, device=upsf.device)
    m, info, st = model_map(job.wcs, src, expo, upsf, partial, job.logEs, net, check_tol=1e-12)
    plain, pinfo = api.point_src_model_map_wcs(job.wcs, src, expo, upsf, partial)
    assert st["values"] == m.numel() and st["maps_fallback"] >= 1 and st["accepted"] == 0
    assert st["checked"] > 0
    assert max_rel(m.cpu().numpy(), plain.cpu().numpy()) < 1e-5
    assert max_rel(info.inv_map_integral.cpu().numpy(), pinfo.inv_map_integral.cpu().numpy()) < 1e-7


def test_fused_surrogate_call_host_and_device(api):
    """xts_point_source_maps_surrogate: the three calls in one with the surrogate's
    map.  From host buffers (the map copied out in groups of sources, each group
    finished on its own) and from device buffers (one group) it gives the map of the
    separate calls, with the same counts."""
    import torch

    from xtsrcmaps_b200.surrogate import Surrogate, model_map, samples
    from xtsrcmaps_b200.synth import make_job

    job = make_job("c1", seed=5, n_sources=20)
    ltf = api.livetime_efficiency_factors(job.logEs, job.effic_front)
    nf = api.normalize_rpsf(job.rpsf_front, job.scale_front)
    nb = api.normalize_rpsf(job.rpsf_back, job.scale_back)
    ex = api.compute_exposure(job.exp_cube, job.wexp_cube, job.logEs, job.src_sph, job.aeff_front,
                              job.aeff_back, ltf)
    ps = api.compute_psf_data(nf, nb, ex, job.logEs, ltf)
    d = torch.device("cuda")
    t = lambda x: torch.as_tensor(np.ascontiguousarray(x), device=d)
    upsf = t(ps.uPsf)
    net = Surrogate(device=d, seed=2)
    X, Y = samples(upsf, job.logEs, 200_000, seed=4)
    net.train(X, Y, epochs=3)
    ref, _, st_ref = model_map(job.wcs, t(job.src_sph), t(ex.exposure), upsf, t(ps.partial_psf_integral),
                               job.logEs, net, check_tol=1e-3)
    ref = ref.cpu().numpy()
    hm, _, st_h = api.point_source_maps_surrogate(job.wcs, job.src_sph, job.exp_cube, job.wexp_cube, job.logEs,
                                                  job.aeff_front, job.aeff_back, nf, nb, ltf, net, check_tol=1e-3)
    assert st_h == st_ref
    assert max_rel(hm, ref) < 1e-6
    from xtsrcmaps_b200.api import ExpCube
    from xtsrcmaps_b200.irf import IrfGrid

    tt = lambda x, dt=torch.float64: torch.as_tensor(np.asarray(x), device=d).to(dt).contiguous()
    grid = lambda g: IrfGrid(tt(g.cosths), tt(g.logEs), tt(g.params), g.min_cos_theta)
    cube = ExpCube(tt(job.exp_cube.cosbins, torch.float32), job.exp_cube.nside, 40, job.exp_cube.cosmin,
                   job.exp_cube.thetabin)
    wcube = ExpCube(tt(job.wexp_cube.cosbins, torch.float32), job.wexp_cube.nside, 40, job.wexp_cube.cosmin,
                    job.wexp_cube.thetabin)
    dm, _, st_d = api.point_source_maps_surrogate(job.wcs, tt(job.src_sph), cube, wcube, tt(job.logEs),
                                                  grid(job.aeff_front), grid(job.aeff_back), grid(nf), grid(nb),
                                                  tt(ltf), net, check_tol=1e-3)
    assert st_d == st_ref
    assert max_rel(dm.cpu().numpy(), ref) < 1e-6


def test_surrogate_map_many_energies(api):
    """More energies than the window path's write pass holds (60 > 52): the rule's
    means come from the FP64 rule per value instead; with a check no network meets,
    the map is the plain map's."""
    import torch

    from xtsrcmaps_b200.surrogate import Surrogate, model_map, samples

    job, upsf, partial, expo = _psf_tables(api, "c1", seed=8, n=3)
    sel = torch.arange(60, device=upsf.device) % upsf.shape[-1]
    u60, p60, e60 = (upsf[..., sel].contiguous(), partial[..., sel].contiguous(), expo[..., sel].contiguous())
    logEs = np.asarray(job.logEs)[sel.cpu().numpy()]
    net = Surrogate(device=upsf.device, seed=0)
    X, Y = samples(upsf, job.logEs, 128 * 64, seed=3)
    net.fit_standardisation(X, Y)
    src = torch.as_tensor(job.src_sph, device=upsf.device)
    m, info, st = model_map(job.wcs, src, e60, u60, p60, logEs, net, check_tol=1e-12)
    plain, pinfo = api.point_src_model_map_wcs(job.wcs, src, e60, u60, p60)
    assert st["values"] == m.numel() and st["accepted"] == 0
    assert max_rel(m.cpu().numpy(), plain.cpu().numpy()) < 1e-5
    assert max_rel(info.inv_map_integral.cpu().numpy(), pinfo.inv_map_integral.cpu().numpy()) < 1e-7


def test_trained_network_gains_over_centre_value(api):
    """Trained on the GPU on 10 M samples of a c2-style job's mean PSFs (separations
    log-uniform in 0.001-30 deg, pixel sizes 0.025-0.2 deg), the network's error on
    fresh samples is compared with the centre value alone (y = 0, the method without
    the network) where the method is meant to serve (rho >= 30); its error cells are
    calibrated on a held-out sample of another job; then the model map of 40 sources
    of a third c2 job must stay within 1e-4 of the plain map everywhere while the
    network serves a share of its values."""
    import torch

    from xtsrcmaps_b200.surrogate import Surrogate, last_stats, model_map, samples

    job, upsf, _, _ = _psf_tables(api, "c2", seed=111)
    X, Y = samples(upsf, job.logEs, 10_000_000, seed=12)
    net = Surrogate(device=upsf.device, seed=11)
    losses = net.train(X, Y, epochs=60)
    assert losses[-1] < 0.1 * losses[0]
    del X, Y
    Xh, Yh = samples(upsf, job.logEs, 400_000, seed=99)
    far = 10.0 ** Xh[:, 0].double() >= 30.0
    yp = net.predict(Xh)
    rho2 = (10.0 ** Xh[:, 0].double()) ** 2
    err_net = ((yp.double() - Yh.double()).abs() / rho2)[far].cpu().numpy()
    err_c = (Yh.double().abs() / rho2)[far].cpu().numpy()
    gain = float(np.sqrt(np.mean(err_c ** 2)) / np.sqrt(np.mean(err_net ** 2)))
    print(f"\nsurrogate (rho >= 30): rms rel error {np.sqrt(np.mean(err_net**2)):.2e} vs centre value "
          f"{np.sqrt(np.mean(err_c**2)):.2e} (gain {gain:.1f}x); within 1e-4: {np.mean(err_net <= 1e-4):.4f}")
    assert gain > 5.0
    cj, cu, _, _ = _psf_tables(api, "c2", seed=211)
    Xc, Yc = samples(cu, cj.logEs, 4_000_000, seed=13)
    cal = net.calibrate(Xc, Yc, tol=1e-4, margin=0.7)
    print(f"calibration: {cal}")
    assert cal["max_rel_err_in_accepted_cells"] <= 0.7e-4 and cal["cells_accepted"] > 0
    del Xc, Yc
    job2, upsf2, partial2, expo2 = _psf_tables(api, "c2", seed=11, n=40)
    src = torch.as_tensor(job2.src_sph, device=upsf2.device)
    m, _, st = model_map(job2.wcs, src, expo2, upsf2, partial2, job2.logEs, net, check_tol=1e-4)
    plain, _ = api.point_src_model_map_wcs(job2.wcs, src, expo2, upsf2, partial2)
    err = ((m.double() - plain.double()).abs() / plain.double().abs().clamp_min(1e-300))
    emax, within = float(err.max()), float((err <= 1e-4).double().mean())
    print(f"surrogate map: {st}; served {st['accepted'] / st['values']:.3f}; max rel err vs plain {emax:.2e}, "
          f"fraction within 1e-4 {within:.6f}")
    assert 0 <= st["accepted"] <= st["values"] == m.numel()
    assert bool(torch.isfinite(m).all())
    assert st["accepted"] > 0.2 * st["values"]
    assert emax <= 1e-4
    # the same call without the stats (no synchronisation): identical map, same counts
    m2, _, none = model_map(job2.wcs, src, expo2, upsf2, partial2, job2.logEs, net, check_tol=1e-4, stats=False)
    assert none is None
    assert last_stats(upsf2.device) == st
    assert torch.equal(m2, m)
    # with the two-warpgroup network kernel in place of the four-tile one: the same map
    # and counts (the kernels' outputs agree bit for bit)
    api.set_tuning(mlp_blocks_per_sm=2)
    try:
        m3, _, st3 = model_map(job2.wcs, src, expo2, upsf2, partial2, job2.logEs, net, check_tol=1e-4)
    finally:
        api.reset_tuning()
    assert st3 == st
    assert torch.equal(m3, m)


def test_surrogate_argument_errors(api):
    """Shapes and parameters the entry points reject with XTS_ERR_ARG (no launch)."""
    import torch

    from xtsrcmaps_b200 import _lib as L
    from xtsrcmaps_b200.surrogate import Surrogate, gemm_bf16

    d = torch.device("cuda")
    a = torch.zeros((100, 128), dtype=torch.bfloat16, device=d)
    b = torch.zeros((128, 128), dtype=torch.bfloat16, device=d)
    with pytest.raises(L.XtsError) as ei:
        gemm_bf16(a, b, 100, 128)  # M not a multiple of 128
    assert ei.value.code == L.XTS_ERR_ARG
    with pytest.raises(L.XtsError) as ei:
        gemm_bf16(torch.zeros((128, 96), dtype=torch.bfloat16, device=d), b[:, :96], 128, 96)  # K % 64
    assert ei.value.code == L.XTS_ERR_ARG
    net = Surrogate(device=d, seed=0)
    X = torch.zeros((200, 5), dtype=torch.float32, device=d)
    Y = torch.zeros((200,), dtype=torch.float32, device=d)
    with pytest.raises(L.XtsError) as ei:
        net.gradient(X, Y)  # 200 rows: not a multiple of 128
    assert ei.value.code == L.XTS_ERR_ARG
    net.in_sd[2] = 0.0
    with pytest.raises(L.XtsError) as ei:
        net.predict(X)
    assert ei.value.code == L.XTS_ERR_ARG


def test_training_is_reproducible(api):
    """Gradient sums run in a fixed order (split-K partials and per-block partials
    reduced in order, no atomics), so two trainings from the same start agree bit
    for bit."""
    import torch

    from xtsrcmaps_b200.surrogate import Surrogate, samples

    job, upsf, _, _ = _psf_tables(api, "c1", seed=10, n=3)
    X, Y = samples(upsf, job.logEs, 128 * 148 * 2 * 3, seed=5)
    out = []
    for _ in range(2):
        net = Surrogate(device=upsf.device, seed=3)
        net.train(X, Y, epochs=2, seed=1)
        torch.cuda.synchronize()
        out.append(net.params.cpu().numpy())
    np.testing.assert_array_equal(out[0], out[1])

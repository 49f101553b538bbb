"""CPU checks of the surrogate network's host side: the numpy oracle's gradient
against finite differences (this pins the oracle the GPU gradients are checked
against), its BF16 rounding, the ctypes layout of xts_mlp and
xts_surrogate_stats against the C header, and the sample oracle's geometry."""
import math
import os
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import mlp_oracle as MO
from oracle import surrogate_oracle as SO

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _net(seed=3):
    rng = np.random.default_rng(seed)
    p = rng.normal(0.0, 0.15, MO.NPARAM)
    X = rng.normal(0.0, 1.0, (16, MO.IN))
    Y = rng.normal(0.0, 1.0, 16)
    return p, X, Y


def test_oracle_gradient_matches_finite_differences():
    p, X, Y = _net()
    mu, sd = np.zeros(MO.IN), np.ones(MO.IN)
    loss, g = MO.loss_and_grads(p, X, Y, mu, sd, 0.0, 1.0, use_bf16=False)
    rng = np.random.default_rng(0)
    idx = np.concatenate([rng.choice(np.arange(lo, hi), 6, replace=False)
                          for lo, hi in ((MO.W1, MO.B1), (MO.B1, MO.W2), (MO.W2, MO.B2), (MO.B2, MO.W3),
                                         (MO.W3, MO.B3), (MO.B3, MO.W4), (MO.W4, MO.B4))] + [[MO.B4]])
    h = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += h
        lp, _ = MO.loss_and_grads(q, X, Y, mu, sd, 0.0, 1.0, use_bf16=False)
        q[i] -= 2 * h
        lm, _ = MO.loss_and_grads(q, X, Y, mu, sd, 0.0, 1.0, use_bf16=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])
    assert loss > 0


def test_bf16_rounding_ties_to_even():
    # 1 + 2^-8 lies halfway between BF16 neighbours 1 and 1 + 2^-7: even mantissa (1) wins
    assert MO.bf16(np.float32(1.0 + 2.0 ** -8))[()] == 1.0
    assert MO.bf16(np.float32(1.0 + 3 * 2.0 ** -8))[()] == 1.0 + 2.0 ** -6
    assert MO.bf16(np.float32(-2.5))[()] == -2.5


def test_struct_layouts_match_the_header():
    from xtsrcmaps_b200 import _lib as L
    import ctypes as C

    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "xtsrcmaps_b200.h"
int main(void) {
    printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(xts_mlp), offsetof(xts_mlp, in_mu),
           offsetof(xts_mlp, out_mu), offsetof(xts_mlp, lo), offsetof(xts_mlp, rho_min),
           offsetof(xts_mlp, cell_lo), offsetof(xts_mlp, cell_hi), offsetof(xts_mlp, cell_ok),
           sizeof(xts_surrogate_stats), offsetof(xts_surrogate_stats, evaluated));
    printf("%zu %zu\n", sizeof(xts_tuning), offsetof(xts_tuning, chunk_sources));
    printf("%d %d %d %d %d %d\n", XTS_MLP_W2, XTS_MLP_W3, XTS_MLP_B4, XTS_MLP_NPARAM, XTS_MLP_CELL_NR,
           XTS_MLP_CELL_NS);
    return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    sizes = [int(v) for v in out[0].split()]
    assert sizes == [C.sizeof(L.XtsMlp), L.XtsMlp.in_mu.offset, L.XtsMlp.out_mu.offset, L.XtsMlp.lo.offset,
                     L.XtsMlp.rho_min.offset, L.XtsMlp.cell_lo.offset, L.XtsMlp.cell_hi.offset,
                     L.XtsMlp.cell_ok.offset, C.sizeof(L.XtsSurrogateStats), L.XtsSurrogateStats.evaluated.offset]
    assert [int(v) for v in out[1].split()] == [C.sizeof(L.XtsTuning), L.XtsTuning.chunk_sources.offset]
    consts = [int(v) for v in out[2].split()]
    assert consts[:4] == [L.MLP_W2, L.MLP_W3, L.MLP_B4, L.MLP_NPARAM] == [MO.W2, MO.W3, MO.B4, MO.NPARAM]
    assert consts[4:] == [L.MLP_CELL_NR, L.MLP_CELL_NS]


def test_sample_oracle_geometry():
    assert abs(SO.RULE[:, 2].sum() - 4.0) < 1e-12
    # a smooth table (u = exp(-theta / 2 deg)) and a sample far from the source:
    # the rule mean approaches the centre value
    seps = np.array([0.0] + [1e-4 * math.exp(k * SO.SEP_STEP) for k in range(400)])
    U = np.exp(-seps / 2.0)[:, None] * np.ones((1, 3))
    upsf = U[None]
    logEs = np.array([2.0, 3.0, 4.0])
    for i in range(20):
        x, y = SO.sample(upsf, logEs, i, seed=5, rho_min=20.0)
        assert 10 ** x[0] >= 20.0 * 0.999  # rho >= rho_min
        assert 0.0 <= x[1] <= 1.0  # offset between table rows
        assert math.log10(0.025 ** 2 * 0.99) <= x[2] <= math.log10(0.2 ** 2 * 1.01)
        assert x[3] in logEs
        assert np.isfinite(y)


def test_surrogate_state_round_trip(tmp_path):
    """Host side of xtsrcmaps_b200.surrogate without a GPU: initialisation, the
    BF16 copies (round to nearest even), standardisation from a training set, and
    save/load of the parameters and standardisation."""
    import torch

    from xtsrcmaps_b200 import _lib as L
    from xtsrcmaps_b200.surrogate import Surrogate

    net = Surrogate(device="cpu", seed=4, rho_min=50.0)
    p = net.params.numpy()
    assert p.shape == (L.MLP_NPARAM,) and np.all(p[L.MLP_B1:L.MLP_W2] == 0)
    w23 = np.concatenate([p[L.MLP_W2:L.MLP_B2], p[L.MLP_W3:L.MLP_B3]])
    bits = net.wbf16.numpy().astype(np.uint16).astype(np.uint32) << 16
    np.testing.assert_array_equal(bits.view(np.float32), MO.bf16(w23).astype(np.float32))
    rng = np.random.default_rng(0)
    X = torch.as_tensor(rng.normal(2.0, 3.0, (4096, 5)).astype(np.float32))
    Y = torch.as_tensor(rng.normal(-1.0, 0.5, 4096).astype(np.float32))
    net.fit_standardisation(X, Y)
    assert np.allclose(net.in_mu, 2.0, atol=0.2) and np.allclose(net.in_sd, 3.0, atol=0.2)
    assert np.all(net.lo <= X.numpy().min(0)) and np.all(net.hi >= X.numpy().max(0))
    assert abs(net.out_mu + 1.0) < 0.05 and abs(net.out_sd - 0.5) < 0.05
    f = str(tmp_path / "net.npz")
    net.save(f)
    back = Surrogate.load(f, device="cpu")
    np.testing.assert_array_equal(back.params.numpy(), p)
    np.testing.assert_array_equal(back.wbf16.numpy(), net.wbf16.numpy())
    for a in ("in_mu", "in_sd", "lo", "hi"):
        np.testing.assert_array_equal(getattr(back, a), getattr(net, a))
    assert (back.out_mu, back.out_sd, back.rho_min) == (net.out_mu, net.out_sd, 50.0)
    s = back.struct()
    assert abs(s.rho_min - 50.0) < 1e-6 and list(s.in_sd) == pytest.approx(list(net.in_sd))
    assert not s.cell_ok  # uncalibrated: no cell restriction (NULL)
    # calibrated error cells travel with the state
    net.cell_lo = np.array([-1.0, -30.0], np.float32)
    net.cell_hi = np.array([3.0, 2.0], np.float32)
    net.cell_ok = torch.as_tensor(rng.integers(0, 2, L.MLP_CELL_NR * L.MLP_CELL_NS).astype(np.uint8))
    net.save(f)
    back = Surrogate.load(f, device="cpu")
    np.testing.assert_array_equal(back.cell_ok.numpy(), net.cell_ok.numpy())
    s = back.struct()
    assert list(s.cell_lo) == [-1.0, -30.0] and list(s.cell_hi) == [3.0, 2.0] and s.cell_ok


def test_cli_and_bench_expose_the_surrogate():
    """The command line and the bench carry the surrogate's options (host side only)."""
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-m", "xtsrcmaps_b200", "--help"], cwd=root, capture_output=True,
                         text=True, check=True).stdout
    for opt in ("--surrogate", "--train-surrogate", "--surrogate-samples", "--check-tol"):
        assert opt in out, opt
    out = subprocess.run([sys.executable, "bench.py", "--help"], cwd=root, capture_output=True, text=True,
                         check=True).stdout
    for opt in ("--no-surrogate", "--surrogate-samples", "--surrogate-epochs", "--surrogate-file", "--no-c4",
                "--no-f64"):
        assert opt in out, opt


def test_bench_gpus_launch_refuses_without_gpus():
    """bench.py --gpus N starts N ranks itself when no launcher did; on a machine
    with fewer CUDA devices it fails loudly instead of running one rank."""
    import sys

    import torch

    if torch.cuda.is_available() and torch.cuda.device_count() >= 2:
        pytest.skip("this machine has the GPUs: the launch would run")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, "bench.py", "--gpus", "2", "--steps", "3"], cwd=root, capture_output=True,
                       text=True, env=env, timeout=300)
    assert r.returncode == 2
    assert "one rank per GPU needs 2" in r.stderr

"""Host logic of the autotuner without a GPU: the library calls and the timer are
replaced by fakes, so what is tested is the choice each tuner makes from the timings
and errors it measures, its restoring and applying of the launch shapes, and its
per-job cache."""
import types

import pytest

torch = pytest.importorskip("torch")

from xtsrcmaps_b200 import api as A  # noqa: E402
from xtsrcmaps_b200 import autotune as T  # noqa: E402


def _job(S=3, H=8, W=6, E=4):
    wcs = types.SimpleNamespace(naxis1=H, naxis2=W, cdelt1=0.1, cdelt2=0.1)
    src = torch.zeros((S, 2), dtype=torch.float64)
    expo = torch.ones((S, E), dtype=torch.float64)
    upsf = torch.ones((S, 401, E), dtype=torch.float64)
    part = torch.ones((S, 401, E), dtype=torch.float64)
    return wcs, src, expo, upsf, part


@pytest.fixture(autouse=True)
def _fresh_cache():
    T._CACHE.clear()
    yield
    T._CACHE.clear()


def test_adaptive_picks_fastest_candidate_meeting_target(monkeypatch):
    wcs, src, expo, upsf, part = _job()
    ref = torch.rand((3, 8, 6, 4), dtype=torch.float32) + 1.0
    state = {}

    def fake_adaptive(wcs_, s, ex, up, pp, rtol, max_depth, with_info=False):
        state["last"] = (rtol, max_depth)
        # error shrinks with rtol and with depth; the converged map is exact
        err = 0.0 if rtol <= 1e-6 else rtol * 4.0 / max_depth
        return ref * (1.0 + err), None

    def fake_timed(fn, reps):
        fn()
        rtol, depth = state["last"]
        return depth * 1e-3 / rtol  # tighter rtol and deeper: slower

    monkeypatch.setattr(A, "point_src_model_map_wcs_adaptive", fake_adaptive)
    monkeypatch.setattr(T, "_timed", fake_timed)
    rtols, depths = (3e-3, 1e-3, 3e-4, 1e-4), (4, 6, 8)
    # target between the candidates' errors (none sits at it): (3e-4, 6) has error 2e-4
    # and is the fastest of those at or below 2.5e-4
    res = T.tune_adaptive(wcs, src, expo, upsf, part, target=2.5e-4, rtols=rtols, depths=depths)
    ok = [(d * 1e-3 / r, r, d) for r in rtols for d in depths if r * 4.0 / d <= 2.5e-4]
    t, r, d = min(ok)
    assert (r, d) == (3e-4, 6)
    assert (res["rtol"], res["max_depth"]) == (r, d)
    assert res["err"] <= 2.5e-4 and abs(res["ms"] - t) < 1e-12
    assert len(res["table"]) == len(rtols) * len(depths)
    # cached per job shape: a second call measures nothing
    monkeypatch.setattr(T, "_timed", lambda fn, reps: pytest.fail("measured again"))
    assert T.tune_adaptive(wcs, src, expo, upsf, part, target=2.5e-4, rtols=rtols, depths=depths) is res
    # a target no candidate meets: None
    T._CACHE.clear()
    monkeypatch.setattr(T, "_timed", fake_timed)
    assert T.tune_adaptive(wcs, src, expo, upsf, part, target=1e-9, rtols=rtols, depths=depths) is None


def test_launch_shapes_choice_restore_and_apply(monkeypatch):
    wcs, src, expo, upsf, part = _job()
    tuning = {"window_blocks_per_sm": 0, "write_blocks_per_sm": 0, "queue_blocks_per_sm": 0,
              "mlp_blocks_per_sm": 0, "chunk_sources": 7}
    applied = []

    def fake_set(**fields):
        tuning.update(fields)
        applied.append(dict(fields))

    cost = {(1, 1): 5.0, (1, 2): 4.2, (2, 1): 5.1, (2, 2): 4.1, (3, 1): 5.0, (3, 2): 4.05}
    mlp_cost = {0: 0.22, 1: 0.36, 2: 0.26}

    def fake_timed(fn, reps):
        fn()
        if state["what"] == "map":
            return cost[(tuning["window_blocks_per_sm"], tuning["write_blocks_per_sm"])]
        return mlp_cost[tuning["mlp_blocks_per_sm"]]

    state = {"what": "map"}

    def fake_map(*args, **kw):
        state["what"] = "map"
        return None, None

    class FakeNet:
        in_mu = [0.0] * 5
        in_sd = [1.0] * 5

        def predict(self, X):
            state["what"] = "mlp"
            assert X.shape == (1 << 20, 5)
            return X[:, 0]

    monkeypatch.setattr(A, "get_tuning", lambda: dict(tuning))
    monkeypatch.setattr(A, "set_tuning", fake_set)
    monkeypatch.setattr(A, "point_src_model_map_wcs", fake_map)
    monkeypatch.setattr(T, "_timed", fake_timed)
    res = T.tune_launch_shapes(wcs, src, expo, upsf, part, net=FakeNet())
    assert res["choice"] == {"window_blocks_per_sm": 3, "write_blocks_per_sm": 2, "mlp_blocks_per_sm": 0}
    assert res["ms"]["window3/write2"] == 4.05 and res["ms"]["mlp1"] == 0.36
    # the shapes in force before are restored, then the choice applied; other fields kept
    assert applied[-2]["window_blocks_per_sm"] == 0 and applied[-2]["chunk_sources"] == 7
    assert applied[-1] == res["choice"]
    assert tuning["chunk_sources"] == 7
    # cached: the choice is applied again without measuring
    applied.clear()
    monkeypatch.setattr(T, "_timed", lambda fn, reps: pytest.fail("measured again"))
    assert T.tune_launch_shapes(wcs, src, expo, upsf, part, net=FakeNet()) is res
    assert applied == [res["choice"]]


def test_write_pass_picks_fastest_kernel(monkeypatch):
    wcs, src, expo, upsf, part = _job()
    state = {}

    def fake_map(*args, kernel="windows", **kw):
        state["k"] = kernel
        return None, None

    times = {"windows": 4.0, "cuda_cores": 19.0, "tcgen05": 28.5}

    def fake_timed(fn, reps):
        fn()
        return times[state["k"]]

    monkeypatch.setattr(A, "point_src_model_map_wcs", fake_map)
    monkeypatch.setattr(T, "_timed", fake_timed)
    res = T.tune_write_pass(wcs, src, expo, upsf, part)
    assert res == {"kernel": "windows", "ms": times}
    times["windows"] = 30.0
    T._CACHE.clear()
    assert T.tune_write_pass(wcs, src, expo, upsf, part)["kernel"] == "cuda_cores"

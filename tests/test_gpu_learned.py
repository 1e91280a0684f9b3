"""GPU learned CDEF strength selection against the CPU oracle and against the
exhaustive search (pf_mlp.cu, pf_search.cu).

* features, forward probabilities and training gradients agree with
  oracle/learned_oracle.cpp (fp32; the only differences are exp/log2
  rounding, so the tolerances are a few ulps);
* training lowers the loss and is bit-for-bit repeatable;
* the masked search measures exactly the exhaustive search's SSE for every
  tested trial and records the untested figure elsewhere, and with every
  block falling back it is the exhaustive search;
* the committed network keeps the luma SSE within 0.5 % of the exhaustive
  search's on average over all 50 held-out frames and beats the same trial
  budget spent without it."""

import ctypes as C
import json
import os

import numpy as np
import pytest

from goav1_b200 import abi, learned, synth

pytestmark = pytest.mark.gpu

F, O = abi.PF_MLP_FEATURES, abi.PF_MLP_OUTPUTS
UNTESTED = 1040400 * 64


@pytest.fixture(scope="module")
def runner():
    from goav1_b200.postfilter import PostFilterRunner

    r = PostFilterRunner()
    yield r
    r.close()


def _pair(runner, seed, w, h):
    src, rec, side, _ = synth.make_search_pair(seed, w, h)
    runner.apply(rec.pf(), side.side)
    return src, rec, learned.noskip_of(side, rec)


def _rand_model(seed, n):
    rng = np.random.default_rng(seed)
    X = (rng.standard_normal((n, F)) * 2 + 0.5).astype(np.float32)
    m = learned.init_model(X, seed=seed)
    np.ctypeslib.as_array(m.b3)[:] = (rng.standard_normal(O) * 0.2).astype(np.float32)
    Y = rng.integers(0, 64, (n, 2)).astype(np.uint8)
    return m, X, Y


def constant_model(luma, chroma):
    """A network whose output ignores the features: the given trials of each
    head in the given order (logits 10, 9, 8, ...; the first at probability
    about 0.7), every other trial far below."""
    m = abi.pf_cdef_mlp()
    b3 = np.ctypeslib.as_array(m.b3)
    b3[:] = 0
    for i, (l, c) in enumerate(zip(luma, chroma)):
        b3[l], b3[64 + c] = 10.0 - i, 10.0 - i
    np.ctypeslib.as_array(m.feat_scale)[:] = 1.0
    return m


@pytest.mark.parametrize("w,h,use_ns", [(256, 192, True), (200, 130, True), (640, 360, False)])
def test_features_match_oracle(runner, oracle, w, h, use_ns):
    _, rec, ns = _pair(runner, 31 + w, w, h)
    ns = ns if use_ns else None
    Xg = runner.cdef_features(rec.pf(), ns, 150)
    Xo = np.zeros_like(Xg)
    assert oracle.oracle_cdef_features(C.byref(rec.pf()), ns.ctypes.data if ns is not None else None, 150, 0,
                                       Xo.ctypes.data) == 0
    assert np.allclose(Xg, Xo, rtol=4e-7, atol=1e-7), np.abs(Xg - Xo).max()


def test_forward_matches_oracle(runner, oracle):
    m, X, _ = _rand_model(1, 100)
    Pg = runner.mlp_forward(m, X)
    Po = np.zeros_like(Pg)
    oracle.oracle_mlp_forward(C.byref(m), X.ctypes.data, X.shape[0], Po.ctypes.data)
    assert np.abs(Pg - Po).max() <= 2e-7


@pytest.mark.parametrize("n", [32, 100])
def test_gradients_match_oracle(runner, oracle, n):
    m, X, Y = _rand_model(2 + n, n)
    loss_g, g = runner.mlp_gradients(m, X, Y)
    gg = np.ctypeslib.as_array(C.cast(C.byref(g), C.POINTER(C.c_float)), (abi.PF_MLP_PARAMS,)).copy()
    loss_o = C.c_float()
    go = np.zeros(abi.PF_MLP_PARAMS, np.float32)
    oracle.oracle_mlp_gradients(C.byref(m), X.ctypes.data, Y.ctypes.data, n, C.byref(loss_o), go.ctypes.data)
    assert abs(loss_g - loss_o.value) <= 1e-6 * abs(loss_o.value)
    assert np.abs(gg - go).max() <= 1e-5 * np.abs(go).max()


def test_training_lowers_loss_and_repeats_exactly(runner):
    rng = np.random.default_rng(5)
    X = rng.standard_normal((2048, F)).astype(np.float32)
    # Learnable labels: each head is the argmax of a fixed linear map.
    A = rng.standard_normal((F, 2, 64)).astype(np.float32)
    Y = np.stack([(X @ A[:, p]).argmax(1) for p in range(2)], 1).astype(np.uint8)
    m1 = learned.init_model(X, seed=3)
    m2 = abi.pf_cdef_mlp.from_buffer_copy(bytes(m1))
    l1 = runner.mlp_train(m1, X, Y, epochs=15, batch=256, lr=3e-3)
    l2 = runner.mlp_train(m2, X, Y, epochs=15, batch=256, lr=3e-3)
    assert l1[-1] < 0.5 * l1[0]
    assert bytes(m1) == bytes(m2) and np.array_equal(l1, l2)


def test_all_fallback_is_the_exhaustive_search(runner):
    src, rec, ns = _pair(runner, 77, 640, 360)
    m, _, _ = _rand_model(9, 64)
    r0, m0, i0 = runner.cdef_search(src.pf(), rec.pf(), ns, 128, 4000.0)
    r1, m1, i1, st = runner.cdef_search_learned(src.pf(), rec.pf(), ns, 128, 4000.0, m, threshold=2.0, refine=True)
    assert np.array_equal(m0, m1) and np.array_equal(i0, i1)
    assert bytes(r0) == bytes(r1)
    assert st.fallback_luma == st.fallback_chroma == st.blocks and st.trials_luma == 64 * st.blocks


def test_masked_search_measures_tested_trials_exactly(runner):
    src, rec, ns = _pair(runner, 78, 640, 360)
    _, m0, _ = runner.cdef_search(src.pf(), rec.pf(), ns, 128, 4000.0)
    m = constant_model([63, 60], [60, 57])
    _, m1, idx, st = runner.cdef_search_learned(src.pf(), rec.pf(), ns, 128, 4000.0, m, threshold=0.5, candidates=2)
    live = m0[0].sum(1) > 0
    assert st.fallback_luma == st.fallback_chroma == 0
    assert st.trials_luma == 2 * st.blocks and st.trials_chroma == 2 * st.blocks
    for p, tested in ((0, [60, 63]), (1, [57, 60])):
        mask = np.zeros(64, bool)
        mask[tested] = True
        assert np.array_equal(m1[p][live][:, mask], m0[p][live][:, mask])
        assert (m1[p][live][:, ~mask] == UNTESTED).all()
    assert (m1[:, ~live] == 0).all()


def test_committed_network_on_eval_frames(runner):
    """All 50 held-out frames (seeds 2000-2049): the network's luma SSE
    increase over the exhaustive search must be at most 0.5 % on average (the
    bar), and must beat the same measurement budget (three trials per head,
    no fallback) spent on the training set's three most frequent best trials,
    the method without the network.  The worst frame is printed."""
    model = learned.load_model()
    with open(os.path.splitext(learned.DEFAULT_MODEL)[0] + ".json") as f:
        rep = json.load(f)
    prior = constant_model(rep["prior_luma"][:3], rep["prior_chroma"][:3])
    inc_net, inc_prior = [], []
    for seed, src, rec, side, _ in learned.search_frames(range(2000, 2050), 1920, 1080, workers=8):
        runner.apply(rec.pf(), side.side)
        ns = learned.noskip_of(side, rec)
        q = learned.frame_qindex(seed)
        r0, m0, i0 = runner.cdef_search(src.pf(), rec.pf(), ns, q, learned.LAMBDA)
        r1, _, i1, st = runner.cdef_search_learned(src.pf(), rec.pf(), ns, q, learned.LAMBDA, model)
        r2, _, i2, _ = runner.cdef_search_learned(src.pf(), rec.pf(), ns, q, learned.LAMBDA, prior, candidates=3)
        base = learned.luma_sse(r0, i0, m0)
        inc_net.append(learned.luma_sse(r1, i1, m0) / base - 1)
        inc_prior.append(learned.luma_sse(r2, i2, m0) / base - 1)
        assert st.blocks > 0
    worst = int(np.argmax(inc_net))
    print("learned luma SSE increase over 50 eval frames: mean %.4f %%, worst %.4f %% (seed %d)"
          % (100 * np.mean(inc_net), 100 * inc_net[worst], 2000 + worst))
    assert np.mean(inc_net) <= 0.005, inc_net
    assert np.mean(inc_net) <= np.mean(inc_prior), (inc_net, inc_prior)


@pytest.mark.parametrize("w,h,cand,refine", [(640, 360, 1, False), (1280, 720, 2, False), (1280, 720, 3, True)])
def test_learned_selection_matches_oracle_finish(runner, oracle, w, h, cand, refine):
    """The greedy selection over the learned search's own table (tested
    trials measured, the rest at the untested figure) equals the oracle's
    finish() over that table, with or without the refinement passes."""
    src, rec, ns = _pair(runner, 90 + w, w, h)
    model = learned.load_model()
    res, mse, idx, st = runner.cdef_search_learned(src.pf(), rec.pf(), ns, 128, 4000.0, model, candidates=cand,
                                                   refine=refine)
    skip = (mse[0].sum(1) == 0).astype(np.uint8)
    res_o = abi.pf_cdef_search_result()
    idx_o = np.zeros_like(idx)
    prm = abi.pf_cdef_search_params(qindex=128, damping=0, max_presets=8, lam=4000.0)
    assert oracle.oracle_cdef_select_ex(mse.ctypes.data, skip.ctypes.data, mse.shape[1], C.byref(prm), int(refine),
                                        idx_o.ctypes.data, C.byref(res_o)) == 0
    assert bytes(res) == bytes(res_o) and np.array_equal(idx, idx_o)
    assert st.trials_luma < 64 * st.blocks

"""CPU checks of the learned CDEF selection's oracle and host helpers
(oracle/learned_oracle.cpp, goav1_b200/learned.py): the oracle's gradients
against finite differences, the fp32 oracle against its double twin, bf16
rounding, label canonicalisation, side-information pickling and the model
file format."""

import ctypes as C
import pickle

import numpy as np
import pytest

from goav1_b200 import abi, learned, synth

NP = abi.PF_MLP_PARAMS
F, H, O = abi.PF_MLP_FEATURES, abi.PF_MLP_HIDDEN, abi.PF_MLP_OUTPUTS


def _rand_model(seed, n=64):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, F)).astype(np.float32) * 3 + 1
    m = learned.init_model(X, seed=seed)
    # Non-zero biases so every path of the gradient is exercised.
    np.ctypeslib.as_array(m.b1)[:] = rng.standard_normal(H).astype(np.float32) * 0.1
    np.ctypeslib.as_array(m.b2)[:] = rng.standard_normal(H).astype(np.float32) * 0.1
    np.ctypeslib.as_array(m.b3)[:] = rng.standard_normal(O).astype(np.float32) * 0.1
    Y = rng.integers(0, 64, (n, 2)).astype(np.uint8)
    return m, X, Y


def _flat(m):
    a = learned.model_arrays(m)
    return np.concatenate([a["w1"].ravel(), a["w2"].ravel(), a["w3"].ravel(), a["b1"], a["b2"], a["b3"]]).astype(
        np.float64), a["shift"].astype(np.float64), a["scale"].astype(np.float64)


def _f64(lib, P, shift, scale, X, Y):
    loss = C.c_double()
    g = np.zeros(NP, np.float64)
    lib.oracle_mlp_loss_grad_f64(P.ctypes.data, shift.ctypes.data, scale.ctypes.data, X.ctypes.data, Y.ctypes.data,
                                 X.shape[0], C.byref(loss), g.ctypes.data)
    return loss.value, g


def test_oracle_gradient_matches_finite_differences(oracle):
    m, X, Y = _rand_model(3, n=12)
    P, shift, scale = _flat(m)
    _, g = _f64(oracle, P, shift, scale, X, Y)
    rng = np.random.default_rng(9)
    idx = np.concatenate([rng.choice(H * F, 12, replace=False),
                          H * F + rng.choice(H * H, 12, replace=False),
                          H * F + H * H + rng.choice(O * H, 12, replace=False),
                          NP - O - 2 * H + rng.choice(2 * H + O, 12, replace=False)])
    eps = 1e-6
    for i in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += eps
        Pm[i] -= eps
        num = (_f64(oracle, Pp, shift, scale, X, Y)[0] - _f64(oracle, Pm, shift, scale, X, Y)[0]) / (2 * eps)
        assert abs(num - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), (i, num, g[i])


def test_fp32_oracle_gradient_close_to_double(oracle):
    m, X, Y = _rand_model(5, n=70)  # three tiles, the last one partial
    P, shift, scale = _flat(m)
    l64, g64 = _f64(oracle, P, shift, scale, X, Y)
    loss = C.c_float()
    g32 = np.zeros(NP, np.float32)
    oracle.oracle_mlp_gradients(C.byref(m), X.ctypes.data, Y.ctypes.data, X.shape[0], C.byref(loss), g32.ctypes.data)
    assert abs(loss.value - l64) <= 1e-5 * abs(l64)
    assert np.abs(g32 - g64).max() <= 1e-4 * np.abs(g64).max()


def test_forward_probabilities_sum_to_one(oracle):
    m, X, _ = _rand_model(7, n=40)
    P = np.zeros((40, O), np.float32)
    oracle.oracle_mlp_forward(C.byref(m), X.ctypes.data, 40, P.ctypes.data)
    assert np.allclose(P[:, :64].sum(1), 1, atol=1e-5) and np.allclose(P[:, 64:].sum(1), 1, atol=1e-5)


def test_bf16_rounding_is_nearest_even():
    vals = np.array([1.0, 1.00390625, 1.01171875, -2.5, 3.0e-3, 65504.0, 1.0 + 2 ** -9], np.float32)
    bits = learned.bf16_bits(vals)
    # 1 + 2^-8 is a tie between 0x3F80 and 0x3F81: even wins; 1 + 3*2^-8 rounds
    # up to the even 0x3F82; 1 + 2^-9 is below the tie.
    assert bits[0] == 0x3F80 and bits[1] == 0x3F80 and bits[2] == 0x3F82 and bits[6] == 0x3F80
    assert np.allclose(learned.bf16_float(bits), vals, rtol=2 ** -8)


def test_canonical_labels_break_near_ties_by_prior():
    mse = np.zeros((2, 3, 64), np.uint64)
    mse[:] = 1000000
    mse[0, 0, 10] = 500000
    mse[0, 0, 20] = 500400  # within 0.2 % of the minimum
    mse[0, 1, 10] = 500000
    mse[0, 1, 20] = 520000  # clearly worse
    mse[1, :, 5] = 100
    keep = np.array([True, True, False])
    prior = np.stack([np.r_[20, 10, np.setdiff1d(np.arange(64), [10, 20])], np.arange(64)])
    y = learned.canonical_labels(mse, keep, prior, tie=0.002)
    assert y.shape == (2, 2)
    assert y[0, 0] == 20 and y[1, 0] == 10 and (y[:, 1] == 5).all()


def test_default_labels_follow_the_frame_ranking():
    mse = np.full((2, 3, 64), 1000000, np.uint64)
    # Block 0 prefers 10 by 0.4 %, blocks 1 and 2 prefer 20 by a lot: the
    # frame ranks 20 first, so block 0's near-tie goes to 20.
    mse[0, 0, 10], mse[0, 0, 20] = 500000, 502000
    mse[0, 1, 20], mse[0, 2, 20] = 100000, 100000
    mse[1, :, 7] = 5
    keep = np.ones(3, bool)
    y = learned.canonical_labels(mse, keep, tie=0.01)
    assert (y[:, 0] == 20).all() and (y[:, 1] == 7).all()
    assert learned.canonical_labels(mse, keep, tie=0.001)[0, 0] == 10


def test_argmin_prior_orders_by_frequency():
    mse = np.full((2, 4, 64), 10, np.uint64)
    mse[0, 0, 3] = mse[0, 1, 3] = mse[0, 2, 7] = 1
    mse[1, :, 9] = 1
    keep = np.array([True, True, True, False])
    pr = learned.argmin_prior([(mse, keep)])
    assert pr[0][0] == 3 and pr[0][1] == 7 and pr[1][0] == 9


def test_strength_trial_inverts_the_trial_order():
    def trial_strength(g):
        return g * 4 if g < 16 else ((g - 16) // 3) * 4 + (g - 16) % 3 + 1

    assert [learned.strength_trial(trial_strength(g)) for g in range(64)] == list(range(64))


def test_model_file_round_trip(tmp_path):
    m, _, _ = _rand_model(11, n=16)
    p = tmp_path / "m.bin"
    learned.save_model(m, str(p))
    m2 = learned.load_model(str(p))
    assert bytes(m) == bytes(m2)
    (tmp_path / "bad.bin").write_bytes(b"x" * 100)
    with pytest.raises(ValueError):
        learned.load_model(str(tmp_path / "bad.bin"))


def test_side_info_pickles(oracle):
    fr, si = synth.make_frame(1, 5, width=320, height=192)
    si2 = pickle.loads(pickle.dumps(si))
    outs = []
    for s in (si, si2):
        a, d = fr.copy(), fr.like()
        assert oracle.oracle_frame_apply(C.byref(a.pf()), C.byref(s.side), C.byref(d.pf())) == 0
        outs.append(a.planes + d.planes)
    assert all(np.array_equal(x, y) for x, y in zip(*outs))


def test_features_oracle_invariants(oracle):
    src, rec, side, _ = synth.make_search_pair(21, 200, 130)
    assert oracle.oracle_loop_filter(C.byref(rec.pf()), C.byref(side.side)) == 0
    ns = learned.noskip_of(side, rec)
    nfb = 4 * 3
    X = np.zeros((nfb, F), np.float32)
    assert oracle.oracle_cdef_features(C.byref(rec.pf()), ns.ctypes.data, 128, 0, X.ctypes.data) == 0
    live = X[:, 29] > 0
    assert live.any()
    assert np.allclose(X[live, 0:8].sum(1), 1, atol=1e-5) and np.allclose(X[live, 8:16].sum(1), 1, atol=1e-6)
    assert np.allclose(X[live, 30], 128 / 255) and np.allclose(X[live, 31], (5 - 3) / 3)
    for j, f in enumerate((16, 19, 22, 23, 24, 25, 27)):
        assert np.allclose(X[:, 33 + j], X[live, f].astype(np.float64).mean(), rtol=1e-6)

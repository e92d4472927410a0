"""RT surrogate: the tcgen05 BF16 GEMM it is built from, its forward and backward passes against
the CPU oracle (oracle_mlp: float64 with the same bf16 rounding points), its training on columns
the plain RT logged, and the in-step re-check / fallback against the plain RT."""
import numpy as np
import pytest

import thor_b200
from thorx_testlib import (RT_WASP43B, RefGrid, grid_dict, hot_jupiter_params, initial_state,
                           oracle_mlp, rel_err, thorx_params)

GLEVEL, NV, DT, H = 4, 20, 300.0, 512


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (256, 128, 192), (384, 512, 512)])
def test_tensor_core_gemm_matches_float64(M, N, K):
    rng = np.random.default_rng(M + N + K)
    A = thor_b200.bf16_bits(rng.standard_normal((M, K)))
    B = thor_b200.bf16_bits(rng.standard_normal((N, K)))
    D = thor_b200.bf16_gemm(A, B)
    a = thor_b200.bf16_value(A).astype(np.float64)
    b = thor_b200.bf16_value(B).astype(np.float64)
    ref, scale = a @ b.T, np.abs(a) @ np.abs(b).T
    # FP32 accumulation of K products: a few float32 ulp of sum |a||b|
    assert np.all(np.abs(D - ref) <= 1e-5 * scale), np.max(np.abs(D - ref) / scale)


def make_ctx(**sur):
    p, c = hot_jupiter_params(GLEVEL, DT)
    g = RefGrid(GLEVEL, NV, A=c["A"], top=c["Top_altitude"])
    x = thor_b200.Thorx(grid_dict(g), GLEVEL, thorx_params(c, DT))
    ic = initial_state(g.arrays, g.point_num, NV, c, amp=1.0)
    for k, v in ic.items():
        x.set(k, v)
    x.rt_enable(RT_WASP43B)
    x.sur_create(hidden=H, **sur)
    return x, g


def layers(x):
    return [x.sur_layer(l) for l in range(4)]


@pytest.mark.gpu
def test_forward_matches_oracle():
    x, g = make_ctx(train_batch=256)
    rng = np.random.default_rng(1)
    B = 200  # not a multiple of 128: padding rows
    xin = rng.standard_normal((B, 2 * NV + 1)).astype(np.float32)
    Ls = layers(x)
    # non-zero biases so that they are exercised
    for l in range(4):
        W, b = Ls[l]
        b[: (NV if l == 3 else H)] = rng.standard_normal(NV if l == 3 else H) * 0.1
        x.sur_set_layer(l, W, b)
    Ls = layers(x)
    y = x.sur_forward(xin, NV)
    x.close(), g.close()
    yo, _, _, _ = oracle_mlp(NV, H, [w for w, _ in Ls], [b for _, b in Ls], xin)
    # both sides round the same quantities to bf16; what remains is FP32-vs-FP64 accumulation,
    # which can flip an occasional bf16 rounding of a hidden activation
    assert rel_err(y, yo) <= 2e-3, rel_err(y, yo)


@pytest.mark.gpu
def test_gradients_match_oracle():
    x, g = make_ctx(train_batch=256)
    rng = np.random.default_rng(2)
    B = 256
    xin = rng.standard_normal((B, 2 * NV + 1)).astype(np.float32)
    tgt = rng.standard_normal((B, NV)).astype(np.float32)
    loss = x.sur_gradients(xin, tgt)
    Ls = layers(x)
    grads = [x.sur_grad(l) for l in range(4)]
    x.close(), g.close()
    _, lo, gW, gb = oracle_mlp(NV, H, [w for w, _ in Ls], [b for _, b in Ls], xin, tgt)
    assert abs(loss - lo) <= 1e-4 * lo, (loss, lo)
    for l in range(4):
        eW = np.linalg.norm(grads[l][0] - gW[l]) / np.linalg.norm(gW[l])
        eb = np.linalg.norm(grads[l][1] - gb[l]) / np.linalg.norm(gb[l])
        assert eW <= 5e-3 and eb <= 5e-3, (l, eW, eb)
        # padding stays exactly zero
        if l == 0:
            assert np.all(grads[l][0][:, 2 * NV + 1:] == 0.0)
        if l == 3:
            assert np.all(grads[l][0][NV:, :] == 0.0) and np.all(grads[l][1][NV:] == 0.0)


@pytest.mark.gpu
def test_training_on_logged_columns_and_in_step_use():
    """Log the plain RT over 48 physics steps from a state S0, train on the GPU, then run the
    first 16 of those steps again from S0 twice, with the plain RT and with the surrogate (the
    states the surrogate sees are then of the kind it was trained on). Every column is
    re-checked once per 16 steps, failed re-checks fall back to the plain RT, and the temperature
    change over the 16 steps matches the plain RT's. The gain: the fraction of column-steps the
    expensive RT still runs on."""
    nlog, nuse = 48, 16
    x, g = make_ctx(train_batch=2048, log_capacity=nlog * 2562, recheck_period=16,
                    tolerance=0.05, seed=7)
    N = g.point_num
    fields = ["Rho", "pressure", "Mh", "Wh", "W", "temperature"]
    x.step(4)  # leave the isothermal start
    x.sync()
    s0 = {f: x.get(f) for f in fields}
    x.sur_mode(thor_b200.SUR_LOG)
    x.step(nlog)
    x.sync()
    assert x.sur_logged() == nlog * N
    first, last = x.sur_train(2000, 2048, lr=1e-3)

    def run(mode):
        for f, v in s0.items():
            x.set(f, v)
        x.sur_mode(mode)
        x.sur_stats()
        x.step(nuse)
        x.sync()
        return {f: x.get(f) for f in fields}, x.sur_stats()

    plain, _ = run(thor_b200.SUR_OFF)
    used, st = run(thor_b200.SUR_USE)
    x.close(), g.close()
    rt_fraction = st["rt_columns"] / (nuse * N)
    dT_plain = plain["temperature"] - s0["temperature"]
    dT_used = used["temperature"] - s0["temperature"]
    change_err = np.max(np.abs(dT_used - dT_plain)) / np.max(np.abs(dT_plain))
    print("surrogate: loss %.3g -> %.3g, stats %s, RT fraction %.3f, dT error %.3g"
          % (first, last, st, rt_fraction, change_err))
    assert last < 0.05 * first, (first, last)
    assert st["rechecked"] == N, st  # each column exactly once in 16 steps
    assert st["failed"] <= st["rechecked"]
    for f in fields:
        assert np.all(np.isfinite(used[f])), f
    # surrogate columns are within the tolerance when re-checked; one that drifts out between
    # two re-checks is caught at the next one
    assert change_err < 0.2, change_err
    assert rt_fraction < 0.5, (st, rt_fraction)


@pytest.mark.gpu
def test_surrogate_from_a_state_it_was_not_trained_on():
    """Train on 48 logged plain-RT steps, run 32 more plain steps to a state S1 that was never
    logged, then run 32 steps from S1 three ways: the plain RT (the judge), the surrogate as
    trained, and the surrogate with online learning (THORX_SUR_USE_LOG: the columns the plain RT
    re-checks or falls back to go into the log, and the network trains 200 Adam steps every 8
    physics steps). States the fraction of column-steps the plain RT still ran on and the error of
    the temperature change against the judge's, for both."""
    nlog, nfree, nuse = 48, 32, 32
    x, g = make_ctx(train_batch=2048, log_capacity=nlog * 2562, recheck_period=16,
                    tolerance=0.05, seed=7)
    N = g.point_num
    fields = ["Rho", "pressure", "Mh", "Wh", "W", "temperature"]
    x.step(4)
    x.sur_mode(thor_b200.SUR_LOG)
    x.step(nlog)
    x.sync()
    first, last = x.sur_train(2000, 2048, lr=1e-3)
    x.sur_mode(thor_b200.SUR_OFF)
    x.step(nfree)
    x.sync()
    s1 = {f: x.get(f) for f in fields}
    W0 = [x.sur_layer(l) for l in range(4)]

    def run(mode, online=False):
        for f, v in s1.items():
            x.set(f, v)
        for l, (W, b) in enumerate(W0):  # every run starts from the same trained network
            x.sur_set_layer(l, W, b)
        x.sur_mode(mode)
        x.sur_stats()
        rt_cols, re, fa = 0, 0, 0
        for _ in range(nuse // 8):
            x.step(8)
            x.sync()
            st = x.sur_stats()
            rt_cols, re, fa = rt_cols + st["rt_columns"], re + st["rechecked"], fa + st["failed"]
            if online:
                x.sur_train(200, 2048, lr=2e-4)
        return {f: x.get(f) for f in fields}, rt_cols / (nuse * N), (re, fa)

    plain, _, _ = run(thor_b200.SUR_OFF)
    used, frac_used, st_used = run(thor_b200.SUR_USE)
    online, frac_online, st_online = run(thor_b200.SUR_USE_LOG, online=True)
    x.close(), g.close()
    dT_plain = plain["temperature"] - s1["temperature"]

    def change_err(r):
        return np.max(np.abs((r["temperature"] - s1["temperature"]) - dT_plain)) / np.max(np.abs(dT_plain))

    e_used, e_online = change_err(used), change_err(online)
    print("surrogate from an unlogged state: loss %.3g -> %.3g; as trained: RT fraction %.3f, "
          "re-checks %s, dT error %.3g; online: RT fraction %.3f, re-checks %s, dT error %.3g"
          % (first, last, frac_used, st_used, e_used, frac_online, st_online, e_online))
    for r in (used, online):
        for f in fields:
            assert np.all(np.isfinite(r[f])), f
    assert st_used[0] == 2 * N and st_online[0] == 2 * N  # every column re-checked twice
    # measured on a B200: as trained, every re-check from S1 fails (the network does not
    # generalise beyond the logged states); the plain RT runs on 0.77 of the column-steps and the
    # temperature change is off by 0.25 of itself before the fallbacks catch up. With online
    # learning nearly every column falls back (0.99) and the error stays at 0.06.
    assert e_used < 0.5 and e_online < 0.2, (e_used, e_online)
    assert frac_used < 1.0 and frac_online <= 1.0

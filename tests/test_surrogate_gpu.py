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

"""Tile-scoring MLP: the device forward/backward (BF16 tensor cores, FP32
accumulation; and the FP32 debug path) against the FP64 CPU restatement in
mlp_ref.py, training, prediction and save/load."""
import numpy as np
import pytest

import mlp_ref

pytestmark = pytest.mark.gpu


def _data(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0.0, 1.0, (n, mlp_ref.IN)).astype(np.float32)
    y = (np.sin(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2] + 0.1 * x[:, 3:8].sum(1)).astype(np.float32)
    return x, y


def _rel_err_per_block(g, ref):
    gb, rb = mlp_ref.blocks(g), mlp_ref.blocks(ref)
    return {k: np.linalg.norm(gb[k] - rb[k]) / max(np.linalg.norm(rb[k]), 1e-30) for k in rb}


def test_gradient_fp32_path_matches_fp64(gpu_dtwj):
    net = gpu_dtwj.MLP(seed=7)
    x, y = _data(777, 1)  # not a multiple of the 16-row tiles
    ref, ref_loss = mlp_ref.grad(net.params, x, y)
    g, loss = net.grad(x, y, precise=True)
    errs = _rel_err_per_block(g, ref)
    assert max(errs.values()) <= 1e-4, errs
    assert loss == pytest.approx(ref_loss, rel=1e-4)


def test_gradient_bf16_path_matches_fp64(gpu_dtwj):
    # the tensor-core path rounds every GEMM operand to bfloat16: against the
    # FP64 gradient with the same operands rounded, it must agree to 1e-2
    # (in practice to FP32 accumulation error); against unrounded FP64 math
    # the rounding itself shows (a few percent on the first layer)
    net = gpu_dtwj.MLP(seed=7)
    x, y = _data(777, 1)
    p = net.params
    g, loss = net.grad(x, y, precise=False)
    ref_b, loss_b = mlp_ref.grad(p, x, y, bf16_operands=True)
    errs_b = _rel_err_per_block(g, ref_b)
    assert max(errs_b.values()) <= 1e-2, errs_b
    assert loss == pytest.approx(loss_b, rel=1e-3)
    ref, _ = mlp_ref.grad(p, x, y)
    errs = _rel_err_per_block(g, ref)
    assert max(errs.values()) <= 1e-1, errs


def test_training_reduces_the_loss_and_predicts_like_the_reference(gpu_dtwj, tmp_path):
    net = gpu_dtwj.MLP(seed=3)
    x, y = _data(20000, 2)
    xt, yt = _data(2000, 3)
    before = float(np.mean((net.predict(xt) - yt) ** 2))
    last = net.train(x, y, epochs=8, batch=1024, lr=2e-3, seed=5)
    after = float(np.mean((net.predict(xt) - yt) ** 2))
    assert last < 0.2 * float(np.var(y)) and after < 0.3 * before, (before, after, last)
    # device inference (BF16 operands) against the FP64 forward of the same weights
    ref = mlp_ref.forward(net.params, xt)[0]
    np.testing.assert_allclose(net.predict(xt), ref, rtol=0, atol=5e-2 * np.std(ref) + 1e-3)
    path = str(tmp_path / "tile_mlp.bin")
    net.save(path)
    net2 = gpu_dtwj.MLP.load_file(path)
    np.testing.assert_array_equal(net2.params, net.params)
    np.testing.assert_array_equal(net2.predict(xt), net.predict(xt))

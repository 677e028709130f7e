"""The seed network: its CPU reference against finite differences, the library's
gradients against that reference, training on pairs from the exact evaluator, and
what its Newton starts gain over the sub-patch-centre start with the same answers."""
import numpy as np
import pytest

from implicitcam_b200 import part_gpu, parts

import seednet_ref as ref


def random_theta(seed):
    rng = np.random.default_rng(seed)
    th = rng.normal(0, 0.3, ref.N_PARAMS)
    p = ref.unpack(th)
    p["W1"][19:] = 0  # padded inputs
    p["W4"][:, 3:] = 0  # padded outputs
    return ref.pack(p)


def test_reference_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    th = random_theta(1)
    x = np.zeros((7, 32))
    x[:, :19] = rng.normal(0, 1, (7, 19))
    y = np.c_[rng.uniform(0, 1, (7, 2)), rng.uniform(0, 0.5, 7), np.ones(7)]
    loss, g = ref.loss_and_grad(th, x, y)
    idx = rng.choice(ref.N_PARAMS, 200, replace=False)
    for i in idx:
        e = np.zeros_like(th)
        e[i] = 1e-6
        fd = (ref.loss_only(th + e, x, y) - ref.loss_only(th - e, x, y)) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * (1 + abs(fd)), i
    assert abs(loss - ref.loss_only(th, x, y)) < 1e-12


@pytest.fixture(scope="module")
def freeform():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    g = part_gpu.PartGpu(parts.freeform_top(seed=0))
    yield g
    g.close()


@pytest.mark.gpu
def test_samples_are_exact_feet(freeform):
    x, y = freeform.seednet_samples(4096, seed=5)
    assert np.isfinite(x).all() and np.isfinite(y).all()
    assert (x[:, 19:] == 0).all()
    assert (y[:, :2] >= 0).all() and (y[:, :2] <= 1).all() and (y[:, 3] == 1).all()
    assert (y[:, 2] >= 0).all()


@pytest.mark.gpu
def test_gradients_match_the_cpu_reference(freeform):
    th = random_theta(2).astype(np.float32)
    freeform.seednet_params(th)
    x, y = freeform.seednet_samples(1000, seed=9)
    g, loss = freeform.seednet_grad(x, y)
    rl, rg = ref.loss_and_grad(th.astype(np.float64), x, y)
    assert abs(loss - rl) <= 1e-4 * (1 + abs(rl))
    scale = np.abs(rg).max()
    assert np.abs(g - rg).max() <= 2e-4 * scale, np.abs(g - rg).max() / scale


@pytest.mark.gpu
def test_training_lowers_the_loss_and_the_seeds_save_newton_steps(freeform):
    loss = freeform.seednet_train(1500, batch=4096, seed=11, lr=2e-3)
    first, last = loss[:50].mean(), loss[-50:].mean()
    assert last < 0.2 * first, (first, last)
    ab = freeform.seednet_ab(1 << 16, seed=12)
    # the net's starts converge in fewer steps than the centre's, to the same feet
    assert ab["mean_iters_net"] < ab["mean_iters_centre"] - 0.5, ab
    assert ab["fallback_rate"] < 0.01, ab
    assert ab["pairs_differing"] <= 1e-3 * ab["pairs"], ab

"""The learned warm start of the saturation adjustment.

* the GPU training kernels' gradient equals the oracle's FP64 gradient
  (relative 1e-4: FP32 accumulation);
* FP32 inference matches the oracle's forward pass; the BF16 tensor-core
  inference stays within 2e-2 of it (normalised units);
* a trained network reproduces the converged temperature to ~1 K;
* the learned solve returns the plain solve's answer (T to 1e-9 K, species
  to 1e-12 relative) and needs fewer evaluations of the energy residual --
  what the network gains (printed);
* the gated start on the GPU equals the oracle's gated start given the
  GPU's guesses.
"""
import numpy as np
import pytest

from canoe_b200 import learned, thermo

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def th():
    return thermo.earth_moist()


@pytest.fixture(scope="module")
def net(th):
    return learned.train_warm_start(th, n=1 << 20, epochs=30, batch=4096)


def test_gradient_matches_oracle(oracle_mod):
    rng = np.random.Generator(np.random.PCG64(1))
    netr = learned.WarmStartNet(seed=3)
    p = netr.params().astype(np.float64)
    x = rng.standard_normal((4096, 4)).astype(np.float32)
    y = rng.standard_normal(4096).astype(np.float32)
    loss, g = netr.loss_grad(x, y)
    lref, gref = oracle_mod.mlp_loss_grad(p, 64, x.astype(np.float64), y.astype(np.float64))
    assert abs(loss - lref) <= 1e-5 * abs(lref)
    assert np.linalg.norm(g - gref) <= 1e-4 * np.linalg.norm(gref)


def test_inference_fp32_and_tensor_core(oracle_mod):
    rng = np.random.Generator(np.random.PCG64(2))
    netr = learned.WarmStartNet(seed=5)
    p = netr.params().astype(np.float64)
    x = rng.standard_normal((5000, 4)).astype(np.float32)
    ref = oracle_mod.mlp_forward(p, 64, x.astype(np.float64))
    y32 = netr.forward(x, tensor_core=False)
    ytc = netr.forward(x, tensor_core=True)
    assert np.max(np.abs(y32 - ref)) < 1e-4
    assert np.max(np.abs(ytc - ref)) < 2e-2


def test_training_fits_converged_temperature(th, net):
    x, T = learned.training_pairs(th, 1 << 16, seed=99)
    err = learned.predict(net, th, x) - T
    assert np.sqrt(np.mean(err ** 2)) < 0.3, np.sqrt(np.mean(err ** 2))


def test_learned_solve_same_answer_fewer_evaluations(th, net):
    u = learned.perturbed_states(th, 1 << 16, seed=31)
    uc, Tc, itc, stc, _ = learned.satadj_gpu(th, u, mode=0)
    ul, Tl, itl, stl, guess = learned.satadj_gpu(th, u, mode=2, net=net)
    assert np.max(np.abs(Tl - Tc)) < 1e-9
    scale = np.abs(uc[1:4]).max()
    assert np.max(np.abs(ul[1:4] - uc[1:4])) <= 1e-12 * scale
    assert stc[3] == 0 and stl[3] == 0
    sat = uc[2] + uc[3] > 0  # cells that end with condensate
    assert sat.sum() > 1000
    print(f"evaluations of f per cell: cold {itc.mean():.3f} learned {itl.mean():.3f}; "
          f"saturated cells cold {itc[sat].mean():.3f} learned {itl[sat].mean():.3f}")
    assert itl[sat].mean() < itc[sat].mean(), (itl[sat].mean(), itc[sat].mean())
    assert itl.mean() < itc.mean()


def test_gated_start_matches_oracle(th, net, oracle_mod):
    u = learned.perturbed_states(th, 20000, seed=41)
    ul, Tl, itl, _, guess = learned.satadj_gpu(th, u, mode=2, net=net)
    ref = u.copy()
    Tr, itr, _ = oracle_mod.satadj(th, ref, t_guess=guess, mode=2)
    assert np.max(np.abs(Tl - Tr)) < 1e-9
    # cells that stay all vapour end at their first evaluation
    run = itl > 1
    assert (ref[2][~run] == 0).all() and (ref[3][~run] == 0).all()
    assert (itl[run] == itr[run]).mean() > 0.99

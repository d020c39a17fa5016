"""Learned Newton guess: device forward/backward vs the CPU oracle, training,
and what the trained network gains over the guess without it."""

import numpy as np
import pytest
import torch

from mirgecom_b200.eos import PyrometheusMixture
from mirgecom_b200.fluid import ConservedVars
from mirgecom_b200.gas_model import GasModel, make_fluid_state
from mirgecom_b200.learned_guess import TemperatureMLP
from mirgecom_b200.thermochemistry import UIUC_7SP
from oracle import mlp as omlp

pytestmark = pytest.mark.gpu


def _batch(cuda, n=4096, seed=1):
    e, y, t = TemperatureMLP.training_pairs(UIUC_7SP, n, cuda, seed=seed)
    return e, y, t


def test_device_gradient_matches_oracle(cuda):
    net = TemperatureMLP(cuda, seed=3)
    e, y, t = _batch(cuda)
    net.set_normalisation(e, y)
    x = net.features(e, y)
    tn = ((t.float() - net.out_shift) / net.out_scale).contiguous()
    loss, grad = net.loss_and_grad(x, tn)
    p = net.numpy_params()
    ref_loss, ref = omlp.loss_and_grad(p, x.cpu().numpy().astype(np.float64),
                                       tn.cpu().numpy().astype(np.float64), emulate_bf16=True)
    assert abs(float(loss.item()) - ref_loss) <= 1e-4 * ref_loss
    g = grad.cpu().numpy().astype(np.float64)
    from mirgecom_b200 import learned_guess as lg
    dev = {"w1": g[lg.P_W1:lg.P_B1].reshape(64, 16)[:, :8], "b1": g[lg.P_B1:lg.P_W2],
           "w2": g[lg.P_W2:lg.P_B2].reshape(64, 64), "b2": g[lg.P_B2:lg.P_W3],
           "w3": g[lg.P_W3:lg.P_B3], "b3": g[lg.P_B3]}
    for k in ref:
        err = np.linalg.norm(np.ravel(dev[k] - ref[k])) / np.linalg.norm(np.ravel(ref[k]))
        assert err < 2e-3, (k, err)


def test_training_and_iteration_gain(cuda):
    net = TemperatureMLP(cuda, seed=0)
    e, y, t = TemperatureMLP.training_pairs(UIUC_7SP, 1 << 18, cuda, seed=0)
    hist = net.fit(e, y, t, steps=1500, batch=32768, lr=3e-3)
    assert hist[-1] < 0.05 * hist[0]
    # held-out states, as a conserved state (rho = 1, at rest)
    e2, y2, t2 = TemperatureMLP.training_pairs(UIUC_7SP, 20000, cuda, seed=9)
    q = torch.cat([torch.ones_like(e2)[None], e2[None], torch.zeros((3, e2.numel()),
                  dtype=torch.float64, device=cuda), y2]).float().contiguous()
    cv = ConservedVars(q, 3)
    guess = net.predict(cv)
    rms = float(((guess.double() - t2) ** 2).mean().sqrt())
    assert rms < 60.0, rms
    # device inference against the oracle forward with the same weights
    p = net.numpy_params()
    x = net.features(e2, y2).cpu().numpy().astype(np.float64)
    ref = net.out_shift + net.out_scale * omlp.forward(p, x, emulate_bf16=True)["y"]
    # inference evaluates tanh with tanh.approx.f16x2 (about 2^-11 relative
    # error per activation, which also moves some bf16 roundings of the
    # layer-1 activations by one step), and the device derives the features
    # from the float32 state, the oracle from float64 (e, Y): a few kelvin at
    # most, against the hundreds of kelvin a fragment-layout error would give
    d = np.abs(guess.cpu().numpy() - ref)
    assert np.quantile(d, 0.99) < 5.0 and d.max() < 25.0, (np.quantile(d, 0.99), d.max())
    # Newton iterations: reference default cold guess (300 K) vs learned guess
    gas_plain = GasModel(eos=PyrometheusMixture(UIUC_7SP))
    gas_learn = GasModel(eos=PyrometheusMixture(UIUC_7SP, learned_guess=net))
    cold = torch.full_like(t2, 300.0)
    it_plain = torch.zeros(q[0].shape, dtype=torch.int32, device=cuda)
    it_learn = torch.zeros_like(it_plain)
    tp = make_fluid_state(cv, gas_plain, temperature_seed=cold,
                          newton_iterations=it_plain).temperature
    tl = make_fluid_state(cv, gas_learn, temperature_seed=cold,
                          newton_iterations=it_learn).temperature
    ok_p = it_plain < 1000
    ok_l = it_learn < 1000
    assert bool(ok_l.all())
    mean_plain = float(it_plain.float().mean())
    mean_learn = float(it_learn.float().mean())
    assert mean_learn < mean_plain, (mean_learn, mean_plain)
    both = ok_p & ok_l
    assert float(((tp - tl).abs() / tl)[both].max()) < 2e-6
    assert float(((tl.double() - t2).abs() / t2).max()) < 2e-6
    # seeds within one small Newton step (time marching): every warp skips
    # the network (+100 marker) and the temperatures are those of the plain
    # solve from the same seeds
    warm = t2 + 1.0
    it_w = torch.zeros_like(it_plain)
    it_wp = torch.zeros_like(it_plain)
    tw = make_fluid_state(cv, gas_learn, temperature_seed=warm,
                          newton_iterations=it_w).temperature
    twp = make_fluid_state(cv, gas_plain, temperature_seed=warm,
                           newton_iterations=it_wp).temperature
    assert bool(((it_w >= 100) & (it_w < 1000)).all())
    assert float((it_w - 100 != it_wp).float().mean()) < 1e-3
    assert float(((tw - twp).abs() / twp).max()) < 2e-6

"""The learned FWI preconditioner end to end on a small layered case: pairs
from the Born operators, training on the GPU kernels, and what the trained
network gains over the plain gradient.

* On held-out perturbations, the Born data of the learned update fit those of
  the true perturbation better than the data of the gradient do (each at its
  best scale: the exact Born residual decides).
* In FWI from a perturbed start, L-BFGS with learned steps (each accepted only
  when the exact misfit drops) reaches a lower misfit in the same number of
  iterations than plain L-BFGS."""
import numpy as np
import pytest

from elastic_isotropic_operators_b200 import fwi, precond, prop, synthetic

pytestmark = pytest.mark.gpu


def _setup(nts=450):
    # 0.45 s records the reflections of the whole 400 m deep interior
    w = synthetic.small(nts=nts, nshots=6)
    src, rec = w.geometry()
    sig = w.source_signal()
    nl = prop.nonlinearFwiPropElasticShotsGpu(w.elastic, w.par, sig[None], *src, *rec)
    born = prop.BornElasticShotsGpu(w.elastic, w.par, [sig], *src, *rec)
    return w, nl, born


def _start(true, seed=11):
    rng = np.random.default_rng(seed)
    nx, nz = true.shape[1:]
    interior = (16, nx - 16, 16, nz - 16)
    m0 = true.copy()
    for c in range(3):
        f = precond.smooth_perturbation((nx, nz), rng, 4.0, interior)
        m0[c] *= (1.0 - 0.02 * f)
    return m0


def _data_residual(born, dm_hat, dm):
    """Relative Born data residual of the best multiple of dm_hat:
    min_a ||a J dm_hat - J dm|| / ||J dm|| (the line search picks a)."""
    shape = born.dataSpace().getNdArray().shape
    d_hat, d = np.zeros(shape, np.float32), np.zeros(shape, np.float32)
    born.forward(False, np.ascontiguousarray(dm_hat, np.float32), d_hat)
    born.forward(False, np.ascontiguousarray(dm, np.float32), d)
    a64, b64 = d_hat.ravel().astype(np.float64), d.ravel().astype(np.float64)
    a = (a64 @ b64) / (a64 @ a64)
    return np.linalg.norm(a * a64 - b64) / np.linalg.norm(b64)


def test_learned_update_beats_the_scaled_gradient_on_held_out_perturbations():
    """Judged by the exact Born residual: the data of the learned update fit the
    data of the true perturbation better than those of the gradient (each at
    its best scale)."""
    w, nl, born = _setup()
    m0 = w.elastic.getNdArray().copy()
    P = precond.LearnedPreconditioner(born, m0, sigma=3.0, seed=0)
    X, T, _, _ = P.make_pairs(64, seed=1)
    hist = P.train(X, T, epochs=60, batch=8, lr=3e-3)
    print("training loss", hist[0], hist[len(hist) // 2], hist[-1])
    assert hist[-1] < 0.9 * hist[0], hist
    _, _, _, Dh = P.make_pairs(6, seed=99)
    res_net, res_g = [], []
    for k in range(6):
        g = P._normal(Dh[k])
        res_net.append(_data_residual(born, P.predict(g), Dh[k]))
        res_g.append(_data_residual(born, g, Dh[k]))
    print("held-out Born residual: learned", np.mean(res_net), "gradient", np.mean(res_g))
    assert np.mean(res_net) < 0.9 * np.mean(res_g), (res_net, res_g)


def test_fwi_with_learned_steps_reaches_a_lower_misfit():
    w, nl, born = _setup()
    true = w.elastic.getNdArray().copy()
    d = nl.dataSpace()
    nl.forward(False, true, d)
    d_obs = d.getNdArray().copy()
    m0 = _start(true)
    obj = fwi.FwiObjective(nl, born, d_obs)
    niter = 4
    _, plain = fwi.lbfgs(obj, m0, niter=niter, scale=m0)
    P = precond.LearnedPreconditioner(born, m0, sigma=4.0, seed=0)
    X, T, _, _ = P.make_pairs(64, seed=2)
    P.train(X, T, epochs=60, batch=8, lr=3e-3)
    stats = {}
    _, learned = fwi.lbfgs(obj, m0, niter=niter, scale=m0, precond=P, stats=stats)
    print("plain", plain, "learned", learned, stats)
    assert stats["learned"] >= 1, stats
    assert learned[-1] < plain[-1], (learned, plain)


def test_unet_preconditioner_learns_the_normal_operator_inverse():
    """The four-level U-Net in the same role (grids off its size multiple of
    8 are padded for the network and cut back): trained on Born pairs, its
    update fits held-out perturbations' data better than the gradient does."""
    w, nl, born = _setup()
    m0 = w.elastic.getNdArray().copy()
    P = precond.LearnedPreconditioner(born, m0, sigma=3.0, seed=0, arch="unet")
    assert isinstance(P.net, precond.UNet)
    X, T, _, _ = P.make_pairs(64, seed=1)
    hist = P.train(X, T, epochs=60, batch=8, lr=1e-3)
    print("U-Net training loss", hist[0], hist[len(hist) // 2], hist[-1])
    assert hist[-1] < 0.9 * hist[0], hist
    _, _, _, Dh = P.make_pairs(6, seed=99)
    res_net, res_g = [], []
    for k in range(6):
        g = P._normal(Dh[k])
        dm_hat = P.predict(g)
        assert dm_hat.shape == g.shape
        res_net.append(_data_residual(born, dm_hat, Dh[k]))
        res_g.append(_data_residual(born, g, Dh[k]))
    print("held-out Born residual: U-Net", np.mean(res_net), "gradient", np.mean(res_g))
    assert np.mean(res_net) < 0.9 * np.mean(res_g), (res_net, res_g)

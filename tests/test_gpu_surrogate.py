"""GPU checks of the learned surrogate: site features against the CPU oracle,
the training kernels' parameter gradient against the numpy reference, a
training run that lowers the loss, the fused surrogate site energies against
the numpy ensemble on oracle features, forces against finite differences of
the surrogate energy, exact agreement with plain ACE when every site falls
back (tau = 0), and a speed gain over plain ACE."""
import dataclasses
import time

import numpy as np
import pytest

from oracle import oracle as O
from pfw_b200 import ace_generate as G
from pfw_b200 import lib
from pfw_b200 import surrogate as S
from pfw_b200 import workloads as WL
from pfw_b200.ace_model import read_resolved

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def models():
    m = read_resolved(G.generate_b2_model())
    feat, sel = S.restrict_model(m)
    return m, feat, sel


@pytest.fixture(scope="module")
def trained(models):
    m, feat, sel = models
    h = lib.Handle(lib.FP64)
    X, E, Z = S.training_set(h, m, feat, n_lattices=4, nc=6, seed=31)
    sur = S.train(h, feat, sel, X, E, Z, epochs=30, batch=256, lr=3e-3, lr_final=1e-4, seed=5)
    return sur, (X, E, Z)


def test_site_features_match_oracle(models):
    m, feat, sel = models
    s = WL.b2(seed=2, nc=4, sigma=0.12)
    h = lib.Handle(lib.FP64)
    h.surrogate(feat)
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    f = h.surrogate_features()
    r = O.AceOracle(feat).evaluate(s.X, s.H, s.pbc, s.species, request=1, features=True)["features"]
    nz, nb, nQ = feat.nz, feat.nbasis, feat.pair.nchannels
    for i, z in enumerate(s.species):
        ref = np.concatenate([r[i, z * nb:(z + 1) * nb], r[i, nz * nb + z * nQ:nz * nb + (z + 1) * nQ]])
        assert np.allclose(f[i], ref, rtol=1e-10, atol=1e-10)


def test_param_grad_matches_numpy():
    nz, M, nin, H = 2, 2, 64, S.HIDDEN
    P = S.init_params(nz, M, nin, H, seed=9)
    rng = np.random.default_rng(4)
    P += rng.normal(0, 0.01, P.shape).astype(np.float32)  # nonzero biases
    n = 150
    X = rng.normal(size=(n, nin)).astype(np.float32)
    y = rng.normal(size=n).astype(np.float32)
    Z = (np.arange(n) % 3 == 0).astype(np.int32)
    h = lib.Handle(lib.FP64)
    loss, grad = h.mlp_param_grad(P, X, y, Z)
    for z in range(nz):
        idx = Z == z
        for m in range(M):
            l_ref, g_ref = S.mlp_param_grad_reference(P[z, m].astype(np.float64), X[idx].astype(np.float64),
                                                      y[idx].astype(np.float64), nin, H)
            assert abs(loss[z, m] - l_ref) <= 1e-4 * l_ref
            assert np.abs(grad[z, m] - g_ref).max() <= 1e-4 * np.abs(g_ref).max()


def test_training_lowers_loss(trained):
    sur, _ = trained
    h = sur.history
    assert h[-1] < 0.5 * h[0]


def ungated(sur):
    return dataclasses.replace(sur, x_lo=np.full_like(sur.x_lo, -np.inf), x_hi=np.full_like(sur.x_hi, np.inf),
                               tau=np.inf)


def test_surrogate_energies_match_numpy_ensemble(models, trained):
    m, feat, _ = models
    sur, _ = trained
    s = WL.b2(seed=40, nc=4, sigma=0.1)
    h = lib.Handle(lib.FP64)
    h.ace(m)
    h.surrogate(feat, ungated(sur))
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    E, F, W = h.evaluate(lib.MODEL_SURROGATE, 7)
    es = h.site_energies()
    r = O.AceOracle(feat).evaluate(s.X, s.H, s.pbc, s.species, request=1, features=True)["features"]
    nz, nb, nQ = feat.nz, feat.nbasis, feat.pair.nchannels
    f = np.array([np.concatenate([r[i, z * nb:(z + 1) * nb], r[i, nz * nb + z * nQ:nz * nb + (z + 1) * nQ]])
                  for i, z in enumerate(s.species)])
    e_ref, _, _ = sur.predict(f, s.species)
    e_ref = e_ref + feat.reference[s.species]
    assert np.abs(es - e_ref).max() <= 1e-5 * max(1.0, np.abs(e_ref).max())
    assert abs(E - es.sum()) <= 1e-9 * abs(E)
    fb, n = h.surrogate_stats()
    assert n == len(s.species) and fb == 0


def test_surrogate_forces_are_energy_gradients(models, trained):
    m, feat, _ = models
    sur, _ = trained
    s = WL.b2(seed=41, nc=2, sigma=0.1)
    h = lib.Handle(lib.FP64)
    h.ace(m)
    h.surrogate(feat, ungated(sur))
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    E, F, W = h.evaluate(lib.MODEL_SURROGATE, 7)
    step = 1e-3
    for i in range(0, len(s.species), 3):
        for a in range(3):
            Xp, Xm = s.X.copy(), s.X.copy()
            Xp[i, a] += step
            Xm[i, a] -= step
            h.set_geometry(Xp, s.H, s.pbc, s.species)
            ep = h.evaluate(lib.MODEL_SURROGATE, 1)[0]
            h.set_geometry(Xm, s.H, s.pbc, s.species)
            em = h.evaluate(lib.MODEL_SURROGATE, 1)[0]
            fd = -(ep - em) / (2 * step)
            assert abs(fd - F[i, a]) <= 2e-3 + 2e-3 * abs(F[i, a]), (i, a, fd, F[i, a])


def test_full_fallback_equals_ace(models, trained):
    m, feat, _ = models
    sur, _ = trained
    s = WL.b2(seed=42, nc=4, sigma=0.1)
    h = lib.Handle(lib.FP64)
    h.ace(m)
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    E0, F0, W0 = h.evaluate(lib.MODEL_ACE, 7)
    h.surrogate(feat, sur, tau=0.0)
    E1, F1, W1 = h.evaluate(lib.MODEL_SURROGATE, 7)
    fb, n = h.surrogate_stats()
    assert fb == n
    assert E1 == E0 and np.array_equal(F1, F0) and np.array_equal(W1, W0)


def test_gate_flags_out_of_range_sites(models, trained):
    m, feat, _ = models
    sur, _ = trained
    # a strongly compressed cell leaves the training range: every site falls back
    s = WL.b2(seed=43, nc=4, sigma=0.05, a=2.3)
    h = lib.Handle(lib.FP64)
    h.ace(m)
    h.surrogate(feat, sur)
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    E1, F1, _ = h.evaluate(lib.MODEL_SURROGATE, 7)
    fb, n = h.surrogate_stats()
    assert fb == n
    E0, F0, _ = h.evaluate(lib.MODEL_ACE, 7)
    assert E1 == E0 and np.array_equal(F1, F0)


def test_surrogate_faster_than_ace(models, trained):
    m, feat, _ = models
    sur, _ = trained
    s = WL.b2(seed=44, nc=16, sigma=0.08)
    h = lib.Handle(lib.FP64)
    h.ace(m)
    h.surrogate(feat, ungated(sur))
    h.set_geometry(s.X, s.H, s.pbc, s.species)

    def best(model):
        h.evaluate(model, 7)
        ts = []
        for _ in range(3):
            t = time.perf_counter()
            h.evaluate(model, 7)
            ts.append(time.perf_counter() - t)
        return min(ts)

    assert best(lib.MODEL_ACE) > 1.5 * best(lib.MODEL_SURROGATE)


def test_mixed_surrogate_matches_fp64_surrogate(models, trained):
    """A mixed workspace runs the surrogate's two site passes in FP32: the
    same surrogate energies and forces as the FP64 workspace to FP32
    accuracy (far below the surrogate's own error against ACE)."""
    m, feat, _ = models
    sur, _ = trained
    s = WL.b2(seed=45, nc=4, sigma=0.1)
    out = {}
    for prec in (lib.FP64, lib.MIXED):
        h = lib.Handle(prec)
        h.ace(m)
        h.surrogate(feat, ungated(sur))
        h.set_geometry(s.X, s.H, s.pbc, s.species)
        out[prec] = h.evaluate(lib.MODEL_SURROGATE, 7)
    (E64, F64, W64), (E32, F32, W32) = out[lib.FP64], out[lib.MIXED]
    assert abs(E32 - E64) <= 1e-5 * max(1.0, abs(E64))
    assert float(np.sqrt(np.mean((F32 - F64) ** 2))) <= 1e-4
    assert float(np.abs(W32 - W64).max()) <= 1e-4 * max(1.0, float(np.abs(W64).max()))

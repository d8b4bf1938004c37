"""GPU checks of the surrogate's energy + force training: the kernel's
energy + force gradient and the members' input gradients against the FP64
numpy reference, the feature pull-back against central differences of a
linear function of the features, and force training on B2 lattices
(displacements 0.03-0.25 Å) that lowers the held-out force RMSE against plain
ACE by at least a quarter relative to the energy-only ensemble it starts
from, and meets the 2e-2 eV/Å bar on the small-displacement lattice.  (The
64 order-1/2 features cannot carry the model's order-3 part, which holds
most of its site-energy variation, so the larger displacements stay above
that bar without fallback.)  The gate calibrated on force error
(surrogate.calibrate_gate) then brings the pooled held-out force RMSE to
2e-2 eV/Å or below with part of the sites falling back to plain ACE."""
import ctypes
import dataclasses

import numpy as np
import pytest

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


def test_ef_gradient_and_input_gradient_match_numpy():
    import torch
    nz, M, nin, H = 2, 2, 64, S.HIDDEN
    rng = np.random.default_rng(8)
    P = S.init_params(nz, M, nin, H, seed=2) + rng.normal(0, 0.01, (nz, M, S.nparams(nin, H))).astype(np.float32)
    n = 150
    X = rng.normal(size=(n, nin)).astype(np.float32)
    y = rng.normal(size=n).astype(np.float32)
    V = rng.normal(size=(M, n, nin)).astype(np.float32)
    c = rng.normal(size=n).astype(np.float32)
    Z = (np.arange(n) % 3 == 0).astype(np.int32)
    h = lib.Handle(lib.FP64)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)  # the library and the tensors in one stream (not handle 0)
    h.set_stream(ctypes.c_void_p(stream.cuda_stream))
    with torch.cuda.stream(stream):
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        shape = S.pfw_mlp_shape(nz, M, nin, H)
        Pd = t(P)
        grad = torch.zeros_like(Pd)
        h.mlp_ef_step(shape, Pd, None, None, t(X), t(y), Z, t(V), t(c), wE=0.8, lr=0.0, step=1, grad=grad)
        Gd = torch.zeros((M, n, nin), dtype=torch.float32, device=dev)
        h.mlp_input_grad(shape, Pd, t(X), Z, Gd)
        grad, Gh = grad.cpu().numpy(), Gd.cpu().numpy()
    h.set_stream(None)
    for z in range(nz):
        idx = Z == z
        for m in range(M):
            p64 = P[z, m].astype(np.float64)
            g_ref = S.mlp_ef_grad_reference(p64, X[idx].astype(np.float64), y[idx].astype(np.float64),
                                            V[m][idx].astype(np.float64), c[idx].astype(np.float64), 0.8, nin, H)
            assert np.abs(grad[z, m] - g_ref).max() <= 1e-4 * np.abs(g_ref).max()
            _, dydx = S.mlp_forward(p64, X[idx].astype(np.float64), nin, H)
            assert np.abs(Gh[m][idx] - dydx).max() <= 1e-4 * np.abs(dydx).max()


def test_pullback_is_minus_gradient_of_linear_feature_energy(models):
    # E(r) = Σ_i w_i·x_i(r) with fixed w: the pull-back of w is -∂E/∂r
    import torch
    m, feat, _ = models
    s = WL.b2(seed=6, nc=3, sigma=0.15)
    h = lib.Handle(lib.FP64)
    h.surrogate(feat)
    rng = np.random.default_rng(1)
    w = rng.normal(size=(len(s), S.NIN))
    dev = torch.device("cuda", 0)
    F = torch.zeros((len(s), 3), dtype=torch.float64, device=dev)
    wd = torch.from_numpy(w).to(dev)
    torch.cuda.synchronize()  # the library runs on its own stream
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    h.surrogate_pullback(wd, F)
    F = F.cpu().numpy()

    def energy(X):
        h.set_geometry(X, s.H, s.pbc, s.species)
        return float(np.sum(w * h.surrogate_features()))

    eps = 1e-5
    for k in (0, 5, 17, len(s) - 1):
        for a in range(3):
            Xp, Xm = s.X.copy(), s.X.copy()
            Xp[k, a] += eps
            Xm[k, a] -= eps
            fd = -(energy(Xp) - energy(Xm)) / (2 * eps)
            assert abs(F[k, a] - fd) <= 1e-6 * max(1.0, abs(fd)), (k, a, F[k, a], fd)


def ungated(sur):
    """The surrogate alone: no feature-range or ensemble gate, so no site falls back."""
    return dataclasses.replace(sur, x_lo=np.full_like(sur.x_lo, -np.inf), x_hi=np.full_like(sur.x_hi, np.inf),
                               tau=np.inf)


def test_force_training_lowers_the_force_error(models):
    m, feat, sel = models
    h = lib.Handle(lib.FP64)
    lat = S.force_training_set(h, m, feat, n_lattices=8, nc=10, seed=41)
    X = np.concatenate([L["X"] for L in lat])
    E = np.concatenate([L["E"] for L in lat])
    Z = np.concatenate([L["Z"] for L in lat])
    sur = S.train(h, feat, sel, X, E, Z, epochs=40, batch=512, lr=2e-3, lr_final=2e-5, seed=5)

    def force_rmse(s_, systems):
        ho = lib.Handle(lib.FP64)
        ho.ace(m)
        ho.surrogate(feat, ungated(s_))
        out = []
        for sy in systems:
            ho.set_geometry(sy.X, sy.H, sy.pbc, sy.species)
            _, Fa, _ = ho.evaluate(lib.MODEL_ACE, 7)
            _, Fs, _ = ho.evaluate(lib.MODEL_SURROGATE, 7)
            out.append(float(np.sqrt(np.mean((Fs - Fa) ** 2))))
        return np.array(out)

    held_out = [WL.b2(seed=900 + k, nc=10, sigma=sg) for k, sg in enumerate((0.03, 0.1, 0.17, 0.25))]
    before = force_rmse(sur, held_out)
    h.surrogate(feat)
    hist = S.train_forces(h, sur, lat, epochs=30)
    after = force_rmse(sur, held_out)
    print("held-out force rmse by displacement, energy-only", before, "energy + force", after)
    assert hist[-1][1] < 0.9 * hist[0][1]
    rms = lambda a: float(np.sqrt(np.mean(a ** 2)))
    assert rms(after) <= 0.75 * rms(before), (before, after)
    assert after[0] <= 2e-2, (before, after)

    # the gate calibrated on force error (other held-out lattices over the same sigma range): with
    # its fallback the pooled held-out force RMSE meets 2e-2 eV/Å while some sites stay surrogate
    calib = [WL.b2(seed=800 + k, nc=10, sigma=sg) for k, sg in enumerate((0.03, 0.1, 0.17, 0.25))]
    curve = S.calibrate_gate(h, sur, m, feat, calib, target=1.8e-2)
    assert curve[-1]["force_rmse"] <= 1.8e-2 and curve[0]["force_rmse"] > 1.8e-2
    ho = lib.Handle(lib.FP64)
    ho.ace(m)
    ho.surrogate(feat, sur)
    se = cnt = fb = ns = 0
    for sy in held_out:
        ho.set_geometry(sy.X, sy.H, sy.pbc, sy.species)
        _, Fa, _ = ho.evaluate(lib.MODEL_ACE, 7)
        _, Fs, _ = ho.evaluate(lib.MODEL_SURROGATE, 7)
        f, n = ho.surrogate_stats()
        se += float(np.sum((Fs - Fa) ** 2))
        cnt += Fs.size
        fb += f
        ns += n
    pooled, frac = float(np.sqrt(se / cnt)), fb / ns
    print("calibrated gate: tau", sur.tau, "pooled held-out force rmse", pooled, "fallback fraction", frac)
    assert pooled <= 2e-2, (pooled, frac)
    assert 0.05 < frac < 0.9, (pooled, frac)

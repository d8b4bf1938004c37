"""Host side of the learned surrogate: the restricted feature model reproduces
the selected invariants and pair sums of the full ACE model exactly (CPU
oracle), the numpy MLP reference that the GPU gradient check uses agrees with
finite differences, and BF16 rounding is round-to-nearest-even."""
import numpy as np
import pytest

from oracle import oracle as O
from pfw_b200 import ace_generate as G
from pfw_b200 import surrogate as S
from pfw_b200 import workloads as WL
from pfw_b200.ace_model import read_resolved


@pytest.fixture(scope="module")
def models():
    m = read_resolved(G.generate_b2_model())
    feat, sel = S.restrict_model(m)
    return m, feat, sel


def test_feature_model_shape(models):
    m, feat, sel = models
    order = S.invariant_orders(m)
    assert feat.nbasis + feat.pair.nchannels == S.NIN
    assert all(order[b] in (1, 2) for b in sel)
    assert sel == sorted(sel, key=lambda b: (order[b], b))
    assert feat.lmax <= m.lmax and feat.ndensity < m.ndensity and feat.nproducts < m.nproducts


def test_feature_model_reproduces_selected_invariants(models):
    m, feat, sel = models
    s = WL.b2(seed=1, nc=3)
    rf = O.AceOracle(m).evaluate(s.X, s.H, s.pbc, s.species, request=1, features=True)["features"]
    rr = O.AceOracle(feat).evaluate(s.X, s.H, s.pbc, s.species, request=1, features=True)["features"]
    nz, nB, nQ, nb = m.nz, m.nbasis, m.pair.nchannels, feat.nbasis
    for z in range(nz):
        full = np.concatenate([rf[:, z * nB + np.array(sel)], rf[:, nz * nB + z * nQ:nz * nB + (z + 1) * nQ]], 1)
        red = np.concatenate([rr[:, z * nb:(z + 1) * nb], rr[:, nz * nb + z * nQ:nz * nb + (z + 1) * nQ]], 1)
        assert np.array_equal(full, red)


def test_numpy_mlp_reference_gradients():
    nin, H = 8, S.HIDDEN
    P = S.init_params(1, 1, nin, H, seed=3)[0, 0].astype(np.float64)
    P[H * nin:H * nin + H] = 0.1  # nonzero biases
    rng = np.random.default_rng(0)
    x = rng.normal(size=(5, nin))
    t = rng.normal(size=5)
    loss, g = S.mlp_param_grad_reference(P, x, t, nin, H)
    for k in rng.choice(len(P), 12, replace=False):
        e = np.zeros_like(P)
        e[k] = 1e-6
        fd = (S.mlp_param_grad_reference(P + e, x, t, nin, H)[0] - S.mlp_param_grad_reference(P - e, x, t, nin, H)[0]) / 2e-6
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(g[k])
    y, dydx = S.mlp_forward(P, x, nin, H)
    for i in range(nin):
        e = np.zeros(nin)
        e[i] = 1e-6
        fd = (S.mlp_forward(P, x + e, nin, H)[0] - S.mlp_forward(P, x - e, nin, H)[0]) / 2e-6
        assert np.allclose(fd, dydx[:, i], rtol=1e-5, atol=1e-7)


def test_bf16_rounding():
    vals = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.0e-3, 65504.0], np.float32)
    b = S.to_bf16_bits(vals)
    assert b[0] == 0x3F80
    assert b[1] == 0x3F80  # 1 + 2^-8: tie, rounds to even
    assert b[2] == 0x3F81  # 1 + 3·2^-9: above the tie
    back = S.from_bf16_bits(b)
    assert np.all(np.abs(back - vals) <= np.abs(vals) * 2.0 ** -8)


def test_energy_force_gradient_reference_matches_finite_differences():
    # the energy + force objective wE·MSE + Σ c·(v·∇_x y): the analytic
    # gradient (energy backward plus the reverse of the tangent pass) against
    # central differences of the objective, every parameter of a small model
    nin, H, n = 5, 4, 7
    rng = np.random.default_rng(3)
    p = S.init_params(1, 1, nin, H, 9)[0, 0].astype(np.float64)
    p[nin * H:nin * H + H] = rng.normal(0, 0.3, H)  # nonzero biases
    x = rng.normal(0, 1, (n, nin))
    v = rng.normal(0, 1, (n, nin))
    t = rng.normal(0, 1, n)
    c = rng.normal(0, 1, n)
    g = S.mlp_ef_grad_reference(p, x, t, v, c, 0.7, nin, H)
    fd = np.zeros_like(p)
    for k in range(len(p)):
        d = np.zeros_like(p)
        d[k] = 1e-6
        fd[k] = (S.mlp_ef_objective(p + d, x, t, v, c, 0.7, nin, H)
                 - S.mlp_ef_objective(p - d, x, t, v, c, 0.7, nin, H)) / 2e-6
    assert np.abs(g - fd).max() <= 1e-7 * max(1.0, np.abs(fd).max())
    # without the force term it is the energy gradient
    _, ge = S.mlp_param_grad_reference(p, x, t, nin, H)
    assert np.allclose(S.mlp_ef_grad_reference(p, x, t, v, np.zeros(n), 1.0, nin, H), ge, rtol=1e-12, atol=1e-14)


class FakeHandle:
    """Stands in for lib.Handle in calibrate_gate: the surrogate's force error
    is the ACE force scaled by the fraction of sites whose ensemble spread
    does not exceed tau (those stay surrogate), so the RMSE falls as tau
    falls and is zero at tau = 0."""

    def __init__(self, sd):
        self.sd, self.tau, self.n = sd, np.inf, len(sd)

    def ace(self, model):
        pass

    def surrogate(self, feat, sur=None, tau=None):
        self.tau = np.inf if tau is None else tau

    def set_geometry(self, X, H, pbc, species):
        pass

    def evaluate(self, model, request):
        F = np.ones((self.n, 3))
        if model == 1:  # MODEL_ACE
            return 0.0, F, None
        keep = self.sd <= self.tau
        return 0.0, F + 0.1 * keep.mean(), None

    def surrogate_features(self):
        return self.sd[:, None]

    def surrogate_stats(self):
        return int(np.sum(self.sd > self.tau)), self.n


class FakeSurrogate:
    def __init__(self, sd):
        self.sd, self.tau = sd, 1.0

    def predict(self, feats, species):
        return None, feats[:, 0], None


def test_calibrate_gate_keeps_the_largest_tau_that_meets_the_target():
    from pfw_b200 import lib
    assert lib.MODEL_ACE == 1
    sd = np.linspace(0.01, 1.0, 100)
    sys1 = WL.System(np.zeros((100, 3)), np.eye(3), (True, True, True), np.zeros(100, np.int32))
    sur = FakeSurrogate(sd)
    curve = S.calibrate_gate(FakeHandle(sd), sur, None, None, [sys1], target=0.0501)
    # RMSE = 0.1 × (fraction kept): the first quantile keeping at most half of the sites is 0.5
    assert curve[0]["quantile"] == 1.0 and abs(curve[0]["force_rmse"] - 0.1) < 1e-12
    assert curve[-1]["force_rmse"] <= 0.0501 < curve[-2]["force_rmse"]
    assert sur.tau == curve[-1]["tau"] == pytest.approx(np.quantile(sd, 0.5))
    # an unreachable target walks down to tau = 0 (every site falls back)
    curve = S.calibrate_gate(FakeHandle(sd), sur, None, None, [sys1], target=-1.0)
    assert sur.tau == 0.0 and curve[-1]["fallback_fraction"] == 1.0

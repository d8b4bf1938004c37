"""Learned per-atom surrogate of an ACE model with a gated ACE fallback.

There is no GPU surrogate in the reference; its nearest analogue is the CPU
invariant head ACEFeatureEnergy (ACE/feature_energy.jl:1-86), trained through
Lux.  This module builds the pieces the library's surrogate path consumes:

  restrict_model   the feature model: the ACE model cut down to its order-1
                   invariants, then its order-2 invariants in index order, up
                   to nin - nQ of them, plus its nQ pair radial sums; only the
                   densities, radial channels and harmonics those need
  training_set     site features (pfw_surrogate_features) and site energies of
                   the full model (plain FP64 GPU ACE) on seeded B2 lattices
                   with displacement sigma spread over [0.03, 0.25] Å
  train            standardisation, seeded Xavier initialisation, training with
                   the library's kernels (pfw_mlp_train), BF16 rounding, gate
  Surrogate        the trained ensemble; params() gives the pfw_mlp_params view
  train_forces     fine-tuning of every member on energies and forces
  calibrate_gate   tau chosen from the force error the gate leaves behind

Gate rule (recorded with each surrogate): per species and feature, the
standardised training range widened by 5 % of its width on each side; and the
ensemble standard deviation of a site energy at most tau.  train() sets tau
to 1.5 × the 99.5th percentile over the training sites (an energy-only
rule); calibrate_gate() replaces it by the largest tau whose evaluation
meets a force-RMSE target against plain ACE on held-out systems.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from .ace_model import PackedACE, RadialFamily

NIN = 64
HIDDEN = 64
MEMBERS = 4


# ---------------------------------------------------------------------------
# feature model
# ---------------------------------------------------------------------------
def invariant_orders(packed: PackedACE):
    """Correlation order of every invariant (its products' factor count)."""
    order = np.zeros(packed.nbasis, np.int32)
    for r, c in zip(packed.coupling_rows, packed.coupling_cols):
        order[int(r)] = max(order[int(r)], len(packed.products[int(c)]))
    return order


def restrict_model(packed: PackedACE, nin=NIN):
    """Feature model of nin features: (restricted PackedACE, selected invariant indices)."""
    nQ = packed.pair.nchannels
    order = invariant_orders(packed)
    sel = [b for b in range(packed.nbasis) if order[b] == 1] + [b for b in range(packed.nbasis) if order[b] == 2]
    sel = sel[: nin - nQ]
    if len(sel) != nin - nQ:
        raise ValueError("the model has too few order-1/2 invariants for the feature count")
    selmap = {b: i for i, b in enumerate(sel)}
    entries = [(int(r), int(c), float(v)) for r, c, v in zip(packed.coupling_rows, packed.coupling_cols,
                                                              packed.coupling_vals) if int(r) in selmap]
    K = sorted({c for _, c, _ in entries})
    kmap = {k: i for i, k in enumerate(K)}
    Dset = sorted({a for k in K for a in packed.products[k]})
    dmap = {a: i for i, a in enumerate(Dset)}
    Nset = sorted({int(packed.density[a][0]) for a in Dset})
    nmap = {n: i for i, n in enumerate(Nset)}
    lmax = max(int(np.floor(np.sqrt(int(packed.density[a][1])) + 1e-9)) for a in Dset)
    R = packed.radial
    radial = RadialFamily(spec=[R.spec[n] for n in Nset], lengths=R.lengths.copy(), nodes=R.nodes.copy(),
                          coeff=np.ascontiguousarray(R.coeff[:, :, Nset, :]), transform=R.transform.copy(),
                          powers=R.powers.copy(), envelope_kind=R.envelope_kind.copy(), envelope=R.envelope.copy())
    density = np.array([[nmap[int(packed.density[a][0])], int(packed.density[a][1])] for a in Dset], np.int32)
    products = [[dmap[a] for a in packed.products[k]] for k in K]
    entries.sort(key=lambda e: (kmap[e[1]], selmap[e[0]]))
    nz = packed.nz
    feat = PackedACE(
        atomic_numbers=list(packed.atomic_numbers), lmax=lmax, radial=radial, pair=packed.pair, density=density,
        products=products, coupling_rows=np.array([selmap[r] for r, _, _ in entries], np.int32),
        coupling_cols=np.array([kmap[c] for _, c, _ in entries], np.int32),
        coupling_vals=np.array([v for _, _, v in entries], np.float64), nbasis=len(sel),
        WB=np.zeros((nz, len(sel))), Wpair=np.zeros((nz, nQ)), reference=packed.reference.copy(),
        pair_allowed=packed.pair_allowed.copy())
    return feat, sel


# ---------------------------------------------------------------------------
# ctypes view of pfw_mlp_params
# ---------------------------------------------------------------------------
class pfw_mlp_params(C.Structure):
    _fields_ = [("nz", C.c_int32), ("members", C.c_int32), ("nin", C.c_int32), ("hidden", C.c_int32),
                ("W1", C.POINTER(C.c_uint16)), ("b1", C.POINTER(C.c_float)),
                ("W2", C.POINTER(C.c_uint16)), ("b2", C.POINTER(C.c_float)),
                ("w3", C.POINTER(C.c_uint16)), ("b3", C.POINTER(C.c_float)),
                ("x_mean", C.POINTER(C.c_double)), ("x_std", C.POINTER(C.c_double)),
                ("x_lo", C.POINTER(C.c_float)), ("x_hi", C.POINTER(C.c_float)),
                ("y_mean", C.POINTER(C.c_double)), ("y_std", C.POINTER(C.c_double)), ("tau", C.c_double)]


class pfw_mlp_shape(C.Structure):
    _fields_ = [("nz", C.c_int32), ("members", C.c_int32), ("nin", C.c_int32), ("hidden", C.c_int32)]


class pfw_mlp_train_options(C.Structure):
    _fields_ = [("epochs", C.c_int32), ("batch", C.c_int32), ("lr", C.c_float), ("lr_final", C.c_float),
                ("seed", C.c_uint64)]


def to_bf16_bits(a):
    """Round FP32 to BF16 (nearest, ties to even); returns the uint16 bit patterns."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return u.astype(np.uint16)


def from_bf16_bits(b):
    return (np.asarray(b, np.uint32) << 16).view(np.float32)


def nparams(nin, H):
    return H * nin + H * H + 3 * H + 1


def split_params(p, nin, H):
    """FP32 parameter vector → (W1 [H,nin], b1, W2 [H,H], b2, w3, b3)."""
    o = 0
    W1 = p[o:o + H * nin].reshape(H, nin); o += H * nin
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    return W1, b1, W2, b2, w3, p[o]


def init_params(nz, members, nin, H, seed):
    """Xavier-uniform weights, zero biases, one stream per (species, member)."""
    out = np.zeros((nz, members, nparams(nin, H)), np.float32)
    for z in range(nz):
        for m in range(members):
            rng = np.random.default_rng([seed, z, m])
            a1, a2, a3 = np.sqrt(6.0 / (nin + H)), np.sqrt(6.0 / (2 * H)), np.sqrt(6.0 / (H + 1))
            W1 = rng.uniform(-a1, a1, (H, nin))
            W2 = rng.uniform(-a2, a2, (H, H))
            w3 = rng.uniform(-a3, a3, H)
            out[z, m] = np.concatenate([W1.ravel(), np.zeros(H), W2.ravel(), np.zeros(H), w3, [0.0]])
    return out


def silu(z):
    return z / (1.0 + np.exp(-z))


def mlp_forward(params, x, nin, H):
    """FP64 numpy reference of one member: y and dy/dx for x [n, nin]."""
    W1, b1, W2, b2, w3, b3 = (np.asarray(v, np.float64) for v in split_params(params, nin, H))
    z1 = x @ W1.T + b1
    s1 = 1.0 / (1.0 + np.exp(-z1))
    h1 = z1 * s1
    z2 = h1 @ W2.T + b2
    s2 = 1.0 / (1.0 + np.exp(-z2))
    h2 = z2 * s2
    y = h2 @ w3 + b3
    d2 = w3 * (s2 * (1 + z2 * (1 - s2)))
    d1 = (d2 @ W2) * (s1 * (1 + z1 * (1 - s1)))
    return y, d1 @ W1


def mlp_param_grad_reference(params, x, t, nin, H):
    """FP64 numpy gradient of mean((y - t)^2) with respect to the parameter vector."""
    W1, b1, W2, b2, w3, b3 = (np.asarray(v, np.float64) for v in split_params(params, nin, H))
    z1 = x @ W1.T + b1
    s1 = 1.0 / (1.0 + np.exp(-z1))
    h1 = z1 * s1
    z2 = h1 @ W2.T + b2
    s2 = 1.0 / (1.0 + np.exp(-z2))
    h2 = z2 * s2
    y = h2 @ w3 + b3
    n = len(t)
    dy = 2.0 * (y - t) / n
    D2 = dy[:, None] * w3[None, :] * (s2 * (1 + z2 * (1 - s2)))
    D1 = (D2 @ W2) * (s1 * (1 + z1 * (1 - s1)))
    g = np.concatenate([(D1.T @ x).ravel(), D1.sum(0), (D2.T @ h1).ravel(), D2.sum(0), dy @ h2, [dy.sum()]])
    return float(np.mean((y - t) ** 2)), g


def _silu_parts(z):
    a = 1.0 / (1.0 + np.exp(-z))
    return z * a, a * (1 + z * (1 - a)), a * (1 - a) * (2 + z * (1 - 2 * a))


def mlp_ef_objective(params, x, t, v, c, wE, nin, H):
    """wE·mean((y - t)²) + Σ_s c_s·(v_s·∇_x y(x_s)): the energy + force
    training objective of one model in FP64 (v: the force error pulled back
    into standardised feature space, c: the per-sample force weight)."""
    y, dydx = mlp_forward(params, x, nin, H)
    return wE * float(np.mean((y - t) ** 2)) + float(np.sum(c * np.einsum("si,si->s", v, dydx)))


def mlp_ef_grad_reference(params, x, t, v, c, wE, nin, H):
    """FP64 numpy gradient of mlp_ef_objective with respect to the parameter
    vector: the energy backward pass plus the reverse of the tangent pass
    t1 = W1 v, u1 = s1'⊙t1, t2 = W2 u1, u2 = s2'⊙t2, ẏ = w3·u2."""
    W1, b1, W2, b2, w3, b3 = (np.asarray(q, np.float64) for q in split_params(params, nin, H))
    z1 = x @ W1.T + b1
    h1, s1, q1 = _silu_parts(z1)
    t1 = v @ W1.T
    u1 = s1 * t1
    z2 = h1 @ W2.T + b2
    h2, s2, q2 = _silu_parts(z2)
    t2 = u1 @ W2.T
    u2 = s2 * t2
    y = h2 @ w3 + b3
    dy = wE * 2.0 * (y - t) / len(t)
    G2 = dy[:, None] * w3 * s2 + c[:, None] * w3 * t2 * q2
    B2 = c[:, None] * w3 * s2
    bh, bu = G2 @ W2, B2 @ W2
    G1 = bh * s1 + bu * t1 * q1
    B1 = bu * s1
    return np.concatenate([(G1.T @ x + B1.T @ v).ravel(), G1.sum(0), (G2.T @ h1 + B2.T @ u1).ravel(), G2.sum(0),
                           dy @ h2 + c @ u2, [dy.sum()]])


# ---------------------------------------------------------------------------
# the trained surrogate
# ---------------------------------------------------------------------------
@dataclass
class Surrogate:
    feature_model: PackedACE
    selected: list
    params: np.ndarray      # FP32 [nz, M, nparams] (training result)
    x_mean: np.ndarray      # [nz, nin]
    x_std: np.ndarray
    x_lo: np.ndarray        # standardised accepted range, margin included
    x_hi: np.ndarray
    y_mean: np.ndarray      # [nz]
    y_std: np.ndarray
    tau: float
    history: list = field(default_factory=list)
    _keep: list = field(default_factory=list, repr=False)

    @property
    def shape(self):
        nz, M, _ = self.params.shape
        return nz, M, self.x_mean.shape[1], HIDDEN

    def bf16_members(self):
        """Per (z, m): the FP32 parameter vector with every weight rounded to BF16."""
        nz, M, nin, H = self.shape
        out = self.params.copy()
        for z in range(nz):
            for m in range(M):
                W1, b1, W2, b2, w3, b3 = split_params(out[z, m], nin, H)
                W1[...] = from_bf16_bits(to_bf16_bits(W1))
                W2[...] = from_bf16_bits(to_bf16_bits(W2))
                w3[...] = from_bf16_bits(to_bf16_bits(w3))
        return out

    def mlp_struct(self, tau=None):
        nz, M, nin, H = self.shape
        W1 = np.zeros((nz, M, H, nin), np.float32)
        W2 = np.zeros((nz, M, H, H), np.float32)
        w3 = np.zeros((nz, M, H), np.float32)
        b1 = np.zeros((nz, M, H), np.float32)
        b2 = np.zeros((nz, M, H), np.float32)
        b3 = np.zeros((nz, M), np.float32)
        for z in range(nz):
            for m in range(M):
                a = split_params(self.params[z, m], nin, H)
                W1[z, m], b1[z, m], W2[z, m], b2[z, m], w3[z, m], b3[z, m] = a
        arrs = dict(W1=to_bf16_bits(W1), W2=to_bf16_bits(W2), w3=to_bf16_bits(w3), b1=b1, b2=b2, b3=b3,
                    x_mean=np.ascontiguousarray(self.x_mean, np.float64),
                    x_std=np.ascontiguousarray(self.x_std, np.float64),
                    x_lo=np.ascontiguousarray(self.x_lo, np.float32), x_hi=np.ascontiguousarray(self.x_hi, np.float32),
                    y_mean=np.ascontiguousarray(self.y_mean, np.float64),
                    y_std=np.ascontiguousarray(self.y_std, np.float64))
        self._keep = list(arrs.values())
        s = pfw_mlp_params()
        s.nz, s.members, s.nin, s.hidden = nz, M, nin, H
        for k, v in arrs.items():
            ct = {np.dtype(np.uint16): C.c_uint16, np.dtype(np.float32): C.c_float, np.dtype(np.float64): C.c_double}[v.dtype]
            setattr(s, k, v.ctypes.data_as(C.POINTER(ct)))
        s.tau = float(self.tau if tau is None else tau)
        return s

    def predict(self, feats, species):
        """numpy reference of the deployed ensemble (BF16 weights): site energy minus the
        reference energy, ensemble std (eV) and dE/dfeature, for features [n, nin]."""
        nz, M, nin, H = self.shape
        P = self.bf16_members()
        n = len(species)
        e = np.zeros(n)
        sd = np.zeros(n)
        g = np.zeros((n, nin))
        for z in range(nz):
            idx = np.nonzero(species == z)[0]
            if not len(idx):
                continue
            x = (feats[idx] - self.x_mean[z]) / self.x_std[z]
            ys, gs = [], []
            for m in range(M):
                y, dydx = mlp_forward(P[z, m], x, nin, H)
                ys.append(y)
                gs.append(dydx)
            ys = np.array(ys)
            e[idx] = self.y_mean[z] + self.y_std[z] * ys.mean(0)
            sd[idx] = self.y_std[z] * ys.std(0)
            g[idx] = self.y_std[z] * np.mean(gs, axis=0) / self.x_std[z]
        return e, sd, g


def training_set(h, full: PackedACE, feat: PackedACE, n_lattices=13, nc=20, seed=11, sigma=(0.03, 0.25)):
    """Site features and full-model site energies on B2 lattices, sigma evenly spread."""
    from . import lib
    from . import workloads as WL
    X, E, Z = [], [], []
    h.ace(full)
    h.surrogate(feat, None)
    for k, sg in enumerate(np.linspace(sigma[0], sigma[1], n_lattices)):
        s = WL.b2(seed=seed + k, nc=nc, sigma=float(sg))
        h.set_geometry(s.X, s.H, s.pbc, s.species)
        h.evaluate(lib.MODEL_ACE, 1)
        E.append(h.site_energies())
        X.append(h.surrogate_features())
        Z.append(s.species.copy())
    return np.concatenate(X), np.concatenate(E), np.concatenate(Z)


def train(h, feat: PackedACE, selected, X, E, Z, *, members=MEMBERS, epochs=40, batch=512, lr=2e-3,
          lr_final=2e-5, seed=7, margin=0.05, tau_quantile=0.995, tau_factor=1.5):
    """Train the ensemble on (features X, site energies E, species Z) with pfw_mlp_train."""
    nz, nin = feat.nz, X.shape[1]
    ref = feat.reference
    x_mean = np.zeros((nz, nin))
    x_std = np.ones((nz, nin))
    y_mean = np.zeros(nz)
    y_std = np.ones(nz)
    Xs = np.zeros_like(X, dtype=np.float32)
    ys = np.zeros(len(E), np.float32)
    x_lo = np.zeros((nz, nin))
    x_hi = np.zeros((nz, nin))
    for z in range(nz):
        idx = np.nonzero(Z == z)[0]
        if not len(idx):
            continue
        x_mean[z] = X[idx].mean(0)
        x_std[z] = np.maximum(X[idx].std(0), 1e-12 * np.maximum(1.0, np.abs(x_mean[z])))
        t = E[idx] - ref[z]
        y_mean[z] = t.mean()
        y_std[z] = max(t.std(), 1e-12)
        Xs[idx] = (X[idx] - x_mean[z]) / x_std[z]
        ys[idx] = (t - y_mean[z]) / y_std[z]
        lo, hi = Xs[idx].min(0), Xs[idx].max(0)
        w = hi - lo
        x_lo[z], x_hi[z] = lo - margin * w - 1e-6, hi + margin * w + 1e-6
    P = init_params(nz, members, nin, HIDDEN, seed)
    hist = h.mlp_train(P, Xs, ys, Z.astype(np.int32), epochs=epochs, batch=batch, lr=lr, lr_final=lr_final,
                       seed=seed)
    sur = Surrogate(feature_model=feat, selected=list(selected), params=P, x_mean=x_mean, x_std=x_std, x_lo=x_lo,
                    x_hi=x_hi, y_mean=y_mean, y_std=y_std, tau=np.inf, history=list(map(float, hist)))
    _, sd, _ = sur.predict(X, Z)
    sur.tau = float(tau_factor * np.quantile(sd, tau_quantile))
    return sur


# ---------------------------------------------------------------------------
# energy + force fine-tuning
# ---------------------------------------------------------------------------
def force_training_set(h, full: PackedACE, feat: PackedACE, n_lattices=13, nc=20, seed=11, sigma=(0.03, 0.25)):
    """B2 lattices with the full model's site energies and forces (plain FP64
    GPU ACE) and the site features: one dict per lattice."""
    from . import lib
    from . import workloads as WL
    out = []
    h.ace(full)
    h.surrogate(feat, None)
    for k, sg in enumerate(np.linspace(sigma[0], sigma[1], n_lattices)):
        s = WL.b2(seed=seed + k, nc=nc, sigma=float(sg))
        h.set_geometry(s.X, s.H, s.pbc, s.species)
        _, F, _ = h.evaluate(lib.MODEL_ACE, 7)
        out.append(dict(sys=s, E=h.site_energies(), F=F, X=h.surrogate_features(), Z=s.species.copy()))
    return out


def train_forces(h, sur: "Surrogate", lattices, *, epochs=40, inner=1, batch=1 << 30, lr=1e-3, lr_final=1e-5,
                 warmup=50, wE=1.0, wF=1.0, step_disp=1e-4, seed=3, log=None):
    """Fine-tune every member of the ensemble on energies AND forces with the
    library's kernels.  Per lattice visit: ∂y/∂x of every member at every
    site (pfw_mlp_input_grad), each member's forces through the feature model
    (pfw_surrogate_pullback), the force error ΔF_m against the full model,
    and its pull-back into feature space v = D_ΔF x (central difference of
    the features along ΔF, largest displacement step_disp Å).  Then `inner`
    Adam steps (pfw_mlp_ef_step) on random batches of `batch` sites of the
    lattice, each on wE·MSE(energy) + wF·Σ|ΔF|²/(3 n σ_F²) with v held at
    the visit's value (the force term's gradient is exact at the first step
    and linearised after it).  Fine-tuning starts from a converged energy
    fit, so the learning rate ramps up linearly over `warmup` steps (Adam's
    first steps move every weight by the full rate) and then decays as a
    cosine to lr_final.  The feature model must be loaded in h
    (h.surrogate).  Returns the history of (energy MSE, force RMSE in eV/Å
    at the visits) per epoch."""
    import torch

    dev = torch.device("cuda", h.device)
    # The library's kernels and the torch glue must run in one stream, in
    # order.  A stream of its own: the legacy default stream's handle is 0,
    # which pfw_set_stream reads as "the workspace's own stream".
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.synchronize(dev)
    h.set_stream(C.c_void_p(stream.cuda_stream))
    try:
        with torch.cuda.stream(stream):
            return _train_forces(h, sur, lattices, dev, epochs=epochs, inner=inner, batch=batch, lr=lr,
                                 lr_final=lr_final, warmup=warmup, wE=wE, wF=wF, step_disp=step_disp, seed=seed,
                                 log=log)
    finally:
        torch.cuda.synchronize(dev)
        h.set_stream(None)


def _train_forces(h, sur, lattices, dev, *, epochs, inner, batch, lr, lr_final, warmup, wE, wF, step_disp, seed,
                  log):
    import torch

    nz, M, nin, H = sur.shape
    shape = pfw_mlp_shape(nz, M, nin, H)
    P = torch.from_numpy(np.ascontiguousarray(sur.params, np.float32)).to(dev)
    m1 = torch.zeros_like(P)
    m2 = torch.zeros_like(P)
    xm = torch.from_numpy(sur.x_mean).to(dev)
    xs = torch.from_numpy(sur.x_std).to(dev)
    ym, ys = sur.y_mean, sur.y_std
    sigF = float(np.sqrt(np.mean(np.concatenate([L["F"].ravel() for L in lattices]) ** 2)))
    data = []
    for L in lattices:
        Z = L["Z"].astype(np.int32)
        zt = torch.from_numpy(Z.astype(np.int64)).to(dev)
        Xd = torch.from_numpy(L["X"]).to(dev)
        t = (L["E"] - sur.feature_model.reference[Z] - ym[Z]) / ys[Z]
        data.append(dict(Z=Z, zt=zt, Xs=((Xd - xm[zt]) / xs[zt]).float().contiguous(),
                         y=torch.from_numpy(t.astype(np.float32)).to(dev), F=torch.from_numpy(L["F"]).to(dev),
                         sys=L["sys"], n=len(Z), yscale=torch.from_numpy(ys[Z]).to(dev)))
    rng = np.random.default_rng(seed)
    total = epochs * len(data) * inner
    step = 0
    hist = []
    for ep in range(epochs):
        e_mse, f_sq, f_cnt = 0.0, 0.0, 0
        for li in rng.permutation(len(data)):
            d = data[li]
            n, s = d["n"], d["sys"]
            G = torch.empty((M, n, nin), dtype=torch.float32, device=dev)
            h.mlp_input_grad(shape, P, d["Xs"], d["Z"], G)
            V = torch.empty((M, n, nin), dtype=torch.float32, device=dev)
            scale = d["yscale"][:, None] / xs[d["zt"]]  # dE/dx = y_std ∂y/∂x̃ / x_std
            for m in range(M):
                dEdx = (G[m].double() * scale).contiguous()
                Fp = torch.empty((n, 3), dtype=torch.float64, device=dev)
                h.set_geometry(s.X, s.H, s.pbc, s.species)
                h.surrogate_pullback(dEdx, Fp)
                dF = (Fp - d["F"]).cpu().numpy()
                f_sq += float((dF ** 2).sum())
                f_cnt += dF.size
                eps = step_disp / max(float(np.abs(dF).max()), 1e-30)
                h.set_geometry(s.X + eps * dF, s.H, s.pbc, s.species)
                xp = torch.from_numpy(h.surrogate_features()).to(dev)
                h.set_geometry(s.X - eps * dF, s.H, s.pbc, s.species)
                xn = torch.from_numpy(h.surrogate_features()).to(dev)
                V[m] = ((xp - xn) / (2.0 * eps) / xs[d["zt"]]).float()
            B = min(batch, n)
            # the force weight of a site in a batch of B of the lattice's n sites (unbiased in expectation)
            c_all = -2.0 * wF / (3.0 * B * sigF ** 2) * d["yscale"]
            for _ in range(inner):
                idx = np.sort(rng.choice(n, B, replace=False))
                it = torch.from_numpy(idx).to(dev)
                frac = step / max(total - 1, 1)
                lr_t = (lr_final + 0.5 * (lr - lr_final) * (1.0 + np.cos(np.pi * frac))) * min(1.0, (step + 1) / warmup)
                step += 1
                loss = h.mlp_ef_step(shape, P, m1, m2, d["Xs"][it].contiguous(), d["y"][it].contiguous(),
                                     d["Z"][idx], V[:, it].contiguous(), c_all[it].float().contiguous(), wE=wE,
                                     lr=lr_t, step=step, with_loss=True)
                e_mse += float(np.mean(loss)) / inner
        hist.append((e_mse / len(data), float(np.sqrt(f_sq / max(f_cnt, 1)))))
        if log:
            log(f"epoch {ep}: energy mse {hist[-1][0]:.3e}, force rmse {hist[-1][1]:.4f} eV/A")
    torch.cuda.synchronize()
    sur.params = P.cpu().numpy().reshape(sur.params.shape)
    sur.force_history = hist
    return hist


def calibrate_gate(h, sur: "Surrogate", full: PackedACE, feat: PackedACE, systems, target=2e-2,
                   quantiles=(1.0, 0.95, 0.9, 0.85, 0.8, 0.75, 0.7, 0.6, 0.5, 0.4, 0.3, 0.2, 0.1)):
    """Choose the ensemble-disagreement threshold tau from forces.

    On the calibration systems (held out from training), plain FP64 ACE
    forces are the reference.  tau runs down the quantiles of the sites' ensemble
    standard deviation (numpy restatement of the deployed BF16 ensemble on
    the library's features; quantile 1 means no disagreement gate); for each,
    the surrogate is evaluated with its feature-range gate and that tau, and
    the force RMSE against ACE over all systems is measured together with the
    fallback fraction.  The first (largest) tau whose RMSE meets `target` is
    kept in sur.tau; tau = 0 (every site falls back) reproduces ACE exactly,
    so the walk ends there at the latest.  Returns the curve as a list of
    dicts (quantile, tau, fallback_fraction, force_rmse)."""
    from . import lib
    h.ace(full)
    h.surrogate(feat, sur, tau=np.inf)
    refs, sds = [], []
    for sy in systems:
        h.set_geometry(sy.X, sy.H, sy.pbc, sy.species)
        _, Fa, _ = h.evaluate(lib.MODEL_ACE, 7)
        refs.append(Fa)
        _, sd, _ = sur.predict(h.surrogate_features(), np.asarray(sy.species))
        sds.append(sd)
    sd_all = np.concatenate(sds)
    curve = []
    chosen = 0.0
    for q in list(quantiles) + [None]:
        tau = 0.0 if q is None else (np.inf if q >= 1.0 else float(np.quantile(sd_all, q)))
        h.surrogate(feat, sur, tau=tau)
        se, cnt, fb, ns = 0.0, 0, 0, 0
        for sy, Fa in zip(systems, refs):
            h.set_geometry(sy.X, sy.H, sy.pbc, sy.species)
            _, Fs, _ = h.evaluate(lib.MODEL_SURROGATE, 7)
            se += float(np.sum((Fs - Fa) ** 2))
            cnt += Fs.size
            f, n = h.surrogate_stats()
            fb += f
            ns += n
        rmse = float(np.sqrt(se / max(cnt, 1)))
        curve.append(dict(quantile=0.0 if q is None else float(q), tau=float(tau),
                          fallback_fraction=fb / max(ns, 1), force_rmse=rmse))
        if rmse <= target:
            chosen = tau
            break
    sur.tau = float(chosen)
    return curve

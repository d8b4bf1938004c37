"""Resolved ACE model import and packing for the device.

`read_resolved` restates the schema-v1 reader of the reference
(ACE/resolved.jl:57-142): it validates the same fields and produces the same
model tables (radial/pair spline channels per species pair, density list,
products, sparse coupling, readout WB/Wpair, reference energies).
`PackedACE` restates `pack_model`/`pack_radials` (ACE/adaptation.jl:57-98):
ragged spline tables are padded along the model dimensions, indices become
0-based, and the invariant mask is folded into WB.  `tables()` returns the
C struct `pfw_ace_tables` expected by `pfw_ace_model_load`.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import copy
import dataclasses
from dataclasses import dataclass, field

import numpy as np

from .errors import argument_error, dimension_mismatch

# factors per product the device records hold (ushort4 with a sentinel)
MAX_ORDER = 4

ENVELOPE_KIND = {"PolyEnvelope2sX": 1, "ACE1_PolyEnvelope1sR": 2, "PolyEnvelope1sR": 3}


class pfw_radial_family(C.Structure):
    _fields_ = [
        ("nchannels", C.c_int32),
        ("nknots", C.c_int32),
        ("lengths", C.POINTER(C.c_int32)),
        ("nodes", C.POINTER(C.c_double)),
        ("coeff", C.POINTER(C.c_double)),
        ("transform", C.POINTER(C.c_double)),
        ("powers", C.POINTER(C.c_int32)),
        ("envelope_kind", C.POINTER(C.c_int32)),
        ("envelope", C.POINTER(C.c_double)),
    ]


class pfw_ace_tables(C.Structure):
    _fields_ = [
        ("nz", C.c_int32),
        ("lmax", C.c_int32),
        ("radial", pfw_radial_family),
        ("pair", pfw_radial_family),
        ("ndensity", C.c_int32),
        ("density", C.POINTER(C.c_int32)),
        ("nproducts", C.c_int32),
        ("product_offsets", C.POINTER(C.c_int32)),
        ("product_factors", C.POINTER(C.c_int32)),
        ("nbasis", C.c_int32),
        ("ncoupling", C.c_int32),
        ("coupling_rows", C.POINTER(C.c_int32)),
        ("coupling_cols", C.POINTER(C.c_int32)),
        ("coupling_vals", C.POINTER(C.c_double)),
        ("WB", C.POINTER(C.c_double)),
        ("Wpair", C.POINTER(C.c_double)),
        ("reference", C.POINTER(C.c_double)),
        ("pair_allowed", C.POINTER(C.c_uint8)),
        ("cutoff", C.c_double),
        ("angular_kind", C.c_int32),
    ]


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


@dataclass
class RadialFamily:
    """One radial family (R or pair Q) over nz×nz species pairs."""

    spec: list  # [(n, l)]
    lengths: np.ndarray  # int32 [nz*nz]
    nodes: np.ndarray  # f64 [nz*nz, nknots]
    coeff: np.ndarray  # f64 [nz*nz, nknots-1, nch, 4]
    transform: np.ndarray  # f64 [nz*nz, 6]
    powers: np.ndarray  # int32 [nz*nz, 2]
    envelope_kind: np.ndarray  # int32 [nz*nz]
    envelope: np.ndarray  # f64 [nz*nz, 5]

    @property
    def nchannels(self):
        return self.coeff.shape[2]

    @property
    def nknots(self):
        return self.nodes.shape[1]

    @property
    def cutoff(self):
        return float(self.transform[:, 5].max())

    def scaled(self, scale, nz):
        """The family with channel n of species pair (iz, jz) multiplied by
        scale[n, iz, jz] (the trainable ps.radial.scale / ps.pair.scale of
        ACE/serial.jl:12-17, applied by the reference at run time as
        scale · R, gpu.jl:74-91).  Splines are linear in their coefficients,
        so the scale is folded into the coefficient table."""
        s = np.asarray(scale, dtype=np.float64)
        if s.shape != (self.nchannels, nz, nz):
            raise dimension_mismatch("radial scale dimensions")
        if not np.all(np.isfinite(s)):
            raise argument_error("nonfinite radial scale")
        per_pair = s.transpose(1, 2, 0).reshape(nz * nz, 1, self.nchannels, 1)  # k = iz*nz + jz
        return dataclasses.replace(self, coeff=np.ascontiguousarray(self.coeff * per_pair))

    def to_dict(self, nz):
        """The family as the resolved schema's radial table (the inverse of
        read_radial, ACE/resolved.jl:57-92)."""
        names = {v: k for k, v in ENVELOPE_KIND.items()}
        channels = []
        for ci in range(nz):
            for ni in range(nz):
                k = ci * nz + ni
                K = int(self.lengths[k])
                t = self.transform[k]
                kind = names[int(self.envelope_kind[k])]
                e = self.envelope[k]
                if kind == "PolyEnvelope2sX":
                    env = {"x1": float(e[0]), "x2": float(e[1]), "p1": int(e[2]), "p2": int(e[3]), "s": float(e[4])}
                elif kind == "PolyEnvelope1sR":
                    env = {"rcut": float(e[0]), "p": int(e[1])}
                else:
                    env = {"rcut": float(e[0]), "r0": float(e[1]), "p": int(e[2])}
                channels.append({
                    "centre": ci + 1, "neighbour": ni + 1,
                    "transform": {"p": int(self.powers[k, 0]), "q": int(self.powers[k, 1]), "a": float(t[0]),
                                  "rin": float(t[1]), "r0": float(t[2]), "yin": float(t[3]), "ycut": float(t[4]),
                                  "rcut": float(t[5]), "normalization_rin": float(t[1])},
                    "envelope_kind": kind, "envelope": env,
                    "nodes": [float(v) for v in self.nodes[k, :K]],
                    "coefficient_shape": [4, self.nchannels, K - 1],
                    # [interval][channel][power] row-major = Julia column-major (4, nch, K-1)
                    "coefficients": [float(v) for v in self.coeff[k, :K - 1].ravel()]})
        return {"kind": "piecewise_cubic_agnesi", "spec": [{"n": int(n), "l": int(l)} for n, l in self.spec],
                "channels": channels}

    def struct(self):
        return pfw_radial_family(
            self.nchannels, self.nknots, _ptr(self.lengths, C.c_int32), _ptr(self.nodes, C.c_double),
            _ptr(self.coeff, C.c_double), _ptr(self.transform, C.c_double), _ptr(self.powers, C.c_int32),
            _ptr(self.envelope_kind, C.c_int32), _ptr(self.envelope, C.c_double))


@dataclass
class PackedACE:
    atomic_numbers: list
    lmax: int
    radial: RadialFamily
    pair: RadialFamily
    density: np.ndarray  # int32 [D, 2] 0-based (radial channel, harmonic)
    products: list  # list of lists of 0-based density indices
    coupling_rows: np.ndarray  # int32, CSC order
    coupling_cols: np.ndarray  # int32
    coupling_vals: np.ndarray  # f64
    nbasis: int
    WB: np.ndarray  # f64 [nz, nbasis] (mask applied)
    Wpair: np.ndarray  # f64 [nz, nQ]
    reference: np.ndarray  # f64 [nz]
    pair_allowed: np.ndarray  # uint8 [nz]
    source_sha256: str = ""
    _keep: list = field(default_factory=list, repr=False)
    angular_kind: int = 0  # 0 real spherical, 1 real solid r^l·Y_lm (angular_blocks.jl:25-48)
    # the resolved-schema model tree it was read from, without "parameters"
    # (written back by save_calculator); None when built from packed tables
    resolved: dict | None = field(default=None, repr=False)
    # invariant mask of the basis policy (interface.jl:1-16); None = all rows
    mask: np.ndarray | None = field(default=None, repr=False)
    # readout as read, Julia shapes WB (nbasis, nz) and Wpair (nQ, nz), unmasked
    parameters0: dict | None = field(default=None, repr=False)

    @property
    def nz(self):
        return len(self.atomic_numbers)

    @property
    def cutoff(self):
        # NI.search_cutoff(::ResolvedModel) = max rcut over both families (ACE/cpu.jl:316)
        return max(self.radial.cutoff, self.pair.cutoff)

    @property
    def ndensity(self):
        return self.density.shape[0]

    @property
    def nproducts(self):
        return len(self.products)

    def product_csr(self):
        offs = np.zeros(len(self.products) + 1, dtype=np.int32)
        offs[1:] = np.cumsum([len(p) for p in self.products])
        facs = np.array([a for p in self.products for a in p], dtype=np.int32)
        return offs, facs

    def channel_of(self, z: int) -> int:
        return self.atomic_numbers.index(z)

    def tables(self) -> pfw_ace_tables:
        """C struct view; the arrays stay owned by this object.  The device
        kernels hold a product's factors in one 4-wide record, so products of
        more than 4 densities (correlation order above 4) are rejected here,
        as the library rejects them; every shipped model has order <= 3."""
        if any(len(p) > MAX_ORDER for p in self.products):
            raise argument_error(f"ACE correlation order above {MAX_ORDER} is not supported on the device")
        if any(len(p) == 0 for p in self.products):
            raise argument_error("empty ACE product")
        offs, facs = self.product_csr()
        dens = np.ascontiguousarray(self.density, dtype=np.int32)
        self._keep = [offs, facs, dens]
        t = pfw_ace_tables()
        t.nz = self.nz
        t.lmax = self.lmax
        t.radial = self.radial.struct()
        t.pair = self.pair.struct()
        t.ndensity = dens.shape[0]
        t.density = _ptr(dens, C.c_int32)
        t.nproducts = len(self.products)
        t.product_offsets = _ptr(offs, C.c_int32)
        t.product_factors = _ptr(facs, C.c_int32)
        t.nbasis = self.nbasis
        t.ncoupling = len(self.coupling_vals)
        t.coupling_rows = _ptr(self.coupling_rows, C.c_int32)
        t.coupling_cols = _ptr(self.coupling_cols, C.c_int32)
        t.coupling_vals = _ptr(self.coupling_vals, C.c_double)
        t.WB = _ptr(self.WB, C.c_double)
        t.Wpair = _ptr(self.Wpair, C.c_double)
        t.reference = _ptr(self.reference, C.c_double)
        t.pair_allowed = _ptr(self.pair_allowed, C.c_uint8)
        t.cutoff = self.cutoff
        t.angular_kind = self.angular_kind
        return t

    def readout_mask(self) -> np.ndarray:
        return np.ones(self.nbasis, bool) if self.mask is None else np.asarray(self.mask, bool)

    def default_parameters(self) -> dict:
        """The model's own parameters (WB, Wpair) in the reference's shapes."""
        if self.parameters0 is not None:
            return {k: np.array(v) for k, v in self.parameters0.items()}
        return {"WB": self.WB.T.copy(), "Wpair": self.Wpair.T.copy()}

    def with_parameters(self, ps) -> "PackedACE":
        """Device tables for explicit parameters: WB (nbasis, nz) masked by the
        policy (effective_WB, interface.jl:125), Wpair (nQ, nz), and optional
        radial/pair scales {"scale": (n, nz, nz)} folded into the splines
        (checkpoint_read_model's shape checks, persistence.jl:83-99)."""
        if not (isinstance(ps, dict) and "WB" in ps and "Wpair" in ps):
            raise argument_error("ACE parameters require WB and Wpair")
        nz, m, nq = self.nz, self.nbasis, self.pair.nchannels
        WB = np.asarray(ps["WB"], dtype=np.float64)
        Wp = np.asarray(ps["Wpair"], dtype=np.float64)
        if WB.shape != (m, nz) or Wp.shape != (nq, nz):
            raise dimension_mismatch("ACE readout shapes")
        if not (np.all(np.isfinite(WB)) and np.all(np.isfinite(Wp))):
            raise argument_error("nonfinite ACE readout")
        radial, pair = self.radial, self.pair
        for key, fam in (("radial", radial), ("pair", pair)):
            if key in ps:
                block = ps[key]
                if not (isinstance(block, dict) and "scale" in block):
                    raise dimension_mismatch(f"{key} scale dimensions")
                if np.asarray(block["scale"]).shape != (fam.nchannels, nz, nz):
                    raise dimension_mismatch(f"{key} scale dimensions")
                if key == "radial":
                    radial = fam.scaled(block["scale"], nz)
                else:
                    pair = fam.scaled(block["scale"], nz)
        return dataclasses.replace(
            self, radial=radial, pair=pair, _keep=[],
            WB=np.ascontiguousarray((WB * self.readout_mask()[:, None]).T),
            Wpair=np.ascontiguousarray(Wp.T))

    def resolved_dict(self) -> dict:
        """The model as a resolved schema-v1 tree without "parameters"
        (the "model" entry of a checkpoint, persistence.jl:70-80)."""
        if self.resolved is not None:
            return copy.deepcopy(self.resolved)
        if not np.all(self.pair_allowed == 1):
            raise argument_error("a model without its resolved source needs the default pair policy")
        return {
            "schema": "PotentialFrameWork.resolved_ACE", "schema_version": 1,
            "source_sha256": self.source_sha256, "coordinate_kind": "invariant",
            "coefficient_precision": "Float64",
            "species_atomic_numbers": [int(v) for v in self.atomic_numbers],
            "reference_eV": [float(v) for v in self.reference],
            "angular": {"kind": ("real_spherical", "real_solid")[self.angular_kind], "normalization": "L2",
                        "ordering": "l*l+l+m+1", "lmax": int(self.lmax)},
            "radial": self.radial.to_dict(self.nz), "pair_radial": self.pair.to_dict(self.nz),
            "density_indices": [[int(a) + 1, int(b) + 1] for a, b in self.density],
            "products": [[int(i) + 1 for i in p] for p in self.products],
            "coupling": {"shape": [int(self.nbasis), len(self.products)],
                         "rows": [int(v) + 1 for v in self.coupling_rows],
                         "columns": [int(v) + 1 for v in self.coupling_cols],
                         "values": [float(v) for v in self.coupling_vals]}}

    def weights(self) -> np.ndarray:
        """Precontracted product weights w[z, k] = Σ_b C[b,k]·WB[z,b] (ACE/cpu.jl:265-268)."""
        w = np.zeros((self.nz, self.nproducts))
        for z in range(self.nz):
            np.add.at(w[z], self.coupling_cols, self.coupling_vals * self.WB[z, self.coupling_rows])
        return w

    # --- persistence of the packed form (npz) ---------------------------
    def to_npz_dict(self, prefix=""):
        offs, facs = self.product_csr()
        d = {}
        for fam_name, fam in (("radial", self.radial), ("pair", self.pair)):
            for k in ("lengths", "nodes", "coeff", "transform", "powers", "envelope_kind", "envelope"):
                d[f"{prefix}{fam_name}_{k}"] = getattr(fam, k)
            d[f"{prefix}{fam_name}_spec"] = np.array(fam.spec, dtype=np.int32).reshape(-1, 2)
        d.update({
            f"{prefix}atomic_numbers": np.array(self.atomic_numbers, dtype=np.int32),
            f"{prefix}lmax": np.array(self.lmax),
            f"{prefix}density": self.density,
            f"{prefix}product_offsets": offs,
            f"{prefix}product_factors": facs,
            f"{prefix}coupling_rows": self.coupling_rows,
            f"{prefix}coupling_cols": self.coupling_cols,
            f"{prefix}coupling_vals": self.coupling_vals,
            f"{prefix}nbasis": np.array(self.nbasis),
            f"{prefix}WB": self.WB,
            f"{prefix}Wpair": self.Wpair,
            f"{prefix}reference": self.reference,
            f"{prefix}pair_allowed": self.pair_allowed,
            f"{prefix}angular_kind": np.array(self.angular_kind),
        })
        return d

    @classmethod
    def from_npz_dict(cls, d, prefix=""):
        fams = {}
        for fam_name in ("radial", "pair"):
            g = lambda k: np.ascontiguousarray(d[f"{prefix}{fam_name}_{k}"])
            fams[fam_name] = RadialFamily(
                spec=[tuple(int(v) for v in r) for r in g("spec")], lengths=g("lengths").astype(np.int32),
                nodes=g("nodes").astype(np.float64), coeff=g("coeff").astype(np.float64),
                transform=g("transform").astype(np.float64), powers=g("powers").astype(np.int32),
                envelope_kind=g("envelope_kind").astype(np.int32), envelope=g("envelope").astype(np.float64))
        offs = d[f"{prefix}product_offsets"]
        facs = d[f"{prefix}product_factors"]
        products = [list(map(int, facs[offs[k]:offs[k + 1]])) for k in range(len(offs) - 1)]
        return cls(
            atomic_numbers=[int(z) for z in d[f"{prefix}atomic_numbers"]], lmax=int(d[f"{prefix}lmax"]),
            radial=fams["radial"], pair=fams["pair"],
            density=np.ascontiguousarray(d[f"{prefix}density"], dtype=np.int32), products=products,
            coupling_rows=np.ascontiguousarray(d[f"{prefix}coupling_rows"], dtype=np.int32),
            coupling_cols=np.ascontiguousarray(d[f"{prefix}coupling_cols"], dtype=np.int32),
            coupling_vals=np.ascontiguousarray(d[f"{prefix}coupling_vals"], dtype=np.float64),
            nbasis=int(d[f"{prefix}nbasis"]), WB=np.ascontiguousarray(d[f"{prefix}WB"], dtype=np.float64),
            Wpair=np.ascontiguousarray(d[f"{prefix}Wpair"], dtype=np.float64),
            reference=np.ascontiguousarray(d[f"{prefix}reference"], dtype=np.float64),
            pair_allowed=np.ascontiguousarray(d[f"{prefix}pair_allowed"], dtype=np.uint8),
            angular_kind=int(d[f"{prefix}angular_kind"]) if f"{prefix}angular_kind" in d else 0)

    def save(self, path):
        np.savez_compressed(path, **self.to_npz_dict())

    @classmethod
    def load(cls, path):
        with np.load(path) as d:
            return cls.from_npz_dict(d)


def _read_family(D: dict, nz: int) -> RadialFamily:
    """read_radial (ACE/resolved.jl:57-92) + pack_radials (adaptation.jl:57-75)."""
    if D.get("kind") != "piecewise_cubic_agnesi":
        raise argument_error("unsupported resolved radial kind")
    spec = [(int(b["n"]), int(b["l"])) for b in D["spec"]]
    seen = {}
    for ch in D["channels"]:
        ij = (int(ch["centre"]), int(ch["neighbour"]))
        if not all(1 <= i <= nz for i in ij) or ij in seen:
            raise argument_error("invalid/duplicate radial species channel")
        seen[ij] = ch
    if len(seen) != nz * nz:
        raise argument_error("missing radial species channels")
    nk = max(len(ch["nodes"]) for ch in D["channels"])
    nch = len(spec)
    lengths = np.zeros(nz * nz, np.int32)
    nodes = np.zeros((nz * nz, nk))
    coeff = np.zeros((nz * nz, nk - 1, nch, 4))
    transform = np.zeros((nz * nz, 6))
    powers = np.zeros((nz * nz, 2), np.int32)
    env_kind = np.zeros(nz * nz, np.int32)
    env = np.zeros((nz * nz, 5))
    for (ci, ni), ch in seen.items():
        k = (ci - 1) * nz + (ni - 1)
        t = ch["transform"]
        if t["normalization_rin"] != t["rin"]:
            raise argument_error("unsupported differing transform origins")
        p, q = int(t["p"]), int(t["q"])
        if not (p > 0 and q >= p and t["a"] > 0 and t["rcut"] > t["r0"] > t["rin"]):
            raise argument_error("invalid Agnesi transform")
        kind = ch["envelope_kind"]
        e = ch["envelope"]
        if kind == "PolyEnvelope2sX":
            ep = [e["x1"], e["x2"], e["p1"], e["p2"], e["s"]]
        elif kind == "PolyEnvelope1sR":
            ep = [e["rcut"], e["p"]]
        elif kind == "ACE1_PolyEnvelope1sR":
            ep = [e["rcut"], e["r0"], e["p"]]
        else:
            raise argument_error(f"unsupported resolved envelope {kind}")
        nd = np.asarray(ch["nodes"], dtype=np.float64)
        if not (len(nd) >= 2 and nd[0] == -1 and nd[-1] == 1 and np.all(np.diff(nd) > 0)):
            raise argument_error("invalid spline nodes")
        shape = tuple(int(s) for s in ch["coefficient_shape"])
        if shape != (4, nch, len(nd) - 1):
            raise dimension_mismatch("invalid spline coefficients")
        # Julia column-major reshape of the flat coefficient list to (4, nch, K-1)
        c = np.asarray(ch["coefficients"], dtype=np.float64).reshape(shape[::-1]).transpose(2, 1, 0)
        if not np.all(np.isfinite(c)):
            raise argument_error("nonfinite spline coefficients")
        lengths[k] = len(nd)
        nodes[k, :len(nd)] = nd
        coeff[k, :len(nd) - 1] = c.transpose(2, 1, 0)  # [interval, channel, power]
        transform[k] = [t["a"], t["rin"], t["r0"], t["yin"], t["ycut"], t["rcut"]]
        powers[k] = [p, q]
        env_kind[k] = ENVELOPE_KIND[kind]
        env[k, :len(ep)] = ep
    return RadialFamily(spec, lengths, nodes, coeff, transform, powers, env_kind, env)


def read_resolved(D: dict) -> PackedACE:
    """Read the schema-v1 dict (ACE/resolved.jl:103-142) into packed tables."""
    if not (D.get("schema") == "PotentialFrameWork.resolved_ACE" and D.get("schema_version") == 1):
        raise argument_error("unsupported resolved ACE schema")
    z = [int(v) for v in D["species_atomic_numbers"]]
    nz = len(z)
    if len(set(z)) != nz or not all(v > 0 for v in z):
        raise argument_error("invalid species channels")
    ang = D["angular"]
    if not (ang["kind"] in ("real_spherical", "real_solid") and ang["normalization"] == "L2"
            and ang["ordering"] == "l*l+l+m+1"):
        raise argument_error("unsupported angular convention")
    angular_kind = 1 if ang["kind"] == "real_solid" else 0
    lmax = int(ang["lmax"])
    if lmax < 0:
        raise argument_error("invalid lmax")
    radial = _read_family(D["radial"], nz)
    pair = _read_family(D["pair_radial"], nz)
    density = [tuple(int(x) for x in v) for v in D["density_indices"]]
    if not all(len(v) == 2 and 1 <= v[0] <= len(radial.spec) and 1 <= v[1] <= (lmax + 1) ** 2 for v in density):
        raise argument_error("invalid density indices")
    products = [[int(x) for x in v] for v in D["products"]]
    if not all(len(v) > 0 and all(1 <= i <= len(density) for i in v) for v in products):
        raise argument_error("invalid product indices")
    c = D["coupling"]
    m, n = (int(s) for s in c["shape"])
    if n != len(products):
        raise dimension_mismatch("coupling/product dimensions")
    rows = np.asarray(c["rows"], dtype=np.int64) - 1
    cols = np.asarray(c["columns"], dtype=np.int64) - 1
    vals = np.asarray(c["values"], dtype=np.float64)
    # sparse(rows, cols, vals): duplicates are summed; store in CSC order
    key = cols * m + rows
    order = np.argsort(key, kind="stable")
    key, vals = key[order], vals[order]
    ukey, inv = np.unique(key, return_inverse=True)
    uvals = np.zeros(len(ukey))
    np.add.at(uvals, inv, vals)
    crow = (ukey % m).astype(np.int32)
    ccol = (ukey // m).astype(np.int32)
    params = D["parameters"]
    if params["ordering"] != "vec(WB), vec(Wpair); Julia column-major":
        raise argument_error("unsupported parameter ordering")
    nq = len(pair.spec)
    if list(params["WB_shape"]) != [m, nz] or list(params["Wpair_shape"]) != [nq, nz]:
        raise dimension_mismatch("readout dimensions")
    flat = np.asarray(params["flat"], dtype=np.float64)
    if len(flat) != (m + nq) * nz:
        raise dimension_mismatch("parameter length")
    ref = np.asarray(D["reference_eV"], dtype=np.float64)
    if len(ref) != nz:
        raise dimension_mismatch("reference energy channels")
    if not (np.all(np.isfinite(flat)) and np.all(np.isfinite(ref)) and np.all(np.isfinite(uvals))):
        raise argument_error("nonfinite model values")
    WB = flat[: m * nz].reshape(nz, m).copy()  # column-major (m, nz) -> [z][b]
    Wpair = flat[m * nz:].reshape(nz, nq).copy()
    parameters0 = {"WB": WB.T.copy(), "Wpair": Wpair.T.copy()}
    mask = None
    pair_allowed = np.ones(nz, np.uint8)
    if "interface_policy" in D:
        mask, use_pair, use_ref = _read_policy(D["interface_policy"], m, len(products), len(density),
                                               len(radial.spec), nz)
        # pack_model drops masked coupling entries (adaptation.jl:84-87) and
        # effective_WB zeroes their readout (interface.jl:125)
        keep = mask[crow]
        crow, ccol, uvals = crow[keep], ccol[keep], uvals[keep]
        WB *= mask[None, :]
        if not use_pair:
            pair_allowed[:] = 0
        if not use_ref:
            ref = np.zeros_like(ref)
    if D.get("coordinate_kind") == "legacy_PI" or D.get("conversion", {}).get("kind") == "exact_legacy_complex_PI_to_real":
        pass  # numerics identical; descriptor selection is outside the device path
    return PackedACE(
        atomic_numbers=z, lmax=lmax, radial=radial, pair=pair,
        density=np.array([[v[0] - 1, v[1] - 1] for v in density], dtype=np.int32).reshape(-1, 2),
        products=[[i - 1 for i in p] for p in products],
        coupling_rows=crow, coupling_cols=ccol, coupling_vals=uvals, nbasis=m,
        WB=np.ascontiguousarray(WB), Wpair=np.ascontiguousarray(Wpair), reference=ref.copy(),
        pair_allowed=pair_allowed, source_sha256=str(D.get("source_sha256", "")), angular_kind=angular_kind,
        resolved={k: copy.deepcopy(v) for k, v in D.items() if k != "parameters"}, mask=mask,
        parameters0=parameters0)


def _read_policy(d, nrows, nproducts, ndensity, nradial, nz):
    """read_policy (ACE/interface_persistence.jl:8-24) for the device: the
    provenance maps are validated as the reference does; the invariant mask,
    the pair flag and the reference flag are applied; a species/order
    projection (selected storage) is not packed for the device."""
    if d.get("version") != 1:
        raise argument_error("unsupported basis policy version")
    for key, n in (("rows", nrows), ("products", nproducts), ("density", ndensity), ("radial", nradial)):
        v = d[key]
        if not (len(v) == n and all(isinstance(x, int) and not isinstance(x, bool) and x > 0 for x in v)
                and len(set(v)) == n):
            raise argument_error(f"invalid {key} provenance map")
    mask = d["mask"]
    if not (len(mask) == nrows and all(isinstance(x, bool) for x in mask)):
        raise argument_error("invalid invariant mask")
    sp = [int(x) for x in d["species"]]
    if not (all(1 <= i <= nz for i in sp) and len(set(sp)) == len(sp)):
        raise argument_error("invalid projected species")
    o = d["orders"]
    if not (len(o) == 0 or (len(o) == 2 and 0 <= o[0] <= o[1])):
        raise argument_error("invalid projected orders")
    if len(d["origin"]) != 64:
        raise argument_error("invalid basis namespace")
    if sp or o:
        raise argument_error("projected species/order policies are not packed for the device")
    return np.array(mask, bool), bool(d["pair"]), bool(d["reference"])


def load_resolved(path) -> PackedACE:
    """load_resolved(path) (ACE/resolved.jl:98-102) — TOML file to packed tables."""
    import tomllib

    with open(path, "rb") as f:
        raw = f.read()
    m = read_resolved(tomllib.loads(raw.decode()))
    m.file_sha256 = hashlib.sha256(raw).hexdigest()
    return m

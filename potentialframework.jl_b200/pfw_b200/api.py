"""Host-side mirror of the reference's public API for the force-evaluation path.

Same names, argument meaning and error behaviour as PotentialFrameWork.jl:

  Workspace(width=4, precision="Float64", bruteforce_threshold=32)
                                    NeighbourList/storage.jl:59-65
  evaluate_(w, sys, p, request=EnergyForcesVirial())   (Julia `evaluate!`)
  evaluate(sys, p, width=4, precision=..., bruteforce_threshold=32)
                                    PairPotentials/evaluation.jl:31-52,64-66
  SmoothPair(labels, amplitudes, radius), lennard_jones(epsilon, sigma, radius)
                                    PairPotentials/models.jl:28-44, lennard_jones.jl:19-24
  neighbour_list(sys, cutoff) / neighbour_list(X, cutoff, cell, pbc), neighbours(list, i)
                                    NeighbourList/interface.jl:47-151
  potential_energy / forces / virial / energy_forces / energy_forces_virial and the
  in-place forces_ / energy_forces_ / energy_forces_virial_ (which ADD into the
  destination)                      PairPotentials/calculators.jl:54-94
  ACECalculator(model | path), load_resolved(path), save_calculator(path, calc),
  trainable_parameters(model, ps)   ACE/calculators.jl, ACE/resolved.jl:98-102,
                                    ACE/persistence.jl:101-167, ACE/serial.jl:12-16

Systems are numeric (Å): any object with X (n,3), H (3,3, columns = cell
vectors), pbc (3 flags) and species (channel ints, the model's labels, or
element symbols for ACE models, which are labelled by atomic number).  Unit
handling is the caller's: the Julia shim strips Unitful units at the boundary
exactly where the reference does (storage.jl:74-78).  Every evaluation runs
on the GPU through libpfw_b200.so; there is no CPU path.
"""
from __future__ import annotations

import copy
import os

import numpy as np

from . import checkpoint as _checkpoint
from . import lib as _lib
from .ace_model import PackedACE
from .ace_model import load_resolved as _load_resolved
from .lib import ArgumentError, DimensionMismatch, DomainError  # noqa: F401


class EnergyOnly:
    pass


class EnergyForcesVirial:
    pass


class Energy:
    pass


class Forces:
    pass


class Virial:
    pass


def _request_bits(request):
    """normalize_properties (NeighbourList/execution.jl:155-163)."""
    if isinstance(request, EnergyOnly) or request is EnergyOnly:
        return _lib.REQ_E
    if isinstance(request, EnergyForcesVirial) or request is EnergyForcesVirial:
        return 7
    props = request if isinstance(request, (tuple, list)) else (request,)
    bits = 0
    for p in props:
        p = p() if isinstance(p, type) else p
        if isinstance(p, Energy) or p == "energy":
            bits |= _lib.REQ_E
        elif isinstance(p, Forces) or p == "forces":
            bits |= _lib.REQ_F
        elif isinstance(p, Virial) or p == "virial":
            bits |= _lib.REQ_V
        else:
            raise ArgumentError(_lib.EINVAL, "supported properties are Energy(), Forces() and Virial()")
    return bits


_ELEMENTS = ("H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn Ga Ge As Se Br Kr "
             "Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe Cs Ba La Ce Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm Yb "
             "Lu Hf Ta W Re Os Ir Pt Au Hg Tl Pb Bi Po At Rn Fr Ra Ac Th Pa U Np Pu Am Cm Bk Cf Es Fm Md No Lr Rf "
             "Db Sg Bh Hs Mt Ds Rg Cn Nh Fl Mc Lv Ts Og").split()


def species_channels(species, labels):
    """Species of a system → the model's channel indices (bind_species,
    PairPotentials/models.jl:50-58; ACE channels by atomic number).  Integer
    arrays are channel indices already.  Other entries are matched to the
    labels by equality; for models labelled by atomic number (ACE) an element
    symbol is matched through its atomic number.  An entry the model has no
    parameters for raises ArgumentError."""
    sp = np.asarray(species)
    if sp.dtype.kind in "iu":
        return sp.astype(np.int32)
    labels = list(labels)
    numeric = all(isinstance(v, (int, np.integer)) for v in labels)
    ids = []
    for s in sp:
        key = s
        if numeric and isinstance(s, str) and s in _ELEMENTS:
            key = _ELEMENTS.index(s) + 1
        if key not in labels:
            raise ArgumentError(_lib.EINVAL, f"potential has no parameters for species {s}")
        ids.append(labels.index(key))
    return np.array(ids, np.int32)


class SmoothPair:
    """U_ab(r) = A_ab (1 - r²/c²)³ for r < c (PairPotentials/models.jl:28-44)."""

    def __init__(self, labels, amplitudes, radius):
        labels = list(labels)
        A = np.asarray(amplitudes, dtype=np.float64)
        n = len(labels)
        if A.shape != (n, n):
            raise ArgumentError(_lib.EINVAL, "parameter table size must match species labels")
        if len(set(labels)) != n:
            raise ArgumentError(_lib.EINVAL, "species labels must be unique")
        if not (np.all(np.isfinite(A)) and np.array_equal(A, A.T)):
            raise ArgumentError(_lib.EINVAL, "amplitude table must be finite and symmetric")
        if not (np.isfinite(radius) and radius > 0):
            raise ArgumentError(_lib.EINVAL, "cutoff must be finite and positive")
        self.labels, self.amplitudes, self.radius = labels, A, float(radius)

    def cutoff(self):
        return self.radius

    def get_parameters(self):
        """AC.get_parameters (PairPotentials/parameters.jl:34-37): the upper
        triangle of the amplitude table in column order, A[i, j] for
        j = 1..n, i = 1..j."""
        n = len(self.labels)
        return {"amplitudes": np.array([self.amplitudes[i, j] for j in range(n) for i in range(j + 1)])}

    def set_parameters(self, parameters):
        """AC.set_parameters! (parameters.jl:54): a new model, as with_parameters."""
        return with_parameters(self, parameters)


class LennardJones:
    """Energy-shifted LJ (PairPotentials/lennard_jones.jl:5-33)."""

    def __init__(self, epsilon, sigma, radius):
        self.epsilon, self.sigma, self.radius = float(epsilon), float(sigma), float(radius)
        if not all(np.isfinite(v) and v > 0 for v in (self.epsilon, self.sigma, self.radius)):
            raise ArgumentError(_lib.EINVAL, "LJ parameters must be positive and finite")

    def cutoff(self):
        return self.radius

    def get_parameters(self):
        """AC.get_parameters (PairPotentials/lennard_jones.jl:23)."""
        return {"epsilon": self.epsilon, "sigma": self.sigma}

    def set_parameters(self, parameters):
        return with_parameters(self, parameters)


def lennard_jones(epsilon=0.0103, sigma=3.4, radius=8.5):
    return LennardJones(epsilon, sigma, radius)


class Workspace:
    """GPU workspace: the drop-in for NeighbourList.Workspace (one per thread).

    `width` is accepted for API compatibility (the GPU kernels have no SIMD
    lane width); `precision` is "Float64" (plain path) or "mixed"
    (FP32 arithmetic, FP64 wrap, Kahan FP64 energy/virial).  `skin` > 0
    keeps a pair list of all images within cutoff + skin between calls on
    the same structure and rebuilds it only once an atom has moved more than
    skin/2 (the GPU skin list of NeighbourList/gpu.jl:404-549); pairs within
    about one ulp of the cutoff may then differ from a rebuild."""

    def __init__(self, width=4, precision="Float64", bruteforce_threshold=32, device=0, skin=0.0):
        if width not in (1, 2, 4, 8, 16):
            raise ArgumentError(_lib.EINVAL, "width must be 1, 2, 4, 8 or 16")
        if precision in ("Float64", np.float64, float):
            prec = _lib.FP64
        elif precision in ("mixed", "Float32", np.float32):
            prec = _lib.MIXED
        else:
            raise ArgumentError(_lib.EINVAL, "precision must be Float64 or mixed")
        if not (isinstance(bruteforce_threshold, (int, np.integer)) and bruteforce_threshold >= 0):
            raise ArgumentError(_lib.EINVAL, "bruteforce_threshold must be a nonnegative integer")
        self.width = width
        self.precision = precision
        self.handle = _lib.Handle(prec, bruteforce_threshold, device)
        if not (np.isfinite(skin) and skin >= 0):
            raise ArgumentError(_lib.EINVAL, "skin must be finite and nonnegative")
        if skin:
            self.handle.pair_skin(skin)
        self._model_key = None

    # geometry/model binding -------------------------------------------
    def _species(self, sys, labels):
        return species_channels(sys.species, labels)

    def bind(self, sys, p):
        if isinstance(p, SmoothPair):
            species = self._species(sys, p.labels)
            self.handle.smooth(p.amplitudes, p.radius)
        elif isinstance(p, LennardJones):
            species = np.zeros(len(sys.X), np.int32)
            self.handle.lj(p.epsilon, p.sigma, p.radius)
        elif isinstance(p, ACECalculator):
            species = self._species(sys, p.model.atomic_numbers)
            dev = p.device_model()
            if self._model_key is not dev:
                self.handle.ace(dev)
                self._model_key = dev
        else:
            raise ArgumentError(_lib.EINVAL, "pair evaluation requires SmoothPair or lennard_jones")
        self.handle.set_geometry(sys.X, sys.H, sys.pbc, species)
        return _lib.MODEL_ACE if isinstance(p, ACECalculator) else _lib.MODEL_PAIR


def evaluate_(w: Workspace, sys, p, request=EnergyForcesVirial(), parallel=False, parameters=None):
    """evaluate!(w, sys, p; request) — rebuilds topology on every call and returns
    owning, original-order outputs (energy eV, forces (n,3) eV/Å, virial 3×3 eV)."""
    if parameters is not None:
        p = with_parameters(p, parameters)
    bits = _request_bits(request)
    model = w.bind(sys, p)
    E, F, W = w.handle.evaluate(model, bits)
    if isinstance(request, EnergyOnly) or request is EnergyOnly:
        return dict(energy=E)
    if isinstance(request, EnergyForcesVirial) or request is EnergyForcesVirial:
        return dict(energy=E, forces=F, virial=W)
    out = {}
    if bits & _lib.REQ_E:
        out["energy"] = E
    if bits & _lib.REQ_F:
        out["forces"] = F
    if bits & _lib.REQ_V:
        out["virial"] = W
    return out


def evaluate(sys, p, width=4, precision="Float64", bruteforce_threshold=32, **kw):
    return evaluate_(Workspace(width=width, precision=precision, bruteforce_threshold=bruteforce_threshold), sys, p,
                     **kw)


def with_parameters(p, parameters):
    """with_parameters (PairPotentials/parameters.jl:38-53, lennard_jones.jl:24-27)."""
    if isinstance(p, SmoothPair):
        if set(parameters) != {"amplitudes"}:
            raise ArgumentError(_lib.EINVAL, "SmoothPair parameters must contain only amplitudes; cutoff is fixed")
        a = np.asarray(parameters["amplitudes"], dtype=np.float64)
        n = len(p.labels)
        if a.shape != (n * (n + 1) // 2,):
            raise ArgumentError(_lib.EINVAL, "amplitudes must be a real vector of length n*(n+1)/2")
        if not np.all(np.isfinite(a)):
            raise ArgumentError(_lib.EINVAL, "amplitudes must be finite")
        A = np.zeros((n, n))
        for j in range(n):
            for i in range(j + 1):
                A[i, j] = A[j, i] = a[j * (j + 1) // 2 + i]  # upper triangle, column order
        return SmoothPair(p.labels, A, p.radius)
    if isinstance(p, LennardJones):
        if set(parameters) != {"epsilon", "sigma"}:
            raise ArgumentError(_lib.EINVAL, "LJ parameters require epsilon and sigma; cutoff is fixed")
        return LennardJones(parameters["epsilon"], parameters["sigma"], p.radius)
    if isinstance(p, ACECalculator):
        return ACECalculator(p.model, parameters, p.state)
    raise ArgumentError(_lib.EINVAL, f"{type(p).__name__} does not implement with_parameters")


# ---- neighbour snapshot ----------------------------------------------------
class NeighbourSnapshot:
    def __init__(self, offsets, j, S, R):
        self.offsets, self.j, self.S, self.R = offsets, j, S, R

    def __len__(self):
        return len(self.offsets) - 1

    def npairs(self):
        return int(self.offsets[-1])


class _RawSystem:
    def __init__(self, X, H, pbc):
        self.X = X
        self.H = H
        self.pbc = pbc
        self.species = np.zeros(len(X), np.int32)


def neighbour_list(X_or_sys, cutoff, cell=None, pbc=None, width=4, precision="Float64", bruteforce_threshold=32,
                   int_type=np.int32, workspace=None):
    """neighbour_list (NeighbourList/interface.jl:47-83).  Raw form: cell has the
    lattice vectors in ROWS (NeighbourLists.jl convention); AtomsBase-like form:
    sys.H columns are cell vectors."""
    if cell is not None:
        cell = np.asarray(cell, dtype=np.float64)
        if cell.shape != (3, 3):
            raise DimensionMismatch(_lib.ESHAPE, "cell must be 3×3 with vectors in rows")
        if len(pbc) != 3:
            raise DimensionMismatch(_lib.ESHAPE, "pbc must contain three flags")
        X = np.asarray(X_or_sys, dtype=np.float64)
        if X.ndim == 2 and X.shape[1] != 3 and X.shape[0] == 3:
            X = X.T
        if X.size and X.shape[-1] != 3:
            raise DimensionMismatch(_lib.ESHAPE, "positions must be 3-vectors")
        sys = _RawSystem(X.reshape(-1, 3), cell.T, pbc)
    else:
        sys = X_or_sys
    if np.dtype(int_type) not in (np.int8, np.int16, np.int32, np.int64):
        raise ArgumentError(_lib.EINVAL, "int_type must be a signed built-in integer type")
    if len(sys.X) > np.iinfo(int_type).max:
        raise ArgumentError(_lib.EINVAL, "int_type cannot represent all atom indices")
    c = float(cutoff)
    if not (np.isfinite(c) and c > 0):
        raise ArgumentError(_lib.EINVAL, "cutoff must be finite and positive (Å)")
    w = workspace or Workspace(width=width, precision=precision, bruteforce_threshold=bruteforce_threshold)
    w.handle.set_geometry(sys.X, sys.H, sys.pbc, np.zeros(len(sys.X), np.int32))
    offs, j, S, R = w.handle.neighbour_list(c)
    info = np.iinfo(int_type)
    if len(S) and (S.max() > info.max or -S.max() < info.min or S.min() < info.min or -S.min() > info.max):
        raise OverflowError("image shift does not fit int_type")
    return NeighbourSnapshot(offs, j.astype(int_type), S.astype(int_type), R)


def neighbours(lst: NeighbourSnapshot, i):
    """neighbours(list, i) → (js, Rs, Ss), independent arrays, 0-based i and js."""
    if not (0 <= i < len(lst)):
        raise IndexError(i)
    a, b = lst.offsets[i], lst.offsets[i + 1]
    return lst.j[a:b].copy(), lst.R[a:b].copy(), lst.S[a:b].copy()


# ---- ACE ------------------------------------------------------------------
class ACECalculator:
    """GPU ACE calculator (ACE/calculators.jl:1-40, persistence.jl:101-124).

    ACECalculator(model, parameters=None, state=None) over a packed resolved
    model, or ACECalculator(path) for a checkpoint written by save_calculator
    or a resolved TOML export (the file's content decides).  `parameters`
    ({"WB": (nbasis, nz), "Wpair": (nQ, nz)} and optionally
    {"radial": {"scale": (nR, nz, nz)}, "pair": {"scale": (nQ, nz, nz)}}) is
    authoritative; replace it with set_parameters.  Execution keywords of the
    reference (width, slots, angular_backend, ...) configure CPU scratch and
    are accepted and ignored; nothing of the execution state is saved."""

    def __init__(self, model, parameters=None, state=None, **execution):
        if isinstance(model, (str, os.PathLike)):
            model, ps0, st0 = _checkpoint.load(model)
            parameters = ps0 if parameters is None else parameters
            state = st0 if state is None else state
        if not isinstance(model, PackedACE):
            raise ArgumentError(_lib.EINVAL, "ACECalculator needs a resolved ACE model")
        self.model = model
        self.parameters = copy.deepcopy(model.default_parameters() if parameters is None else parameters)
        self.state = copy.deepcopy({} if state is None else state)
        self._device = model.with_parameters(self.parameters)

    def device_model(self):
        """Packed tables for the installed parameters (mask and scales applied)."""
        return self._device

    def get_parameters(self):
        return copy.deepcopy(self.parameters)

    def set_parameters(self, ps):
        """AC.set_parameters! (calculators.jl:38-42): same readout shapes or
        DimensionMismatch; the calculator keeps its own copy."""
        cur = self.parameters
        if np.shape(ps["WB"]) != np.shape(cur["WB"]) or np.shape(ps["Wpair"]) != np.shape(cur["Wpair"]):
            raise DimensionMismatch(_lib.ESHAPE, "ACE readout shapes")
        self._device = self.model.with_parameters(ps)
        self.parameters = copy.deepcopy(ps)
        return self

    def cutoff(self):
        return self.model.cutoff


def cutoff(p):
    """cutoff(p) (PairPotentials/models.jl:44 and RadialPotential): the model's
    cutoff radius in Å, for SmoothPair, Lennard-Jones and ACECalculator."""
    if not hasattr(p, "cutoff"):
        raise ArgumentError(_lib.EINVAL, f"{type(p).__name__} has no cutoff")
    return p.cutoff()


def get_parameters(p):
    """AtomsCalculators.get_parameters for the pair models and ACECalculator."""
    if not hasattr(p, "get_parameters"):
        raise ArgumentError(_lib.EINVAL, f"{type(p).__name__} has no parameters")
    return p.get_parameters()


def set_parameters(p, parameters):
    """AtomsCalculators.set_parameters!: the pair models are immutable and
    return a new model (parameters.jl:54); ACECalculator installs the
    parameters in place and returns itself (ACE/calculators.jl:38-42)."""
    if not hasattr(p, "set_parameters"):
        raise ArgumentError(_lib.EINVAL, f"{type(p).__name__} has no parameters")
    return p.set_parameters(parameters)


def load_resolved(path):
    return _load_resolved(path)


def save_calculator(path, calc, parameters=None, state=None):
    """save_calculator (ACE/persistence.jl:139-167)."""
    return _checkpoint.save_calculator(path, calc, parameters, state)


def trainable_parameters(model, ps):
    """trainable_parameters (ACE/serial.jl:12-16)."""
    return _checkpoint.trainable_parameters(model.model if isinstance(model, ACECalculator) else model, ps)


# ---- AtomsCalculators methods (PairPotentials/calculators.jl:54-94) --------
_default_ws = {}


def _ws(neighbourlist=None):
    if neighbourlist is not None:
        return neighbourlist
    import threading
    key = threading.get_ident()
    if key not in _default_ws:
        _default_ws[key] = Workspace()
    return _default_ws[key]


def potential_energy(sys, p, neighbourlist=None, **kw):
    return evaluate_(_ws(neighbourlist), sys, p, request=EnergyOnly())["energy"]


def forces(sys, p, neighbourlist=None, **kw):
    return evaluate_(_ws(neighbourlist), sys, p, request=(Forces(),))["forces"]


def virial(sys, p, neighbourlist=None, **kw):
    return evaluate_(_ws(neighbourlist), sys, p, request=(Virial(),))["virial"]


def energy_forces(sys, p, neighbourlist=None, **kw):
    r = evaluate_(_ws(neighbourlist), sys, p, request=(Energy(), Forces()))
    return dict(energy=r["energy"], forces=r["forces"])


def energy_forces_virial(sys, p, neighbourlist=None, **kw):
    return evaluate_(_ws(neighbourlist), sys, p)


def _add_into(dest, value):
    dest = np.asarray(dest)
    if dest.shape != value.shape:
        raise DimensionMismatch(_lib.ESHAPE, "force destination has the wrong shape")
    dest += value
    return dest


def forces_(F, sys, p, neighbourlist=None, **kw):
    """In-place: ADDS the forces into F (calculators.jl:79-94)."""
    _add_into(F, forces(sys, p, neighbourlist))
    return F


def energy_forces_(F, sys, p, neighbourlist=None, **kw):
    r = energy_forces(sys, p, neighbourlist)
    _add_into(F, r["forces"])
    return dict(energy=r["energy"], forces=F)


def energy_forces_virial_(F, sys, p, neighbourlist=None, **kw):
    r = energy_forces_virial(sys, p, neighbourlist)
    _add_into(F, r["forces"])
    return dict(energy=r["energy"], forces=F, virial=r["virial"])


def calculate(props, sys, p, parameters=None, state=None, neighbourlist=None):
    """AtomsCalculators.calculate (PairPotentials/calculators.jl:100-143,
    ACE/calculators.jl:113-129): the requested properties plus `state`
    (the calculator's own state for ACE when none is given)."""
    if isinstance(p, ACECalculator) and state is None:
        state = p.state
    if parameters is not None and not (isinstance(parameters, dict) and not parameters):
        p = with_parameters(p, parameters)
    out = {} if isinstance(props, (tuple, list)) and len(props) == 0 else \
        evaluate_(_ws(neighbourlist), sys, p, request=props)
    out["state"] = state
    return out

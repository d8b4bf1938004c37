"""Linear fitting rows of the ACE model on the GPU (ACE/fitting.jl).

  design_matrix(systems, calc, fit_pair=True)
        design_matrix_impl (fitting.jl:18-67): energy, vec(forces) and
        vec(virial) rows of every structure, stacked structure after structure
        (the assembly ACEfit builds), computed by one batched launch of the
        design kernel (pfw_ace_design_matrix).  Returns dict(matrix, baseline):
        `baseline` holds the reference energies on the energy rows and, with
        fit_pair=False, the pair term of the installed Wpair on every row
        (whose columns are then dropped), exactly as the reference.
  linear_parameters(ps), install_readout(ps, coefficients, fit_pair)
        fitting.jl:1-11
  training_rows(design, labels, weights)
        fitting.jl:118-145 for one structure's design

The radial scales of the calculator's parameters (trainable_parameters) are
part of the basis and are applied; its WB and Wpair are not used except for
the fit_pair=False baseline.
"""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from . import lib as _lib
from .errors import argument_error, dimension_mismatch


def _systems(systems):
    if hasattr(systems, "X"):
        return [systems], True
    return list(systems), False


def design_matrix(systems, calc, fit_pair=True, handle=None):
    """Design rows for one structure or a list of structures (see module doc)."""
    sys_list, single = _systems(systems)
    model = calc.device_model()
    h = handle or _lib.Handle(_lib.FP64)
    h.ace(model)
    species = []
    for s in sys_list:
        sp = np.asarray(s.species)
        if sp.dtype.kind not in "iu":
            sp = np.array([model.atomic_numbers.index(int(z)) if not isinstance(z, str) else -1 for z in sp], np.int32)
            if np.any(sp < 0):
                raise argument_error("species must be channel indices or atomic numbers of the model")
        species.append(sp.astype(np.int32))
    if single:
        s = sys_list[0]
        h.set_geometry(s.X, s.H, s.pbc, species[0])
    else:
        h.set_batch([SimpleNamespace(X=s.X, H=s.H, pbc=s.pbc, species=z) for s, z in zip(sys_list, species)])
    A, base = h.design_matrix()
    rows = A.shape[0]
    baseline = np.zeros(rows)
    r0 = 0
    for k, s in enumerate(sys_list):
        baseline[r0] = base[k]
        r0 += 10 + 3 * len(s.X)
    if not fit_pair:
        nb = model.nz * model.nbasis
        Wp = np.asarray(calc.parameters["Wpair"], np.float64)
        baseline += A[:, nb:] @ Wp.ravel(order="F")
        A = np.ascontiguousarray(A[:, :nb])
    return dict(matrix=A, baseline=baseline)


def linear_parameters(ps):
    """vcat(vec(WB), vec(Wpair)) (fitting.jl:1)."""
    return np.concatenate([np.asarray(ps["WB"], np.float64).ravel(order="F"),
                           np.asarray(ps["Wpair"], np.float64).ravel(order="F")])


def install_readout(ps, coefficients, fit_pair=True):
    """install_readout (fitting.jl:2-11): new parameters with the fitted readout."""
    c = np.asarray(coefficients, np.float64)
    WB = np.asarray(ps["WB"])
    n = WB.size
    out = dict(ps)
    if not fit_pair:
        if c.size != n:
            raise dimension_mismatch("ACE readout length")
        out["WB"] = c.reshape(WB.shape, order="F").copy()
        return out
    Wp = np.asarray(ps["Wpair"])
    if c.size != n + Wp.size:
        raise dimension_mismatch("readout length")
    out["WB"] = c[:n].reshape(WB.shape, order="F").copy()
    out["Wpair"] = c[n:].reshape(Wp.shape, order="F").copy()
    return out


def training_rows(design, labels, weights=None):
    """training_rows (fitting.jl:118-145) for one structure: labels is a dict
    with optional energy (eV), forces ((n,3) or 3n, eV/Å) and virial (3×3, eV);
    a missing or None label omits its rows.  Returns dict(matrix, labels,
    row_weights) with labels minus the design's baseline."""
    w_all = dict(energy=1.0, forces=1.0, virial=1.0)
    w_all.update(weights or {})
    A, base = design["matrix"], design["baseline"]
    n3 = A.shape[0] - 10
    idx, vals, rw = [], [], []
    for key, rng in (("energy", range(0, 1)), ("forces", range(1, 1 + n3)), ("virial", range(1 + n3, 10 + n3))):
        v = labels.get(key)
        if v is None:
            continue
        if key == "energy":
            v = np.array([float(v)])
        elif key == "virial":
            v = np.asarray(v, np.float64).reshape(3, 3).ravel(order="F")
        else:
            v = np.asarray(v, np.float64)
            if v.ndim == 2 and v.shape[1] != 3:
                raise dimension_mismatch("forces need three components per atom")
            v = v.ravel()
        if v.size != len(rng):
            raise dimension_mismatch(f"{key} label dimensions")
        w = float(w_all[key])
        if not (np.isfinite(w) and w >= 0):
            raise argument_error(f"invalid {key} weight")
        idx.extend(rng)
        vals.extend(v.tolist())
        rw.extend([w] * len(rng))
    idx = np.array(idx, dtype=np.int64)
    return dict(matrix=A[idx], labels=np.array(vals) - base[idx], row_weights=np.array(rw))

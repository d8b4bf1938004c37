"""pfw_b200 — host side of libpfw_b200.so, the B200-native force-evaluation
hot path of PotentialFrameWork.jl (cell lists, SmoothPair/LJ pairs, ACE)."""
from .api import (ACECalculator, Energy, EnergyForcesVirial, EnergyOnly, Forces, LennardJones, SmoothPair,  # noqa
                  Virial, Workspace, calculate, cutoff, energy_forces, energy_forces_, energy_forces_virial,
                  energy_forces_virial_, evaluate, evaluate_, forces, forces_, get_parameters, lennard_jones,
                  load_resolved, neighbour_list, neighbours, potential_energy, save_calculator, set_parameters,
                  trainable_parameters, virial, with_parameters)
from .lib import ArgumentError, DimensionMismatch, DomainError, PFWError  # noqa: F401
from .precision import compare_precision  # noqa: F401

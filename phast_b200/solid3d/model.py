"""3D cell description: voxel grid, phase materials, load case and solver settings.

Mirrors the data classes of ``phast.solid3d.model`` (src/phast/solid3d/model.py:183-895)
that the hot path reads.  Objects of the reference package with the same fields
are accepted wherever these are.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

VOIGT = ("xx", "yy", "zz", "yz", "xz", "xy")


@dataclass(frozen=True)
class VoxelGrid:
    """``shape`` (nx, ny, nz), voxel size ``h``; voxel arrays are (nz, ny, nx) (model.py:183-300)."""
    shape: tuple
    h: tuple
    origin: tuple = (0.0, 0.0, 0.0)
    periodic: tuple = (True, True, True)

    @property
    def n_elements(self):
        nx, ny, nz = self.shape
        return nx * ny * nz

    @property
    def lengths(self):
        return tuple(n * h for n, h in zip(self.shape, self.h))

    @property
    def volume(self):
        lx, ly, lz = self.lengths
        return lx * ly * lz

    @property
    def voxel_volume(self):
        return self.h[0] * self.h[1] * self.h[2]


@dataclass(frozen=True)
class PhaseMaterial:
    """Isotropic phase: E, nu (MPa), Gc (N/mm), damage driver ('spectral', 'full' or 'none')."""
    name: str
    E: float
    nu: float
    Gc: float
    driver: str = "spectral"
    kind: str = "isotropic"


@dataclass(frozen=True)
class LoadCase:
    """Mixed macro-strain control (model.py:589-681)."""
    name: str
    controlled: int
    targets: tuple
    free: tuple = ()
    fixed_zero: tuple = ()

    def __post_init__(self):
        comps = sorted([int(self.controlled), *self.free, *self.fixed_zero])
        if comps != list(range(6)):
            raise ValueError("{controlled}, free and fixed_zero must partition {0,...,5}")

    @property
    def n_increments(self):
        return len(self.targets)

    @classmethod
    def ramp(cls, name, controlled, to, increments, fixed_zero=None):
        fz = tuple(i for i in range(6) if i != controlled) if fixed_zero is None else tuple(fixed_zero)
        return cls(name, controlled, tuple(to * k / increments for k in range(1, increments + 1)), (), fz)


@dataclass(frozen=True)
class SolverConfig:
    """Staggered settings (model.py:706-895); defaults are PhAST's."""
    kappa: float = 1.0e-6
    stagger_tol: float = 1.0e-4
    max_stagger: int = 2000
    min_stagger: int = 2
    pcg_rtol_mech: float = 1.0e-8
    pcg_maxit_mech: int = 20000
    preconditioner: str = "jacobi"
    check_every: int = 10
    damage_linear_tol: float = 1.0e-10
    damage_kkt_tol: float = 1.0e-8
    damage_maxit: int = 4000
    damage_max_active_set: int = 64
    energy_split_isotropic: str = "spectral"
    final_mechanics_resolve: bool = True
    damaged_threshold: float = 0.95
    max_cutbacks: int = 1
    on_stagger_failure: str = "cutback"


def sphere_pore_phase(shape, radius_fraction, matrix_id=0, pore_id=1):
    """Phase ids (nz, ny, nx): pore where the voxel-centre distance to the cell centre < r * L."""
    nx, ny, nz = shape
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    c = np.stack([(i + 0.5) / nx - 0.5, (j + 0.5) / ny - 0.5, (k + 0.5) / nz - 0.5], -1)
    phase = np.full((nz, ny, nx), matrix_id, dtype=np.uint8)
    phase[np.linalg.norm(c, axis=-1) < radius_fraction] = pore_id
    return phase


def isotropic_C(E, nu):
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    C = np.zeros((6, 6))
    C[:3, :3] = lam
    C[[0, 1, 2], [0, 1, 2]] = lam + 2 * mu
    C[[3, 4, 5], [3, 4, 5]] = mu
    return C, lam, mu

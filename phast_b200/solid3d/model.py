"""3D cell description: voxel grid, phase materials, load case and solver settings.

Mirrors the data classes of ``phast.solid3d.model`` (src/phast/solid3d/model.py:37-897)
and ``build_element_arrays`` (src/phast/solid3d/materials.py:474-547) with the same
names, fields, defaults and validation errors, so a caller written against the
reference builds the same objects here.  Objects of the reference package with
the same fields are accepted wherever these are (the operator reads attributes
only).  Options of the reference that this backend does not run (smeared-laminate
phases with their band closure, the interface driver) are accepted by the data classes and refused
with ``NotImplementedError`` when an operator or solver is built from them.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any, Mapping

import numpy as np
import torch

VOIGT = ("xx", "yy", "zz", "yz", "xz", "xy")
PHASE_NAMES = ("fibre", "bn_band", "cvi_sic", "mi_matrix", "pore")  # model.py:42-48
PHASE_ID = {name: index for index, name in enumerate(PHASE_NAMES)}
DRIVER_NONE, DRIVER_FULL, DRIVER_SPECTRAL = 0, 1, 2  # model.py:52
DRIVER_INTERFACE = 3
MATERIAL_KINDS = ("isotropic", "smeared_laminate")
DRIVER_NAMES = ("spectral", "full", "none", "interface")
_PFCZM_EXPONENTS = {"linear": 2, "exponential": 2.5}  # Wu's softening exponents (physics/pfczm.py:12)


def _set(obj, name, value):
    object.__setattr__(obj, name, value)


def _finite(name, value):
    v = float(value)
    if not math.isfinite(v):
        raise ValueError(f"{name} must be finite, got {value!r}")
    return v


def _positive(name, value):
    v = _finite(name, value)
    if v <= 0.0:
        raise ValueError(f"{name} must be positive, got {value!r}")
    return v


def _positive_int(name, value):
    if isinstance(value, bool) or int(value) != value or int(value) < 1:
        raise ValueError(f"{name} must be a positive integer, got {value!r}")
    return int(value)


def _choice(name, value, allowed):
    if value not in allowed:
        raise ValueError(f"{name} must be one of {tuple(allowed)}, got {value!r}")
    return value


def _triple(name, value, cast):
    items = tuple(value)
    if len(items) != 3:
        raise ValueError(f"{name} must have three entries, got {value!r}")
    return tuple(cast(v) for v in items)


@dataclass(frozen=True)
class VoxelGrid:
    """Structured voxel grid (model.py:183-300): ``shape`` (nx, ny, nz), voxel size ``h``;
    voxel arrays are (nz, ny, nx)."""
    shape: tuple
    h: tuple
    origin: tuple = (0.0, 0.0, 0.0)
    periodic: tuple = (True, True, True)

    def __post_init__(self):
        _set(self, "shape", tuple(_positive_int(f"shape[{a}]", v) for a, v in enumerate(_triple("shape", self.shape,
                                                                                              lambda v: v))))
        _set(self, "h", tuple(_positive(f"h[{a}]", v) for a, v in enumerate(_triple("h", self.h, float))))
        _set(self, "origin", tuple(_finite(f"origin[{a}]", v) for a, v in enumerate(_triple("origin", self.origin,
                                                                                              float))))
        periodic = _triple("periodic", self.periodic, lambda v: v)
        for axis, flag in enumerate(periodic):
            if not isinstance(flag, (bool, np.bool_)):
                raise TypeError(f"periodic[{axis}] must be a bool, got {flag!r}")
        _set(self, "periodic", tuple(bool(f) for f in periodic))

    @property
    def nx(self):
        return self.shape[0]

    @property
    def ny(self):
        return self.shape[1]

    @property
    def nz(self):
        return self.shape[2]

    @property
    def n_elements(self):
        nx, ny, nz = self.shape
        return nx * ny * nz

    @property
    def n_nodes_full(self):
        nx, ny, nz = self.shape
        return (nx + 1) * (ny + 1) * (nz + 1)

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

    @property
    def array_shape(self):
        nx, ny, nz = self.shape
        return (nz, ny, nx)


@dataclass(frozen=True)
class PhaseMaterial:
    """Constitutive and fracture data of one phase (model.py:345-421).

    ``kind`` 'isotropic' needs ``E`` and ``nu`` (MPa); ``Gc`` in N/mm; ``driver`` is the
    nominal damage driver ('spectral', 'full', 'none' or 'interface').
    """
    name: str
    kind: str
    Gc: float
    driver: str
    E: float | None = None
    nu: float | None = None
    sources: Mapping[str, str] = field(default_factory=dict)
    layers: tuple | None = None
    tensile_strength: float | None = None

    def __post_init__(self):
        _choice("phase name", self.name, PHASE_NAMES)
        if self.tensile_strength is not None:
            _set(self, "tensile_strength", _positive(f"{self.name}: tensile_strength", self.tensile_strength))
        _choice(f"{self.name}: kind", self.kind, MATERIAL_KINDS)
        _choice(f"{self.name}: driver", self.driver, DRIVER_NAMES)
        _set(self, "Gc", _positive(f"{self.name}: Gc", self.Gc))
        if self.kind == "smeared_laminate":
            if self.layers is None or len(self.layers) < 1:
                raise ValueError(f"{self.name}: smeared_laminate phases need layers")
            layers = []
            for i, layer in enumerate(self.layers):
                if len(layer) != 3:
                    raise ValueError(f"{self.name}: layer {i} must be (fraction, E, nu)")
                nu_i = _finite(f"{self.name}: layer {i} nu", layer[2])
                if not -1.0 < nu_i < 0.5:
                    raise ValueError(f"{self.name}: layer {i} nu must lie in (-1, 0.5)")
                layers.append((_positive(f"{self.name}: layer {i} fraction", layer[0]),
                               _positive(f"{self.name}: layer {i} E", layer[1]), nu_i))
            if abs(sum(f for f, _, _ in layers) - 1.0) > 1.0e-12:
                raise ValueError(f"{self.name}: layer fractions must sum to 1")
            _set(self, "layers", tuple(layers))
        elif self.layers is not None:
            raise ValueError(f"{self.name}: layers apply to smeared_laminate phases only")
        if self.E is None or self.nu is None:
            raise ValueError(f"{self.name}: {self.kind} phases need E and nu")
        _set(self, "E", _positive(f"{self.name}: E", self.E))
        nu = _finite(f"{self.name}: nu", self.nu)
        if not -1.0 < nu < 0.5:
            raise ValueError(f"{self.name}: nu must lie in (-1, 0.5), got {nu!r}")
        _set(self, "nu", nu)
        _set(self, "sources", {str(k): str(v) for k, v in dict(self.sources).items()})

    @property
    def phase_id(self):
        return PHASE_ID[self.name]

    @property
    def is_isotropic(self):
        return self.kind == "isotropic"

    @property
    def is_laminate(self):
        return self.kind == "smeared_laminate"


@dataclass(frozen=True)
class MaterialTable:
    """Phase materials of one scale with the uniform length scale ``ell`` in mm (model.py:424-493)."""
    phases: Mapping[str, PhaseMaterial]
    length_scale: float
    scale: str = "micro"
    notes: tuple = ()

    def __post_init__(self):
        phases = dict(self.phases)
        if not phases:
            raise ValueError("MaterialTable needs at least one phase")
        for key, material in phases.items():
            if getattr(material, "name", None) != key:
                raise ValueError(f"phase key {key!r} differs from material name {getattr(material, 'name', None)!r}")
        _set(self, "phases", {name: phases[name] for name in PHASE_NAMES if name in phases})
        _set(self, "length_scale", _positive("length_scale", self.length_scale))
        _choice("scale", self.scale, ("micro",))
        _set(self, "notes", tuple(str(n) for n in self.notes))


@dataclass
class VoxelModel:
    """Phase-labelled voxel cell (model.py:496-586): ``phase_id`` (nz, ny, nx) uint8 with ids
    from ``PHASE_ID``; ``tangent`` (nz, ny, nx, 3) (used by smeared-laminate phases only)."""
    grid: VoxelGrid
    phase_id: np.ndarray
    tangent: np.ndarray
    materials: MaterialTable
    metadata: dict = field(default_factory=dict)
    aux: dict = field(default_factory=dict)

    def __post_init__(self):
        self.validate()

    def validate(self):
        shape = tuple(self.grid.array_shape)
        phase = np.asarray(self.phase_id)
        if phase.shape != shape:
            raise ValueError(f"phase_id must have shape {shape}, got {phase.shape}")
        if not np.issubdtype(phase.dtype, np.integer):
            raise TypeError(f"phase_id must be an integer array, got {phase.dtype}")
        if phase.size and (int(phase.min()) < 0 or int(phase.max()) >= len(PHASE_NAMES)):
            raise ValueError("phase_id contains an unknown phase id")
        self.phase_id = np.ascontiguousarray(phase, dtype=np.uint8)
        tangent = np.asarray(self.tangent, dtype=np.float64)
        if tangent.shape != (*shape, 3):
            raise ValueError(f"tangent must have shape {(*shape, 3)}, got {tangent.shape}")
        if not np.isfinite(tangent).all():
            raise ValueError("tangent contains non-finite values")
        self.tangent = np.ascontiguousarray(tangent)
        present = self.phases_present()
        missing = [name for name in present if name not in self.materials.phases]
        if missing:
            raise ValueError(f"phases {missing} are present but have no material")
        for name in present:
            if self.materials.phases[name].kind == "isotropic":
                continue
            norms = np.linalg.norm(self.tangent[self.phase_id == PHASE_ID[name]], axis=-1)
            if norms.size and float(np.abs(norms - 1.0).max()) > 1.0e-8:
                raise ValueError(f"phase {name!r}: tangents must be unit vectors")
        if "interface_nodes" in self.aux:
            mask = np.asarray(self.aux["interface_nodes"])
            if mask.shape != (self.grid.n_nodes_full,) or mask.dtype != np.bool_:
                raise ValueError(f"aux['interface_nodes'] must be a bool array of shape ({self.grid.n_nodes_full},)")

    def phases_present(self):
        return tuple(PHASE_NAMES[int(i)] for i in np.unique(np.asarray(self.phase_id)))

    def volume_fractions(self):
        counts = np.bincount(np.asarray(self.phase_id).reshape(-1), minlength=len(PHASE_NAMES))
        total = float(counts.sum())
        return {name: float(counts[PHASE_ID[name]]) / total for name in self.phases_present()}


@dataclass(frozen=True)
class LoadCase:
    """Mixed macro-strain control (model.py:589-681): ``targets[n-1]`` is E[controlled]
    after increment n; ``free`` components carry zero macro stress, ``fixed_zero`` ones
    zero strain."""
    name: str
    controlled: int
    targets: tuple
    free: tuple = ()
    fixed_zero: tuple = ()

    def __post_init__(self):
        if isinstance(self.controlled, bool) or int(self.controlled) != self.controlled:
            raise ValueError(f"controlled must be an integer, got {self.controlled!r}")
        controlled = int(self.controlled)
        free = tuple(int(v) for v in self.free)
        fixed_zero = tuple(int(v) for v in self.fixed_zero)
        if sorted([controlled, *free, *fixed_zero]) != list(range(6)):
            raise ValueError("{controlled}, free and fixed_zero must partition {0,...,5}; got "
                             f"controlled={controlled}, free={free}, fixed_zero={fixed_zero}")
        targets = tuple(float(v) for v in self.targets)
        if not targets:
            raise ValueError("a LoadCase needs at least one target")
        previous = 0.0
        for index, target in enumerate(targets):
            if not math.isfinite(target):
                raise ValueError(f"target {index} is not finite: {target!r}")
            if target == previous:
                raise ValueError(f"target {index} repeats the previous value {target!r}")
            previous = target
        _set(self, "name", str(self.name))
        _set(self, "controlled", controlled)
        _set(self, "targets", targets)
        _set(self, "free", free)
        _set(self, "fixed_zero", fixed_zero)

    @classmethod
    def from_schedule(cls, name, *, controlled, schedule, free, fixed_zero):
        """Targets from ``[(upto, inc), ...]`` segments starting at zero (model.py:634-671)."""
        targets, start = [], 0.0
        for index, segment in enumerate(schedule):
            upto, inc = (float(v) for v in segment)
            if not (math.isfinite(upto) and math.isfinite(inc)) or inc == 0.0:
                raise ValueError(f"schedule segment {index} is invalid: {segment!r}")
            n_steps = int(round(abs(upto - start) / abs(inc)))
            if n_steps < 1:
                raise ValueError(f"schedule segment {index} ({segment!r}) has no step from {start!r}")
            span = upto - start
            targets.extend(start + span * (s / n_steps) for s in range(1, n_steps))
            targets.append(upto)
            start = upto
        return cls(name=name, controlled=controlled, targets=tuple(targets), free=tuple(free),
                   fixed_zero=tuple(fixed_zero))

    @classmethod
    def ramp(cls, name, controlled, to, increments, fixed_zero=None):
        """``increments`` equal steps from zero to ``to``; by default every other component is held at zero."""
        fz = tuple(i for i in range(6) if i != controlled) if fixed_zero is None else tuple(fixed_zero)
        free = tuple(i for i in range(6) if i != controlled and i not in fz)
        return cls(name, controlled, tuple(to * k / increments for k in range(1, increments + 1)), free, fz)

    @property
    def n_increments(self):
        return len(self.targets)

    def increments(self):
        previous = (0.0, *self.targets[:-1])
        return tuple(t - s for s, t in zip(previous, self.targets))


@dataclass(frozen=True)
class SolverConfig:
    """Numerical settings of the staggered solve (model.py:706-897); defaults are PhAST's.

    ``dtype`` is 'float64' only, as in the reference (the chosen mechanics form may compute in
    FP32 under FP64 refinement; see ``StaggeredSolver(form=...)``).  The GPU backend runs
    ``damage_law`` 'at2' or 'pfczm', ``irreversibility`` 'box_kkt' or 'history_only', ``history``
    'max' or 'current', ``crack_closure`` 'none' or 'axes' and ``anderson_depth`` 0-6; ``device``
    names the CUDA device (the default here, where the reference's is 'cpu').  Invalid settings
    and combinations raise the reference's ``ValueError`` at construction.
    """
    device: str = "cuda"
    dtype: str = "float64"
    num_threads: int | None = None
    batch_size: int = 65536
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
    irreversibility: str = "box_kkt"
    history: str = "max"
    energy_split_isotropic: str = "spectral"
    on_stagger_failure: str = "cutback"
    max_cutbacks: int = 1
    final_mechanics_resolve: bool = True
    damaged_threshold: float = 0.95
    energy_split_band: str = "isotropic"
    band_stress: str = "hybrid"
    anderson_depth: int = 0
    anderson_start: int = 2
    crack_closure: str = "none"
    damage_law: str = "at2"
    pfczm_softening: str = "linear"
    pfczm_p: float = 2
    pfczm_max_newton: int = 100

    def __post_init__(self):
        for key in ("batch_size", "max_stagger", "pcg_maxit_mech", "check_every", "damage_maxit",
                    "damage_max_active_set"):
            _set(self, key, _positive_int(key, getattr(self, key)))
        if isinstance(self.min_stagger, bool) or int(self.min_stagger) != self.min_stagger or self.min_stagger < 0:
            raise ValueError(f"min_stagger must be an integer >= 0, got {self.min_stagger!r}")
        if self.min_stagger > self.max_stagger:
            raise ValueError("min_stagger must not exceed max_stagger")
        if isinstance(self.max_cutbacks, bool) or int(self.max_cutbacks) != self.max_cutbacks or self.max_cutbacks < 0:
            raise ValueError(f"max_cutbacks must be an integer >= 0, got {self.max_cutbacks!r}")
        kappa = _finite("kappa", self.kappa)
        if not 0.0 <= kappa < 1.0:
            raise ValueError(f"kappa must lie in [0, 1), got {kappa!r}")
        _set(self, "kappa", kappa)
        for key in ("stagger_tol", "pcg_rtol_mech", "damage_linear_tol", "damage_kkt_tol"):
            _set(self, key, _positive(key, getattr(self, key)))
        threshold = _finite("damaged_threshold", self.damaged_threshold)
        if not 0.0 < threshold <= 1.0:
            raise ValueError("damaged_threshold must lie in (0, 1]")
        # the reference refuses every dtype but float64 and every device but cpu/cuda at
        # construction (model.py:806-809, 683-700, 1441-1446)
        if not (self.dtype == "float64" or self.dtype is torch.float64):
            raise ValueError(f"only float64 is supported, got {self.dtype!r}")
        try:
            dev = torch.device(self.device)
        except (RuntimeError, TypeError) as exc:
            raise ValueError(f"device must be cpu or cuda, got {self.device!r}") from exc
        if dev.type not in ("cpu", "cuda"):
            raise ValueError(f"device must be cpu or cuda, got {self.device!r}")
        if self.num_threads is not None:
            _positive_int("num_threads", self.num_threads)
        _choice("preconditioner", self.preconditioner, ("jacobi",))
        _choice("irreversibility", self.irreversibility, ("box_kkt", "history_only"))
        _choice("history", self.history, ("max", "current"))
        _choice("energy_split_isotropic", self.energy_split_isotropic, ("spectral", "full"))
        _choice("energy_split_band", self.energy_split_band, ("isotropic", "interface"))
        _choice("band_stress", self.band_stress, ("hybrid", "variational"))
        _choice("on_stagger_failure", self.on_stagger_failure, ("cutback", "raise"))
        _choice("crack_closure", self.crack_closure, ("none", "axes"))
        _choice("damage_law", self.damage_law, ("at2", "pfczm"))
        _choice("pfczm_softening", self.pfczm_softening, ("linear", "exponential"))
        if isinstance(self.anderson_depth, bool) or int(self.anderson_depth) != self.anderson_depth or \
                self.anderson_depth < 0:
            raise ValueError(f"anderson_depth must be an integer >= 0, got {self.anderson_depth!r}")
        _set(self, "anderson_depth", int(self.anderson_depth))
        _set(self, "damaged_threshold", threshold)
        # the cross-option rules of solid3d/model.py:840-895: a mix needs two residuals, the
        # closure's line-searched mechanics is not covered by the mixing safeguard, the
        # variational band stress is the derivative of the interface split, and the PF-CZM
        # settings belong to that law (its exponent fixed by the softening curve)
        start = self.anderson_start
        if isinstance(start, bool) or int(start) != start or start < 2:
            raise ValueError(f"anderson_start must be an integer >= 2 (a mix needs two staggered residuals), "
                             f"got {start!r}")
        _set(self, "anderson_start", int(start))
        if self.band_stress == "variational" and self.energy_split_band != "interface":
            raise ValueError("band_stress 'variational' needs energy_split_band 'interface'")
        if self.crack_closure != "none" and self.anderson_depth > 0:
            raise ValueError("crack_closure 'axes' is not available with Anderson mixing (anderson_depth > 0)")
        p = self.pfczm_p
        if isinstance(p, bool) or not isinstance(p, (int, float)) or not math.isfinite(p) or p < 2:
            raise ValueError(f"pfczm_p must be a number >= 2, got {p!r}")
        p = int(p) if float(p).is_integer() else float(p)
        _set(self, "pfczm_p", p)
        _set(self, "pfczm_max_newton", _positive_int("pfczm_max_newton", self.pfczm_max_newton))
        if self.damage_law == "at2":
            changed = [k for k in ("pfczm_softening", "pfczm_p", "pfczm_max_newton")
                       if getattr(self, k) != getattr(SolverConfig, k)]
            if changed:
                raise ValueError(f"{', '.join(changed)} apply to damage_law 'pfczm' only")
        else:
            if self.irreversibility != "box_kkt":
                raise ValueError("damage_law 'pfczm' needs irreversibility 'box_kkt' (the crack function "
                                 "2d - d^2 is unbounded below for d < 0)")
            wu_p = _PFCZM_EXPONENTS[self.pfczm_softening]
            if p != wu_p:
                raise ValueError(f"pfczm_softening {self.pfczm_softening!r} is Wu's law with pfczm_p = {wu_p}, "
                                 f"got {p!r}")


def unsupported_options(cfg):
    """Names of ``cfg`` settings this backend does not run (empty when it runs them all)."""
    out = []
    if getattr(cfg, "anderson_depth", 0) > 6:
        out.append(f"anderson_depth={cfg.anderson_depth!r} (the B200 backend mixes at most 6 pairs)")
    if getattr(cfg, "energy_split_band", "isotropic") != "isotropic":
        out.append(f"energy_split_band={cfg.energy_split_band!r}")
    return out


def lame(E, nu):
    """Lame parameters (materials.py:162-167)."""
    return E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), E / (2.0 * (1.0 + nu))


def isotropic_C(E, nu):
    lam, mu = lame(E, nu)
    C = np.zeros((6, 6))
    C[:3, :3] = lam
    C[[0, 1, 2], [0, 1, 2]] = lam + 2 * mu
    C[[3, 4, 5], [3, 4, 5]] = mu
    return C, lam, mu


def resolve_driver(material, cfg):
    """Element driver code of a phase under ``cfg`` (materials.py:450-471)."""
    if material.name == "pore" or material.driver == "none":
        return DRIVER_NONE
    if material.name == "bn_band" and getattr(cfg, "energy_split_band", "isotropic") == "interface":
        return DRIVER_INTERFACE
    return DRIVER_SPECTRAL if getattr(cfg, "energy_split_isotropic", "spectral") == "spectral" else DRIVER_FULL


@dataclass(frozen=True)
class ElementMaterialArrays:
    """Per-element material data on the device (materials.py:400-440 field names).

    ``stiffness_bank`` (S, 6, 6) holds one isotropic stiffness per present phase in
    phase-id order and ``stiffness_index`` (E,) its slot per element; ``Gc``, ``lam``,
    ``mu`` (E,) float64, ``driver`` (E,) int8, ``phase`` (E,) int64 and ``tangent`` (E, 3).
    """
    stiffness_bank: torch.Tensor
    stiffness_index: torch.Tensor
    Gc: torch.Tensor
    driver: torch.Tensor
    lam: torch.Tensor
    mu: torch.Tensor
    phase: torch.Tensor
    tangent: torch.Tensor

    @property
    def n_elements(self):
        return int(self.stiffness_index.shape[0])

    @property
    def device(self):
        return self.stiffness_index.device


def build_element_arrays(model, cfg, *, device=None):
    """Per-element material arrays on ``device`` (default ``cfg.device``), materials.py:474-547.

    Only isotropic phases are supported by the GPU kernels; a smeared-laminate phase
    raises ``NotImplementedError``.
    """
    model.validate()
    target = torch.device(getattr(cfg, "device", "cuda") if device is None else device)
    phase_flat = np.asarray(model.phase_id).reshape(-1).astype(np.int64)
    materials = model.materials.phases
    present = model.phases_present()
    framed = [name for name in present if not materials[name].is_isotropic]
    if framed:
        raise NotImplementedError(f"smeared-laminate phases {framed} are not supported by the GPU backend")
    slot = np.empty(phase_flat.shape[0], dtype=np.int64)
    bank = []
    n_ids = len(PHASE_NAMES)
    by_id = {k: np.zeros(n_ids) for k in ("Gc", "lam", "mu")}
    driver_by_id = np.zeros(n_ids, dtype=np.int8)
    for s, name in enumerate(present):
        m = materials[name]
        C, lam, mu = isotropic_C(float(m.E), float(m.nu))
        bank.append(C)
        slot[phase_flat == PHASE_ID[name]] = s
        pid = PHASE_ID[name]
        by_id["Gc"][pid], by_id["lam"][pid], by_id["mu"][pid] = float(m.Gc), lam, mu
        driver_by_id[pid] = resolve_driver(m, cfg)

    def element(values):
        return torch.as_tensor(values[phase_flat], dtype=torch.float64, device=target)

    return ElementMaterialArrays(
        stiffness_bank=torch.as_tensor(np.stack(bank), dtype=torch.float64, device=target),
        stiffness_index=torch.as_tensor(slot, dtype=torch.long, device=target),
        Gc=element(by_id["Gc"]), driver=torch.as_tensor(driver_by_id[phase_flat], device=target),
        lam=element(by_id["lam"]), mu=element(by_id["mu"]),
        phase=torch.as_tensor(phase_flat, dtype=torch.long, device=target),
        tangent=torch.as_tensor(np.asarray(model.tangent).reshape(-1, 3), dtype=torch.float64, device=target))


def sphere_pore_model(shape, radius_fraction, *, E=3000.0, nu=0.35, Gc=0.5, ell_voxels=2.0, pore_stiffness=1e-6,
                      tensile_strength=None, pore_tensile_strength=None):
    """A cubic-voxel cell of ``mi_matrix`` with one central spherical ``pore`` (E x ``pore_stiffness``);
    the tensile strengths (MPa) are those of the PF-CZM law."""
    nx, ny, nz = shape
    h = 1.0 / nz
    phase = sphere_pore_phase(shape, radius_fraction, PHASE_ID["mi_matrix"], PHASE_ID["pore"])
    phases = {"mi_matrix": PhaseMaterial("mi_matrix", "isotropic", Gc, "spectral", E, nu,
                                         tensile_strength=tensile_strength),
              "pore": PhaseMaterial("pore", "isotropic", Gc, "spectral", E * pore_stiffness, nu,
                                    tensile_strength=pore_tensile_strength)}
    tangent = np.zeros((nz, ny, nx, 3))
    tangent[..., 2] = 1.0
    return VoxelModel(VoxelGrid(shape, (h, h, h)), phase, tangent, MaterialTable(phases, ell_voxels * h, "micro"))


def sphere_pore_phase(shape, radius_fraction, matrix_id=PHASE_ID["mi_matrix"], pore_id=PHASE_ID["pore"]):
    """Phase ids (nz, ny, nx): pore where the voxel-centre distance to the cell centre < r * L."""
    nx, ny, nz = shape
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    c = np.stack([(i + 0.5) / nx - 0.5, (j + 0.5) / ny - 0.5, (k + 0.5) / nz - 0.5], -1)
    phase = np.full((nz, ny, nx), matrix_id, dtype=np.uint8)
    phase[np.linalg.norm(c, axis=-1) < radius_fraction] = pore_id
    return phase


@dataclass
class ClosurePattern:
    """Sign pattern of the crack-closure terms at every quadrature point (model.py:1200-1223).

    ``iso`` ``(E, 8, 4)`` bool holds the bits ``[tr eps < 0], [eps_xx < 0], [eps_yy < 0],
    [eps_zz < 0]`` of the isotropic closure (False outside the group); ``band`` is the
    smeared-laminate group, ``None`` here (laminate phases are not run by this backend).  For a
    fixed pattern the closure stress is linear in the strain.
    """
    iso: torch.Tensor | None = None
    band: torch.Tensor | None = None

    def groups(self):
        return (self.iso, self.band)

    def equals(self, other):
        """Whether both patterns hold the same bits in every group."""
        for mine, theirs in zip(self.groups(), other.groups()):
            if (mine is None) != (theirs is None):
                return False
            if mine is not None and not torch.equal(mine, theirs):
                return False
        return True

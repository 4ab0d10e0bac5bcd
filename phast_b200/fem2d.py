"""2D structured-Q4 operators behind PhAST's ``FEMOperators`` interface.

Mirrors ``phast.core.fem_operators.FEMOperators`` (src/phast/core/fem_operators.py)
for Q4 meshes laid out by ``structured_q4_mesh`` (src/phast/core/quad_elements.py:458),
i.e. the meshes of the SENT and dynamic-branching benchmarks.  Every operator is
one launch of a kernel in ``libphastb.so``; tensors stay on the GPU.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr, stream


# ----------------------------------------------------------------------------
# material, mesh, boundary conditions (the data the hot path reads)
# ----------------------------------------------------------------------------

@dataclass
class Material:
    """``phast.physics.material.Material`` (physics/material.py:80-257): the same fields in the
    same order with the same defaults, and the same construction checks and normalisation
    (``eta_residual <= 0`` becomes 1e-7, ``pf_model`` upper-cased).  The GPU kernels read the
    elastic, fracture and split fields; the solvers refuse, with ``NotImplementedError``, the
    laws and couplings they do not run (PF-CZM, Allen-Cahn, non-standard degradation,
    plasticity, the principal-stress driver, the ``sigma_ts`` nucleation scaling)."""
    E: float = 210000.0
    nu: float = 0.3
    Gc: float = 2.7
    l0: float = 0.005
    rho: float = 7.8e-9
    eta_residual: float = 1e-7
    energy_split: str = "amor"
    pf_model: str = "AT2"
    gamma_correction: bool = False
    degradation_type: str = "standard"
    stress_degradation: str = "split"
    cubic_s: float = 1.0
    sigma_ts: float = 0.0
    pfczm_p: int = 2
    pfczm_softening: str = "linear"
    driving_force: str = "strain_energy"
    plane_stress: bool = False
    at1_threshold: object = "auto"
    plasticity_model: str = "none"
    yield_stress: float = 0.0
    hardening_modulus: float = 0.0
    hardening_type: str = "none"
    voce_q_inf: Optional[float] = None
    voce_b: Optional[float] = None
    swift_K: Optional[float] = None
    swift_n: Optional[float] = None
    swift_eps0: Optional[float] = None

    def __post_init__(self):
        # the reference's rules (material.py:176-257), restated
        if self.eta_residual <= 0.0:
            self.eta_residual = 1e-7
        model = str(self.pf_model)
        self.pf_model = "allencahn" if model.lower() == "allencahn" else model.upper()
        if self.pf_model not in ("AT1", "AT2", "PFCZM", "allencahn"):
            raise ValueError(f"pf_model must be 'AT1', 'AT2', 'PFCZM', or 'allencahn', got {self.pf_model!r}")
        if self.stress_degradation not in ("split", "full"):
            raise ValueError(f"stress_degradation must be 'split' or 'full', got {self.stress_degradation!r}")
        if self.degradation_type == "rational_at2" and self.pf_model != "AT2":
            raise ValueError(f"degradation_type='rational_at2' is defined for pf_model='AT2', got {self.pf_model!r}")
        if isinstance(self.pfczm_p, bool) or not isinstance(self.pfczm_p, int) or self.pfczm_p < 2:
            raise ValueError(f"pfczm_p must be an integer >= 2, got {self.pfczm_p!r}")
        if self.pfczm_softening not in ("linear", "exponential"):
            raise ValueError(f"pfczm_softening must be 'linear' or 'exponential', got {self.pfczm_softening!r}")
        if self.energy_split == "spectral_plane_stress_condensed" and not self.plane_stress:
            raise ValueError("energy_split='spectral_plane_stress_condensed' requires plane_stress=True")
        if self.pf_model == "PFCZM" and self.sigma_ts <= 0.0:
            raise ValueError("pf_model='PFCZM' requires sigma_ts > 0")
        if self.pf_model == "PFCZM" and self.degradation_type != "standard":
            raise ValueError("pf_model='PFCZM' requires degradation_type='standard'")
        t = self.at1_threshold
        if isinstance(t, str):
            if t != "auto":
                raise ValueError(f"at1_threshold must be 'auto' or a float, got {t!r}")
        elif not isinstance(t, (int, float)):
            raise ValueError(f"at1_threshold must be 'auto' or a float, got type {type(t).__name__}")
        elif t < 0.0:
            raise ValueError(f"at1_threshold must be non-negative, got {t}")
        if self.cubic_s < 0.0:
            raise ValueError(f"cubic_s must be non-negative, got {self.cubic_s}")
        if self.plasticity_model != "none":
            if self.yield_stress <= 0.0:
                raise ValueError(f"plasticity_model={self.plasticity_model!r} requires yield_stress > 0")
            if self.hardening_modulus < 0.0:
                raise ValueError(f"hardening_modulus must be non-negative, got {self.hardening_modulus}")
            if self.hardening_type == "voce":
                if self.voce_q_inf is None or self.voce_b is None:
                    raise ValueError("hardening_type='voce' requires voce_q_inf and voce_b to be set")
                if self.voce_b <= 0.0:
                    raise ValueError(f"voce_b must be > 0, got {self.voce_b}")
            if self.hardening_type == "swift":
                if self.swift_K is None or self.swift_n is None:
                    raise ValueError("hardening_type='swift' requires swift_K and swift_n to be set")
                if self.swift_K <= 0.0 or self.swift_n <= 0.0:
                    raise ValueError(f"swift_K and swift_n must be > 0, got K={self.swift_K}, n={self.swift_n}")

    @property
    def lam(self):
        if self.plane_stress:
            return self.E * self.nu / (1.0 - self.nu ** 2)
        return self.E * self.nu / ((1 + self.nu) * (1 - 2 * self.nu))

    @property
    def mu(self):
        return self.E / (2 * (1 + self.nu))

    @property
    def at1_source(self):
        """The AT1 source S_H of the damage right-hand side 2H - S_H: 3 Gc / (8 l0) unless
        ``at1_threshold`` overrides it; 0 for AT2 (material.py:259-271)."""
        if self.pf_model != "AT1":
            return 0.0
        if isinstance(self.at1_threshold, str) and self.at1_threshold == "auto":
            return 3.0 * self.Gc / (8.0 * self.l0)
        return float(self.at1_threshold)

    @property
    def kappa(self):
        return self.E / (3.0 * (1.0 - 2.0 * self.nu))

    @property
    def c_p(self):
        return math.sqrt((self.lam + 2 * self.mu) / self.rho)

    def effective_stress_split(self):
        if self.stress_degradation == "full":
            return "isotropic"
        return self.energy_split

    def degradation(self, d):
        return (1.0 - d) ** 2 * (1.0 - self.eta_residual) + self.eta_residual


def stress_split_of(material):
    f = getattr(material, "effective_stress_split", None)
    return f() if callable(f) else getattr(material, "energy_split", "isotropic")


@dataclass
class StructuredQ4Mesh:
    nodes: torch.Tensor
    quads: torch.Tensor
    node_sets: dict
    nx: int
    ny: int


def structured_q4_mesh(width, height, nx, ny, *, dtype=torch.float64):
    """Same numbering as PhAST's structured_q4_mesh (quad_elements.py:458-487)."""
    xs = torch.linspace(0.0, float(width), int(nx) + 1, dtype=dtype)
    ys = torch.linspace(0.0, float(height), int(ny) + 1, dtype=dtype)
    yy, xx = torch.meshgrid(ys, xs, indexing="ij")
    nodes = torch.stack([xx.reshape(-1), yy.reshape(-1)], dim=1)
    j, i = torch.meshgrid(torch.arange(ny), torch.arange(nx), indexing="ij")
    n0 = (j * (nx + 1) + i).reshape(-1)
    quads = torch.stack([n0, n0 + 1, n0 + nx + 2, n0 + nx + 1], 1)
    sets = {
        "left": torch.arange(0, (ny + 1) * (nx + 1), nx + 1),
        "right": torch.arange(nx, (ny + 1) * (nx + 1), nx + 1),
        "bottom": torch.arange(0, nx + 1),
        "top": torch.arange(ny * (nx + 1), (ny + 1) * (nx + 1)),
    }
    return StructuredQ4Mesh(nodes, quads, sets, nx, ny)


class FEMMesh:
    """Minimal ``FEMMesh.from_tensors`` (core/mesh.py:84-155) for Q4 grids on the GPU."""

    def __init__(self, nodes, elements, element_type="Q4", device=None, dtype=torch.float64, node_sets=None):
        if element_type not in ("Q4", "T3"):
            raise NotImplementedError("the B200 backend implements structured Q4 and unstructured T3 meshes")
        device = torch.device(device) if device is not None else torch.device("cuda")
        self.element_type = element_type
        self.dtype = dtype
        self.device = device
        self.nodes = torch.as_tensor(nodes, dtype=dtype).to(device)
        self.elements = torch.as_tensor(elements, dtype=torch.long).to(device)
        self.node_sets = node_sets or {}
        self.n_nodes = int(self.nodes.shape[0])
        self.n_elems = int(self.elements.shape[0])

    @classmethod
    def from_tensors(cls, nodes, elements, node_sets=None, device=None, dtype=torch.float64, element_type="T3"):
        return cls(nodes, elements, element_type=element_type, device=device, dtype=dtype, node_sets=node_sets)


def detect_structured(mesh):
    """Return (nx, ny, hx, hy) when ``mesh`` has the structured_q4_mesh layout, else raise."""
    nodes = mesh.nodes.detach().to("cpu", torch.float64).numpy()
    el = mesh.elements.detach().to("cpu", torch.long).numpy()
    if el.ndim != 2 or el.shape[1] != 4 or el.shape[0] == 0:
        raise NotImplementedError("expected (E, 4) Q4 connectivity")
    nx = int(el[0, 3]) - 1
    if nx < 1 or el.shape[0] % nx:
        raise NotImplementedError("Q4 mesh is not a structured_q4_mesh grid")
    ny = el.shape[0] // nx
    if nodes.shape[0] != (nx + 1) * (ny + 1):
        raise NotImplementedError("Q4 mesh is not a structured_q4_mesh grid")
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    n0 = (j * (nx + 1) + i).reshape(-1)
    ref = np.stack([n0, n0 + 1, n0 + nx + 2, n0 + nx + 1], 1)
    if not np.array_equal(ref, el):
        raise NotImplementedError("Q4 connectivity differs from structured_q4_mesh numbering")
    x0, y0 = nodes[0]
    hx = (nodes[nx, 0] - x0) / nx
    hy = (nodes[-1, 1] - y0) / ny
    jj, ii = np.meshgrid(np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    grid = np.stack([x0 + ii.reshape(-1) * hx, y0 + jj.reshape(-1) * hy], 1)
    scale = max(abs(hx) * nx, abs(hy) * ny)
    if hx <= 0 or hy <= 0 or np.abs(grid - nodes).max() > 1e-9 * scale:
        raise NotImplementedError("Q4 mesh is not a uniform rectangular grid")
    return nx, ny, float(hx), float(hy)


def q4_material_struct(material, dtype=torch.float64):
    split = getattr(material, "energy_split", "isotropic")
    ssplit = stress_split_of(material)
    for s in (split, ssplit):
        if s not in _lib.SPLITS:
            raise NotImplementedError(f"energy split {s!r} is not implemented by the B200 backend")
    if getattr(material, "degradation_type", "standard") != "standard":
        raise NotImplementedError("only the standard AT2 degradation (1-d)^2 (1-eta) + eta is implemented")
    m = _lib.Q4Material()
    m.E, m.nu = float(material.E), float(material.nu)
    m.lam, m.mu, m.kappa = float(material.lam), float(material.mu), float(material.kappa)
    m.eta = float(material.eta_residual)
    # FP64 floor of the spectral split (fem_operators.py:126) in both precisions: the FP32
    # kernels are checked against the FP64 reference, so they keep its regularisation.
    m.spectral_eps = 1e-12
    m.plane_stress = int(bool(getattr(material, "plane_stress", False)))
    m.stress_split = _lib.SPLITS[ssplit]
    m.psi_split = _lib.SPLITS[split]
    return m


def _dtype_code(t):
    if t.dtype == torch.float64:
        return _lib.F64
    if t.dtype == torch.float32:
        return _lib.F32
    raise ValueError(f"unsupported dtype {t.dtype}")


class FEMOperators:
    """GPU ``FEMOperators`` for structured Q4 grids (core/fem_operators.py:35-1530).

    A mesh whose ``element_type`` is ``'T3'`` gets the triangle operators of
    ``phast_b200.t3`` instead.
    """

    def __new__(cls, mesh, material, ctx=None):
        if getattr(mesh, "element_type", "Q4") == "T3":
            from .t3 import T3FEMOperators
            return T3FEMOperators(mesh, material)
        return super().__new__(cls)

    def __init__(self, mesh, material, ctx=None):
        self.mesh = mesh
        self.material = material
        self.device = torch.device(getattr(mesh, "device", "cuda"))
        if self.device.type != "cuda":
            raise ValueError("the B200 backend needs the mesh on a CUDA device")
        self.dtype = getattr(mesh, "dtype", torch.float64)
        nx, ny, hx, hy = detect_structured(mesh)
        self.nx, self.ny, self.hx, self.hy = nx, ny, hx, hy
        self.n_nodes = (nx + 1) * (ny + 1)
        self.n_elems = nx * ny
        self.grid = _lib.Q4Grid(nx, ny, hx, hy)
        self._mat = {torch.float64: q4_material_struct(material, torch.float64),
                     torch.float32: q4_material_struct(material, torch.float32)}
        lam, mu = material.lam, material.mu
        self.C = torch.tensor([[lam + 2 * mu, lam, 0.0], [lam, lam + 2 * mu, 0.0], [0.0, 0.0, mu]],
                              dtype=self.dtype, device=self.device)
        i = torch.arange(nx + 1, device=self.device)
        j = torch.arange(ny + 1, device=self.device)
        ci = 1 + ((i > 0) & (i < nx)).to(self.dtype)
        cj = 1 + ((j > 0) & (j < ny)).to(self.dtype)
        # lumped mass sum_e sum_q N_a w (mesh.py:_precompute_q4): hx hy / 4 per adjacent element
        self.M_scalar = (cj[:, None] * ci[None, :]).reshape(-1) * (0.25 * hx * hy)
        self.M_vec = material.rho * self.M_scalar.unsqueeze(1).expand(-1, 2).flatten()
        self.M_vec_inv = 1.0 / (self.M_vec + 1e-30)
        self.h_min = min(hx, hy)
        self.dt_cfl = self.h_min / material.c_p
        self.diff_E_field = None
        self._zeros_q = torch.zeros(self.n_elems, 4, dtype=torch.float64, device=self.device)
        self._ws = _lib.Workspace(self.device)

    # -- helpers ------------------------------------------------------------
    def mat(self, dtype=None):
        return self._mat[dtype or self.dtype]

    def _check_nodal(self, t, comps, name):
        shape = (self.n_nodes, comps) if comps > 1 else (self.n_nodes,)
        if tuple(t.shape) != shape:
            raise ValueError(f"{name} must have shape {shape}, got {tuple(t.shape)}")
        _lib.require_cuda(t, name)
        return t.contiguous()

    # -- strain / stress / force --------------------------------------------
    def compute_strain(self, u):
        """Q4 strain at 2x2 Gauss points, three (E, 4) tensors (fem_operators.py:244-254)."""
        u = self._check_nodal(u, 2, "u")
        out = [torch.empty(self.n_elems, 4, dtype=u.dtype, device=u.device) for _ in range(3)]
        call("phastb_q4_strain", self.grid, _dtype_code(u), ptr(u), *[ptr(o) for o in out], stream())
        return tuple(out)

    def internal_force(self, u, d):
        """Degraded internal force (N, 2) (fem_operators.py:598-612)."""
        u = self._check_nodal(u, 2, "u")
        d = self._check_nodal(d, 1, "d").to(u.dtype)
        f = torch.empty_like(u)
        call("phastb_q4_internal_force", self.grid, self.mat(u.dtype), _dtype_code(u), ptr(u), ptr(d), ptr(f),
             stream())
        return f

    def internal_force_linear(self, u):
        u = self._check_nodal(u, 2, "u")
        f = torch.empty_like(u)
        call("phastb_q4_internal_force", self.grid, self.mat(u.dtype), _dtype_code(u), ptr(u), None, ptr(f),
             stream())
        return f

    def stiffness_diagonal(self, d=None):
        """Jacobi diagonal (N, 2) of K(d) (fem_operators.py:1284-1320)."""
        diag = torch.empty(self.n_nodes, 2, dtype=self.dtype, device=self.device)
        dd = None if d is None else self._check_nodal(d, 1, "d").to(self.dtype)
        call("phastb_q4_stiffness_diagonal", self.grid, self.mat(), _dtype_code(diag), ptr(dd), ptr(diag), stream())
        return diag

    # -- energies -------------------------------------------------------------
    def compute_psi_plus(self, u, strain=None, d=None):
        """Tensile energy at Gauss points (E, 4) (fem_operators.py:951-1025)."""
        u = self._check_nodal(u, 2, "u")
        psi = torch.empty(self.n_elems, 4, dtype=u.dtype, device=u.device)
        call("phastb_q4_psi_history", self.grid, self.mat(u.dtype), _dtype_code(u), ptr(u), None, None, ptr(psi),
             stream())
        return psi

    def compute_driving_force(self, u, strain=None, d=None):
        mode = getattr(self.material, "driving_force", "strain_energy")
        if mode != "strain_energy":
            raise NotImplementedError("only the strain-energy driving force is implemented")
        return self.compute_psi_plus(u, strain=strain, d=d)

    def psi_history(self, u, H_in, H_out):
        """Fused psi+ and history max: H_out = max(H_in, psi+(u))."""
        call("phastb_q4_psi_history", self.grid, self.mat(u.dtype), _dtype_code(u), ptr(u), ptr(H_in), ptr(H_out),
             None, stream())
        return H_out

    # -- adjoint pieces (isotropic split) -------------------------------------------
    def psi_grad_t(self, u, wq):
        """sum_{e,q} wq[e,q] (d psi+_{e,q} / du): the transpose of the Gauss-point energy map, (N, 2)."""
        u = self._check_nodal(u, 2, "u").double()
        wq = wq.to(torch.float64).contiguous()
        f = torch.empty_like(u)
        call("phastb_q4_psi_grad_t", self.grid, self.mat(torch.float64), ptr(u), ptr(wq), ptr(f), stream())
        return f

    def force_dd_t(self, u, z, d):
        """d/dd [z . f_int(u, d)], (N,)."""
        u = self._check_nodal(u, 2, "u").double()
        z = self._check_nodal(z, 2, "z").double()
        d = self._check_nodal(d, 1, "d").double()
        out = torch.empty_like(d)
        call("phastb_q4_force_dd_t", self.grid, self.mat(torch.float64), ptr(u), ptr(z), ptr(d), ptr(out), stream())
        return out

    def laplacian_matvec(self, d):
        """K_lap d (fem_operators.py:1253-1266)."""
        d = self._check_nodal(d, 1, "d").double()
        y = torch.empty_like(d)
        call("phastb_q4_damage_apply", self.grid, ptr(d), ptr(self._zeros_q), 0.0, 0.0, None, 1.0, None, ptr(y),
             stream())
        return y

    def _q4_mass_matvec(self, d):
        """Consistent Q4 mass times d (fem_operators.py:1268-1277)."""
        d = self._check_nodal(d, 1, "d").double()
        y = torch.empty_like(d)
        call("phastb_q4_damage_apply", self.grid, ptr(d), ptr(self._zeros_q), 0.0, 1.0, None, 0.0, None, ptr(y),
             stream())
        return y

    def _energy_sums(self, u, d, v=None):
        u = self._check_nodal(u, 2, "u").double()
        d = self._check_nodal(d, 1, "d").double()
        vv = None if v is None else self._check_nodal(v, 2, "v").double()
        out = (ctypes_double4 := (_lib.C.c_double * 4)())
        wsz = _lib.load().phastb_reduce_workspace_bytes()
        wp, wn = self._ws.get(wsz)
        call("phastb_q4_energy_sums", self.grid, self.mat(torch.float64), ptr(u), ptr(d), ptr(vv), out, wp, wn,
             stream())
        return [float(x) for x in ctypes_double4]

    def compute_energy_components(self, u, d, v=None, strain=None, psi_plus=None):
        """Elastic / kinetic / fracture energies, AT2 (fem_operators.py:1430-1496)."""
        if getattr(self.material, "pf_model", "AT2") != "AT2":
            raise NotImplementedError("energy components are implemented for AT2")
        el, dMd, dKd, vMv = self._energy_sums(u, d, v)
        mat = self.material
        frac = mat.Gc / (2.0 * mat.l0) * dMd + mat.Gc * mat.l0 / 2.0 * dKd
        kin = 0.5 * mat.rho * vMv if v is not None else 0.0
        return {"elastic": el, "kinetic": kin, "fracture": frac, "total": el + kin + frac}

    def compute_total_energy(self, u, d, strain=None, psi_plus=None):
        e = self.compute_energy_components(u, d)
        return e["elastic"] + e["fracture"]

    def compute_reaction_force(self, u, d, node_indices, component=1, f_ext=None):
        """Sum of f_int (- f_ext) over nodes, FP64 (fem_operators.py:1502-1530); returns a float."""
        u = self._check_nodal(u, 2, "u").double()
        d = self._check_nodal(d, 1, "d").double()
        idx = torch.as_tensor(node_indices, dtype=torch.long).to(self.device).contiguous()
        fe = None if f_ext is None else self._check_nodal(f_ext, 2, "f_ext").double()
        out = _lib.C.c_double(0.0)
        wp, wn = self._ws.get(_lib.load().phastb_q4_reaction_workspace_bytes(self.n_nodes))
        call("phastb_q4_reaction", self.grid, self.mat(torch.float64), ptr(u), ptr(d), ptr(idx), int(idx.numel()),
             int(component), ptr(fe), _lib.C.byref(out), wp, wn, stream())
        return float(out.value)

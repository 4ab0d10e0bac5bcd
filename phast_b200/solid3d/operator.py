"""Periodic voxel H8 phase-field operator on the GPU.

Mirrors ``phast.solid3d.operator.PeriodicVoxelPhaseFieldOperator`` (AT2 parts,
src/phast/solid3d/operator.py:133-1544): the same reduced periodic numbering
(periodic.py:61-113), the same 2x2x2 Gauss rule and Voigt order, the same
``x = [u~ (3 n_red), E (6)]`` layout.  The elastic and damage actions are
one launch each of ``libphastb.so``'s tiled z-marching kernels.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from .. import _lib
from .._lib import call, ptr, stream
from .model import SolverConfig, build_element_arrays, isotropic_C, unsupported_options

PORE = "pore"


def pfczm_softening_parameters(softening):
    """``(a2, a3)`` of Wu's softening laws (pfczm.py:57-65)."""
    if softening == "linear":
        return -0.5, 0.0
    if softening == "exponential":
        return 2.0 ** (5.0 / 3.0) - 3.0, 0.0
    raise ValueError(f"PF-CZM softening must be one of ('linear', 'exponential'), got {softening!r}")


def _driver_code(phase, split_isotropic):
    """resolve_driver (solid3d/materials.py:454-471) for isotropic phases."""
    if getattr(phase, "name", "") == PORE or getattr(phase, "driver", "spectral") == "none":
        return _lib.DRIVER_NONE
    return _lib.DRIVER_SPECTRAL if split_isotropic == "spectral" else _lib.DRIVER_FULL


class PeriodicVoxelPhaseFieldOperator:
    """Matrix-free mechanics and damage operators of one periodic voxel cell (AT2).

    ``PeriodicVoxelPhaseFieldOperator(model, load, cfg, *, materials=None, pinned_node=None,
    pfczm_strengths=None)`` as PhAST's constructor (operator.py:172-320): ``model`` a
    ``VoxelModel`` (grid, phase ids, material table with the length scale ``ell``), ``load``
    a ``LoadCase``, ``cfg`` a ``SolverConfig`` (``kappa``, ``energy_split_isotropic``,
    ``device``), ``materials`` the ``build_element_arrays`` result (built from ``model`` and
    ``cfg`` when omitted), ``pinned_node`` the reduced node whose fluctuation is fixed
    (default: the first node touching no pore voxel, periodic.py:224-249).  The reference's
    data classes are accepted as well as this package's.  Options the GPU kernels do not
    run (see ``model.unsupported_options``) raise ``NotImplementedError``.
    """

    def __init__(self, model, load, cfg, *, materials=None, pinned_node=None, pfczm_strengths=None):
        bad = unsupported_options(cfg)
        if bad:
            raise NotImplementedError(f"the B200 backend does not run {', '.join(bad)}")
        if pfczm_strengths is not None and getattr(cfg, "damage_law", "at2") != "pfczm":
            raise ValueError("pfczm_strengths applies to damage_law 'pfczm' only")
        model.validate()
        if materials is None:
            materials = build_element_arrays(model, cfg)
        if int(materials.stiffness_index.shape[0]) != int(model.grid.n_elements):
            raise ValueError(f"materials describe {int(materials.stiffness_index.shape[0])} elements, the grid has "
                             f"{model.grid.n_elements}")
        present = model.phases_present()
        phases = [model.materials.phases[name] for name in present]
        framed = [p.name for p in phases if getattr(p, "kind", "isotropic") != "isotropic"]
        if framed:
            raise NotImplementedError(f"smeared-laminate phases {framed} are not supported by the GPU backend")
        slot = materials.stiffness_index.detach().to("cpu").numpy().astype(np.int64)
        self.model = model
        self.cfg = cfg
        self.mat_arrays = materials
        self._setup(model.grid, slot, phases, float(model.materials.length_scale), float(cfg.kappa), load,
                    cfg.energy_split_isotropic, pinned_node, materials.stiffness_index.device)
        if getattr(cfg, "damage_law", "at2") == "pfczm":
            self._build_pfczm(cfg, pfczm_strengths)
        if getattr(cfg, "crack_closure", "none") == "axes":
            self._build_closure()

    @classmethod
    def from_slots(cls, grid, slot, phases, ell, kappa, load, *, split_isotropic="spectral", pinned_node=None,
                   device="cuda"):
        """An operator from per-voxel material slots: ``slot`` (nz, ny, nx) or (E,) indexes ``phases``
        (objects with ``name``, ``E``, ``nu``, ``Gc``, ``driver``); ``ell`` and ``kappa`` given directly."""
        self = cls.__new__(cls)
        self.model = None
        self.cfg = SolverConfig(device=str(device), kappa=float(kappa), energy_split_isotropic=split_isotropic)
        self.mat_arrays = None
        self._setup(grid, np.asarray(slot).reshape(-1).astype(np.int64), list(phases), float(ell), float(kappa),
                    load, split_isotropic, pinned_node, device)
        return self

    def _setup(self, grid, slot_np, phases, ell, kappa, load, split_isotropic, pinned_node, device):
        self.grid = grid
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("the B200 backend needs a CUDA device")
        if self.device.index is None:  # tensors made on "cuda" report the current device's index
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.dtype = torch.float64
        nx, ny, nz = (int(v) for v in grid.shape)
        hx, hy, hz = (float(v) for v in grid.h)
        px, py, pz = (bool(v) for v in getattr(grid, "periodic", (True, True, True)))
        self.shape = (nx, ny, nz)
        self.h = (hx, hy, hz)
        self.vgrid = _lib.VoxelGrid(nx, ny, nz, int(px), int(py), int(pz), hx, hy, hz)
        self.reduced_shape = (nx if px else nx + 1, ny if py else ny + 1, nz if pz else nz + 1)
        rx, ry, rz = self.reduced_shape
        self.n_red = rx * ry * rz
        self.n_mech = 3 * self.n_red + 6
        self.n_elements = nx * ny * nz
        self.volume = nx * ny * nz * hx * hy * hz
        self.ell = float(ell)
        self.kappa = float(kappa)
        self.load = load
        if slot_np.shape[0] != self.n_elements:
            raise ValueError(f"slot must hold {self.n_elements} entries")
        if len(phases) > _lib.MAX_SLOTS or slot_np.min() < 0 or slot_np.max() >= len(phases):
            raise ValueError("bad material slots")
        self.phases = list(phases)
        self.slot_np = slot_np
        self.slot = torch.as_tensor(slot_np.astype(np.uint8), device=self.device)
        m = _lib.VoxelMaterial()
        m.n_slots = len(phases)
        m.isotropic = 1
        self._lam, self._mu, self._Gc = [], [], []
        for s, ph in enumerate(phases):
            Cm, lam, mu = isotropic_C(float(ph.E), float(ph.nu))
            for k in range(36):
                m.C[s][k] = float(Cm.reshape(-1)[k])
            m.lam[s], m.mu[s], m.Gc[s] = lam, mu, float(ph.Gc)
            m.driver[s] = _driver_code(ph, split_isotropic)
            self._lam.append(lam)
            self._mu.append(mu)
            self._Gc.append(float(ph.Gc))
        m.kappa = self.kappa
        m.ell = self.ell
        self.mat = m
        Ge = np.asarray(self._Gc)[slot_np]
        if not np.all(np.isfinite(Ge)) or not np.all(Ge > 0):
            raise ValueError("Gc must be finite and positive at every element")
        self.damage_scale = self.ell / (float(Ge.min()) * hx * hy * hz)  # operator.py:238
        if pinned_node is None:
            pinned_node = self._choose_pinned_node()
        self.pinned_node = int(pinned_node)
        self._ws = _lib.Workspace(self.device)
        self._scratch64 = None
        self._scratch32 = None
        self._red = _lib.Workspace(self.device)
        self._rec = _lib.Workspace(self.device)
        self._resid = _lib.Workspace(self.device)
        self._pf = None
        self._pfws = _lib.Workspace(self.device)
        self._closure = False
        self._clws = _lib.Workspace(self.device)
        self._kgws = _lib.Workspace(self.device)
        self.pfczm_bound = None
        self.pfczm_phases = {}
        self.pfczm_strengths = {}

    # -- construction helpers -----------------------------------------------------------
    def _choose_pinned_node(self):
        """choose_pinned_node (periodic.py:224-249): first reduced node touching no pore voxel."""
        pore_slots = [s for s, p in enumerate(self.phases) if getattr(p, "name", "") == PORE]
        if not pore_slots:
            return 0
        nx, ny, nz = self.shape
        rx, ry, rz = self.reduced_shape
        px, py, pz = self.vgrid.px, self.vgrid.py, self.vgrid.pz
        ke, je, ie = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        pore = np.isin(self.slot_np, pore_slots)
        count = np.zeros(self.n_red, dtype=np.int64)
        for L in range(8):
            i = ie.reshape(-1) + (L & 1)
            j = je.reshape(-1) + ((L >> 1) & 1)
            k = ke.reshape(-1) + (L >> 2)
            if px:
                i = i % nx
            if py:
                j = j % ny
            if pz:
                k = k % nz
            nodes = i + rx * (j + ry * k)
            np.add.at(count, nodes[pore], 1)
        return int(np.argmin(count))

    def _build_pfczm(self, cfg, strengths):
        """Per-slot ``a1`` of the PF-CZM law and the onset check (operator.py:326-439).

        ``a1 = 4 E Gc / (pi ell f_t^2 (1 - kappa))`` (pfczm.py:16-31) with ``f_t`` the phase's
        ``tensile_strength`` or its ``pfczm_strengths`` override; raises ``ValueError`` when a present
        phase has no strength, or when ``a1 < p + a2`` (``g''(0) < 0``) in a phase with a damage driver.
        """
        a2, a3 = pfczm_softening_parameters(cfg.pfczm_softening)
        p = float(cfg.pfczm_p)
        bound = p + a2
        scale = max(1.0 - self.kappa, 1.0e-30)
        law = _lib.PfczmLaw()
        law.a2, law.a3, law.p = a2, a3, p
        strengths = dict(strengths or {})
        names = {ph.name for ph in self.phases}
        for name, value in strengths.items():
            if name not in names:
                raise ValueError(f"pfczm_strengths phase {name!r} is not present in the cell")
            f = float(value)
            if not (math.isfinite(f) and f > 0.0):
                raise ValueError(f"pfczm_strengths[{name!r}] must be finite and positive")
            self.pfczm_strengths[name] = f
        missing, violations = [], []
        for s, ph in enumerate(self.phases):
            f = self.pfczm_strengths.get(ph.name, getattr(ph, "tensile_strength", None))
            if f is None:
                missing.append(ph.name)
                continue
            E, Gc, f = float(ph.E), float(ph.Gc), float(f)
            a1 = 4.0 * E * Gc / (math.pi * self.ell * f ** 2 * scale)
            law.a1[s] = a1
            checked = int(self.mat.driver[s]) != _lib.DRIVER_NONE
            f_max = (4.0 * E * Gc / (math.pi * self.ell * scale) / bound) ** 0.5
            ell_max = 4.0 * E * Gc / (math.pi * f ** 2 * scale) / bound
            ok = (not checked) or a1 >= bound
            if not ok:
                violations.append(f"{ph.name}: a1 = {a1:.4g} < {bound:g} (f_t = {f:g} MPa; largest admissible f_t "
                                  f"{f_max:.4g} MPa at this ell, largest admissible ell {ell_max:.4g} mm at this f_t)")
            self.pfczm_phases[ph.name] = {"f_t": f, "E_ref_min": E, "E_ref_max": E, "Gc_min": Gc, "Gc_max": Gc,
                                          "a1_min": a1, "a1_max": a1, "a1_bound": bound, "f_t_max": f_max,
                                          "ell_max": ell_max, "onset_checked": checked, "onset_ok": ok}
        if missing:
            raise ValueError("damage_law 'pfczm' needs a tensile strength for every phase of the cell "
                             f"(material.tensile_strength); missing: {', '.join(missing)}")
        if violations:
            raise ValueError(f"damage_law 'pfczm': the onset condition a1 >= p + a2 = {bound:g} (g''(0) >= 0, i.e. "
                             "ell <= 4 E Gc / (pi f_t^2 (1 - kappa)(p + a2)), 8 l_ch / (3 pi) for linear softening) "
                             f"fails at ell = {self.ell:g} mm in: " + "; ".join(violations))
        self._pf = law
        self.pfczm_bound = bound
        self._a1 = torch.as_tensor(np.array([law.a1[s] for s in range(len(self.phases))])[self.slot_np],
                                   dtype=torch.float64, device=self.device)

    @property
    def is_pfczm(self):
        """Whether the damage law is the PF-CZM law (``damage_law = 'pfczm'``)."""
        return self._pf is not None

    def scratch(self, dtype=torch.float64):
        code = _lib.F64 if dtype == torch.float64 else _lib.F32
        nbytes = _lib.load().phastb_h8_scratch_bytes(self.vgrid, code)
        attr = "_scratch64" if code == _lib.F64 else "_scratch32"
        buf = getattr(self, attr)
        if buf is None or buf.numel() < nbytes:
            buf = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            setattr(self, attr, buf)
        return C.c_void_p(buf.data_ptr())

    def _check(self, name, t, shape, dtype=None):
        if not isinstance(t, torch.Tensor):
            raise TypeError(f"{name} must be a torch.Tensor")
        if tuple(t.shape) != shape:
            raise ValueError(f"{name} must have shape {shape}, got {tuple(t.shape)}")
        _lib.require_cuda(t, name)
        if dtype is not None and t.dtype != dtype:
            raise ValueError(f"{name} must be {dtype}")
        return t.contiguous()

    def _dt(self, t):
        return _lib.F64 if t.dtype == torch.float64 else _lib.F32

    # -- layout --------------------------------------------------------------------------
    def split_mech(self, x):
        n = 3 * self.n_red
        return x[:n].reshape(self.n_red, 3), x[n:]

    def pack_mech(self, u, E):
        u = torch.as_tensor(u, dtype=torch.float64, device=self.device).reshape(-1)
        E = torch.as_tensor(E, dtype=torch.float64, device=self.device).reshape(-1)
        return torch.cat((u, E))

    def mech_fixed_mask(self):
        """Pinned-node dofs, the controlled and the fixed_zero E components (operator.py:905-915)."""
        mask = torch.zeros(self.n_mech, dtype=torch.bool, device=self.device)
        b = 3 * self.pinned_node
        mask[b:b + 3] = True
        off = 3 * self.n_red
        mask[off + int(self.load.controlled)] = True
        for c in self.load.fixed_zero:
            mask[off + int(c)] = True
        return mask

    def mech_fixed_values(self, e_c):
        vals = torch.zeros(self.n_mech, dtype=torch.float64, device=self.device)
        vals[3 * self.n_red + int(self.load.controlled)] = float(e_c)
        return vals

    # -- mechanics -------------------------------------------------------------------------
    def degradation(self, d):
        """Gauss-point degradation g (E, 8) with d_q = d_e N^T (operator.py:939-946): AT2
        (1-kappa)(1-d_q)^2 + kappa, or the PF-CZM rational law (FP64) with ``damage_law='pfczm'``."""
        d = self._check("d", d, (self.n_red,))
        if self._pf is not None:
            dd = d.to(torch.float64).contiguous()
            g = torch.empty(self.n_elements, 8, dtype=torch.float64, device=self.device)
            call("phastb_h8_pfczm_degradation", self.vgrid, self.mat, C.byref(self._pf), ptr(self.slot), ptr(dd),
                 ptr(g), stream())
            return g.to(d.dtype)
        g = torch.empty(self.n_elements, 8, dtype=d.dtype, device=self.device)
        call("phastb_h8_degradation", self.vgrid, self._dt(d), ptr(d), self.kappa, ptr(g), stream())
        return g

    def _law_g(self, g, d, dtype):
        """``(g, d)`` for the kernels: the PF-CZM law and the closure add-back need ``g`` itself."""
        if (self._pf is not None or self._closure) and g is None and d is not None:
            return self.degradation(d).to(dtype), None
        return g, d

    def _no_closure(self, opening=None, closure=None):
        """The packed (E, 8) sign pattern of ``closure`` (None: each point's own signs)."""
        if opening is not None:
            raise NotImplementedError("interface opening patterns are not supported by the GPU backend")
        if closure is None:
            return None
        if not self._closure:
            raise ValueError("closure applies with crack_closure 'axes' only; this operator has none")
        return self._packed(closure)

    def mech_action(self, x, g=None, *, opening=None, closure=None, d=None, mask=None, out=None):
        """A(g) x (operator.py:1171-1194); ``g=None`` means undamaged.  ``d`` instead of ``g`` fuses
        the degradation into the action; ``mask`` zeroes rows; ``out`` receives the result.  With the
        crack closure the (1 - g) add-back of ``closure``'s pattern joins (each point's own signs when
        ``closure`` is None)."""
        pattern = self._no_closure(opening, closure)
        x = self._check("x", x, (self.n_mech,))
        g, d = self._law_g(g, d, x.dtype)
        gq = None if g is None else self._check("g", g, (self.n_elements, 8), x.dtype)
        dd = None if d is None else self._check("d", d, (self.n_red,)).to(x.dtype)
        mk = None if mask is None else mask.to(torch.uint8).contiguous()
        if out is None:
            y = torch.empty_like(x)
        else:
            y = out
            if y.shape != x.shape or y.dtype != x.dtype or not y.is_contiguous() or y.data_ptr() == x.data_ptr():
                raise ValueError("out must be a distinct contiguous tensor like x")
        call("phastb_h8_mech_apply", self.vgrid, self.mat, ptr(self.slot), self._dt(x), ptr(x), ptr(gq), ptr(dd),
             ptr(mk), ptr(y), self.scratch(x.dtype), stream())
        if self._closure and gq is not None:
            self._fp64_closure(x)
            wp, wn = self._cl_ws()
            call("phastb_h8_closure_apply_add", self.vgrid, self.mat, ptr(self.slot), ptr(x), ptr(gq), ptr(pattern),
                 ptr(mk), ptr(y), wp, wn, stream())
        return y

    def mech_operator(self, g=None, *, d=None):
        """The action ``v -> A(g) v`` as a callable that ``solve_constrained`` recognises."""
        g, d = self._law_g(g, d, torch.float64)
        return MechOperator(self, g, d)

    def tile_shape(self, dtype=torch.float64, shape=None):
        """Tile shape (ox, oy, kz) of the elastic-action kernel; ``shape`` records a new one."""
        arr = (C.c_int * 3)(*(shape if shape is not None else (0, 0, 0)))
        code = _lib.F32 if dtype == torch.float32 else _lib.F64
        call("phastb_h8_tile_shape", self.vgrid, code, int(shape is not None), arr)
        return tuple(arr)

    def autotune(self, dtype=torch.float64, seed=0):
        """Time the elastic action over the candidate tile shapes and keep the fastest for this grid.

        Returns ``(shape, ms_per_action)``.
        """
        gen = torch.Generator(device="cpu").manual_seed(seed)
        x = torch.rand(self.n_mech, generator=gen, dtype=torch.float64).to(self.device, dtype) * 1e-3
        d = torch.rand(self.n_red, generator=gen, dtype=torch.float64).to(self.device, dtype) * 0.5
        y = torch.empty_like(x)
        shape = (C.c_int * 3)()
        ms = C.c_float(0.0)
        wn = _lib.load().phastb_h8_scratch_bytes(self.vgrid, self._dt(x))
        call("phastb_h8_autotune", self.vgrid, self.mat, self._dt(x), ptr(self.slot), ptr(x), ptr(d), ptr(y),
             self.scratch(dtype), wn, shape, C.byref(ms), stream())
        return tuple(shape), float(ms.value)

    def mech_diagonal(self, g=None, *, opening=None, closure=None, d=None):
        """Jacobi diagonal of A(g) (operator.py:1196-1302); with the crack closure the add-back's terms
        of ``closure``'s bits (every bit when None)."""
        pattern = self._no_closure(opening, closure)
        dtype = g.dtype if g is not None else (d.dtype if d is not None else torch.float64)
        g, d = self._law_g(g, d, dtype)
        gq = None if g is None else self._check("g", g, (self.n_elements, 8), dtype)
        dd = None if d is None else self._check("d", d, (self.n_red,), dtype)
        y = torch.empty(self.n_mech, dtype=dtype, device=self.device)
        call("phastb_h8_mech_diagonal", self.vgrid, self.mat, ptr(self.slot), self._dt(y), ptr(gq), ptr(dd), ptr(y),
             self.scratch(dtype), stream())
        if self._closure and gq is not None:
            self._fp64_closure(y)
            wp, wn = self._cl_ws()
            call("phastb_h8_closure_diagonal_add", self.vgrid, self.mat, ptr(self.slot), ptr(gq), ptr(pattern), ptr(y),
                 wp, wn, stream())
        return y

    def _stress_energy(self, x, g=None, d=None, pattern=None):
        x = self._check("x", x, (self.n_mech,), torch.float64)
        g, d = self._law_g(g, d, torch.float64)
        gq = None if g is None else self._check("g", g, (self.n_elements, 8), torch.float64)
        dd = None if d is None else self._check("d", d, (self.n_red,), torch.float64)
        rE = (C.c_double * 6)()
        en = C.c_double(0.0)
        call("phastb_h8_stress_energy", self.vgrid, self.mat, ptr(self.slot), ptr(x), ptr(gq), ptr(dd), rE,
             C.byref(en), self.scratch(torch.float64), stream())
        rE, en = np.array(list(rE)), float(en.value)
        if self._closure and gq is not None:
            out = self._closure_energy(x, gq, pattern)
            rE[:3] += out[1:4]
            en += out[0]
        return rE, en

    def _closure_energy(self, x, gq, pattern=None):
        out = (C.c_double * 4)()
        wp, wn = self._cl_ws()
        call("phastb_h8_closure_energy", self.vgrid, self.mat, ptr(self.slot), ptr(x), ptr(gq), ptr(pattern), out,
             wp, wn, stream())
        return np.array(list(out))

    def macro_stress(self, x, g=None, *, opening=None, closure=None, d=None):
        """Sigma = r_E / V (operator.py:1303-1316)."""
        pattern = self._no_closure(opening, closure)
        rE, _ = self._stress_energy(x, g, d, pattern)
        return torch.as_tensor(rE / self.volume, dtype=torch.float64, device=self.device)

    def elastic_energy(self, x, g=None, *, opening=None, closure=None, d=None):
        """0.5 x . A(g) x in mJ, a 0-dim tensor (operator.py:1318-1340)."""
        pattern = self._no_closure(opening, closure)
        _, en = self._stress_energy(x, g, d, pattern)
        return torch.tensor(en, dtype=torch.float64, device=self.device)

    def mean_strain(self, x):
        """Volume-average total strain <eps> (6,) (operator.py:1342-1389): E on a triply periodic cell."""
        if not all(bool(p) for p in getattr(self.grid, "periodic", (True, True, True))):
            raise NotImplementedError("mean_strain of a cell with free faces is not supported by the GPU backend")
        x = self._check("x", x, (self.n_mech,))
        return self.split_mech(x)[1].clone()

    def hill_mandel(self, x, g=None, *, closure=None):
        """``mean_work = 2 E_el / V``, ``macro_work = Sigma . E`` and their relative gap (operator.py:1390-1413)."""
        pattern = self._no_closure(None, closure)
        rE, en = self._stress_energy(x, g, None, pattern)
        E = self.split_mech(x)[1].detach().cpu().numpy()
        mean = 2.0 * en / self.volume
        macro = float(np.dot(rE / self.volume, E))
        scale = max(abs(mean), abs(macro))
        return {"mean_work": mean, "macro_work": macro, "relative": abs(mean - macro) / scale if scale > 0 else 0.0}

    # -- crack closure ('axes', isotropic group) ---------------------------------------------
    def _build_closure(self):
        """The isotropic closure group (operator.py:673-727): every element with a damage driver, rows
        (trace, e_x, e_y, e_z), moduli (lam, 2 mu, 2 mu, 2 mu) of its slot."""
        for s, ph in enumerate(self.phases):
            if int(self.mat.driver[s]) != _lib.DRIVER_NONE and self._lam[s] < 0.0:
                raise ValueError("crack_closure 'axes' needs lam >= 0 in every isotropic phase")
        self._closure = True

    @property
    def has_closure(self):
        """Whether the crack closure is on (``crack_closure != 'none'``)."""
        return self._closure

    @property
    def n_closure_band(self):
        """Number of smeared-laminate band elements with the band closure (none here)."""
        return 0

    # -- the interface driver (operator.py:634-655, 991-1008): this backend refuses the
    # interface driver, so there are no interface elements and the queries say so
    @property
    def has_interface(self):
        """Whether any element uses the directional interface driver (never here)."""
        return False

    @property
    def n_interface(self):
        """Number of interface-driver elements (0 here)."""
        return 0

    @property
    def has_interface_stress(self):
        """Whether interface elements carry the variational band stress (never here)."""
        return False

    def interface_normal_traction(self, x):
        """Normal interface traction ``(n_interface, 8)`` of the interface elements: empty here."""
        self._check("x", x, (self.n_mech,))
        return torch.empty((0, 8), dtype=self.dtype, device=self.device)

    def interface_opening(self, x):
        """Normal-opening pattern ``(n_interface, 8)`` bool: empty here."""
        return self.interface_normal_traction(x) > 0.0

    def reduced_of_full(self):
        """Reduced node of every full grid node ``(N_full,)`` (periodic.py:40-123): full node
        ``i + (nx+1)(j + (ny+1) k)`` maps to ``i' + rx (j' + ry k')`` with periodic axes wrapped."""
        if getattr(self, "_rof", None) is None:
            nx, ny, nz = self.shape
            rx, ry, _ = self.reduced_shape
            px, py, pz = bool(self.vgrid.px), bool(self.vgrid.py), bool(self.vgrid.pz)
            i = np.arange(nx + 1) % nx if px else np.arange(nx + 1)
            j = np.arange(ny + 1) % ny if py else np.arange(ny + 1)
            k = np.arange(nz + 1) % nz if pz else np.arange(nz + 1)
            idx = i[None, None, :] + rx * (j[None, :, None] + ry * k[:, None, None])
            self._rof = torch.as_tensor(idx.reshape(-1), dtype=torch.long, device=self.device)
        return self._rof

    def expand_damage(self, d):
        """Full nodal damage ``P d`` ``(N_full,)`` (operator.py:1546-1550)."""
        d = self._check("d", d, (self.n_red,))
        return d[self.reduced_of_full()]

    def _cl_ws(self):
        return self._clws.get(_lib.load().phastb_h8_closure_workspace_bytes(self.vgrid))

    @staticmethod
    def _fp64_closure(t):
        if t.dtype != torch.float64:
            raise NotImplementedError("the crack closure runs in FP64")

    def _packed(self, closure):
        """(E, 8) uint8 bits of a ClosurePattern (bit k: row k active)."""
        packed = getattr(closure, "_packed", None)
        if packed is not None:
            return packed
        iso = getattr(closure, "iso", None)
        if getattr(closure, "band", None) is not None:
            raise ValueError("closure.band must be None: the model has no band closure group")
        if not isinstance(iso, torch.Tensor) or iso.dtype != torch.bool:
            raise TypeError("closure.iso must be a torch.bool tensor")
        if tuple(iso.shape) != (self.n_elements, 8, 4) or iso.device != self.device:
            raise ValueError(f"closure.iso must have shape {(self.n_elements, 8, 4)} on {self.device}")
        weights = torch.tensor([1, 2, 4, 8], dtype=torch.uint8, device=self.device)
        return (iso.to(torch.uint8) * weights).sum(-1).to(torch.uint8).contiguous()

    def _pattern_object(self, packed):
        from .model import ClosurePattern
        bits = torch.tensor([1, 2, 4, 8], dtype=torch.uint8, device=self.device)
        out = ClosurePattern(iso=(packed.unsqueeze(-1) & bits) != 0, band=None)
        out._packed = packed
        return out

    def _closure_pattern_packed(self, x):
        x = self._check("x", x, (self.n_mech,), torch.float64)
        out = torch.empty(self.n_elements, 8, dtype=torch.uint8, device=self.device)
        call("phastb_h8_closure_pattern", self.vgrid, self.mat, ptr(self.slot), ptr(x), ptr(out), stream())
        return out

    def _closure_change_packed(self, x, old, g, tolerance):
        x = self._check("x", x, (self.n_mech,), torch.float64)
        g = self._check("g", g, (self.n_elements, 8), torch.float64)
        new = torch.empty_like(old)
        changed = (C.c_int * 1)()
        wp, wn = self._cl_ws()
        call("phastb_h8_closure_pattern_change", self.vgrid, self.mat, ptr(self.slot), ptr(x), ptr(g), ptr(old),
             float(tolerance), ptr(new), changed, wp, wn, stream())
        return new, bool(changed[0])

    def closure_pattern(self, x):
        """Sign pattern ``v . eps < 0`` of every closure term at state ``x`` (operator.py:821-834)."""
        if not self._closure:
            raise ValueError("closure_pattern needs crack_closure 'axes'")
        return self._pattern_object(self._closure_pattern_packed(x))

    def closure_pattern_change(self, x, pattern, g, *, tolerance=1.0e-8):
        """New closure pattern of state ``x`` and whether it changed materially (operator.py:836-873):
        a flipped bit counts where its stress jump ``(1 - g) k |v . eps|`` exceeds ``tolerance`` times
        the largest ``k |v . eps|``."""
        old = self._no_closure(None, pattern)
        if old is None:
            raise ValueError("closure_pattern_change needs a pattern")
        new, changed = self._closure_change_packed(x, old, g, tolerance)
        return self._pattern_object(new), changed

    def kinematic_guard(self, x, d):
        """Smallest element-mean normal strain, principal strain of the element-mean strain and
        Gauss-point ``det(I + grad u)`` of state ``x``, and the same over the elements whose mean nodal
        damage exceeds ``cfg.damaged_threshold`` (``damaged_*``, None when there are none)
        (operator.py:1713-1770)."""
        x = self._check("x", x, (self.n_mech,), torch.float64)
        d = self._check("d", d, (self.n_red,), torch.float64)
        out = (C.c_double * 6)()
        wp, wn = self._kgws.get(_lib.load().phastb_reduce_workspace_bytes())
        call("phastb_h8_kinematic_guard", self.vgrid, ptr(x), ptr(d), float(self.cfg.damaged_threshold), out, wp, wn,
             stream())
        v = [float(a) for a in out]
        damaged = math.isfinite(v[3])
        return {"min_normal_strain": v[0], "min_principal_strain": v[1], "min_det_F": v[2],
                "damaged_min_normal_strain": v[3] if damaged else None,
                "damaged_min_principal_strain": v[4] if damaged else None,
                "damaged_min_det_F": v[5] if damaged else None}

    def driving_force(self, x):
        """Undamaged driving energy Y (E, 8) (operator.py:1415-1444)."""
        return self.driving_history(x, None, want_Y=True)[0]

    def driving_history(self, x, H_prev, want_Y=False):
        """(Y or None, H = max(H_prev, Y)) in one kernel."""
        x = self._check("x", x, (self.n_mech,), torch.float64)
        Hp = None if H_prev is None else self._check("H_prev", H_prev, (self.n_elements, 8), torch.float64)
        Y = torch.empty(self.n_elements, 8, dtype=torch.float64, device=self.device) if want_Y else None
        H = None if (H_prev is None and want_Y) else torch.empty(self.n_elements, 8, dtype=torch.float64,
                                                                 device=self.device)
        call("phastb_h8_driving_history", self.vgrid, self.mat, ptr(self.slot), ptr(x), ptr(Hp), ptr(Y), ptr(H),
             stream())
        return Y, H

    # -- damage ----------------------------------------------------------------------------
    def damage_action(self, d, H=None, *, scale=1.0):
        """Unscaled damage operator (operator.py:1450-1466)."""
        d = self._check("d", d, (self.n_red,), torch.float64)
        Hq = None if H is None else self._check("H", H, (self.n_elements, 8), torch.float64)
        y = torch.empty_like(d)
        call("phastb_h8_damage_apply", self.vgrid, self.mat, ptr(self.slot), ptr(d), ptr(Hq), float(scale), ptr(y),
             self.scratch(), stream())
        return y

    def damage_rhs(self, H, *, scale=1.0):
        Hq = None if H is None else self._check("H", H, (self.n_elements, 8), torch.float64)
        y = torch.empty(self.n_red, dtype=torch.float64, device=self.device)
        call("phastb_h8_damage_rhs_diag", self.vgrid, self.mat, ptr(self.slot), ptr(Hq), float(scale), ptr(y), None,
             self.scratch(), stream())
        return y

    def damage_diagonal(self, H=None, *, scale=1.0):
        Hq = None if H is None else self._check("H", H, (self.n_elements, 8), torch.float64)
        y = torch.empty(self.n_red, dtype=torch.float64, device=self.device)
        call("phastb_h8_damage_rhs_diag", self.vgrid, self.mat, ptr(self.slot), ptr(Hq), float(scale), None, ptr(y),
             self.scratch(), stream())
        return y

    def fracture_energy(self, d):
        """Fracture energy in mJ (operator.py:1511-1545): per element Gc/(2 ell) d.M d ('local') plus
        Gc ell/2 d.L d ('gradient'), and 'by_phase' over the present phases (pores included).  With
        the PF-CZM law the functional is Gc/(pi ell) int (2d - d^2) + Gc ell/pi int |grad d|^2
        (_pfczm_fracture_energy, operator.py:608-631)."""
        out = self.increment_record(None, d, None, 1.0)
        return {"total": out["local"] + out["gradient"], "local": out["local"], "gradient": out["gradient"],
                "by_phase": out["by_phase"]}

    def increment_record(self, x, d, H, threshold):
        """All scalars of an accepted increment in one kernel pair and one host read (``x`` may be None):
        E, r_E, elastic energy, fracture energy (total, parts, by phase), element-mean damage sum,
        damaged-element count, max H and max d."""
        d = self._check("d", d, (self.n_red,), torch.float64)
        xx = None if x is None else self._check("x", x, (self.n_mech,), torch.float64)
        Hq = None if H is None else self._check("H", H, (self.n_elements, 8), torch.float64)
        out = (C.c_double * _lib.RECORD_WORDS)()
        wp, wn = self._rec.get(_lib.load().phastb_h8_record_workspace_bytes(self.vgrid))
        if self._pf is not None:
            # elastic part at the PF-CZM degradation, surface energy of the PF-CZM functional
            gq = None if xx is None else self.degradation(d)
            call("phastb_h8_increment_record_ex", self.vgrid, self.mat, ptr(self.slot), ptr(xx), ptr(gq), ptr(d),
                 ptr(Hq), float(threshold), C.byref(self._pf), out, wp, wn, stream())
        else:
            call("phastb_h8_increment_record", self.vgrid, self.mat, ptr(self.slot), ptr(xx), ptr(d), ptr(Hq),
                 float(threshold), out, wp, wn, stream())
        v = list(out)
        if self._closure and xx is not None:
            # the closure add-back at each point's own signs joins r_E and the elastic energy
            extra = self._closure_energy(xx, self.degradation(d))
            v[6:9] = [a + b for a, b in zip(v[6:9], extra[1:4])]
            v[12] += extra[0]
        S = _lib.MAX_SLOTS
        return {"E": np.array(v[0:6]), "rE": np.array(v[6:12]), "energy": v[12],
                "by_phase": {p.name: v[13 + s] for s, p in enumerate(self.phases)},
                "local": v[13 + S], "gradient": v[14 + S], "sum_element_d": v[15 + S], "damaged": v[16 + S],
                "max_H": v[17 + S], "max_d": v[18 + S]}

    def damage_residual_norm(self, H, d):
        """||rhs - A d|| of the scaled damage system of history ``H`` (staggered.py:766-770)."""
        d = self._check("d", d, (self.n_red,), torch.float64)
        Hq = None if H is None else self._check("H", H, (self.n_elements, 8), torch.float64)
        r = C.c_double(0.0)
        wp, wn = self._resid.get(_lib.load().phastb_h8_damage_residual_workspace_bytes(self.vgrid))
        call("phastb_h8_damage_residual_norm", self.vgrid, self.mat, ptr(self.slot), ptr(Hq), self.damage_scale,
             ptr(d), C.byref(r), wp, wn, stream())
        return float(r.value)

    # -- PF-CZM damage law ------------------------------------------------------------------
    def _pf_law(self):
        if self._pf is None:
            raise ValueError("the PF-CZM damage operators need damage_law 'pfczm'")
        return C.byref(self._pf)

    def _pf_ws(self):
        return self._pfws.get(_lib.load().phastb_h8_pfczm_workspace_bytes(self.vgrid))

    def _pf_H(self, H):
        return None if H is None else self._check("H", H, (self.n_elements, 8), torch.float64)

    def pfczm_damage_energy(self, d, H):
        """PF-CZM damage energy in mJ as a 0-dim tensor (operator.py:465-489):
        ``sum_q w H_q g(d_q) + Gc/(pi ell) int (2d - d^2) + Gc ell/pi int |grad d|^2``; ``H=None``
        drops the history term."""
        law = self._pf_law()
        d = self._check("d", d, (self.n_red,), torch.float64)
        out = (C.c_double * _lib.PFCZM_ENERGY_WORDS)()
        wp, wn = self._pf_ws()
        call("phastb_h8_pfczm_energy", self.vgrid, self.mat, law, ptr(self.slot), ptr(d), ptr(self._pf_H(H)), out,
             wp, wn, stream())
        return torch.tensor(float(out[0]), dtype=torch.float64, device=self.device)

    def pfczm_damage_gradient(self, d, H, *, scale=1.0):
        """Unscaled gradient (n_red,) of :meth:`pfczm_damage_energy` (operator.py:491-513)."""
        law = self._pf_law()
        d = self._check("d", d, (self.n_red,), torch.float64)
        y = torch.empty(self.n_red, dtype=torch.float64, device=self.device)
        wp, wn = self._pf_ws()
        call("phastb_h8_pfczm_gradient", self.vgrid, self.mat, law, ptr(self.slot), ptr(d), ptr(self._pf_H(H)),
             float(scale), ptr(y), wp, wn, stream())
        return y

    def pfczm_tangent_weights(self, d, H):
        """Gauss-point curvatures (E, 8) of the Newton tangent (operator.py:515-539):
        ``max(H g''(d_q) - 2 Gc/(pi ell), 0.25 * 2 Gc/(pi ell))``."""
        law = self._pf_law()
        d = self._check("d", d, (self.n_red,), torch.float64)
        W = torch.empty(self.n_elements, 8, dtype=torch.float64, device=self.device)
        call("phastb_h8_pfczm_tangent_weights", self.vgrid, self.mat, law, ptr(self.slot), ptr(d),
             ptr(self._pf_H(H)), ptr(W), stream())
        return W

    def pfczm_tangent_action(self, field, weights, *, scale=1.0):
        """Unscaled tangent action ``Gc (2 ell/pi) L f + sum_q w c_q N_q N_q^T f`` (operator.py:541-553)."""
        self._pf_law()
        f = self._check("field", field, (self.n_red,), torch.float64)
        W = self._check("weights", weights, (self.n_elements, 8), torch.float64)
        y = torch.empty(self.n_red, dtype=torch.float64, device=self.device)
        wp, wn = self._pf_ws()
        call("phastb_h8_pfczm_tangent_apply", self.vgrid, self.mat, ptr(self.slot), ptr(W), ptr(f), float(scale),
             ptr(y), wp, wn, stream())
        return y

    def pfczm_tangent_diagonal(self, weights, *, scale=1.0):
        """Unscaled Jacobi diagonal of :meth:`pfczm_tangent_action` (operator.py:555-566)."""
        self._pf_law()
        W = self._check("weights", weights, (self.n_elements, 8), torch.float64)
        y = torch.empty(self.n_red, dtype=torch.float64, device=self.device)
        wp, wn = self._pf_ws()
        call("phastb_h8_pfczm_tangent_diagonal", self.vgrid, self.mat, ptr(self.slot), ptr(W), float(scale), ptr(y),
             wp, wn, stream())
        return y

    def pfczm_newton_system(self, d, H, *, scaled=True, correction=False):
        """SPD Newton subproblem at ``d`` and the gradient there, both times ``damage_scale`` when
        ``scaled`` (operator.py:568-606): the tangent ``K`` of the curvature weights and the
        right-hand side ``K d - gradient`` (``-gradient`` with ``correction=True``)."""
        scale = self.damage_scale if scaled else 1.0
        W = self.pfczm_tangent_weights(d, H)
        gradient = self.pfczm_damage_gradient(d, H, scale=scale)
        system = PfczmNewtonSystem(self, W, scale)
        system.rhs = -gradient if correction else system.apply(d) - gradient
        return system, gradient

    def damage_system(self, H, *, scaled=True):
        """The scaled damage system; solved by ``solve_h8_scalar_box_kkt`` (operator.py:1495-1509)."""
        return H8DamageSystem(self, H, self.damage_scale if scaled else 1.0)


class MechOperator:
    """``v -> A(g) v`` of one operator and degradation (``g`` (E, 8) or the damage ``d``), as a callable.

    ``solve_constrained`` runs its whole solve as one fused C-ABI call when given this
    object (or the bound ``op.mech_action``) instead of an arbitrary function.
    """

    def __init__(self, op, g=None, d=None):
        self.op, self.g, self.d = op, g, d

    def __call__(self, v):
        return self.op.mech_action(v, self.g, d=self.d)


class H8DamageSystem:
    """``H8ScalarSPDSystem`` of one history field (box_kkt_h8.py:64-122), evaluated on the device."""

    def __init__(self, op, H, scale):
        self.op, self.H, self.scale = op, H, float(scale)

    @property
    def n_dofs(self):
        return self.op.n_red

    def apply(self, field):
        return self.op.damage_action(field, self.H, scale=self.scale)

    action = apply

    @property
    def rhs(self):
        return self.op.damage_rhs(self.H, scale=self.scale)

    @property
    def diagonal(self):
        return self.op.damage_diagonal(self.H, scale=self.scale)


class PfczmNewtonSystem:
    """The SPD Newton subproblem of the PF-CZM damage solve (operator.py:568-606): ``apply``,
    ``rhs`` and ``diagonal`` like PhAST's ``H8ScalarSPDSystem``; ``weights`` are the tangent's
    Gauss-point curvatures."""

    def __init__(self, op, weights, scale):
        self.op, self.weights, self.scale = op, weights, float(scale)
        self.rhs = None

    @property
    def n_dofs(self):
        return self.op.n_red

    def apply(self, field):
        return self.op.pfczm_tangent_action(field, self.weights, scale=self.scale)

    action = apply

    @property
    def diagonal(self):
        return self.op.pfczm_tangent_diagonal(self.weights, scale=self.scale)

"""Writes tests/golden/validation.json: which constructor arguments the reference's 3D data
classes (VoxelGrid, PhaseMaterial, MaterialTable, VoxelModel, LoadCase, SolverConfig;
src/phast/solid3d/model.py:183-897), its 2D ``Material`` (src/phast/physics/material.py:80-257)
and 2D ``SolverConfig`` (src/phast/solvers/staggered_solver.py:45-162) accept and which they refuse, with the exception class (and, for an accepted 2D material, the
fields it normalises).

Usage: python tests/golden/make_golden_validation.py <path to the reference's src directory>

Each case is plain JSON data; ``build(mod, case)`` turns it into a constructor call on the
classes of ``mod`` (the reference's classes here, ``phast_b200``'s in the test),
so the test replays the same calls on this backend's classes.
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

ISO = dict(name="mi_matrix", kind="isotropic", Gc=0.5, driver="spectral", E=3000.0, nu=0.35)
PORE = dict(name="pore", kind="isotropic", Gc=0.5, driver="none", E=1e-3, nu=0.35)
LAM = dict(name="bn_band", kind="smeared_laminate", Gc=0.1, driver="spectral", E=100.0, nu=0.2,
           layers=[[0.5, 100.0, 0.2], [0.5, 50.0, 0.25]])
GRID = dict(shape=[3, 2, 4], h=[0.1, 0.1, 0.1])
LOAD = dict(name="zz", controlled=2, targets=[0.001, 0.002], free=[], fixed_zero=[0, 1, 3, 4, 5])


def _with(base, **kw):
    out = dict(base)
    out.update(kw)
    return out


def _without(base, key):
    return {k: v for k, v in base.items() if k != key}


CASES = []


def _case(cls, **kw):
    CASES.append({"cls": cls, "kw": kw})


# VoxelGrid (model.py:183-216)
_case("VoxelGrid", **GRID)
_case("VoxelGrid", **_with(GRID, periodic=[True, False, True], origin=[1.0, -2.0, 0.5]))
_case("VoxelGrid", **_with(GRID, shape=[3, 2]))
_case("VoxelGrid", **_with(GRID, shape=[3, 0, 4]))
_case("VoxelGrid", **_with(GRID, shape=[3, 2.5, 4]))
_case("VoxelGrid", **_with(GRID, shape=[3, True, 4]))
_case("VoxelGrid", **_with(GRID, h=[0.1, -0.1, 0.1]))
_case("VoxelGrid", **_with(GRID, h=[0.1, math.nan, 0.1]))
_case("VoxelGrid", **_with(GRID, origin=[0.0, math.inf, 0.0]))
_case("VoxelGrid", **_with(GRID, periodic=[1, 1, 1]))
_case("VoxelGrid", **_with(GRID, periodic=[True, True]))

# PhaseMaterial (model.py:345-421)
_case("PhaseMaterial", **ISO)
_case("PhaseMaterial", **_with(ISO, tensile_strength=30.0))
_case("PhaseMaterial", **_with(ISO, tensile_strength=0.0))
_case("PhaseMaterial", **_with(ISO, name="steel"))
_case("PhaseMaterial", **_with(ISO, kind="orthotropic"))
_case("PhaseMaterial", **_with(ISO, driver="amor"))
_case("PhaseMaterial", **_with(ISO, Gc=0.0))
_case("PhaseMaterial", **_with(ISO, Gc=math.inf))
_case("PhaseMaterial", **_without(ISO, "E"))
_case("PhaseMaterial", **_with(ISO, nu=0.5))
_case("PhaseMaterial", **_with(ISO, nu=-1.0))
_case("PhaseMaterial", **_with(ISO, E=-5.0))
_case("PhaseMaterial", **_with(ISO, layers=[[1.0, 100.0, 0.2]]))
_case("PhaseMaterial", **_with(ISO, driver="interface"))
_case("PhaseMaterial", **LAM)
_case("PhaseMaterial", **_without(LAM, "layers"))
_case("PhaseMaterial", **_with(LAM, layers=[]))
_case("PhaseMaterial", **_with(LAM, layers=[[0.5, 100.0], [0.5, 50.0, 0.25]]))
_case("PhaseMaterial", **_with(LAM, layers=[[0.5, 100.0, 0.2], [0.4, 50.0, 0.25]]))
_case("PhaseMaterial", **_with(LAM, layers=[[0.5, 100.0, 0.2], [0.5, 50.0, 0.6]]))
_case("PhaseMaterial", **_with(LAM, layers=[[0.0, 100.0, 0.2], [1.0, 50.0, 0.25]]))
_case("PhaseMaterial", **_with(LAM, layers=[[0.5, -1.0, 0.2], [0.5, 50.0, 0.25]]))
_case("PhaseMaterial", **_without(LAM, "nu"))

# MaterialTable (model.py:424-446): phases given as {key: PhaseMaterial arguments}
_case("MaterialTable", phases={"mi_matrix": ISO, "pore": PORE}, length_scale=0.3, scale="micro")
_case("MaterialTable", phases={}, length_scale=0.3, scale="micro")
_case("MaterialTable", phases={"fibre": ISO}, length_scale=0.3, scale="micro")
_case("MaterialTable", phases={"mi_matrix": ISO}, length_scale=0.0, scale="micro")
_case("MaterialTable", phases={"mi_matrix": ISO}, length_scale=0.3, scale="meso")

# VoxelModel (model.py:496-572): the phase array is `fill` everywhere (or `phase_dtype`,
# `phase_shape` overrides), the tangent `tangent` everywhere, the materials `phases`
_VM = dict(grid=GRID, fill=3, phases={"mi_matrix": ISO, "pore": PORE}, tangent=[0.0, 0.0, 1.0])
_case("VoxelModel", **_VM)
_case("VoxelModel", **_with(_VM, fill=4))
_case("VoxelModel", **_with(_VM, fill=0))
_case("VoxelModel", **_with(_VM, fill=7))
_case("VoxelModel", **_with(_VM, phase_shape=[4, 2, 2]))
_case("VoxelModel", **_with(_VM, phase_dtype="float64"))
_case("VoxelModel", **_with(_VM, tangent=[0.0, 0.0, math.nan]))
_case("VoxelModel", **_with(_VM, tangent_shape=[4, 2, 3, 2]))
_case("VoxelModel", **_with(_VM, fill=1, phases={"bn_band": LAM}))
_case("VoxelModel", **_with(_VM, fill=1, phases={"bn_band": LAM}, tangent=[0.0, 0.0, 2.0]))
_case("VoxelModel", **_with(_VM, tangent=[0.0, 0.0, 2.0]))
_case("VoxelModel", **_with(_VM, interface_nodes=[60, "bool"]))
_case("VoxelModel", **_with(_VM, interface_nodes=[59, "bool"]))
_case("VoxelModel", **_with(_VM, interface_nodes=[60, "int64"]))

# LoadCase (model.py:589-627)
_case("LoadCase", **LOAD)
_case("LoadCase", **_with(LOAD, targets=[0.001, -0.001, 0.0]))
_case("LoadCase", **_with(LOAD, controlled=1.5))
_case("LoadCase", **_with(LOAD, controlled=True))
_case("LoadCase", **_with(LOAD, controlled=2.0))
_case("LoadCase", **_with(LOAD, free=[1], fixed_zero=[0, 1, 3, 4, 5]))
_case("LoadCase", **_with(LOAD, fixed_zero=[0, 1, 3, 4]))
_case("LoadCase", **_with(LOAD, targets=[]))
_case("LoadCase", **_with(LOAD, targets=[0.0, 0.001]))
_case("LoadCase", **_with(LOAD, targets=[0.001, 0.001]))
_case("LoadCase", **_with(LOAD, targets=[0.001, math.nan]))
_case("LoadCase", **_with(LOAD, free=[0, 1], fixed_zero=[3, 4, 5]))

# SolverConfig (model.py:706-897); the device is named so the two defaults do not differ
for kw in [dict(), dict(kappa=0.0), dict(kappa=1.0), dict(kappa=-1e-3), dict(kappa=math.nan),
           dict(stagger_tol=0.0), dict(pcg_rtol_mech=-1.0), dict(damage_kkt_tol=math.inf),
           dict(max_stagger=0), dict(max_stagger=2.5), dict(min_stagger=3, max_stagger=2), dict(min_stagger=-1),
           dict(min_stagger=0), dict(max_cutbacks=-1), dict(max_cutbacks=0), dict(batch_size=0),
           dict(check_every=True), dict(damage_maxit=0), dict(damage_max_active_set=1),
           dict(damaged_threshold=0.0), dict(damaged_threshold=1.0), dict(damaged_threshold=1.5),
           dict(preconditioner="ilu"), dict(irreversibility="penalty"), dict(irreversibility="history_only"),
           dict(history="min"), dict(history="current"), dict(energy_split_isotropic="amor"),
           dict(energy_split_isotropic="full"), dict(energy_split_band="interface"),
           dict(energy_split_band="laminate"), dict(band_stress="variational"),
           dict(band_stress="variational", energy_split_band="interface"), dict(band_stress="plain"),
           dict(on_stagger_failure="skip"), dict(on_stagger_failure="raise"), dict(final_mechanics_resolve=False),
           dict(anderson_depth=-1), dict(anderson_depth=1.5), dict(anderson_depth=True), dict(anderson_depth=4),
           dict(anderson_start=1), dict(anderson_start=4), dict(anderson_start=2.5),
           dict(crack_closure="axes"), dict(crack_closure="onset"), dict(crack_closure="spectral"),
           dict(crack_closure="full"), dict(crack_closure="axes", anderson_depth=1),
           dict(damage_law="at1"), dict(damage_law="pfczm"), dict(damage_law="pfczm", irreversibility="history_only"),
           dict(damage_law="pfczm", pfczm_softening="exponential"),
           dict(damage_law="pfczm", pfczm_softening="exponential", pfczm_p=2.5),
           dict(damage_law="pfczm", pfczm_softening="cubic"), dict(damage_law="pfczm", pfczm_p=3),
           dict(damage_law="pfczm", pfczm_p=1), dict(damage_law="pfczm", pfczm_p=True),
           dict(damage_law="pfczm", pfczm_max_newton=0), dict(damage_law="pfczm", pfczm_max_newton=10),
           dict(pfczm_max_newton=10), dict(pfczm_p=2.0), dict(pfczm_softening="exponential"),
           dict(dtype="float32"), dict(dtype="float64"), dict(device="mps"), dict(device="cpu"),
           dict(device="npu"), dict(num_threads=0), dict(num_threads=4)]:
    _case("SolverConfig", **({"device": "cuda"} | kw))


# 2D Material (physics/material.py:80-257)
MAT = dict(E=210000.0, nu=0.3, Gc=2.7, l0=0.05)
for kw in [dict(), dict(pf_model="at1"), dict(pf_model="AllenCahn"), dict(pf_model="at3"), dict(pf_model="pfczm"),
           dict(pf_model="PFCZM", sigma_ts=3.0), dict(pf_model="PFCZM", sigma_ts=3.0, degradation_type="cubic"),
           dict(eta_residual=0.0), dict(eta_residual=-1.0), dict(stress_degradation="partial"),
           dict(stress_degradation="full"), dict(degradation_type="rational_at2"),
           dict(degradation_type="rational_at2", pf_model="AT1"), dict(pfczm_p=1), dict(pfczm_p=2.5),
           dict(pfczm_p=True), dict(pfczm_p=3), dict(pfczm_softening="cubic"), dict(pfczm_softening="exponential"),
           dict(energy_split="spectral_plane_stress_condensed"),
           dict(energy_split="spectral_plane_stress_condensed", plane_stress=True),
           dict(at1_threshold="manual"), dict(at1_threshold=-1.0), dict(at1_threshold=2.5), dict(at1_threshold=0),
           dict(at1_threshold=[1.0]), dict(cubic_s=-0.5), dict(plasticity_model="j2_isotropic"),
           dict(plasticity_model="j2_isotropic", yield_stress=300.0),
           dict(plasticity_model="j2_isotropic", yield_stress=300.0, hardening_modulus=-1.0),
           dict(plasticity_model="j2_isotropic", yield_stress=300.0, hardening_type="voce"),
           dict(plasticity_model="j2_isotropic", yield_stress=300.0, hardening_type="voce", voce_q_inf=100.0,
                voce_b=0.0),
           dict(plasticity_model="j2_isotropic", yield_stress=300.0, hardening_type="voce", voce_q_inf=100.0,
                voce_b=5.0),
           dict(plasticity_model="j2_isotropic", yield_stress=300.0, hardening_type="swift", swift_K=500.0),
           dict(plasticity_model="j2_isotropic", yield_stress=300.0, hardening_type="swift", swift_K=500.0,
                swift_n=-0.2),
           dict(hardening_type="swift")]:
    _case("Material2D", **(MAT | kw))

# 2D SolverConfig (solvers/staggered_solver.py:45-162): no checks, one normalisation
for kw in [dict(), dict(solver_type="quasi_static"), dict(solver_type="static"), dict(solver_type="monolithic"),
           dict(solver_type="quasi_static", preconditioner="gmg"), dict(solver_type="explicit", preconditioner="gmg"),
           dict(adaptive_dt=True, print_every=0, h5_every=0, viz_format="pv", dump_every=0),
           dict(time_integrator="verlet", rho_inf=0.8, softmax_H_beta=10.0, H_update_scale=0.5)]:
    _case("Config2D", **kw)

NORMALISED = {"Material2D": ("pf_model", "eta_residual", "at1_threshold", "pfczm_p"),
              "Config2D": ("preconditioner", "solver_type", "time_integrator")}
"""Fields of an accepted 2D object whose stored value the fixture records."""


def build(mod, case):
    """Run the constructor call of ``case`` on the classes of namespace ``mod`` (the 3D data
    classes, ``Material`` and ``Config2D``, the 2D material and solver settings)."""
    cls, kw = case["cls"], dict(case["kw"])

    def phase(args):
        args = dict(args)
        if args.get("layers") is not None:
            args["layers"] = tuple(tuple(layer) for layer in args["layers"])
        return mod.PhaseMaterial(**args)

    def table(phases, length_scale=0.3, scale="micro"):
        return mod.MaterialTable(phases={k: phase(v) for k, v in phases.items()}, length_scale=length_scale,
                                 scale=scale)

    def grid(args):
        return mod.VoxelGrid(**{k: tuple(v) for k, v in args.items()})

    if cls == "VoxelGrid":
        return grid(kw)
    if cls == "PhaseMaterial":
        return phase(kw)
    if cls == "MaterialTable":
        return table(**kw)
    if cls == "VoxelModel":
        g = grid(kw["grid"])
        shape = tuple(kw.get("phase_shape", g.array_shape))
        phase_id = np.full(shape, kw["fill"], dtype=kw.get("phase_dtype", "uint8"))
        if "tangent_shape" in kw:
            tangent = np.zeros(tuple(kw["tangent_shape"]))
        else:
            tangent = np.broadcast_to(np.asarray(kw["tangent"], dtype=np.float64), (*g.array_shape, 3)).copy()
        aux = {}
        if "interface_nodes" in kw:
            length, dtype = kw["interface_nodes"]
            aux["interface_nodes"] = np.zeros(length, dtype=dtype)
        return mod.VoxelModel(grid=g, phase_id=phase_id, tangent=tangent, materials=table(kw["phases"]), aux=aux)
    if cls == "LoadCase":
        return mod.LoadCase(**{k: tuple(v) if isinstance(v, list) else v for k, v in kw.items()})
    if cls == "SolverConfig":
        return mod.SolverConfig(**kw)
    if cls == "Material2D":
        return mod.Material(**kw)
    if cls == "Config2D":
        return mod.Config2D(**kw)
    raise KeyError(cls)


def outcome(mod, case):
    """``'ok'`` (with the normalised fields of a 2D material) or the exception class name."""
    try:
        obj = build(mod, case)
    except (ValueError, TypeError) as exc:
        return type(exc).__name__
    if case["cls"] in NORMALISED:
        return "ok " + json.dumps({k: getattr(obj, k) for k in NORMALISED[case["cls"]]})
    return "ok"


def main(src):
    sys.path.insert(0, HERE)
    from make_golden import _import_reference
    _import_reference(src)
    import types
    import phast.solid3d.model as ref3d
    from phast.physics.material import Material
    from phast.solvers.staggered_solver import SolverConfig as Config2D
    ref = types.SimpleNamespace(**vars(ref3d))
    ref.Material, ref.Config2D = Material, Config2D
    out = [dict(case, outcome=outcome(ref, case)) for case in CASES]
    with open(os.path.join(HERE, "validation.json"), "w") as f:
        json.dump(out, f, indent=0)
    print(f"{len(out)} cases, {sum(not c['outcome'].startswith('ok') for c in out)} refused")


if __name__ == "__main__":
    main(sys.argv[1])

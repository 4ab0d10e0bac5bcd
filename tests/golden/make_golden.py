"""Generate golden vectors by running the PhAST reference implementation.

Run in a container where the reference sources are present, passing the
reference's ``src`` directory::

    python tests/golden/make_golden.py <path-to-reference-src>

The reference is pure Python/PyTorch.  Its I/O-only dependencies (meshio,
gmsh, h5py, zarr, numcodecs, matplotlib) are not needed on the hot path; they
are replaced by permissive stub modules for the import.  Every case uses small
seeded inputs so the fixtures stay a few hundred KB.  The fixtures are the
ground truth the oracle and the CUDA path are pinned against; this script is
never run by the tests.
"""
from __future__ import annotations

import importlib.abc
import importlib.machinery
import os
import sys
from unittest import mock

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
STUBS = ("meshio", "gmsh", "h5py", "zarr", "numcodecs", "matplotlib", "mpl_toolkits")


class _StubFinder(importlib.abc.MetaPathFinder, importlib.abc.Loader):
    def find_spec(self, name, path=None, target=None):
        if name.split(".")[0] in STUBS:
            return importlib.machinery.ModuleSpec(name, self, is_package=True)
        return None

    def create_module(self, spec):
        m = mock.MagicMock(name=spec.name)
        m.__path__ = []
        m.__spec__ = spec
        return m

    def exec_module(self, module):
        pass


def _import_reference(src):
    sys.meta_path.insert(0, _StubFinder())
    sys.path.insert(0, src)
    import phast  # noqa: F401


def t(x):
    import torch
    return torch.as_tensor(np.asarray(x), dtype=torch.float64)


def n(x):
    return x.detach().cpu().numpy()


# ---------------------------------------------------------------------------
# 2D Q4
# ---------------------------------------------------------------------------

def q4_cases():
    import torch
    from phast.core.mesh import FEMMesh
    from phast.core.quad_elements import structured_q4_mesh
    from phast.core.fem_operators import FEMOperators
    from phast.physics.material import Material

    rng = np.random.default_rng(1234)
    sm = structured_q4_mesh(1.2, 1.0, 6, 5)
    mesh = FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4")
    N, E = mesh.n_nodes, mesh.n_elems
    u = rng.normal(size=(N, 2)) * 1e-3
    d = rng.uniform(0, 1, size=N)
    out = {"nodes": n(sm.nodes), "quads": n(sm.quads), "nx": 6, "ny": 5, "width": 1.2, "height": 1.0,
           "u": u, "d": d}
    for split in ("isotropic", "amor", "spectral", "star_convex", "spectral_stress"):
        for ps in (False, True):
            if ps and split in ("spectral", "spectral_stress"):
                continue
            mat = Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.01, eta_residual=1e-8, energy_split=split,
                           plane_stress=ps, rho=2.45e-9)
            fem = FEMOperators(mesh, mat)
            key = f"{split}_{'ps' if ps else 'pe'}"
            out[f"f_{key}"] = n(fem.internal_force(t(u), t(d)))
            out[f"psi_{key}"] = n(fem.compute_psi_plus(t(u)))
    mat = Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.01, eta_residual=1e-8, energy_split="isotropic", rho=2.45e-9)
    fem = FEMOperators(mesh, mat)
    exx, eyy, gxy = fem.compute_strain(t(u))
    out.update(exx=n(exx), eyy=n(eyy), gxy=n(gxy))
    out["f_linear"] = n(fem.internal_force_linear(t(u)))
    out["kdiag"] = n(fem.stiffness_diagonal(t(d)))
    out["kdiag0"] = n(fem.stiffness_diagonal())
    out["lap"] = n(fem.laplacian_matvec(t(d)))
    out["mass"] = n(fem._q4_mass_matvec(t(d)))
    out["M_scalar"] = n(mesh.M_scalar)
    v = rng.normal(size=(N, 2))
    out["v"] = v
    ec = fem.compute_energy_components(t(u), t(d), v=t(v))
    out["energy"] = np.array([ec["elastic"], ec["kinetic"], ec["fracture"], ec["total"]])
    top = sm.node_sets["top"]
    out["top"] = n(top)
    out["reaction"] = np.array([fem.compute_reaction_force(t(u), t(d), top, component=1)])
    out["h_min"] = np.array([mesh.h_min])
    out["dt_cfl"] = np.array([fem.dt_cfl])
    np.savez_compressed(os.path.join(HERE, "q4_ops.npz"), **out)


def q4_damage_cases():
    import torch
    from phast.core.mesh import FEMMesh
    from phast.core.quad_elements import structured_q4_mesh
    from phast.core.fem_operators import FEMOperators
    from phast.physics.material import Material
    from phast.solvers.damage_solver import PhaseFieldDamageSolver

    rng = np.random.default_rng(99)
    sm = structured_q4_mesh(1.0, 1.0, 12, 10)
    mesh = FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4")
    N, E = mesh.n_nodes, mesh.n_elems
    mat = Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.05, eta_residual=1e-8, energy_split="isotropic")
    fem = FEMOperators(mesh, mat)
    out = {"nx": 12, "ny": 10, "width": 1.0, "height": 1.0, "Gc": 2.7, "l0": 0.05}
    H = rng.uniform(0, 400.0, size=(E, 4))
    H[rng.uniform(size=E) < 0.15] *= 40.0
    d_prev = np.clip(rng.uniform(-0.3, 0.5, size=N), 0, 1)
    out.update(H=H, d_prev=d_prev)
    ds = PhaseFieldDamageSolver(fem, tol=1e-10, max_iter=2000, use_multigrid=False, bounds_method="projected_cg")
    x = rng.uniform(0, 1, size=N)
    rd = 2 * t(H) + mat.Gc / mat.l0
    out["x"] = x
    out["Ax"] = n(ds._Ax_q4(t(x), rd))
    prep = ds._prepare_cg(t(H), t(d_prev))
    out["b"] = n(prep[3])
    out["M_inv"] = n(prep[4])
    out["d_solve"] = n(ds.solve(t(H), t(d_prev)))
    out["iters_solve"] = np.array([ds.last_iter])
    # warm start from an initial guess (quasi-static stagger convention)
    guess = np.clip(d_prev + rng.uniform(0, 0.2, size=N), 0, 1)
    out["guess"] = guess
    out["d_solve_guess"] = n(ds.solve(t(H), t(d_prev), initial_guess=t(guess)))
    out["iters_solve_guess"] = np.array([ds.last_iter])
    # phase-field Dirichlet (notch row) pinned to 1
    mask = np.zeros(N, dtype=bool)
    mask[(np.arange(N) // 13 == 5) & (np.arange(N) % 13 < 6)] = True
    out["pf_mask"] = mask
    out["d_solve_pf"] = n(ds.solve(t(H), t(d_prev), pf_dirichlet_mask=torch.as_tensor(mask),
                                   pf_dirichlet_values=t(mask.astype(float))))
    out["iters_solve_pf"] = np.array([ds.last_iter])
    np.savez_compressed(os.path.join(HERE, "q4_damage.npz"), **out)


def q4_dynamics_cases():
    import torch
    from phast.core.mesh import FEMMesh
    from phast.core.quad_elements import structured_q4_mesh
    from phast.core.fem_operators import FEMOperators
    from phast.physics.material import Material
    from phast.solvers.mechanics_solver import ExplicitDynamics, QuasiStaticSolver

    rng = np.random.default_rng(7)
    sm = structured_q4_mesh(10.0, 4.0, 10, 4)
    mesh = FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4")
    N = mesh.n_nodes
    mat = Material(E=32000.0, nu=0.2, Gc=3e-3, l0=0.5, rho=2.45e-9, eta_residual=1e-8, energy_split="spectral")
    fem = FEMOperators(mesh, mat)
    ex = ExplicitDynamics(fem, dt_safety=0.5)
    u = rng.normal(size=(N, 2)) * 1e-4
    v = rng.normal(size=(N, 2)) * 1e-1
    a = rng.normal(size=(N, 2)) * 1e3
    d = rng.uniform(0, 0.5, size=N)
    f_ext = rng.normal(size=(N, 2))
    bc_mask = np.zeros((N, 2), dtype=bool)
    bc_mask[sm.node_sets["left"].numpy(), 0] = True
    bc_vals = np.zeros((N, 2))
    out = {"nx": 10, "ny": 4, "width": 10.0, "height": 4.0, "u": u, "v": v, "a": a, "d": d, "f_ext": f_ext,
           "bc_mask": bc_mask, "dt": np.array([ex.dt])}
    un, vn, an = t(u), t(v), t(a)
    for _ in range(3):
        un, vn, an = ex.step(un, vn, an, t(d), t(f_ext), torch.as_tensor(bc_mask), t(bc_vals))
    out.update(u3=n(un), v3=n(vn), a3=n(an))
    # quasi-static Newton + CG (isotropic split, linear)
    mat2 = Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.01, eta_residual=1e-8, energy_split="isotropic")
    fem2 = FEMOperators(mesh, mat2)
    qs = QuasiStaticSolver(fem2, tol=1e-10, max_iter=50, backend="cg")
    bm = np.zeros((N, 2), dtype=bool)
    bv = np.zeros((N, 2))
    bot, top = sm.node_sets["bottom"].numpy(), sm.node_sets["top"].numpy()
    bm[bot, :] = True
    bm[top, 1] = True
    bv[top, 1] = 1e-3
    uq, conv, nit = qs.solve(t(d), torch.zeros(N, 2, dtype=torch.float64), torch.as_tensor(bm), t(bv))
    out.update(qs_bc_mask=bm, qs_bc_vals=bv, qs_u=n(uq), qs_conv=np.array([bool(conv)]), qs_nit=np.array([nit]))
    np.savez_compressed(os.path.join(HERE, "q4_dynamics.npz"), **out)


def q4_staggered_case():
    """Two quasi-static SENT load steps and three explicit steps through StaggeredSolver."""
    import torch
    from phast.core.mesh import FEMMesh
    from phast.core.quad_elements import structured_q4_mesh
    from phast.physics.material import Material
    from phast.physics.boundary_conditions import BoundaryConditions
    from phast.solvers.staggered_solver import StaggeredSolver, SolverConfig

    nx = ny = 16
    sm = structured_q4_mesh(1.0, 1.0, nx, ny)
    mesh = FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4")
    N = mesh.n_nodes
    mat = Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.1, eta_residual=1e-8, energy_split="isotropic", rho=7.8e-9)
    bcs = BoundaryConditions(N)
    bot, top = sm.node_sets["bottom"], sm.node_sets["top"]
    bcs.fix(bot, 0)
    bcs.fix(bot, 1)
    bcs.add(top, 1, 1.0)
    nodes = sm.nodes.numpy()
    notch = np.nonzero((np.abs(nodes[:, 1] - 0.5) < 1e-12) & (nodes[:, 0] < 0.5))[0]
    bcs.add_pf_dirichlet(torch.as_tensor(notch), 1.0)
    cfg = SolverConfig(solver_type="quasi_static", backend="cg", static_tol=1e-10, damage_tol=1e-10,
                       bounds_method="projected_cg", use_multigrid=False, stagger_tol=1e-6, max_stagger=100)
    s = StaggeredSolver(mesh, mat, bcs, cfg)
    pf_mask, pf_vals = bcs.get_pf_dirichlet_mask_values()
    s.d = torch.where(pf_mask, pf_vals, s.d)
    out = {"nx": nx, "ny": ny, "notch": notch}
    us, ds_, Hs, rf, stag = [], [], [], [], []
    for k in range(1, 4):
        bcs.load_factor = 0.004 * k
        s.step_full()
        us.append(n(s.u))
        ds_.append(n(s.d))
        Hs.append(n(s.H_elem))
        rf.append(s.fem.compute_reaction_force(s.u, s.d, top, component=1))
        stag.append(s._last_stagger_iter)
    out.update(qs_u=np.stack(us), qs_d=np.stack(ds_), qs_H=np.stack(Hs), qs_rf=np.array(rf), qs_stag=np.array(stag))
    # explicit dynamics with a damage solve every step and constant edge tractions set on f_ext
    mat2 = Material(E=32000.0, nu=0.2, Gc=3e-3, l0=0.15, rho=2.45e-9, eta_residual=1e-8, energy_split="spectral")
    bcs2 = BoundaryConditions(N)
    bcs2.add_pf_dirichlet(torch.as_tensor(notch), 1.0)
    cfg2 = SolverConfig(solver_type="explicit", dt_safety=0.5, damage_every=1, damage_tol=1e-10,
                        bounds_method="projected_cg", use_multigrid=False)
    s2 = StaggeredSolver(mesh, mat2, bcs2, cfg2)
    s2.d = torch.where(pf_mask, pf_vals, s2.d)
    f_ext = np.zeros((N, 2))
    hx = 1.0 / nx
    for nodeset, sign in ((top.numpy(), 1.0), (bot.numpy(), -1.0)):
        w = np.full(len(nodeset), hx)
        w[0] = w[-1] = hx / 2
        f_ext[nodeset, 1] = sign * 50.0 * w
    s2.f_ext = t(f_ext)
    eu, ed, eH = [], [], []
    for k in range(6):
        s2.step_full()
        eu.append(n(s2.u))
        ed.append(n(s2.d))
        eH.append(n(s2.H_elem))
    out.update(ex_f_ext=f_ext, ex_dt=np.array([s2.dt]), ex_u=np.stack(eu), ex_d=np.stack(ed), ex_H=np.stack(eH),
               ex_v=n(s2.v), ex_a=n(s2.a))
    np.savez_compressed(os.path.join(HERE, "q4_staggered.npz"), **out)


# ---------------------------------------------------------------------------
# 3D periodic voxels
# ---------------------------------------------------------------------------

def _voxel_model(shape, h, pore_radius_frac, matrix=(3000.0, 0.35, 0.5), ell=None):
    from phast.solid3d.model import VoxelGrid, VoxelModel, MaterialTable, PhaseMaterial, PHASE_ID
    nx, ny, nz = shape
    grid = VoxelGrid(shape=shape, h=(h, h, h))
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    c = np.stack([(i + 0.5) / nx - 0.5, (j + 0.5) / ny - 0.5, (k + 0.5) / nz - 0.5], -1)
    r = np.linalg.norm(c, axis=-1)
    phase = np.full((nz, ny, nx), PHASE_ID["mi_matrix"], dtype=np.uint8)
    phase[r < pore_radius_frac] = PHASE_ID["pore"]
    E, nu, Gc = matrix
    phases = {"mi_matrix": PhaseMaterial(name="mi_matrix", kind="isotropic", Gc=Gc, driver="spectral", E=E, nu=nu),
              "pore": PhaseMaterial(name="pore", kind="isotropic", Gc=Gc, driver="spectral", E=E * 1e-6, nu=nu)}
    table = MaterialTable(phases=phases, length_scale=(2 * h if ell is None else ell), scale="micro")
    tangent = np.zeros((nz, ny, nx, 3))
    tangent[..., 2] = 1.0
    return VoxelModel(grid=grid, phase_id=phase, tangent=tangent, materials=table), phase


def h8_cases():
    import torch
    from phast.solid3d.model import LoadCase, SolverConfig
    from phast.solid3d.operator import PeriodicVoxelPhaseFieldOperator
    from phast.solvers.box_kkt_h8 import solve_h8_scalar_box_kkt
    from phast.solid3d.linalg import solve_constrained

    rng = np.random.default_rng(5)
    shape = (5, 4, 6)
    h = 1.0 / 6
    model, phase = _voxel_model(shape, h, 0.3)
    load = LoadCase(name="zz", controlled=2, targets=(0.01,), free=(), fixed_zero=(0, 1, 3, 4, 5))
    cfg = SolverConfig(device="cpu", kappa=1e-6, energy_split_isotropic="spectral")
    op = PeriodicVoxelPhaseFieldOperator(model, load, cfg)
    nr, E = op.n_red, op.n_elements
    x = rng.normal(size=op.n_mech) * 1e-3
    d = rng.uniform(0, 1, size=nr)
    H = rng.uniform(0, 2.0, size=(E, 8))
    g = op.degradation(t(d))
    out = {"shape": np.array(shape), "h": h, "phase": phase, "pinned": op.pinned_node, "x": x, "d": d, "H": H,
           "g": n(g), "damage_scale": op.damage_scale, "ell": op.ell}
    out["mech_g"] = n(op.mech_action(t(x), g))
    out["mech_1"] = n(op.mech_action(t(x)))
    out["mdiag_g"] = n(op.mech_diagonal(g))
    out["mdiag_1"] = n(op.mech_diagonal())
    out["Y"] = n(op.driving_force(t(x)))
    out["dact"] = n(op.damage_action(t(d), t(H)))
    out["dact0"] = n(op.damage_action(t(d)))
    out["drhs"] = n(op.damage_rhs(t(H)))
    out["ddiag"] = n(op.damage_diagonal(t(H)))
    out["sigma"] = n(op.macro_stress(t(x), g))
    out["energy"] = np.array([float(op.elastic_energy(t(x), g))])
    out["frac"] = np.array([op.fracture_energy(t(d))["total"]])
    # constrained mechanics solve at fixed damage
    mask = op.mech_fixed_mask()
    vals = op.mech_fixed_values(0.01)
    xs, info = solve_constrained(lambda v: op.mech_action(v, g), diag=op.mech_diagonal(g), fixed_mask=mask,
                                 fixed_values=vals, rtol=1e-8, maxiter=5000, check_every=10)
    out["x_solve"] = n(xs)
    out["x_solve_iters"] = np.array([info.iterations])
    # box-KKT damage solve
    Hs = t(H * 30.0)
    system = op.damage_system(Hs)
    lower = t(np.clip(d - 0.5, 0, 1))
    res = solve_h8_scalar_box_kkt(system, lower_bound=lower, upper_bound=1.0, initial=lower,
                                  linear_tolerance=1e-10, kkt_tolerance=1e-8, max_linear_iterations=4000,
                                  max_active_set_iterations=64)
    out["H_kkt"] = H * 30.0
    out["lower_kkt"] = n(lower)
    out["d_kkt"] = n(res.solution)
    out["kkt_pcg"] = np.array([res.total_pcg_iterations])
    out["kkt_sets"] = np.array([res.active_set_iterations])
    np.savez_compressed(os.path.join(HERE, "h8_ops.npz"), **out)


def h8_staggered_case():
    import torch
    from phast.solid3d.model import LoadCase, SolverConfig
    from phast.solid3d.operator import PeriodicVoxelPhaseFieldOperator
    from phast.solid3d.staggered import StaggeredSolver

    shape = (6, 6, 6)
    h = 1.0 / 6
    model, phase = _voxel_model(shape, h, 0.2)
    targets = tuple(0.02 * k / 50 for k in range(1, 51))
    load = LoadCase(name="zz", controlled=2, targets=targets, free=(), fixed_zero=(0, 1, 3, 4, 5))
    cfg = SolverConfig(device="cpu", kappa=1e-6, energy_split_isotropic="spectral", damage_law="at2")
    op = PeriodicVoxelPhaseFieldOperator(model, load, cfg)
    solver = StaggeredSolver(op)
    state = solver.initial_state()
    xs, dsl, Hs, sig, stag, pm, pp = [], [], [], [], [], [], []
    for k in range(3):
        state, rec = solver.advance(state, targets[k])
        xs.append(n(state.x))
        dsl.append(n(state.d))
        Hs.append(n(state.H))
        sig.append(np.array(rec.macro_stress))
        stag.append(rec.stagger_iters)
        pm.append(rec.pcg_iters_mech)
        pp.append(rec.pcg_iters_pf)
    out = {"shape": np.array(shape), "h": h, "phase": phase, "pinned": op.pinned_node, "targets": np.array(targets[:3]),
           "x": np.stack(xs), "d": np.stack(dsl), "H": np.stack(Hs), "sigma": np.stack(sig),
           "stag": np.array(stag), "pcg_mech": np.array(pm), "pcg_pf": np.array(pp)}
    np.savez_compressed(os.path.join(HERE, "h8_staggered.npz"), **out)


# ---------------------------------------------------------------------------
# 2D T3 (unstructured triangles: a perturbed q4_to_triangles twin)
# ---------------------------------------------------------------------------

def t3_cases():
    import torch
    from phast.core.mesh import FEMMesh
    from phast.core.quad_elements import q4_to_triangles, structured_q4_mesh
    from phast.core.fem_operators import FEMOperators
    from phast.physics.material import Material
    from phast.solvers.damage_solver import PhaseFieldDamageSolver

    rng = np.random.default_rng(4321)
    sm = structured_q4_mesh(1.0, 0.8, 9, 7)
    nodes = n(sm.nodes).copy()
    # jitter interior nodes so the element geometry varies (an unstructured mesh)
    inner = (nodes[:, 0] > 1e-9) & (nodes[:, 0] < 1.0 - 1e-9) & (nodes[:, 1] > 1e-9) & (nodes[:, 1] < 0.8 - 1e-9)
    nodes[inner] += rng.uniform(-0.02, 0.02, size=(int(inner.sum()), 2))
    tri = q4_to_triangles(sm.quads)
    mesh = FEMMesh.from_tensors(t(nodes), tri, element_type="T3")
    N, E = mesh.n_nodes, mesh.n_elems
    u = rng.normal(size=(N, 2)) * 1e-3
    d = rng.uniform(0, 1, size=N)
    out = {"nodes": nodes, "tris": n(tri), "u": u, "d": d}
    for split in ("isotropic", "amor", "spectral", "star_convex", "spectral_stress"):
        for ps in (False, True):
            if ps and split in ("spectral", "spectral_stress"):
                continue
            mat = Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.05, eta_residual=1e-8, energy_split=split,
                           plane_stress=ps, rho=2.45e-9)
            fem = FEMOperators(mesh, mat)
            key = f"{split}_{'ps' if ps else 'pe'}"
            out[f"f_{key}"] = n(fem.internal_force(t(u), t(d)))
            out[f"psi_{key}"] = n(fem.compute_psi_plus(t(u)))
    mat = Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.05, eta_residual=1e-8, energy_split="isotropic", rho=2.45e-9)
    fem = FEMOperators(mesh, mat)
    exx, eyy, gxy = fem.compute_strain(t(u))
    out.update(exx=n(exx), eyy=n(eyy), gxy=n(gxy), areas=n(mesh.areas), grad_phi=n(mesh.grad_phi))
    out["f_linear"] = n(fem.internal_force_linear(t(u)))
    out["M_scalar"] = n(mesh.M_scalar)
    # damage system (element H) and the projected solve
    H = rng.uniform(0, 400.0, size=E)
    d_prev = np.clip(rng.uniform(-0.3, 0.5, size=N), 0, 1)
    out.update(H=H, d_prev=d_prev)
    ds = PhaseFieldDamageSolver(fem, tol=1e-10, max_iter=3000, use_multigrid=False, bounds_method="projected_cg")
    prep = ds._prepare_cg(t(H), t(d_prev))
    x = rng.uniform(0, 1, size=N)
    out["x"] = x
    out["rc"] = n(prep[2])
    out["Ax"] = n(ds._Ax(t(x), prep[2]))
    out["b"] = n(prep[3])
    out["M_inv"] = n(prep[4])
    out["d_solve"] = n(ds.solve(t(H), t(d_prev)))
    out["iters_solve"] = np.array([ds.last_iter])
    np.savez_compressed(os.path.join(HERE, "t3_ops.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        raise SystemExit(__doc__)
    _import_reference(sys.argv[1])
    import torch
    torch.set_num_threads(8)
    q4_cases()
    q4_damage_cases()
    q4_dynamics_cases()
    q4_staggered_case()
    h8_cases()
    h8_staggered_case()
    t3_cases()
    print("golden fixtures written to", HERE)

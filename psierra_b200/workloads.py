"""The configured workloads beyond the single-assembly benchmark, run as they are written.

``python -m psierra_b200.workloads cfg3|cfg4|cfg5 [options]`` runs one workload on the
current GPU and prints one JSON record (timings from CUDA events or the host clock
around synchronised device work, iteration counts, accuracy figures).  Inputs are
seeded synthetic meshes and fields (the reference's own meshes are not used).

* cfg3 -- Tet10 compression: cube 30^3 Kuhn cells -> 162,000 Tet10, 226,981 nodes
  (680,943 DOFs), NeoHookean E = 1e4, nu = 0.4; bottom face clamped, top face u_z =
  -0.2 prescribed and ramped over 20 increments; every Newton step solved by Jacobi PCG
  to rtol 1e-8 (psierra ``analysis/nonlinear_static.py:250-404``,
  ``solver/sparse_linear_solver.py:37-68``).  FP64 and FP32-mixed tangents.
  ``--preconditioner block-jacobi|two-level`` swaps the PCG's preconditioner (same
  tolerance, so the same answer to within it).
* cfg4 -- adjoint identification on the ellipsoid (80 x 60 x 70 mm, 2 mm Kuhn grid
  clipped to the ellipsoid: every corner inside), per-element mu ~ LogNormal(ln 1000 Pa,
  0.3), kappa = 50 mu, density 1040, gravity through the consistent mass (a stated
  fraction of 9.81 m/s^2), clamp z < -60 mm; loss 1/2 ||u - u_target||^2 against a second
  seed's equilibrium; the autograd gradient against central differences (h = 1e-6 mu_e
  by default) on random elements.
* cfg5 -- 256 seeded beams (``meshgen.beam_batch``, ~4.1M Tet4), per-instance E and nu,
  FP32-mixed tangent, 8 increments, the batched Newton replayed as one CUDA graph.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from psierra_b200 import meshgen
from psierra_b200.assembler import GPUAssembler
from psierra_b200.material import IsotropicElasticParameters, NeoHookean, NeoHookeanField
from psierra_b200.newton import DeviceNewton


def _nh(E, nu, rho=1000.0):
    p = IsotropicElasticParameters()
    p.set_from_youngs_poisson(youngs_modulus=E, poissons_ratio=nu, mass_density=rho)
    return NeoHookean(p)


def cfg3(cells: int = 30, n_steps: int = 20, precisions=("fp64", "fp32-mixed"), pcg_rtol: float = 1e-8,
         nr_iterations: int = 30, preconditioner: str = "jacobi") -> dict:
    m = meshgen.tet4_to_tet10(meshgen.box_tet4(1.0, 1.0, 1.0, cells, cells, cells))
    bottom = meshgen.nodes_on_plane(m, 2, "min")
    top = meshgen.nodes_on_plane(m, 2, "max")
    fixed = np.concatenate([3 * bottom + c for c in range(3)] + [3 * top + 2])
    dev = torch.device("cuda")
    up = torch.zeros(m.n_dofs, dtype=torch.float64, device=dev)
    up[torch.from_numpy(3 * top + 2).to(dev)] = -0.2
    f_ext = torch.zeros(m.n_dofs, dtype=torch.float64, device=dev)
    out = {"workload": f"cfg3: cube {cells}^3 Kuhn -> {m.n_elements} Tet10, {m.n_nodes} nodes ({m.n_dofs} DOFs), "
                       f"E=1e4 nu=0.4, top u_z=-0.2 over {n_steps} increments, {preconditioner} PCG rtol {pcg_rtol}, "
                       f"at most {nr_iterations} Newton iterations per increment"}
    us = {}
    for prec in precisions:
        asm = GPUAssembler(m.nodes, m.elements, _nh(1e4, 0.4), precision=prec)
        t_setup = time.perf_counter()
        nt = DeviceNewton(asm, fixed, precision=prec, pcg_tol=pcg_rtol, pcg_maxiter=100000,
                          preconditioner=preconditioner)
        torch.cuda.synchronize()
        t_setup = time.perf_counter() - t_setup
        t0 = time.perf_counter()
        res = nt.solve(f_ext, u_prescribed=up, n_steps=n_steps, nr_iterations=nr_iterations, nr_tol=1e-8)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        us[prec] = res.u
        out[prec.replace("-", "_")] = {
            "converged": bool(res.converged), "steps": res.steps_completed, "seconds": dt,
            "solver_setup_seconds": t_setup,
            "newton_iterations": int(sum(res.iteration_history)), "newton_per_step": res.iteration_history,
            "pcg_iterations": int(sum(res.pcg_iterations)),
            "final_relative_residual": (res.residual_history[-1] / max(res.residual_history[0], 1e-300)
                                        if res.residual_history else None),
            "first_residuals": [float(r) for r in res.residual_history[:32]],
            "first_pcg_iterations": [int(i) for i in res.pcg_iterations[:32]],
            "first_step_lengths": [round(a, 6) for a in res.step_lengths[:32]]}
    if "fp64" in us and "fp32-mixed" in us:
        out["u_mixed_vs_fp64_rel2"] = float((us["fp32-mixed"] - us["fp64"]).norm() / us["fp64"].norm())
    return out


def cfg4(h_grid: float = 0.002, gravity_fraction: float = 0.2, n_check: int = 32, rel_step: float = 1e-6,
         seed: int = 41) -> dict:
    import scipy.sparse as spsp

    from psierra_b200.adjoint import static_equilibrium

    t_mesh = time.perf_counter()
    m = meshgen.ellipsoid_tet4(0.08, 0.06, 0.07, h_grid)
    rng = np.random.default_rng(seed)
    mu_t = np.exp(np.log(1000.0) + 0.3 * rng.normal(size=m.n_elements))
    mu0 = np.exp(np.log(1000.0) + 0.3 * np.random.default_rng(seed + 1).normal(size=m.n_elements))
    asm = GPUAssembler(m.nodes, m.elements, NeoHookeanField(mu0, 50.0 * mu0, mass_density=1040.0))
    _, mv = asm.assemble(None, mass=True)
    M = spsp.csr_matrix((mv.cpu().numpy(), asm.pattern.indices, asm.pattern.indptr), shape=(m.n_dofs,) * 2)
    f_ext = torch.from_numpy(gravity_fraction * (M @ np.tile([0.0, 0.0, -9.81], m.n_nodes))).cuda()
    fixed_nodes = np.where(m.nodes[:, 2] < -0.06 + 1e-12)[0]
    fixed = np.concatenate([3 * fixed_nodes + c for c in range(3)])
    nt = DeviceNewton(asm, fixed, precision="fp64", pcg_tol=1e-13, pcg_maxiter=200000)
    t_mesh = time.perf_counter() - t_mesh
    t_tgt = time.perf_counter()
    with torch.no_grad():
        mt = torch.from_numpy(mu_t).cuda()
        u_tgt = static_equilibrium(nt, mt, 50.0 * mt, f_ext, n_steps=2, polish=3)
    torch.cuda.synchronize()
    t_tgt = time.perf_counter() - t_tgt

    def loss_of(mu_np, u0=None):
        mv_ = torch.from_numpy(mu_np).cuda().requires_grad_(True)
        u = static_equilibrium(nt, mv_, 50.0 * mv_, f_ext, n_steps=2 if u0 is None else 1, polish=3, u0=u0)
        return 0.5 * torch.sum((u - u_tgt) ** 2), mv_, u

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    L, mv_, u_base = loss_of(mu0)
    L.backward()
    u_base = u_base.detach()
    torch.cuda.synchronize()
    t_grad = time.perf_counter() - t0
    g = mv_.grad.cpu().numpy()
    picks = rng.choice(m.n_elements, size=n_check, replace=False)
    errs, fds = [], []
    t1 = time.perf_counter()
    for e in picks:
        h = rel_step * mu0[e]
        mp, mm = mu0.copy(), mu0.copy()
        mp[e] += h
        mm[e] -= h
        with torch.no_grad():
            # Newton from the base equilibrium: a 1e-6 relative change of one element's
            # modulus moves u by far less than one increment would
            fd = (float(loss_of(mp, u_base)[0]) - float(loss_of(mm, u_base)[0])) / (2 * h)
        fds.append(fd)
        errs.append(abs(g[e] - fd) / max(abs(fd), 1e-300))
    t_fd = time.perf_counter() - t1
    Lv = float(L.detach())
    return {"workload": f"cfg4: ellipsoid 80x60x70 mm, {1e3 * h_grid:g} mm Kuhn grid clipped (all corners inside): "
                        f"{m.n_elements} Tet4, {m.n_nodes} nodes; mu_e LogNormal(ln 1000, 0.3), kappa = 50 mu, "
                        f"rho 1040, {gravity_fraction:g} x gravity, clamp z < -60 mm",
            "elements": m.n_elements, "setup_seconds": t_mesh, "target_solve_seconds": t_tgt, "loss": Lv,
            "forward_plus_adjoint_seconds": t_grad, "fd_seconds": t_fd, "fd_elements": int(n_check),
            "fd_relative_step": rel_step, "max_rel_error": float(max(errs)), "median_rel_error": float(np.median(errs)),
            "rel_errors": [float(x) for x in errs],
            "relative_sensitivity": [float(abs(fd) * mu0[e] / Lv) for fd, e in zip(fds, picks)],
            # |adjoint - central difference| in units of L / mu_e: a constant floor here means
            # the difference quotient's rounding (the forward solve's error in L over 2h), not
            # the adjoint, sets the relative errors of the least sensitive elements
            "abs_error_rel_units": [float(abs(g[e] - fd) * mu0[e] / Lv) for fd, e in zip(fds, picks)]}


def cfg5(n: int = 256, target_tets: float = 4.1e6, seed: int = 5, pcg_iterations: int | None = None,
         n_steps: int = 8, preconditioner: str = "two-level") -> dict:
    from psierra_b200.batched import BatchedNewton, MeshBatch

    cases = meshgen.beam_batch(n=n, target_tets=target_tets, seed=seed)
    mus, kappas, forces, fixed = [], [], [], []
    for c in cases:
        mu, _, kappa = meshgen.lame_from_young_poisson(c.youngs, c.poisson)
        mus.append(mu)
        kappas.append(kappa)
        forces.append(meshgen.traction_nodal_forces(c.mesh, 0, "max", c.traction))
        clamp = meshgen.nodes_on_plane(c.mesh, 0, "min")
        fixed.append(np.concatenate([3 * clamp + k for k in range(3)]))
    batch = MeshBatch([c.mesh for c in cases], mus, kappas, precision="fp32-mixed")
    if pcg_iterations is None:
        # block-Jacobi needs O(10^4) CG iterations per Newton step on these beams (fewer
        # stall the Newton iteration); the rigid-body-mode coarse correction a few hundred
        pcg_iterations = 16000 if preconditioner == "block-jacobi" else 300
    t_setup = time.perf_counter()
    solver = BatchedNewton(batch, fixed, pcg_iterations=pcg_iterations, use_graph=True, preconditioner=preconditioner)
    t_setup = time.perf_counter() - t_setup
    f_ext = batch.concat(forces)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = solver.solve(f_ext, n_steps=n_steps)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return {"workload": f"cfg5: {n} beams, {batch.mesh.n_elements} Tet4 in total, FP32-mixed, {n_steps} increments, "
                        f"batched Newton as one CUDA graph per iteration, {preconditioner} CG {pcg_iterations} iterations",
            "elements": batch.mesh.n_elements, "seconds": dt, "solver_setup_seconds": t_setup, "replays": res.replays,
            "newton_per_step_max": [int(x) for x in res.iterations.max(axis=1)],
            "converged": int(res.converged.sum()), "instances": n}


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("workload", choices=["cfg3", "cfg4", "cfg5"])
    ap.add_argument("--cells", type=int, default=30, help="cfg3: cube cells per side")
    ap.add_argument("--steps", type=int, default=20, help="cfg3: increments")
    ap.add_argument("--nr-iterations", type=int, default=30, help="cfg3: Newton iterations per increment")
    ap.add_argument("--pcg-rtol", type=float, default=1e-8, help="cfg3: PCG relative tolerance")
    ap.add_argument("--precisions", default="fp64,fp32-mixed", help="cfg3: comma-separated precisions")
    ap.add_argument("--grid", type=float, default=0.002, help="cfg4: grid spacing (m)")
    ap.add_argument("--gravity", type=float, default=0.2, help="cfg4: fraction of gravity")
    ap.add_argument("--fd-elements", type=int, default=32, help="cfg4: elements checked by central differences")
    ap.add_argument("--fd-step", type=float, default=1e-6, help="cfg4: central-difference step / mu_e")
    ap.add_argument("--beams", type=int, default=256, help="cfg5: instances")
    ap.add_argument("--preconditioner", default=None,
                    help="cfg3 (default jacobi, as configured) and cfg5 (default two-level): jacobi, block-jacobi "
                         "or two-level")
    ap.add_argument("--pcg-iterations", type=int, default=None, help="cfg5: CG iterations per Newton step")
    a = ap.parse_args(argv)
    if a.workload == "cfg3":
        rec = cfg3(cells=a.cells, n_steps=a.steps, precisions=tuple(a.precisions.split(",")), pcg_rtol=a.pcg_rtol,
                   nr_iterations=a.nr_iterations, preconditioner=a.preconditioner or "jacobi")
    elif a.workload == "cfg4":
        rec = cfg4(h_grid=a.grid, gravity_fraction=a.gravity, n_check=a.fd_elements, rel_step=a.fd_step)
    else:
        rec = cfg5(n=a.beams, target_tets=4.1e6 * a.beams / 256, preconditioner=a.preconditioner or "two-level",
                   pcg_iterations=a.pcg_iterations)
    print(json.dumps(rec))


if __name__ == "__main__":
    main()

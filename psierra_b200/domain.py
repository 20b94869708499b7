"""Solid domain, Dirichlet constraints and nodal loads, mirroring pSierra's API.

``SolidDomain`` keeps the state vectors and the assembly entry points of psierra
``domain/solid.py:20-325`` and delegates every assembly to its element's hooks
(``assemble_internal_forces(mesh, displacement)``, ``assemble_tangent_stiffness_matrix
(mesh, displacement)``, ``assemble_stiffness_matrix(mesh)``), exactly the delegation the
reference performs at ``solid.py:180-181, 238-241, 288-291``.  Unlike the reference it
does not pre-allocate ``(E, d, d)`` host buffers (7 GB at 3 M elements), because the GPU
elements never use them.  The reference's own ``SolidDomain`` works with the GPU
elements unchanged; this mirror exists so the drivers run where the reference is not
installed.

``DirichletConstraint``/``DirichletManager`` follow ``boundary/dirichlet.py:8-147`` and
``NodalForce`` follows ``boundary/load.py:9-43``.
"""
from __future__ import annotations

from collections.abc import Sequence

import numpy as np


class SolidDomain:
    def __init__(self, mesh, material, element) -> None:
        self.mesh = mesh
        self.material = material
        self.element = element
        self.element.material = self.material
        n = self.mesh.n_dofs
        self.u = np.zeros(n, dtype=np.float64)
        self.v = np.zeros(n, dtype=np.float64)
        self.a = np.zeros(n, dtype=np.float64)

    @property
    def n_dofs(self) -> int:
        return self.mesh.n_dofs

    @property
    def displacement(self) -> np.ndarray:
        return self.u.reshape(-1, 3)

    @property
    def velocity(self) -> np.ndarray:
        return self.v.reshape(-1, 3)

    @property
    def acceleration(self) -> np.ndarray:
        return self.a.reshape(-1, 3)

    @property
    def current_nodes(self) -> np.ndarray:
        return self.mesh.nodes + self.displacement

    def update_state(self, u=None, v=None, a=None) -> None:
        if u is not None:
            self.u[:] = u
        if v is not None:
            self.v[:] = v
        if a is not None:
            self.a[:] = a

    def reset_state(self) -> None:
        self.u.fill(0.0)
        self.v.fill(0.0)
        self.a.fill(0.0)

    def commit_state(self) -> None:
        pass

    def assemble_stiffness_matrix(self):
        return self.element.assemble_stiffness_matrix(self.mesh)

    def assemble_internal_forces(self) -> np.ndarray:
        return self.element.assemble_internal_forces(self.mesh, self.displacement)

    def assemble_internal_force_vector(self) -> np.ndarray:
        return self.assemble_internal_forces()

    def assemble_tangent_stiffness_matrix(self):
        return self.element.assemble_tangent_stiffness_matrix(self.mesh, self.displacement)

    def assemble_mass_matrix(self):
        """Consistent mass (psierra ``solid.py:209-228``) through the element's hook."""
        return self.element.assemble_mass_matrix(self.mesh)


class DirichletConstraint:
    """Prescribed displacement on nodes (psierra ``boundary/dirichlet.py:8-66``)."""

    def __init__(self, node_indices, components: Sequence[int] = (0, 1, 2), value=0.0, dofs_per_node: int = 3,
                 dof_offset: int = 0) -> None:
        self.node_indices = np.asarray(node_indices, dtype=np.int64)
        self.components = tuple(components)
        self.dofs_per_node = dofs_per_node
        self.dof_offset = int(dof_offset)
        dofs = [self.dof_offset + self.node_indices * dofs_per_node + c for c in self.components]
        self.dofs = np.sort(np.concatenate(dofs)) if dofs else np.array([], dtype=np.int64)
        if np.isscalar(value):
            self.values = np.full(len(self.dofs), float(value))
        else:
            self.values = np.asarray(value, dtype=np.float64)
            if len(self.values) != len(self.dofs):
                raise ValueError(
                    f"Length of values ({len(self.values)}) does not match number of constrained DOFs ({len(self.dofs)}).")


class DirichletManager:
    """Partition of DOFs into free and prescribed (psierra ``boundary/dirichlet.py:89-147``)."""

    def __init__(self, total_dofs: int) -> None:
        self.total_dofs = total_dofs
        self._constraints: list = []

    def add_constraint(self, constraint) -> None:
        self._constraints.append(constraint)

    def remove_constraint(self, constraint) -> None:
        self._constraints.remove(constraint)

    def clear(self) -> None:
        self._constraints.clear()

    @property
    def prescribed_dofs(self) -> np.ndarray:
        if not self._constraints:
            return np.array([], dtype=np.int64)
        return np.unique(np.concatenate([c.dofs for c in self._constraints]))

    @property
    def free_dofs(self) -> np.ndarray:
        p = self.prescribed_dofs
        if len(p) == 0:
            return np.arange(self.total_dofs, dtype=np.int64)
        mask = np.ones(self.total_dofs, dtype=bool)
        mask[p] = False
        return np.where(mask)[0]

    @property
    def prescribed_values(self) -> np.ndarray:
        p = self.prescribed_dofs
        values = np.zeros(len(p), dtype=np.float64)
        for c in self._constraints:
            values[np.searchsorted(p, c.dofs)] = c.values
        return values


class NodalForce:
    """Equal force on each selected node (psierra ``boundary/load.py:9-43``)."""

    def __init__(self, node_indices, force_vector, dofs_per_node: int = 3) -> None:
        self.node_indices = np.asarray(node_indices, dtype=np.int64)
        self.force_vector = np.asarray(force_vector, dtype=np.float64)
        self.dofs_per_node = dofs_per_node
        if self.force_vector.shape != (dofs_per_node,):
            raise ValueError(f"force_vector must have shape ({dofs_per_node},), got {self.force_vector.shape}")

    def compute_force_vector(self, total_dofs: int) -> np.ndarray:
        f = np.zeros(total_dofs, dtype=np.float64)
        for node in self.node_indices:
            f[node * self.dofs_per_node:(node + 1) * self.dofs_per_node] += self.force_vector
        return f

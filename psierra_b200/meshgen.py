"""Structured tetrahedral mesh generators and seeded displacement fields.

These build the synthetic inputs the path is exercised on (the reference ships no
mesh files for it).  Everything here is plain numpy on the host and runs once per
mesh; nothing in this module is on the per-iteration hot path.

* ``box_tet4``: an ``nx x ny x nz`` grid of hexahedral cells, each split into six
  tetrahedra that share the cell's main diagonal (Kuhn split).  Node ids follow
  ``(i * (ny + 1) + j) * (nz + 1) + k``; cell vertices follow the usual hexahedron
  order ``v0=(0,0,0) v1=(1,0,0) v2=(1,1,0) v3=(0,1,0) v4=(0,0,1) v5=(1,0,1)
  v6=(1,1,1) v7=(0,1,1)``; a tetrahedron whose signed volume comes out negative has
  its local nodes 1 and 2 swapped so that every element has positive volume.
* ``tet4_to_tet10``: quadratic upgrade with VTK mid-edge ordering
  (4:(0,1) 5:(1,2) 6:(2,0) 7:(0,3) 8:(1,3) 9:(2,3)); unique edges are numbered in
  lexicographic (min, max) order after the corner nodes, which is the numbering of
  ``compute_tet10_connectivity_and_points`` (psierra ``mesher/order.py:11-81``),
  so the Tet10 sparsity pattern is the reference's.
* ``ellipsoid_tet4``: the box generator clipped to an ellipsoid, keeping the
  tetrahedra whose four corners all lie inside, with unused nodes dropped.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

# Six tetrahedra of a hexahedral cell sharing the diagonal v0 -> v6.
_KUHN_TETS = np.array(
    [[0, 1, 2, 6], [0, 1, 5, 6], [0, 3, 2, 6], [0, 3, 7, 6], [0, 4, 5, 6], [0, 4, 7, 6]],
    dtype=np.int64,
)
_HEX_OFFSETS = np.array(
    [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]],
    dtype=np.int64,
)


@dataclass
class TetMesh:
    """Host-side mesh with the attributes pSierra's ``SolidDomain`` reads.

    ``nodes`` is ``(N, 3)`` float64 and ``elements`` is ``(E, 4)`` or ``(E, 10)``
    int64, exactly the layout of ``VolumetricMesh.nodes`` / ``.elements``
    (psierra ``mesh/volumetric.py:97-124``).
    """

    nodes: np.ndarray
    elements: np.ndarray

    @property
    def n_nodes(self) -> int:
        return int(self.nodes.shape[0])

    @property
    def n_elements(self) -> int:
        return int(self.elements.shape[0])

    @property
    def n_dofs(self) -> int:
        return 3 * self.n_nodes

    @property
    def volumes(self) -> np.ndarray:
        """Reference volume of each element from its four corner nodes."""
        X = self.nodes[self.elements[:, :4]]
        d = X[:, 1:4] - X[:, 0:1]
        return np.abs(np.linalg.det(d)) / 6.0

    def copy(self) -> "TetMesh":
        return TetMesh(self.nodes.copy(), self.elements.copy())


def box_tet4(lx: float, ly: float, lz: float, nx: int, ny: int, nz: int,
             origin=(0.0, 0.0, 0.0)) -> TetMesh:
    """Kuhn-split box ``[0,lx]x[0,ly]x[0,lz]`` (shifted by ``origin``)."""
    xs = origin[0] + np.linspace(0.0, lx, nx + 1)
    ys = origin[1] + np.linspace(0.0, ly, ny + 1)
    zs = origin[2] + np.linspace(0.0, lz, nz + 1)
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    nodes = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)

    ci, cj, ck = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    cells = np.stack([ci.ravel(), cj.ravel(), ck.ravel()], axis=1)  # (C, 3)
    verts = cells[:, None, :] + _HEX_OFFSETS[None, :, :]  # (C, 8, 3)
    vid = (verts[..., 0] * (ny + 1) + verts[..., 1]) * (nz + 1) + verts[..., 2]  # (C, 8)
    tets = vid[:, _KUHN_TETS].reshape(-1, 4)  # (6C, 4), cell-major
    tets = _orient_positive(nodes, tets)
    return TetMesh(nodes, tets)


def _orient_positive(nodes: np.ndarray, tets: np.ndarray) -> np.ndarray:
    X = nodes[tets]
    d = X[:, 1:4] - X[:, 0:1]
    vol = np.linalg.det(d)
    neg = vol < 0.0
    tets = tets.copy()
    tets[neg, 1], tets[neg, 2] = tets[neg, 2].copy(), tets[neg, 1].copy()
    return tets


def tet4_to_tet10(mesh: TetMesh) -> TetMesh:
    """Quadratic upgrade with reference-identical mid-edge numbering."""
    c4 = np.asarray(mesh.elements, dtype=np.int64)
    n = mesh.n_nodes
    pairs = np.array([[0, 1], [1, 2], [2, 0], [0, 3], [1, 3], [2, 3]], dtype=np.int64)
    ends = c4[:, pairs]  # (E, 6, 2)
    lo = ends.min(axis=2)
    hi = ends.max(axis=2)
    key = (lo * n + hi).ravel()
    uniq, inv = np.unique(key, return_inverse=True)
    ulo, uhi = uniq // n, uniq % n
    mid = 0.5 * (mesh.nodes[ulo] + mesh.nodes[uhi])
    c10 = np.hstack([c4, n + inv.reshape(-1, 6)])
    return TetMesh(np.vstack([mesh.nodes, mid]), c10)


def ellipsoid_tet4(ax: float, ay: float, az: float, h: float) -> TetMesh:
    """Kuhn grid of spacing ``h`` clipped to ``x^2/ax^2 + y^2/ay^2 + z^2/az^2 <= 1``."""
    nx, ny, nz = (int(np.ceil(2 * a / h)) for a in (ax, ay, az))
    box = box_tet4(nx * h, ny * h, nz * h, nx, ny, nz,
                   origin=(-0.5 * nx * h, -0.5 * ny * h, -0.5 * nz * h))
    P = box.nodes
    inside = (P[:, 0] / ax) ** 2 + (P[:, 1] / ay) ** 2 + (P[:, 2] / az) ** 2 <= 1.0
    keep = inside[box.elements].all(axis=1)
    tets = box.elements[keep]
    used = np.unique(tets)
    remap = -np.ones(box.n_nodes, dtype=np.int64)
    remap[used] = np.arange(used.size)
    return TetMesh(P[used].copy(), remap[tets])


# ---------------------------------------------------------------------------
# Seeded displacement fields
# ---------------------------------------------------------------------------

def cantilever_seeded_u(mesh: TetMesh, seed: int = 1234) -> np.ndarray:
    """``u = 0.02 x^2 e_z + N(0, 1e-5)`` on every component, shape ``(N, 3)``."""
    rng = np.random.default_rng(seed)
    u = rng.normal(0.0, 1e-5, size=(mesh.n_nodes, 3))
    u[:, 2] += 0.02 * mesh.nodes[:, 0] ** 2
    return u


def cube_smooth_u(mesh: TetMesh, seed: int = 2024) -> np.ndarray:
    """``u = 0.05 sin(pi x) sin(pi y) z e_z + U(-1e-4, 1e-4)``, shape ``(N, 3)``."""
    rng = np.random.default_rng(seed)
    u = rng.uniform(-1e-4, 1e-4, size=(mesh.n_nodes, 3))
    x, y, z = mesh.nodes[:, 0], mesh.nodes[:, 1], mesh.nodes[:, 2]
    u[:, 2] += 0.05 * np.sin(np.pi * x) * np.sin(np.pi * y) * z
    return u


def lame_from_young_poisson(E: float, nu: float) -> tuple[float, float, float]:
    """``(mu, lambda, kappa)`` from Young's modulus and Poisson's ratio.

    Same closed forms as ``IsotropicElasticParameters.set_from_youngs_poisson``
    (psierra ``material/parameters.py:68-70``).
    """
    mu = E / (2.0 * (1.0 + nu))
    lam = (E * nu) / ((1.0 + nu) * (1.0 - 2.0 * nu))
    kappa = E / (3.0 * (1.0 - 2.0 * nu))
    return mu, lam, kappa


def boundary_face_triangles(mesh: TetMesh, axis: int, bound: str, tol: float = 1e-9) -> np.ndarray:
    """Corner-node triangles of the element faces lying on an extremal plane.

    Returns ``(T, 3)`` node ids.  A face belongs to the plane when all three of its
    corners lie within ``tol`` of the plane's coordinate.
    """
    el = np.asarray(mesh.elements[:, :4], dtype=np.int64)
    c = mesh.nodes[:, axis]
    target = c.min() if bound == "min" else c.max()
    on = np.abs(c - target) <= tol
    faces = el[:, [[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]]].reshape(-1, 3)
    return faces[on[faces].all(axis=1)]


def traction_nodal_forces(mesh: TetMesh, axis: int, bound: str, traction) -> np.ndarray:
    """Consistent nodal forces of a uniform traction on a flat boundary face.

    Each face triangle gives ``traction * area / 3`` to each of its corners (exact
    for linear triangles).  Returns the global force vector of length ``n_dofs``.
    """
    tri = boundary_face_triangles(mesh, axis, bound)
    P = mesh.nodes[tri]
    area = 0.5 * np.linalg.norm(np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0]), axis=1)
    f = np.zeros((mesh.n_nodes, 3))
    t = np.asarray(traction, dtype=np.float64)
    np.add.at(f, tri.ravel(), np.repeat(area / 3.0, 3)[:, None] * t[None, :])
    return f.ravel()


def nodes_on_plane(mesh: TetMesh, axis: int, bound: str, tol: float = 1e-4) -> np.ndarray:
    """Nodes on an extremal plane, the selection rule of ``select_nodes_by_plane``
    (psierra ``boundary/selector.py:8-40``)."""
    c = mesh.nodes[:, axis]
    target = c.min() if bound == "min" else c.max()
    return np.where(np.abs(c - target) <= tol)[0].astype(np.int64)


# ---------------------------------------------------------------------------
# Batches of meshes
# ---------------------------------------------------------------------------

def concat_meshes(meshes) -> tuple[TetMesh, np.ndarray, np.ndarray]:
    """Disjoint union of meshes: ``(union, node_offsets, element_offsets)`` (offsets B+1).

    Instance ``i`` owns nodes ``node_offsets[i]:node_offsets[i+1]`` and elements
    ``element_offsets[i]:element_offsets[i+1]`` of the union, in its own order.
    """
    nn = np.array([m.n_nodes for m in meshes], dtype=np.int64)
    ne = np.array([m.n_elements for m in meshes], dtype=np.int64)
    node_off = np.concatenate([[0], np.cumsum(nn)])
    elem_off = np.concatenate([[0], np.cumsum(ne)])
    nodes = np.concatenate([np.asarray(m.nodes, dtype=np.float64) for m in meshes])
    elements = np.concatenate([np.asarray(m.elements, dtype=np.int64) + node_off[i] for i, m in enumerate(meshes)])
    return TetMesh(nodes, elements), node_off, elem_off


@dataclass
class BeamCase:
    mesh: TetMesh
    length: float
    youngs: float
    poisson: float
    traction: np.ndarray  # (3,) Pa on the x = length face
    cells: tuple


def beam_batch(n: int = 256, target_tets: float = 4.1e6, seed: int = 5, section: float = 0.1) -> list[BeamCase]:
    """Seeded batch of clamped cantilever beams of uneven size.

    Length L ~ U[0.5, 2], square section ``section`` x ``section``; cell counts follow
    one seeded size variable s ~ U[0, 1] per beam, (nx, ny, nz) = (8 + 112 s^p,
    2 + 8 s^p, 2 + 8 s^p) rounded, with the exponent p chosen so that the batch holds
    about ``target_tets`` tetrahedra (6 per cell) within the [8x2x2, 120x10x10] range.
    E ~ U[1e3, 1e6] Pa, nu ~ U[0.3, 0.49], traction magnitude |t| ~ U[10, 1000] Pa on
    the tip face: |t| along +x (tension) plus a transverse -z part of min(|t|/2,
    E / (1600 L^2)), which keeps the linear tip-deflection estimate 400 t_z L^2 / E of
    a 0.1 m section at or below L / 4 (a purely transverse |t| would bend many of
    these beams by several times their length).
    """
    rng = np.random.default_rng(seed)
    L = rng.uniform(0.5, 2.0, n)
    s = rng.uniform(0.0, 1.0, n)
    E = rng.uniform(1e3, 1e6, n)
    nu = rng.uniform(0.3, 0.49, n)
    tmag = rng.uniform(10.0, 1000.0, n)

    def cells_for(p):
        sp = s ** p
        nx = np.rint(8 + 112 * sp).astype(np.int64)
        ny = np.rint(2 + 8 * sp).astype(np.int64)
        return nx, ny

    lo, hi = 0.05, 20.0  # total tets decreases as p grows
    for _ in range(60):
        p = np.sqrt(lo * hi)
        nx, ny = cells_for(p)
        tot = float(np.sum(6 * nx * ny * ny))
        if tot > target_tets:
            lo = p
        else:
            hi = p
    nx, ny = cells_for(np.sqrt(lo * hi))
    out = []
    for i in range(n):
        m = box_tet4(float(L[i]), section, section, int(nx[i]), int(ny[i]), int(ny[i]))
        tz = min(0.5 * tmag[i], E[i] / (1600.0 * L[i] ** 2))
        out.append(BeamCase(m, float(L[i]), float(E[i]), float(nu[i]), np.array([tmag[i], 0.0, -tz]),
                            (int(nx[i]), int(ny[i]), int(ny[i]))))
    return out

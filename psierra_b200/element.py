"""Drop-in GPU elements for pSierra's ``SolidDomain`` (Tet4 / Tet10 Total Lagrangian).

``SolidDomain`` delegates to its element when the element defines
``assemble_internal_forces(mesh, displacement)``, ``assemble_tangent_stiffness_matrix
(mesh, displacement)``, ``assemble_stiffness_matrix(mesh)`` or ``prepare_for_assembly``
(psierra ``domain/solid.py:180-181, 238-244, 288-294``; the same hooks ``Tet4Fbar``
uses, ``element/tet4_fbar.py:217-459``).  The classes here implement those hooks on
the GPU, so the reference's unchanged ``SolidDomain``, ``NonlinearStaticAnalysis``,
``DynamicRelaxationAnalysis`` and ``NonlinearDynamicAnalysis`` run on them as they are,
and so does the mirror domain and drivers of this package.

Return values follow the reference: a fresh ``(3N,)`` float64 numpy array for the
internal forces and a canonical ``scipy.sparse.csr_matrix`` (sorted indices, int32
index arrays identical to ``coo_matrix(...).tocsr()``) for the matrices.  In
``precision="fp32-mixed"`` the tangent values are computed and stored in FP32 on
the device and widened to float64 on the way out; f_int stays FP64.
"""
from __future__ import annotations

import weakref

import numpy as np
import scipy.sparse as spsp
import torch

from psierra_b200.assembler import GPUAssembler


class DeviceCSR:
    """A square CSR matrix whose arrays stay on the GPU: ``indptr`` and ``indices`` (int32,
    the canonical pattern of ``coo_matrix(...).tocsr()``, shared by every call on the same
    mesh) and ``data`` (this call's values: float64, or float32 for the FP32-mixed
    tangent).  ``to_scipy()`` gives the float64 host matrix the parity-mode hooks return."""

    def __init__(self, indptr: torch.Tensor, indices: torch.Tensor, data: torch.Tensor, shape) -> None:
        self.indptr, self.indices, self.data, self.shape = indptr, indices, data, tuple(shape)

    @property
    def nnz(self) -> int:
        return int(self.data.numel())

    def to_scipy(self) -> spsp.csr_matrix:
        A = spsp.csr_matrix((self.data.double().cpu().numpy(), self.indices.cpu().numpy(),
                             self.indptr.cpu().numpy()), shape=self.shape, copy=False)
        A.has_sorted_indices = True
        A.has_canonical_format = True
        return A


class _HostStaging:
    """Pinned host buffers for the per-call copies of u (in) and f / K values (out)."""

    def __init__(self):
        self._bufs: dict[tuple, torch.Tensor] = {}

    def get(self, key: str, n: int, dtype) -> torch.Tensor:
        k = (key, dtype)
        b = self._bufs.get(k)
        if b is None or b.numel() < n:
            b = torch.empty(n, dtype=dtype, pin_memory=True)
            self._bufs[k] = b
        return b[:n]


class _ResultPool:
    """Pinned float64 buffers handed out as the backing store of returned arrays.

    A device result is copied straight into a free pinned buffer and returned as a numpy
    view of it; a finalizer on that array returns the buffer to the pool once the caller
    holds no reference to it any more.  Every call therefore still returns a fresh array
    that no other live result aliases (the reference's semantics), without a host-side
    copy.  Past ``cap_bytes`` of buffers in use, results fall back to freshly allocated
    (pageable) arrays.
    """

    def __init__(self, cap_bytes: int = 8 << 30):
        self.cap = cap_bytes
        self.free: list[torch.Tensor] = []
        self.in_use_bytes = 0

    def _release(self, buf: torch.Tensor) -> None:
        self.in_use_bytes -= buf.numel() * 8
        self.free.append(buf)

    def take(self, dev: torch.Tensor) -> np.ndarray:
        n = dev.numel()
        buf = None
        for i, b in enumerate(self.free):
            if b.numel() == n:
                buf = self.free.pop(i)
                break
        if buf is None:
            if self.in_use_bytes + 8 * n > self.cap:
                out = torch.empty(n, dtype=torch.float64)
                out.copy_(dev)
                return out.numpy()
            buf = torch.empty(n, dtype=torch.float64, pin_memory=True)
        self.in_use_bytes += 8 * n
        buf.copy_(dev, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        arr = buf.numpy()
        weakref.finalize(arr, self._release, buf)
        return arr


class _GPUElementBase:
    """Common host <-> device plumbing of the drop-in element classes."""

    supports_element_indexing: bool = True
    _npe = 4

    def __init__(self, material, precision: str = "fp64", device=None) -> None:
        self._material = material
        self.precision = precision
        self.device = device
        self._mesh = None
        self._asm: GPUAssembler | None = None
        self._staging = _HostStaging()
        self._results = _ResultPool()
        self._widen: torch.Tensor | None = None
        self._u_dev: torch.Tensor | None = None
        self._last_u: np.ndarray | None = None
        self._last_f: torch.Tensor | None = None

    # ---------------------------------------------------------------- interface
    @property
    def material(self):
        return self._material

    @material.setter
    def material(self, mat) -> None:
        self._material = mat
        if self._asm is not None:
            self._asm.set_material(mat)
        self.__dict__.pop("_one", None)  # the cached one-element assembler holds the old material
        self._last_u = None

    @property
    def nodes_per_element(self) -> int:
        return self._npe

    @property
    def dofs_per_node(self) -> int:
        return 3

    @property
    def dofs_per_element(self) -> int:
        return 3 * self._npe

    # ---------------------------------------------------------------- setup
    def _make_assembler(self, mesh) -> GPUAssembler:
        return GPUAssembler(mesh.nodes, mesh.elements, self._material, precision=self.precision,
                            device=self.device)

    def _setup(self, mesh) -> GPUAssembler:
        if self._mesh is not mesh or self._asm is None:
            elements = np.asarray(mesh.elements)
            if elements.ndim != 2 or elements.shape[1] != self._npe:
                raise ValueError(f"{type(self).__name__} needs (E, {self._npe}) elements, got {elements.shape}")
            self._asm = self._make_assembler(mesh)
            self._mesh = mesh
            self._u_dev = torch.empty(3 * self._asm.n_nodes, dtype=torch.float64, device=self._asm.device)
            self._last_u = None
        return self._asm

    def prepare_for_assembly(self, mesh, displacement=None) -> None:
        """Build (once per mesh) the device mesh, node graph and CSR pattern."""
        self._setup(mesh)

    def prepare_for_linear_assembly(self, mesh) -> None:
        self._setup(mesh)

    def _upload_u(self, displacement) -> torch.Tensor:
        u = np.ascontiguousarray(displacement, dtype=np.float64).reshape(-1)
        if u.size != self._u_dev.numel():
            raise ValueError(f"displacement has {u.size} entries, expected {self._u_dev.numel()}")
        pin = self._staging.get("u", u.size, torch.float64)
        # torch's copy runs on all host threads (12.8 MB of the 80^3 cube: 0.3 ms instead
        # of the 1.6 ms of a numpy assignment); a read-only array takes the numpy route
        if u.flags.writeable:
            pin.copy_(torch.from_numpy(u))
        else:
            pin.numpy()[:] = u
        self._u_dev.copy_(pin, non_blocking=True)
        return self._u_dev

    def _download(self, t: torch.Tensor, key: str) -> np.ndarray:
        """Device tensor -> a fresh float64 numpy array (the reference returns new arrays).

        The device-to-host copy lands in a reused pinned buffer; the copy out of it (with
        the FP32 -> FP64 widening of mixed-precision K values) runs on all host threads.
        """
        pin = self._staging.get(key, t.numel(), t.dtype)
        pin.copy_(t, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        out = torch.empty(t.numel(), dtype=torch.float64)
        out.copy_(pin)
        return out.numpy()

    def _download_k(self, kvals: torch.Tensor) -> np.ndarray:
        """CSR values -> a fresh float64 host array: FP32 values are widened on the device,
        then copied once into a pooled pinned buffer (``_ResultPool``)."""
        if kvals.dtype != torch.float64:
            if self._widen is None or self._widen.numel() != kvals.numel():
                self._widen = torch.empty(kvals.numel(), dtype=torch.float64, device=kvals.device)
            self._widen.copy_(kvals)
            kvals = self._widen
        return self._results.take(kvals)

    def _csr(self, kvals: torch.Tensor) -> spsp.csr_matrix:
        p = self._asm.pattern
        data = self._download_k(kvals)
        n = p.n_dofs
        A = spsp.csr_matrix((data, p.indices, p.indptr), shape=(n, n), copy=False)
        A.has_sorted_indices = True
        A.has_canonical_format = True
        return A

    # ---------------------------------------------------------------- domain hooks
    def assemble_internal_forces(self, mesh, displacement) -> np.ndarray:
        """f_int(u) as a fresh ``(3N,)`` array (psierra ``domain/solid.py:230-274``)."""
        asm = self._setup(mesh)
        u = self._upload_u(displacement)
        f, _ = asm.assemble(u, want_f=True, want_k=False)
        return self._results.take(f)

    def assemble_tangent_stiffness_matrix(self, mesh, displacement) -> spsp.csr_matrix:
        """K_T(u) as a canonical CSR matrix (psierra ``domain/solid.py:280-325``)."""
        asm = self._setup(mesh)
        u = self._upload_u(displacement)
        _, k = asm.assemble(u, want_f=False, want_k=True)
        return self._csr(k)

    def assemble_stiffness_matrix(self, mesh) -> spsp.csr_matrix:
        """Small-strain K of the reference configuration (psierra ``domain/solid.py:172-207``)."""
        asm = self._setup(mesh)
        _, k = asm.assemble(None, linear=True)
        return self._csr(k)

    def assemble_mass_matrix(self, mesh) -> spsp.csr_matrix:
        """Consistent mass matrix (psierra ``domain/solid.py:209-228`` with ``compute_mass_matrix``)."""
        asm = self._setup(mesh)
        _, k = asm.assemble(None, mass=True)
        return self._csr(k)

    def assemble_force_and_tangent(self, mesh, displacement) -> tuple[np.ndarray, spsp.csr_matrix]:
        """Both outputs from one fused element sweep."""
        asm = self._setup(mesh)
        u = self._upload_u(displacement)
        f, k = asm.assemble(u, want_f=True, want_k=True)
        return self._results.take(f), self._csr(k)

    def assemble_force_and_tangent_device(self, mesh, displacement) -> tuple[torch.Tensor, DeviceCSR]:
        """Throughput form of ``assemble_force_and_tangent``: f_int as a fresh float64
        device tensor and K_T as a ``DeviceCSR`` over fresh device values, with nothing
        copied back to the host.  ``displacement`` is a host array (uploaded) or a
        float64 tensor on the assembler's device (used as it is)."""
        asm = self._setup(mesh)
        if isinstance(displacement, torch.Tensor):
            u = displacement.reshape(-1)
        else:
            u = self._upload_u(displacement)
        f, k = asm.assemble(u, want_f=True, want_k=True)
        n = 3 * asm.n_nodes
        return f, DeviceCSR(asm.dev["indptr"], asm.dev["indices"], k, (n, n))

    # ---------------------------------------------------------------- per-element API
    def compute_nonlinear_force_and_tangent_stiffness(self, node_coords, u_nodes, elem_index=None, **kw):
        """(k_tan, f_int) of one element (psierra ``element/tet4_total_lagrangian.py:77-139``).

        Runs the same GPU kernel on a one-element mesh; it exists for API
        compatibility (reference code that loops over elements, such as the ECSW model or
        a per-element mass loop, calls it once per element), while the domain hooks above
        are the throughput path.  The one-element mesh, its pattern, plan and workspace are
        built on the first call and reused: a later call only uploads the element's
        coordinates, displacements and, with per-element moduli, its mu and kappa.
        """
        one, mesh = self._single_element(node_coords, elem_index)
        f, K = one.assemble_force_and_tangent(mesh, np.asarray(u_nodes, dtype=np.float64).reshape(self._npe, 3))
        return K.toarray(), f

    def _single_element(self, node_coords, elem_index):
        """(element, mesh) of the cached one-element assembler, set to this element."""
        from psierra_b200.material import _host
        from psierra_b200.meshgen import TetMesh

        X = np.asarray(node_coords, dtype=np.float64).reshape(self._npe, 3)
        from psierra_b200.material import NeoHookeanField

        mat = self._material
        one_mat = mat
        if getattr(mat, "mu_e", None) is not None:
            if elem_index is None:
                raise ValueError("per-element moduli need elem_index")
            pick = lambda a: np.asarray(_host(a), dtype=np.float64)[[elem_index]]  # noqa: E731
            lam = getattr(mat, "lam_e", None)
            one_mat = NeoHookeanField(pick(mat.mu_e), pick(mat.kappa_e), mass_density=mat.mass_density,
                                      lam_e=None if lam is None else pick(lam))
        cached = self.__dict__.get("_one")
        if cached is None:
            mesh = TetMesh(X.copy(), np.arange(self._npe, dtype=np.int64)[None, :])
            one = type(self)(one_mat, precision=self.precision, device=self.device)
            one._setup(mesh)
            cached = self._one = (one, mesh)
        one, mesh = cached
        asm = one._setup(mesh)
        mesh.nodes[:] = X
        asm.X.copy_(torch.from_numpy(X))
        if one_mat is not mat:
            asm.set_material(one_mat)
        return one, mesh

    def compute_linear_stiffness_matrix(self, node_coords, elem_index=None, **kw):
        """Small-strain k_e of one element (psierra ``element/tet4_base.py:129-136``), on the
        cached one-element assembler."""
        one, mesh = self._single_element(node_coords, elem_index)
        return one.assemble_stiffness_matrix(mesh).toarray()


class Tet4TotalLagrangian(_GPUElementBase):
    """GPU Tet4 Total-Lagrangian element (psierra ``element/tet4_total_lagrangian.py``)."""

    _npe = 4

    def compute_mass_matrix(self, volume: float) -> np.ndarray:
        """Consistent 12x12 element mass (psierra ``element/tet4_base.py:138-151``)."""
        rho = self._material.mass_density
        m = np.kron(np.ones((4, 4)) + np.identity(4), np.identity(3))
        return (rho * volume / 20.0) * m


# Exact reference mass matrix of the 10-node tetrahedron (entries / 2520), VTK ordering;
# the consistent mass of psierra element/tet10_base.py:12-27, 344-372.
_TET10_MASS_INT = np.array([
    [36, 6, 6, 6, -24, -36, -24, -24, -36, -36],
    [6, 36, 6, 6, -24, -24, -36, -36, -24, -36],
    [6, 6, 36, 6, -36, -24, -24, -36, -36, -24],
    [6, 6, 6, 36, -36, -36, -36, -24, -24, -24],
    [-24, -24, -36, -36, 192, 96, 96, 96, 96, 48],
    [-36, -24, -24, -36, 96, 192, 96, 48, 96, 96],
    [-24, -36, -24, -36, 96, 96, 192, 96, 48, 96],
    [-24, -36, -36, -24, 96, 48, 96, 192, 96, 96],
    [-36, -24, -36, -24, 96, 96, 48, 96, 192, 96],
    [-36, -36, -24, -24, 48, 96, 96, 96, 96, 192]], dtype=np.float64)


class Tet10TotalLagrangian(_GPUElementBase):
    """GPU Tet10 Total-Lagrangian element, 4-point rule (psierra ``element/tet10_total_lagrangian.py``)."""

    _npe = 10

    def __init__(self, material, default_quadrature_order: int = 4, precision: str = "fp64", device=None) -> None:
        if default_quadrature_order != 4:
            raise ValueError("the GPU Tet10 element integrates with the 4-point rule")
        super().__init__(material, precision=precision, device=device)
        self.default_quadrature_order = 4

    def compute_mass_matrix(self, volume: float) -> np.ndarray:
        rho = self._material.mass_density
        return np.kron(_TET10_MASS_INT / 2520.0 * rho * volume, np.identity(3))



class Tet4Fbar(_GPUElementBase):
    """GPU Tet4 F-bar element (psierra ``element/tet4_fbar.py``): nodal volume-averaged
    ``J_bar``, deviatoric element tangent and nodal volumetric blocks on the two-ring
    pattern (``psierra_b200.fbar``).  Same domain hooks and return types as the reference
    class; the tangent's CSR pattern is the reference's (scipy's ``K_dev + K_vol``, exact
    zeros dropped)."""

    _npe = 4

    def __init__(self, material, device=None) -> None:
        super().__init__(material, precision="fp64", device=device)
        self._fbar = None
        self._domain_J_bar: np.ndarray | None = None

    def _make_assembler(self, mesh):
        from psierra_b200.fbar import FbarAssembler

        self._fbar = FbarAssembler(mesh.nodes, mesh.elements, self._material, device=self.device)
        return self._fbar

    @property
    def material(self):
        return self._material

    @material.setter
    def material(self, mat) -> None:
        self._material = mat
        self._mesh = None  # moduli are baked into the assembler
        self._asm = None

    def _setup(self, mesh):
        if self._mesh is not mesh or self._asm is None:
            elements = np.asarray(mesh.elements)
            if elements.ndim != 2 or elements.shape[1] != 4:
                raise ValueError(f"Tet4Fbar needs (E, 4) elements, got {elements.shape}")
            self._asm = self._make_assembler(mesh)
            self._mesh = mesh
            self._u_dev = torch.empty(3 * self._asm.n_nodes, dtype=torch.float64, device=self._asm.device)
        return self._asm

    def _record_jbar(self) -> None:
        self._domain_J_bar = self._fbar.jbar.cpu().numpy().copy()

    def prepare_for_assembly(self, mesh, displacement=None) -> None:
        """Mesh setup and the nodal-averaged J_bar (psierra ``tet4_fbar.py:213-243``)."""
        asm = self._setup(mesh)
        if displacement is not None:
            asm.assemble(self._upload_u(displacement), want_f=True, want_k=False)
            self._record_jbar()

    def assemble_internal_forces(self, mesh, displacement) -> np.ndarray:
        asm = self._setup(mesh)
        f, _ = asm.assemble(self._upload_u(displacement), want_f=True, want_k=False)
        self._record_jbar()
        return self._download(f, "f")

    def assemble_tangent_stiffness_matrix(self, mesh, displacement) -> spsp.csr_matrix:
        asm = self._setup(mesh)
        _, k = asm.assemble(self._upload_u(displacement), want_f=False, want_k=True)
        self._record_jbar()
        return asm.csr(k)

    def assemble_force_and_tangent(self, mesh, displacement):
        asm = self._setup(mesh)
        f, k = asm.assemble(self._upload_u(displacement), want_f=True, want_k=True)
        self._record_jbar()
        return self._download(f, "f"), asm.csr(k)

    def assemble_force_and_tangent_device(self, mesh, displacement):
        """Not offered: the reference's Tet4Fbar tangent is scipy's ``K_dev + K_vol``,
        whose pattern drops the entries that sum to exactly zero, so it depends on the
        values; this element returns it on the host only (``assemble_force_and_tangent``)."""
        raise NotImplementedError("Tet4Fbar returns its value-dependent CSR pattern on the host only")

    def assemble_stiffness_matrix(self, mesh) -> spsp.csr_matrix:
        """The tangent at zero displacement (psierra ``tet4_fbar.py:241-246``)."""
        asm = self._setup(mesh)
        return self.assemble_tangent_stiffness_matrix(mesh, np.zeros((asm.n_nodes, 3)))

    def assemble_mass_matrix(self, mesh) -> spsp.csr_matrix:
        return Tet4TotalLagrangian(self._material, device=self.device).assemble_mass_matrix(mesh)

    def compute_mass_matrix(self, volume: float) -> np.ndarray:
        return Tet4TotalLagrangian(self._material, device=self.device).compute_mass_matrix(volume)

    def compute_linear_stiffness_matrix(self, node_coords, elem_index=None, **kw):
        return Tet4TotalLagrangian(self._material, device=self.device).compute_linear_stiffness_matrix(node_coords)

    def compute_nonlinear_force_and_tangent_stiffness(self, node_coords, u_nodes, elem_index=None, J_bar=None, **kw):
        """(k_tan 12x12, f_int 12) of one element (psierra ``tet4_fbar.py:147-211``)."""
        from psierra_b200.fbar import FbarAssembler

        X = np.asarray(node_coords, dtype=np.float64).reshape(4, 3)
        un = np.asarray(u_nodes, dtype=np.float64).reshape(4, 3)
        if J_bar is None:
            if elem_index is not None and self._domain_J_bar is not None:
                J_bar = float(self._domain_J_bar[elem_index])
            else:
                A = np.ones((4, 4))
                A[:, 1:] = X
                H = np.linalg.inv(A)[1:, :].T
                J_bar = float(np.linalg.det(np.eye(3) + un.T @ H))
        one = FbarAssembler(X, np.arange(4, dtype=np.int64)[None, :], self._material, device=self.device)
        k, f = one.element_matrices(X[None], un[None], np.array([J_bar]))
        return k[0], f[0]

"""Device-resident assembler: mesh, pattern and material on the GPU; one call per sweep.

``GPUAssembler`` owns the device copies of a mesh (coordinates, connectivity, node
graph, CSR pattern) and of its material, and launches the element kernels of
``libpsierra_b200.so`` on the current torch stream.  Inputs and outputs are torch
tensors on the device; the drop-in element classes in ``psierra_b200.element`` add
the host <-> device copies the reference API needs.

Error behaviour matches the reference: an element with non-positive reference
volume raises ``ValueError("Negative or zero element volume detected ...")``
(psierra ``element/tet4_base.py:56-61``) and an inverted element raises
``ValueError("Element inversion detected: det(F) = ... <= 0.")``
(``element/tet4_total_lagrangian.py:110-112``), for the lowest-index bad element,
as the reference's element loop would.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from psierra_b200 import _lib
from psierra_b200._lib import check, lib, ptr
from psierra_b200.material import material_moduli
from psierra_b200.pattern import MeshPattern

PRECISIONS = {"fp64": _lib.PSX_FP64, "fp32-mixed": _lib.PSX_FP32_MIXED}


def _stream_handle() -> int:
    return torch.cuda.current_stream().cuda_stream


WAIT_GAVE_UP = 1  # status flag bit 0: a bounded wait of a persistent kernel gave up


def raise_if_wait_gave_up(flags: int) -> None:
    """Raise when status ``flags`` say a bounded wait gave up: the kernel ran to its end,
    but records may have been read before they were written, so its outputs are invalid."""
    if int(flags) & WAIT_GAVE_UP:
        raise RuntimeError("psierra_b200: a bounded wait in the assembly kernel gave up; results are invalid")


class GPUAssembler:
    """Assembler for one Tet4 or Tet10 mesh with a NeoHookean material (constant or per element)."""

    def __init__(self, nodes: np.ndarray, elements: np.ndarray, material, precision: str = "fp64",
                 device=None, pattern: MeshPattern | None = None):
        if not torch.cuda.is_available():
            raise RuntimeError("psierra_b200 requires a CUDA device (no CPU fallback)")
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}, got {precision!r}")
        lib()  # fail loudly now if the library is missing
        self.device = torch.device(device if device is not None else "cuda")
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        self.pattern = pattern if pattern is not None else MeshPattern(elements, nodes.shape[0])
        self.npe = self.pattern.npe
        self.n_nodes = self.pattern.n_nodes
        self.n_elements = self.pattern.n_elements
        self.precision = precision
        self.dev = self.pattern.device(self.device)
        self.X = torch.from_numpy(nodes).to(self.device)
        nbytes = int(lib().psx_status_bytes())
        self.status = torch.zeros((nbytes + 3) // 4, dtype=torch.int32, device=self.device)
        self._dets = torch.zeros(8, dtype=torch.float64, device=self.device)
        self._work: dict = {}
        self.set_material(material)

    # ------------------------------------------------------------------ material
    def set_material(self, material) -> None:
        self.material = material
        mu, kappa, lam = material_moduli(material)
        self.mu, self.kappa, self.lam = mu, kappa, lam
        self.rho = float(getattr(material, "mass_density", 0.0) or 0.0)
        self.mu_e = self._per_element(getattr(material, "mu_e", None))
        self.kappa_e = self._per_element(getattr(material, "kappa_e", None))
        self._const_mats = {}  # M and K_0 of the composed effective tangent depend on the material

    def _per_element(self, a):
        if a is None:
            return None
        t = a if isinstance(a, torch.Tensor) else torch.from_numpy(np.asarray(a, dtype=np.float64))
        t = t.to(device=self.device, dtype=torch.float64).contiguous()
        if t.numel() != self.n_elements:
            raise ValueError(f"per-element modulus has {t.numel()} entries, mesh has {self.n_elements} elements")
        return t

    # ------------------------------------------------------------------ buffers
    @property
    def nnz(self) -> int:
        return self.pattern.nnz

    def k_dtype(self, precision: str | None = None):
        return torch.float64 if (precision or self.precision) == "fp64" else torch.float32

    def new_f(self) -> torch.Tensor:
        return torch.empty(3 * self.n_nodes, dtype=torch.float64, device=self.device)

    def new_k(self, precision: str | None = None) -> torch.Tensor:
        return torch.empty(self.nnz, dtype=self.k_dtype(precision), device=self.device)

    # ------------------------------------------------------------------ workspace
    def launches_per_call(self, precision: str | None = None) -> int:
        """Kernel launches one assemble() call makes (one persistent kernel)."""
        return 1

    def set_queue(self, lag: int | None = None, blocks_per_sm: int | None = None,
                  ring_slack: int | None = None, lag_f: int | None = None, split: bool | None = None) -> None:
        """Launch shape of the persistent kernel (see ``MeshPattern.set_queue``)."""
        p = self.pattern
        old = (p.lag, p.lag_f, p.ring_slack)
        p.set_queue(lag=lag, blocks_per_sm=blocks_per_sm, ring_slack=ring_slack, lag_f=lag_f, split=split)
        if (p.lag, p.lag_f, p.ring_slack) != old:
            self._work.clear()  # the record ring is sized by the lag and the slack

    def set_wait_limit(self, spins: int) -> None:
        """Polls after which a bounded wait of the persistent kernels gives up (0 = the
        default, about a second); see ``MeshPattern.set_wait_limit``."""
        self.pattern.set_wait_limit(spins)

    def workspace(self, precision: str) -> torch.Tensor:
        w = self._work.get(precision)
        if w is None:
            ring = ctypes.c_int64()
            nbytes = ctypes.c_int64()
            check(lib().psx_work_bytes(ctypes.byref(self.dev["plan"]), PRECISIONS[precision],
                                       ctypes.byref(ring), ctypes.byref(nbytes)), "psx_work_bytes")
            w = torch.empty(int(nbytes.value), dtype=torch.uint8, device=self.device)
            self._work[precision] = w
        return w

    # ------------------------------------------------------------------ kernels
    def assemble(self, u: torch.Tensor | None, want_f: bool = True, want_k: bool = True,
                 precision: str | None = None, f_out: torch.Tensor | None = None,
                 k_out: torch.Tensor | None = None, check_status: bool = True, linear: bool = False,
                 mass: bool = False):
        """One sweep over all elements.  Returns ``(f, k)``; either may be None.

        ``u`` is the ``(N, 3)`` (or ``(3N,)``) float64 displacement on the device.
        ``k`` holds the CSR values in ``pattern.indptr``/``indices`` order (float64,
        or float32 for ``precision="fp32-mixed"``).  With ``linear=True`` the
        small-strain stiffness of the reference configuration is assembled instead, and
        with ``mass=True`` the consistent mass matrix (``u`` is ignored for both).
        """
        prec = precision or self.precision
        if prec not in PRECISIONS:
            raise ValueError(f"unknown precision {prec!r}")
        if linear or mass:
            mode = _lib.PSX_MASS if mass else _lib.PSX_LINEAR
            want_f, want_k, linear = False, True, True
        else:
            mode = (_lib.PSX_WANT_F if want_f else 0) | (_lib.PSX_WANT_K if want_k else 0)
            if mode == 0:
                raise ValueError("nothing requested")
            u = self._check_u(u)
        if want_f and f_out is None:
            f_out = self.new_f()
        if want_k and k_out is None:
            k_out = self.new_k(prec)
        if want_k and k_out.dtype != self.k_dtype(prec):
            raise ValueError(f"k_out must be {self.k_dtype(prec)} for precision {prec}")
        self.status.zero_()
        work = self.workspace(prec)
        entry = lib().psx_tet4_assemble if self.npe == 4 else lib().psx_tet10_assemble
        rc = entry(
            ctypes.byref(self.dev["plan"]), ptr(self.X), ptr(u) if not linear else None,
            ptr(self.mu_e), ptr(self.kappa_e), self.mu, self.kappa, self.rho if mass else self.lam, mode,
            PRECISIONS[prec],
            ptr(f_out) if want_f else None, ptr(k_out) if want_k else None, ptr(work), work.numel(),
            ptr(self.status), _stream_handle())
        check(rc, "psx_tet4_assemble" if self.npe == 4 else "psx_tet10_assemble")
        if check_status:
            self.raise_on_bad_elements(u)
        return (f_out if want_f else None), (k_out if want_k else None)

    def assemble_effective(self, u: torch.Tensor, c_t: float, c_m: float, c_0: float = 0.0, rho: float | None = None,
                           want_f: bool = True, precision: str | None = None, f_out: torch.Tensor | None = None,
                           k_out: torch.Tensor | None = None, check_status: bool = True):
        """``(f_int(u), c_t K_T(u) + c_m M + c_0 K_0)`` from one sweep (Tet4).

        The dynamic effective tangent of ``NonlinearDynamicAnalysis``
        (psierra ``analysis/nonlinear_dynamic.py:640-644``): with generalized-alpha
        constants, ``c_t = 1 - alpha_f``, ``c_m = (1 - alpha_m) a0 + (1 - alpha_f) a1 alpha_R``
        and ``c_0 = (1 - alpha_f) a1 beta_R`` for Rayleigh damping ``alpha_R M + beta_R K_0``.
        ``M`` is the consistent mass of density ``rho`` (default: the material's) and ``K_0``
        the small-strain stiffness of the material.  Tet4 forms all three in one fused
        sweep; Tet10 assembles K_T in one sweep and adds M and K_0, assembled once on the
        same pattern and cached, with one in-place axpy over the CSR values.
        """
        if self.npe != 4:
            return self._effective_composed(u, c_t, c_m, c_0, rho, want_f, precision or self.precision, f_out, k_out,
                                            check_status)
        prec = precision or self.precision
        u = self._check_u(u)
        if want_f and f_out is None:
            f_out = self.new_f()
        if k_out is None:
            k_out = self.new_k(prec)
        if k_out.dtype != self.k_dtype(prec):
            raise ValueError(f"k_out must be {self.k_dtype(prec)} for precision {prec}")
        self.status.zero_()
        work = self.workspace(prec)
        mode = _lib.PSX_WANT_K | (_lib.PSX_WANT_F if want_f else 0)
        check(lib().psx_tet4_assemble_effective(
            ctypes.byref(self.dev["plan"]), ptr(self.X), ptr(u), ptr(self.mu_e), ptr(self.kappa_e), self.mu, self.kappa,
            self.lam, self.rho if rho is None else float(rho), float(c_t), float(c_m), float(c_0), mode, PRECISIONS[prec],
            ptr(f_out) if want_f else None, ptr(k_out), ptr(work), work.numel(), ptr(self.status), _stream_handle()),
            "psx_tet4_assemble_effective")
        if check_status:
            self.raise_on_bad_elements(u)
        return (f_out if want_f else None), k_out

    def _effective_composed(self, u, c_t, c_m, c_0, rho, want_f, prec, f_out, k_out, check_status):
        """c_t K_T(u) + c_m M + c_0 K_0 from one K_T sweep and the cached M, K_0 (Tet10)."""
        if c_0 != 0.0 and self.mu_e is not None:
            raise NotImplementedError("the Tet10 small-strain stiffness takes scalar moduli")
        rho = self.rho if rho is None else float(rho)
        f_out, k_out = self.assemble(u, want_f=want_f, want_k=True, precision=prec, f_out=f_out, k_out=k_out,
                                     check_status=check_status)
        cache = self.__dict__.setdefault("_const_mats", {})
        if c_m != 0.0:
            key = ("M", prec, rho)
            if key not in cache:
                saved, self.rho = self.rho, rho
                try:
                    cache[key] = self.assemble(None, mass=True, precision=prec)[1]
                finally:
                    self.rho = saved
            k_out.mul_(c_t).add_(cache[key], alpha=c_m)
        else:
            k_out.mul_(c_t)
        if c_0 != 0.0:
            key = ("K0", prec)
            if key not in cache:
                cache[key] = self.assemble(None, linear=True, precision=prec)[1]
            k_out.add_(cache[key], alpha=c_0)
        return f_out, k_out

    def kv(self, u: torch.Tensor, v: torch.Tensor, precision: str | None = None,
           y_out: torch.Tensor | None = None, check_status: bool = True) -> torch.Tensor:
        """Matrix-free ``y = K_T(u) v`` (float64 in and out; element math in ``precision``)."""
        prec = precision or self.precision
        u = self._check_u(u)
        v = self._check_u(v)
        if y_out is None:
            y_out = self.new_f()
        self.status.zero_()
        work = self.workspace(prec)
        check(lib().psx_tet4_kv(ctypes.byref(self.dev["plan"]), ptr(self.X), ptr(u), ptr(self.mu_e),
                                ptr(self.kappa_e), self.mu, self.kappa, PRECISIONS[prec], ptr(v), ptr(y_out),
                                ptr(work), work.numel(), ptr(self.status), _stream_handle()), "psx_tet4_kv")
        if check_status:
            self.raise_on_bad_elements(u)
        return y_out

    def adjoint(self, u: torch.Tensor, w: torch.Tensor, want_params: bool = True):
        """Vector-Jacobian product of f_int: ``(gX (3N), gmu (E), gkappa (E))`` for cotangent ``w``.

        FP64; F is recomputed from (X, u).  ``w^T df/du`` is ``kv(u, w)`` (K_T is symmetric).
        """
        u = self._check_u(u)
        w = self._check_u(w)
        gX = self.new_f()
        gmu = torch.empty(self.n_elements, dtype=torch.float64, device=self.device) if want_params else None
        gk = torch.empty(self.n_elements, dtype=torch.float64, device=self.device) if want_params else None
        self.status.zero_()
        work = self.workspace("fp64")
        check(lib().psx_tet4_adjoint(ctypes.byref(self.dev["plan"]), ptr(self.X), ptr(u), ptr(self.mu_e),
                                     ptr(self.kappa_e), self.mu, self.kappa, ptr(w), ptr(gX), ptr(gmu), ptr(gk),
                                     ptr(work), work.numel(), ptr(self.status), _stream_handle()),
              "psx_tet4_adjoint")
        self.raise_on_bad_elements(u)
        return gX, gmu, gk

    def dr_step(self, u: torch.Tensor, b: torch.Tensor, minv: torch.Tensor, x: torch.Tensor, vel: torch.Tensor,
                c1: float, c2: float, dt: float, precision: str | None = None,
                r_out: torch.Tensor | None = None, check_status: bool = True) -> None:
        """One fused dynamic-relaxation pseudo-step on ``K_T(u) x = b`` (updates x, vel in place).

        With ``check_status`` (the default) the sweep's status is read afterwards, which
        synchronises: an inverted element raises the reference's ``ValueError`` and a
        bounded wait that gave up raises ``RuntimeError``.  Loops that check less often
        pass ``check_status=False`` and call ``raise_on_bad_elements`` themselves; the
        status is zeroed before every step either way.
        """
        prec = precision or self.precision
        u = self._check_u(u)
        for t in (b, minv, x, vel):
            self._check_u(t)
        self.status.zero_()
        work = self.workspace(prec)
        check(lib().psx_tet4_dr_step(ctypes.byref(self.dev["plan"]), ptr(self.X), ptr(u), ptr(self.mu_e),
                                     ptr(self.kappa_e), self.mu, self.kappa, PRECISIONS[prec], ptr(b), ptr(minv),
                                     c1, c2, dt, ptr(x), ptr(vel), ptr(r_out), ptr(work), work.numel(),
                                     ptr(self.status), _stream_handle()), "psx_tet4_dr_step")
        if check_status:
            self.raise_on_bad_elements(u)

    def _check_u(self, u: torch.Tensor) -> torch.Tensor:
        if not isinstance(u, torch.Tensor) or u.device != self.X.device or u.dtype != torch.float64:
            raise ValueError("u must be a float64 tensor on the assembler's device")
        if u.numel() != 3 * self.n_nodes:
            raise ValueError(f"u has {u.numel()} entries, expected {3 * self.n_nodes}")
        return u.contiguous()

    # ------------------------------------------------------------------ status
    def status_counts(self) -> tuple[int, int, int, int]:
        """(n_inverted, n_bad_volume, first_bad_element or -1, flags) of the last sweep (synchronises)."""
        s = self.status[:6].cpu().numpy()
        first = int(0x7FFFFFFF - int(s[2])) if s[2] != 0 else -1
        return int(s[0]), int(s[1]), first, int(s[5])

    def last_spins(self) -> int:
        """Spin iterations the bounded waits of the last sweep took (synchronises)."""
        return int(self.status[4].item())

    def raise_on_bad_elements(self, u: torch.Tensor | None) -> None:
        n_inv, n_vol, first, flags = self.status_counts()
        raise_if_wait_gave_up(flags)
        if n_inv == 0 and n_vol == 0:
            return
        if self.npe == 10:
            # tet10_total_lagrangian.py:104-113: quadrature points in order, det J then det F
            check(lib().psx_tet10_element_dets(ptr(self.dev["conn"]), ptr(self.X), ptr(u), first,
                                               ptr(self._dets), _stream_handle()), "psx_tet10_element_dets")
            d = self._dets.cpu().numpy()
            for q in range(4):
                if not d[2 * q] > 0.0:
                    raise ValueError(f"Negative or zero Jacobian determinant: det(J) = {d[2 * q]:.4e}.")
                if not d[2 * q + 1] > 0.0:
                    raise ValueError(f"Element inversion detected: det(F) = {d[2 * q + 1]:.4e} <= 0.")
            raise ValueError("Element inversion detected: det(F) <= 0.")
        check(lib().psx_tet4_element_dets(ptr(self.dev["conn"]), ptr(self.X), ptr(u), first,
                                          ptr(self._dets), _stream_handle()), "psx_tet4_element_dets")
        detA, J = (float(v) for v in self._dets.cpu().numpy()[:2])
        if not detA > 0.0:
            raise ValueError(
                f"Negative or zero element volume detected (det(A) = {detA}). Check element vertex ordering.")
        raise ValueError(f"Element inversion detected: det(F) = {J:.4e} <= 0.")

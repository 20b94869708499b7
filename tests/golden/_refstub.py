"""Import shim for the pSierra reference, used only to generate golden fixtures.

The reference package (tanadul-s/psierra) is pure Python on numpy + scipy, but its
``psierra/__init__.py`` pulls in pyvista, meshio, h5py, vtk, trimesh, pytetwild and
embreex, none of which are installed here.  This shim registers an empty
``psierra`` package whose ``__path__`` points at the reference sources (so the
top-level ``__init__`` is skipped) and inserts inert stand-ins for the missing
third-party modules.  Nothing on the hot path touches those modules.

Only ``tests/golden/make_golden.py`` imports this file, and only in a container
where the reference sources exist.  The GPU tests never read the reference.
"""
from __future__ import annotations

import os
import sys
import types

# the directory holding the reference package ``psierra`` (its ``src`` folder); required
REFERENCE_SRC = os.environ.get("PSIERRA_REFERENCE_SRC", "")


class _Anything:
    """Attribute sink: any attribute access or call returns another sink."""

    def __init__(self, *a, **k):
        pass

    def __getattr__(self, name):
        return _Anything()

    def __call__(self, *a, **k):
        return _Anything()


_STUB_ROOTS: set[str] = set()


def _stub(name: str, **attrs) -> types.ModuleType:
    mod = types.ModuleType(name)
    mod.__path__ = []  # type: ignore[attr-defined]  # a package, so submodules resolve
    for k, v in attrs.items():
        setattr(mod, k, v)
    mod.__getattr__ = lambda attr: _Anything  # type: ignore[attr-defined]
    sys.modules[name] = mod
    _STUB_ROOTS.add(name.split(".")[0])
    return mod


class _StubFinder:
    """Meta-path finder that answers every submodule import of a stubbed package."""

    def find_spec(self, fullname, path=None, target=None):
        import importlib.machinery

        if fullname.split(".")[0] in _STUB_ROOTS and fullname not in sys.modules:
            return importlib.machinery.ModuleSpec(fullname, self, is_package=True)
        return None

    def create_module(self, spec):
        return _stub(spec.name)

    def exec_module(self, module):
        return None


def install() -> None:
    if "psierra" in sys.modules and getattr(sys.modules["psierra"], "_graft_stub", False):
        return
    if not REFERENCE_SRC:
        raise RuntimeError("set PSIERRA_REFERENCE_SRC to the reference's src directory (the one holding psierra/)")
    pkg_dir = os.path.join(REFERENCE_SRC, "psierra")
    if not os.path.isdir(pkg_dir):
        raise RuntimeError(f"reference sources not found at {pkg_dir}")

    class CellType:
        TETRA = 10
        QUADRATIC_TETRA = 24
        TRIANGLE = 5
        QUADRATIC_TRIANGLE = 22
        VERTEX = 1
        LINE = 3

    _stub("pyvista", UnstructuredGrid=_Anything, PolyData=_Anything,
          DataSetAttributes=_Anything, CellType=CellType, MultiBlock=_Anything)
    for name in ("meshio", "h5py", "vtk", "trimesh", "pytetwild", "embreex",
                 "vtkmodules", "vtkmodules.all", "gmsh"):
        if name not in sys.modules:
            _stub(name)

    sys.meta_path.insert(0, _StubFinder())
    ps = types.ModuleType("psierra")
    ps.__path__ = [pkg_dir]  # type: ignore[attr-defined]
    ps._graft_stub = True  # type: ignore[attr-defined]
    sys.modules["psierra"] = ps


class DuckMesh:
    """Minimal stand-in for ``VolumetricMesh`` with the attributes the path reads."""

    def __init__(self, nodes, elements):
        import numpy as np

        self.nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        self.elements = np.ascontiguousarray(elements, dtype=np.int64)

    @property
    def n_nodes(self):
        return int(self.nodes.shape[0])

    @property
    def n_elements(self):
        return int(self.elements.shape[0])

    @property
    def n_dofs(self):
        return 3 * self.n_nodes

    @property
    def volumes(self):
        import numpy as np

        X = self.nodes[self.elements[:, :4]]
        d = np.linalg.det(np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=1))
        return np.abs(d) / 6.0

    def copy(self):
        return DuckMesh(self.nodes.copy(), self.elements.copy())

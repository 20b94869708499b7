"""Command line of the configured-workload runner (CPU): each workload gets its own
options and its own default preconditioner (cfg3 the configured Jacobi PCG, cfg5 the
two-level CG), and the record is printed as one JSON line."""
from __future__ import annotations

import json

import pytest

from psierra_b200 import workloads


@pytest.fixture
def calls(monkeypatch):
    seen = {}

    def fake(name):
        def run(**kw):
            seen[name] = kw
            return {"workload": name}
        return run

    for name in ("cfg3", "cfg4", "cfg5"):
        monkeypatch.setattr(workloads, name, fake(name))
    return seen


def test_cfg3_defaults_to_the_configured_jacobi_pcg(calls, capsys):
    workloads.main(["cfg3"])
    kw = calls["cfg3"]
    assert kw["preconditioner"] == "jacobi"
    assert (kw["cells"], kw["n_steps"], kw["pcg_rtol"], kw["nr_iterations"]) == (30, 20, 1e-8, 30)
    assert kw["precisions"] == ("fp64", "fp32-mixed")
    assert json.loads(capsys.readouterr().out) == {"workload": "cfg3"}


def test_cfg3_options(calls):
    workloads.main(["cfg3", "--steps", "60", "--precisions", "fp64", "--preconditioner", "two-level",
                    "--pcg-rtol", "1e-10"])
    kw = calls["cfg3"]
    assert (kw["n_steps"], kw["precisions"], kw["preconditioner"], kw["pcg_rtol"]) == (60, ("fp64",), "two-level",
                                                                                         1e-10)


def test_cfg5_defaults_to_the_two_level_cg(calls):
    workloads.main(["cfg5"])
    kw = calls["cfg5"]
    assert kw["preconditioner"] == "two-level" and kw["n"] == 256 and kw["pcg_iterations"] is None
    workloads.main(["cfg5", "--preconditioner", "block-jacobi", "--beams", "8", "--pcg-iterations", "50"])
    kw = calls["cfg5"]
    assert (kw["preconditioner"], kw["n"], kw["pcg_iterations"]) == ("block-jacobi", 8, 50)
    assert kw["target_tets"] == pytest.approx(4.1e6 * 8 / 256)


def test_cfg4_options(calls):
    workloads.main(["cfg4", "--grid", "0.004", "--gravity", "1.0", "--fd-elements", "4", "--fd-step", "1e-4"])
    assert calls["cfg4"] == {"h_grid": 0.004, "gravity_fraction": 1.0, "n_check": 4, "rel_step": 1e-4}

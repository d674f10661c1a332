"""CPU tests of the boundary: the CUDA library loads without a GPU and
exports every symbol the public header declares; the Python binding agrees
with the header; the workload generator is frozen."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sdddst_b200.h")


def header_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(sdddst_\w+)\s*\(", txt)))


def test_library_exports_every_header_symbol(engine_lib):
    lib = engine_lib.load()
    names = header_functions()
    assert len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", engine_lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (sdddst_\w+)", out))
    assert set(names) <= exported
    assert set(engine_lib.EXPORTS) == set(names)


def test_header_constants_match_binding(engine_lib):
    txt = open(HEADER).read()
    consts = dict(re.findall(r"#define SDDDST_(\w+) \((-?\d+)\)", txt))
    assert int(consts["ERR_INVALID"]) == engine_lib.ERR_INVALID
    assert int(consts["ERR_SOLVER"]) == engine_lib.ERR_SOLVER
    assert int(consts["ERR_NONFINITE"]) == engine_lib.ERR_NONFINITE


def test_default_params_follow_reference_defaults(engine_lib):
    p = engine_lib.default_params()
    assert p.ic == 2 and p.prec == 1e-8 and p.step_size == 1.0 and p.cutoff_multiplier == 1.0
    assert p.A == 1e-4 * 16.0 and p.KASQR == 1.65 * 1.65 * 1e6 / 256.0
    q = engine_lib.cli_params(4096, 1.0, 1e-7, p=256, pd_scaling=True)
    assert q.A == 1e-4 * 16.0 * (1.0 / np.sqrt(4096.0))
    assert q.KASQR == 1.65 * 1.65 * 1e6 / 256.0 * 4096.0
    # solver defaults of this library (no reference counterpart): cluster-
    # preconditioned GMRES(30), its coupling threshold left to the solver
    assert p.solver == engine_lib.SOLVER_GMRES_CLUSTER and p.gmres_restart == 30
    assert p.precond_theta == 0.0


def test_workload_generator_is_frozen():
    from sdddst_b200 import workloads as w
    xyb, pd = w.dislocations(256, 0)
    assert xyb.shape == (256, 3) and pd.shape == (0, 2)
    assert xyb[:, 2].sum() == 0 and set(np.unique(xyb[:, 2])) == {-1.0, 1.0}
    assert np.all(xyb[:, :2] >= -0.5) and np.all(xyb[:, :2] < 0.5)
    assert xyb[0, 0] == 0.1369616873214543  # first draw of default_rng(0)
    xyb2, pd2 = w.dislocations(4096, 1, 256)
    assert pd2.shape == (256, 2)
    sizes = w.batch_sizes(512, 3)
    assert sizes.min() >= 64 and sizes.max() <= 2048 and len(sizes) == 512


def test_dconf_roundtrip(tmp_path):
    from sdddst_b200 import workloads as w
    xyb, pd = w.dislocations(50, 4, 5)
    w.write_dconf(str(tmp_path / "a.dconf"), xyb)
    w.write_pdconf(str(tmp_path / "a.pdconf"), pd)
    assert np.array_equal(w.read_dconf(str(tmp_path / "a.dconf")), xyb)
    assert np.array_equal(w.read_pdconf(str(tmp_path / "a.pdconf")), pd)


def test_header_enums_match_binding(engine_lib):
    txt = open(HEADER).read()
    enums = dict((k, int(v)) for k, v in re.findall(r"SDDDST_((?:SOLVER|FIELD)_\w+) = (\d+)", txt))
    for name in ("SOLVER_GMRES", "SOLVER_GMRES_JACOBI", "SOLVER_GMRES_CLUSTER", "SOLVER_DIRECT",
                 "SOLVER_GMRES_LEARNED", "SOLVER_GMRES_NEUMANN", "SOLVER_DIRECT_MIXED", "FIELD_ANALYTIC",
                 "FIELD_TABULATED"):
        assert enums[name] == getattr(engine_lib, name), name

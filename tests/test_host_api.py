"""The reference-named host API: sdddstCore C++ classes (sdddst_b200/host)
and the PySdddstCore module (sdddst_b200/python).

CPU: the module imports, its host utilities follow the reference formulas,
the C++ headers compile a reference-style program.  GPU: the README usage of
PySdddstCore and the fine-grained Simulation methods (calculateSpeeds,
calculateJacobian, integrate) against the oracle."""
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import ref
from sdddst_b200 import workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "sdddst_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def psc():
    from sdddst_b200 import build
    build.build_python_module()
    if PKG not in sys.path:
        sys.path.insert(0, PKG)
    import PySdddstCore
    return PySdddstCore


def test_module_surface(psc):
    for name in ["SimulationDataObject", "SimulationData", "Simulation", "AnalyticFieldObject", "FieldObject",
                 "StressProtocolObject", "FixedRateStressProtocolObject", "PrecisionHandler", "Dislocation",
                 "DislocationVector", "PointDefect", "StepType", "normalize", "X", "X2", "E"]:
        assert hasattr(psc, name), name
    assert psc.normalize(0.75) == -0.25 and psc.normalize(-0.5) == -0.5 and psc.normalize(0.5) == -0.5
    assert psc.X(0.25) == np.sin(2 * np.pi * 0.25) * 0.5 / np.pi
    assert psc.X2(0.1) == (1 - np.cos(2 * np.pi * 0.1)) * 0.5 / np.pi / np.pi


def test_precision_handler_semantics(psc):
    ph = psc.PrecisionHandler()
    ph.set_min_precisity(1e-6)
    ph.set_size(3)
    ph.update_tolerance(4e-10, 0)   # 1e-12 = prec^2: not below, unchanged
    ph.update_tolerance(1e-10, 1)   # 2.5e-13 < 1e-12
    ph.update_tolerance(0.0, 2)     # coincident -> EPS
    ph.update_error(1e-6, 1)
    assert ph.get_max_error_ratio_square() == 1e-12 / (1e-10 * 0.25 * 1e-2)
    assert ph.get_new_stepsize(1.0) == 0.9 * min(2.0, (1 / np.sqrt(4.0)) ** (1 / 3))
    ph.reset()
    assert ph.get_max_error_ratio_square() == 0 and ph.get_new_stepsize(1.0) == 2.0


def test_host_field_matches_golden(psc):
    g = np.load(os.path.join(GOLDEN, "field.npz"))
    f = psc.AnalyticFieldObject()
    f.init()
    d = psc.SimulationData("", "")
    d.tau = f
    assert not f.valid()
    tau = d.tau
    xy = np.array([tau.xy(a, b) for a, b in zip(g["dx"], g["dy"])])
    xd = np.array([tau.xy_diff_x(a, b) for a, b in zip(g["dx"], g["dy"])])
    r = np.hypot(g["dx"], g["dy"])
    ok = r > 0
    # relative to the natural scale of each (1/r and 1/r^2)
    assert np.max(np.abs(xy - g["xy"])[ok] * r[ok]) < 1e-12
    assert np.max(np.abs(xd - g["xy_dx"])[ok] * r[ok] ** 2) < 1e-12


def test_simulation_data_files(psc, tmp_path):
    xyb, pd = workloads.dislocations(50, 3, 4)
    workloads.write_dconf(str(tmp_path / "a.dconf"), xyb)
    workloads.write_pdconf(str(tmp_path / "a.pd"), pd)
    obj = psc.SimulationDataObject(str(tmp_path / "a.dconf"), str(tmp_path / "a.pd"))
    sd = obj()
    assert sd.dislocation_count == 50 and sd.point_defect_count == 4
    assert sd.dislocations[7].x == xyb[7, 0] and sd.point_defects[2].y == pd[2, 1]
    sd.cutoff_multiplier = 0.5
    sd.update_cutoff()
    assert sd.cutoff == 1.0 / np.sqrt(50) * 0.5
    sd.write_dislocation_data_to_file(str(tmp_path / "b.dconf"))
    assert np.array_equal(workloads.read_dconf(str(tmp_path / "b.dconf")), xyb)


def test_cpp_headers_compile_reference_style_program(tmp_path):
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-std=c++11", "-fsyntax-only", "-I", os.path.join(PKG, "host", "include"),
                    os.path.join(ROOT, "tests", "cpp", "host_api_check.cpp")], check=True)


@pytest.mark.gpu
def test_readme_usage_matches_oracle(psc, port_lib, tmp_path):
    """PySdddstCore as the reference README uses it, stepped on the GPU,
    against the oracle on the same file."""
    n = 256
    xyb, _ = workloads.dislocations(n, 0)
    path = str(tmp_path / "dislocation.dconf")
    workloads.write_dconf(path, xyb)
    obj = psc.SimulationDataObject(path, "")
    obj().cutoff_multiplier = 0.5
    obj().precision = 1e-6
    obj().step_size = 1e-6
    obj().calculate_strain_during_simulation = True
    obj().update_cutoff()
    stress = psc.StressProtocolObject()
    stress.init()
    obj().external_stress = stress
    field = psc.AnalyticFieldObject()
    field.init()
    obj().tau = field
    sim = psc.Simulation.create(obj)
    o = ref.Sim(xyb, None, ref.params(cutoff_multiplier=0.5, prec=1e-6, step_size=1e-6, calculate_strain=True), "port")
    for k in range(20):
        a = sim.step()
        assert a == o.step(), k
        x = np.array([d.x for d in obj().dislocations])
        assert np.abs(x - o.config(0)[:, 0]).max() <= 1e-9, k
        sc = o.scalars()
        assert obj().successful_steps == sc["successful_steps"] and obj().failed_steps == sc["failed_steps"]
        assert np.isclose(obj().step_size, sc["step_size"], rtol=1e-6)
        assert np.isclose(obj().simulation_time, sc["sim_time"], rtol=1e-12)
        assert np.isclose(obj().total_accumulated_strain_increase, sc["strain"], rtol=1e-6, atol=1e-18)
    assert sim.get_time() == obj().simulation_time


@pytest.mark.gpu
def test_fine_grained_cpp_methods_match_oracle(port_lib, tmp_path):
    from sdddst_b200 import build
    lib = build.build()
    exe = str(tmp_path / "host_api_check")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-std=c++11", "-O1", "-I", os.path.join(PKG, "host", "include"),
                    os.path.join(ROOT, "tests", "cpp", "host_api_check.cpp"), "-o", exe, "-L", PKG, "-lsdddst_b200",
                    "-Wl,-rpath," + PKG], check=True)
    n, m, prec, h = 300, 0.8, 1e-6, 2e-6
    xyb, _ = workloads.dislocations(n, 9)
    path = str(tmp_path / "c.dconf")
    workloads.write_dconf(path, xyb)
    out = subprocess.run([exe, path, str(m), str(prec), str(h)], capture_output=True, text=True, check=True).stdout
    lines = {ln.split()[0]: ln.split()[1:] for ln in out.strip().splitlines()}
    o = ref.Sim(xyb, None, ref.params(cutoff_multiplier=m, prec=prec, step_size=h), "port")
    v_ref, _ = o.speeds(xyb)
    v = np.array(lines["speeds"], dtype=float)
    assert np.all(np.abs(v - v_ref) <= 1e-10 * np.abs(v_ref).max() + 1e-9 * np.abs(v_ref))
    toks = lines["csc"]
    nn, nnz = int(toks[0]), int(toks[1])
    Ap = np.array(toks[2:3 + nn], dtype=np.int32)
    Ai = np.array(toks[3 + nn:3 + nn + nnz], dtype=np.int32)
    Ax = np.array(toks[3 + nn + nnz:3 + nn + 2 * nnz], dtype=float)
    Rp, Ri, Rx, Rd = o.jacobian(h, xyb)
    J = ref.csc_to_dense(Ap, Ai, Ax, n)
    Jr = ref.csc_to_dense(Rp, Ri, Rx, n)
    assert np.abs(J - Jr).max() <= 1e-10 * max(1.0, np.abs(Jr - np.diag(np.diag(Jr))).max())
    # integrate: the oracle's stage I from the same state (first step of a fresh simulation)
    o2 = ref.Sim(xyb, None, ref.params(cutoff_multiplier=m, prec=prec, step_size=h), "port")
    o2.set_state(xyb, h, 0.0, 0.0, 0.0, False)
    x_ref = o2.integrate_stage(1)
    x = np.array(lines["integrate"], dtype=float)
    assert np.abs(x - x_ref).max() <= 1e-10

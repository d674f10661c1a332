"""The `sdddst` command-line drop-in (sdddst_b200/cli/sdddst_main.cpp) for the
reference's simulation mode (src/main.cpp, src/project_parser.cpp:33-298).

CPU: the option checks of ProjectParser and their exit codes.
GPU: the N = 256 workload (seed 0, cutoff multiplier 0.5, precision 1e-6,
200 accepted steps) run through the executable; every line of its 12-column
log (simulation.cpp:463-617: time, successful and failed steps, error ratio^2,
<|v|>, cutoff, order parameter, stress, wall time, strain, sum v^2, energy)
against the oracle stepping the same file, except the wall-time column; the
result configuration file against the oracle's final positions.
"""
import os
import subprocess

import numpy as np
import pytest

from oracle import ref
from sdddst_b200 import workloads


@pytest.fixture(scope="module")
def exe():
    from sdddst_b200 import build
    return build.build_cli()


def _run(exe, *args, **kw):
    return subprocess.run([exe, *args], capture_output=True, text=True, timeout=600, **kw)


def test_option_checks(exe, tmp_path):
    r = _run(exe, "--help")
    assert r.returncode == 0 and "--dislocation-configuration" in r.stdout and "--spring-constant" in r.stdout
    r = _run(exe, "-c")
    assert r.returncode == 255 and "dislocation-configuration is missing!" in r.stderr
    r = _run(exe, "-c", "--dislocation-configuration", "a.dconf")
    assert r.returncode == 255 and "result-dislocation-configuration is missing!" in r.stderr
    r = _run(exe, "-c", "--no-such-option")
    assert r.returncode == 255 and "unrecognised" in r.stderr
    r = _run(exe, "-c", "--ev-analyzation")
    assert r.returncode == 1 and "result-ev-file is not defined" in r.stderr
    r = _run(exe, "-c", "--step-count-limit", "ten")
    assert r.returncode == 255 and "invalid" in r.stderr
    r = _run(exe, "-c", "--calculate-strain=1")
    assert r.returncode == 255
    xyb, _ = workloads.dislocations(8, 1)
    f = str(tmp_path / "d.dconf")
    workloads.write_dconf(f, xyb)
    # both protocols at once: exit(-20) of project_parser.cpp:279-283 (prefix forms accepted)
    r = _run(exe, "-c", "--dislocation-conf", f, "--result-dislocation-configuration=" + str(tmp_path / "o"),
             "--no-external-stress", "--fixed-rate-external-stress", "1.0")
    assert r.returncode == 256 - 20 and "Only one stress protocol" in r.stderr


def _log_rows(path):
    rows = []
    with open(path) as f:
        for line in f:
            rows.append(line.split())
    return rows


@pytest.mark.gpu
def test_cli_run_matches_oracle(exe, port_lib, tmp_path):
    w = workloads.SMALL_256
    xyb, _ = w.state()
    src = str(tmp_path / "start.dconf")
    out = str(tmp_path / "end.dconf")
    log = str(tmp_path / "run.log")
    workloads.write_dconf(src, xyb)
    r = _run(exe, "-c", "--dislocation-configuration", src, "--result-dislocation-configuration", out,
             "--logfile-path", log, "--step-count-limit", str(w.steps), "--cutoff-multiplier",
             str(w.cutoff_multiplier), "--position-precision", str(w.prec), "--initial-stepsize", str(w.step_size),
             "--calculate-strain")
    assert r.returncode == 0, r.stderr
    rows = _log_rows(log)
    assert len(rows) == w.steps + 1 and all(len(rw) == 12 for rw in rows)
    o = ref.Sim(xyb, None, ref.params(cutoff_multiplier=w.cutoff_multiplier, prec=w.prec, step_size=w.step_size,
                                      calculate_strain=True), "port")
    # first line: initial state (simulation.cpp:463-476)
    v0, _ = o.speeds(xyb)
    first = rows[0]
    assert [float(first[0]), int(first[1]), int(first[2]), float(first[3])] == [0.0, 0, 0, 0.0]
    assert np.isclose(float(first[4]), np.abs(v0).mean(), rtol=1e-10)
    assert first[6] == "-" and first[8] == "-"
    assert np.isclose(float(first[10]), np.sum(v0 * v0), rtol=1e-10)
    k = 1
    attempts = 0
    while k <= w.steps and attempts < 2000:
        attempts += 1
        if not o.step():
            continue
        s, rw = o.scalars(), rows[k]
        assert np.isclose(float(rw[0]), s["sim_time"], rtol=1e-9, atol=0), k
        assert int(rw[1]) == s["successful_steps"] and int(rw[2]) == s["failed_steps"], k
        assert np.isclose(float(rw[3]), s["max_error_ratio_sqr"], rtol=1e-5, atol=1e-12), k
        assert np.isclose(float(rw[4]), s["avg_speed"], rtol=1e-9), k
        assert float(rw[5]) == s["cutoff"], k
        assert rw[6] == "-"
        assert float(rw[7]) == s["stress"], k
        assert np.isclose(float(rw[9]), s["strain"], rtol=1e-7, atol=1e-18), k
        # sum v^2 weights the largest velocities, which agree to 1e-10 of the
        # largest: 1e-8 relative
        assert np.isclose(float(rw[10]), s["vsquare"], rtol=1e-8), k
        assert np.isclose(float(rw[11]), s["energy"], rtol=1e-8), k
        k += 1
    assert k == w.steps + 1
    end = workloads.read_dconf(out)
    assert np.abs(end[:, 0] - o.config(0)[:, 0]).max() <= 1e-9
    assert np.array_equal(end[:, 1:], o.config(0)[:, 1:])

"""The eigenvalue analysis (the reference's --ev-analyzation mode:
src/time_series_processor.cpp:21-247, src/spectral_decompositor.cpp:63-201).

CPU: the oracle's Hessian and second field derivative are pinned bit for bit
to the reference compiled in place (oracle/Makefile, with the LAPACKE shim
recording the matrix decompose() hands to LAPACKE_dsyevd), its eigenpairs to
the shim's Jacobi eigensolver; the n^3 form of the eigenvalue derivatives the
device uses (v_m^T M v_m / rate) is checked against the reference's literal
n^4 loop.
GPU: the device Hessian, eigenpairs, observables, derivatives and
correlation matrices against the oracle (numpy.linalg.eigh: LAPACK's syevd,
the driver the reference calls), and the CLI's gzip output against the
oracle line by line.  Eigenvectors are compared up to sign and only for
modes separated from their neighbours (an eigenvector is defined by its
eigenvalue's isolation).
"""
import gzip
import os
import subprocess

import numpy as np
import pytest

from oracle import ref
from sdddst_b200 import workloads


def _wrap(d):
    return d - np.floor(d + 0.5)


def _derivative_matrix(xyb, v):
    """M_ij = b_i b_j xy_diff_x2(x_i - x_j, y_i - y_j) (v_i - v_j),
    M_ii = -sum_{j != i} M_ij (restated with the oracle's field)."""
    n = xyb.shape[0]
    dx = _wrap(xyb[:, 0][:, None] - xyb[:, 0][None, :])
    dy = _wrap(xyb[:, 1][:, None] - xyb[:, 1][None, :])
    F = ref.field(2, dx, dy, "port").reshape(n, n)
    np.fill_diagonal(F, 0.0)
    M = xyb[:, 2][:, None] * xyb[:, 2][None, :] * F * (v[:, None] - v[None, :])
    np.fill_diagonal(M, 0.0)
    M[np.diag_indices(n)] = -M.sum(axis=1)
    return M


def test_ev_oracle_pinned_to_reference(port_lib, ref_available):
    if not ref_available:
        pytest.skip("reference not compiled here (oracle/_ref)")
    for n, seed, p in ((40, 3, 5), (33, 4, 0)):
        xyb, pd = workloads.dislocations(n, seed, p)
        H_ref, w_ref, V_ref = ref.ev_decompose_ref(xyb, pd)
        H = ref.ev_hessian(xyb, pd)
        assert np.array_equal(H, H_ref)
        w, Vc = np.linalg.eigh(H)
        assert np.abs(w - w_ref).max() <= 1e-12 * np.abs(w).max()
        V = Vc.T
        sgn = np.sign(np.sum(V * V_ref, axis=1))
        assert np.abs(V * sgn[:, None] - V_ref).max() <= 1e-10
    rng = np.random.default_rng(11)
    dx, dy = rng.uniform(-0.5, 0.5, 2000), rng.uniform(-0.5, 0.5, 2000)
    assert np.array_equal(ref.field(2, dx, dy, "ref"), ref.field(2, dx, dy, "port"))


def test_ev_derivative_identity(port_lib):
    """sum_ij V_mi V_mj sum_k v_k dH_ij/dx_k / rate (the reference's loop) =
    v_m^T M v_m / rate."""
    n, rate = 24, 3e-3
    xyb, pd = workloads.dislocations(n, 5, 3)
    v = np.random.default_rng(1).standard_normal(n)
    res = ref.ev_analysis(xyb, pd, v, stress_derivative=rate, nvec=0, deriv=True)
    V = res["V"]
    M = _derivative_matrix(xyb, v)
    compact = np.einsum("mi,ij,mj->m", V, M, V) / rate
    assert np.abs(compact - res["derivatives"]).max() <= 1e-11 * np.abs(res["derivatives"]).max()


def _engine(xyb, pd, rate):
    from sdddst_b200 import capi
    n, p = xyb.shape[0], pd.shape[0]
    prm = capi.cli_params(n, 1.0, 1e-6, p=p, pd_scaling=True, stress_kind=capi.STRESS_FIXED_RATE, stress_rate=rate)
    return capi.Engine(prm, xyb, pd if p else None)


def _oracle_speeds(xyb, pd, rate, t):
    o = ref.Sim(xyb, pd if pd.shape[0] else None,
                ref.params(cutoff_multiplier=1.0, prec=1e-6, stress_kind=1, stress_rate=rate, pd_scaling=True), "port")
    v, _ = o.speeds(xyb, t, 0)
    return v


def _separated(w, rel=1e-6):
    gap = np.full(w.shape, np.inf)
    d = np.diff(w)
    gap[:-1] = np.minimum(gap[:-1], d)
    gap[1:] = np.minimum(gap[1:], d)
    return gap > rel * np.abs(w).max()


@pytest.mark.gpu
def test_ev_hessian_matches_oracle(engine_lib, port_lib):
    n, p = 300, 16
    xyb, pd = workloads.dislocations(n, 7, p)
    e = _engine(xyb, pd, 1e-3)
    H = e.ev_hessian(xyb)
    H_ref = ref.ev_hessian(xyb, pd)
    off = H_ref - np.diag(np.diag(H_ref))
    assert np.abs(H - H_ref).max() <= 1e-10 * np.abs(off).max()
    assert np.array_equal(H, H.T)


@pytest.mark.gpu
def test_ev_analysis_matches_oracle(engine_lib, port_lib):
    n, p, rate, t, S = 200, 8, 2e-3, 0.75, 6
    xyb, pd = workloads.dislocations(n, 8, p)
    e = _engine(xyb, pd, rate)
    got = e.ev_analyze(xyb, sim_time=t, nvec=n, corr_bins=S)
    v_ref = _oracle_speeds(xyb, pd, rate, t)
    exp = ref.ev_analysis(xyb, pd, v_ref, stress_derivative=rate, nvec=n, corr_bins=S)
    w, w_ref = got["eigenvalues"], exp["eigenvalues"]
    scale = np.abs(w_ref).max()
    assert np.abs(w - w_ref).max() <= 1e-10 * scale
    assert np.abs(got["speeds"] - v_ref).max() <= 1e-10 * np.abs(v_ref).max()
    ok = _separated(w_ref)
    assert ok.sum() >= 0.9 * n
    V, V_ref = got["eigenvectors"], exp["eigenvectors"]
    sgn = np.sign(np.sum(V * V_ref, axis=1))
    assert np.abs((V * sgn[:, None] - V_ref)[ok]).max() <= 1e-7
    assert np.allclose(got["participation"][ok], exp["participation"][ok], rtol=1e-6)
    s, s_ref = got["burgers_sum"] * sgn, exp["burgers_sum"]
    assert np.abs(s - s_ref)[ok].max() <= 1e-7 * np.sqrt(n)
    g, g_ref = got["gan"], exp["gan"]
    big = ok & (np.abs(w_ref) > 1e-6 * scale)
    assert np.all(np.abs(g - g_ref)[big] <= 1e-6 * np.abs(g_ref)[big] + 1e-9 * np.abs(g_ref[big]).max())
    c, c_ref = got["correlations"], exp["correlations"]
    assert np.abs(c - c_ref)[ok].max() <= 1e-6
    # the all-pairs histogram is the sum of the equal- and opposite-sign ones
    assert np.allclose(c[:, 2], c[:, 0] + c[:, 1], rtol=0, atol=1e-15)


@pytest.mark.gpu
def test_ev_derivatives_match_literal_loop(engine_lib, port_lib):
    n, p, rate, t = 40, 4, 5e-3, 2.0
    xyb, pd = workloads.dislocations(n, 9, p)
    e = _engine(xyb, pd, rate)
    got = e.ev_analyze(xyb, sim_time=t, nvec=0, deriv=True)
    v_ref = _oracle_speeds(xyb, pd, rate, t)
    exp = ref.ev_analysis(xyb, pd, v_ref, stress_derivative=rate, nvec=0, deriv=True)
    ok = _separated(exp["eigenvalues"])
    d, d_ref = got["derivatives"], exp["derivatives"]
    assert np.abs(d - d_ref)[ok].max() <= 1e-7 * np.abs(d_ref).max()


@pytest.mark.gpu
def test_ev_zero_stress_has_no_derivative(engine_lib):
    from sdddst_b200 import capi
    n = 32
    xyb, _ = workloads.dislocations(n, 2)
    e = capi.Engine(capi.cli_params(n, 1.0, 1e-6), xyb)
    got = e.ev_analyze(xyb, nvec=2, deriv=True)
    assert np.all(got["derivatives"] == 0.0) and np.all(np.isfinite(got["eigenvalues"]))


def _write_series(tmp_path, sizes, p, seed):
    lst, configs = [], []
    _, pd = workloads.dislocations(4, seed, p)
    pdf = str(tmp_path / "defects.fconf")
    with open(pdf, "w") as f:
        for q in pd:
            f.write(f"{q[0]:.17g} {q[1]:.17g}\n")
    for k, n in enumerate(sizes):
        xyb, _ = workloads.dislocations(n, seed + 1 + k)
        path = str(tmp_path / f"c{k}.dconf")
        workloads.write_dconf(path, xyb)
        t = 0.5 + 0.75 * k
        lst.append(f"{t:.17g} {path}")
        configs.append((t, workloads.read_dconf(path)))
    fl = str(tmp_path / "files.txt")
    with open(fl, "w") as f:
        f.write("\n".join(lst) + "\n")
    return fl, pdf, pd, configs


def _close(a, b, scale):
    return np.all(np.abs(np.asarray(a) - np.asarray(b)) <= 2e-5 * np.abs(b) + 1e-9 * scale)


def test_ev_cli_option_checks(tmp_path):
    from sdddst_b200 import build
    exe = build.build_cli()
    r = subprocess.run([exe, "-c", "--ev-analyzation"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "result-ev-file is not defined" in r.stderr
    out = str(tmp_path / "o.gz")
    r = subprocess.run([exe, "-c", "--ev-analyzation", "--result-ev-file", out], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode < 0  # getStressProtocol aborts without a fixed-rate protocol
    r = subprocess.run([exe, "-c", "--ev-analyzation", "--result-ev-file", out, "--fixed-rate-external-stress", "1"],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "file-list" in r.stderr


@pytest.mark.gpu
def test_ev_cli_matches_oracle(engine_lib, port_lib, tmp_path):
    from sdddst_b200 import build
    exe = build.build_cli()
    rate, nvec = 2e-3, 3
    fl, pdf, pd, configs = _write_series(tmp_path, (48, 56), 4, 21)
    assert workloads.read_pdconf(pdf).shape == (4, 2)
    out = str(tmp_path / "ev.gz")
    r = subprocess.run([exe, "-c", "--ev-analyzation", "--file-list", fl, "--pd-configuration", pdf,
                        "--result-ev-file", out, "--fixed-rate-external-stress", repr(rate), "--calculate-ev-deriv",
                        "--eigenvector-to-write", str(nvec)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert [float(s) for s in r.stdout.split()] == [t for t, _ in configs]
    with gzip.open(out, "rt") as f:
        lines = f.read().splitlines()
    assert len(lines) == len(configs)
    for (t, xyb), line in zip(configs, lines):
        n = xyb.shape[0]
        tok = np.array([float(s) for s in line.split()])
        assert tok.size == 1 + 6 * n + nvec * n + n and tok[0] == float(f"{t:g}")
        ev, pn, gan, sp, x, sm = (tok[1 + k * n:1 + (k + 1) * n] for k in range(6))
        vecs = tok[1 + 6 * n:1 + 6 * n + nvec * n].reshape(nvec, n)
        der = tok[1 + 6 * n + nvec * n:]
        v_ref = _oracle_speeds(xyb, pd, rate, t)
        exp = ref.ev_analysis(xyb, pd, v_ref, stress_derivative=rate, nvec=nvec, deriv=True)
        ok = _separated(exp["eigenvalues"])
        assert _close(ev, exp["eigenvalues"], np.abs(exp["eigenvalues"]).max())
        assert _close(pn[ok], exp["participation"][ok], 1.0)
        assert _close(sp, v_ref, np.abs(v_ref).max())
        assert _close(x, xyb[:, 0], 1.0)
        assert _close(np.abs(sm[ok]), np.abs(exp["burgers_sum"][ok]), np.sqrt(n))
        big = ok & (np.abs(exp["eigenvalues"]) > 1e-6 * np.abs(exp["eigenvalues"]).max())
        assert _close(gan[big], exp["gan"][big], np.abs(exp["gan"]).max())
        for m in range(nvec):
            if ok[m]:
                s = np.sign(vecs[m] @ exp["eigenvectors"][m])
                assert _close(s * vecs[m], exp["eigenvectors"][m], 1.0)
        assert _close(der[ok], exp["derivatives"][ok], np.abs(exp["derivatives"]).max())


@pytest.mark.gpu
def test_ev_cli_correlation_matrices(engine_lib, port_lib, tmp_path):
    from sdddst_b200 import build
    exe = build.build_cli()
    rate, S = 1e-3, 3
    fl, pdf, pd, configs = _write_series(tmp_path, (30,), 2, 31)
    out = str(tmp_path / "corr.gz")
    r = subprocess.run([exe, "-c", "--ev-analyzation", "--file-list", fl, "--pd-configuration", pdf,
                        "--result-ev-file", out, "--fixed-rate-external-stress", repr(rate),
                        "--write-correlation-matrices", str(S)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    with gzip.open(out, "rt") as f:
        lines = f.read().splitlines()
    t, xyb = configs[0]
    n = xyb.shape[0]
    assert len(lines) == 1 + n * 3 * S
    head = np.array([float(s) for s in lines[0].split()])
    assert head.size == 1 + 3 * n
    v_ref = _oracle_speeds(xyb, pd, rate, t)
    exp = ref.ev_analysis(xyb, pd, v_ref, stress_derivative=rate, nvec=0, corr_bins=S)
    assert _close(head[1:1 + n], exp["eigenvalues"], np.abs(exp["eigenvalues"]).max())
    body = np.array([[float(s) for s in ln.split()] for ln in lines[1:]])
    assert body.shape == (n * 3 * S, S) and lines[1].endswith(" ")
    c = body.reshape(n, 3, S, S)
    ok = _separated(exp["eigenvalues"])
    assert np.all(np.abs(c - exp["correlations"])[ok] <= 2e-5 * np.abs(exp["correlations"])[ok] + 1e-9)

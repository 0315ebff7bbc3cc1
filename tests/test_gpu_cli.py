"""The `dgb` command-line driver against the reference's own driver.

`dgb` (dgpr_b200/csrc/dgb_main.cpp) takes the reference's options and writes
its outputs.  Run with the same arguments as the reference FP64 CPU solver
(`dg`, compiled in place into oracle/_ref/), it must print the same per-step
residual norms (rel 1e-10), write the same checkpoint and final .dg files,
and their states must agree to 1e-12 relative L2 (the bar for the FP64
path).  The bump channel mesh is curved (q = 2), the initial state the
reference's turbulent one, the boundaries freestream and walls."""
import os
import subprocess

import numpy as np
import pytest

import dgpr_b200 as dg

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DGB = os.path.join(ROOT, "dgpr_b200", "_lib", "dgb")
REF = os.path.join(ROOT, "oracle", "_ref", "dg")

ARGS = ["-p", "2", "-q", "2", "-nx", "4", "-ny", "2", "-nz", "2", "-niter", "6", "-chkint", "4", "-dt", "1e-3",
        "-mu", "1e-2", "-u", "0.3", "-scheme", "RK4", "-turb", "-bmx", "freestream", "-bpx", "freestream",
        "-bmy", "no_slip_wall", "-bpy", "inviscid_wall"]


def _run(exe, prefix, cwd, extra=()):
    out = subprocess.run([exe] + ARGS + list(extra) + ["-ofile", prefix], cwd=cwd, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    norms = {}
    for line in out.stdout.splitlines():
        if " : " in line:
            k, v = line.split(" : ")
            norms[int(k)] = float(v)
    return norms


def test_dgb_matches_the_reference_driver(tmp_path):
    if not os.path.exists(REF):
        pytest.skip("reference driver not built here")
    ours = _run(DGB, "ours_", tmp_path)
    ref = _run(REF, "ref_", tmp_path)
    assert sorted(ours) == sorted(ref) == list(range(6))
    for k in ref:
        assert abs(ours[k] - ref[k]) <= 1e-10 * ref[k], (k, ours[k], ref[k])
    for suffix in ("3.dg", ".dg"):
        assert os.path.exists(tmp_path / f"ours_{suffix}")
        ta, _, ua = dg.read_state(str(tmp_path / f"ours_{suffix}"))
        tb, _, ub = dg.read_state(str(tmp_path / f"ref_{suffix}"))
        assert np.linalg.norm(ua - ub) / np.linalg.norm(ub) < 1e-12
        assert ta == tb


def test_dgb_restarts_from_its_own_checkpoint(tmp_path):
    """-ifile continues from a checkpoint like the reference (cudg.cu:58-70):
    the checkpoint written before step 3 holds the state after 3 steps, so 3
    more steps from it give the uninterrupted 6-step run's final state, bit
    for bit (mesh, orders and boundaries come from the file)."""
    _run(DGB, "full_", tmp_path)
    out = subprocess.run([DGB, "-niter", "3", "-dt", "1e-3", "-mu", "1e-2", "-u", "0.3", "-scheme", "RK4",
                          "-ifile", "full_3", "-ofile", "restart_"],
                         cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    a = dg.read_state(str(tmp_path / "restart_.dg"))[2]
    b = dg.read_state(str(tmp_path / "full_.dg"))[2]
    assert np.array_equal(a, b)


def test_dgb_running_mean_matches_the_reference_driver(tmp_path):
    """-mean_start: the running mean (dg.cpp:123-131, output.cpp:39-49) is
    written beside the state in the checkpoint and final files."""
    if not os.path.exists(REF):
        pytest.skip("reference driver not built here")
    extra = ["-mean_start", "2"]
    ours = _run(DGB, "ours_", tmp_path, extra)
    ref = _run(REF, "ref_", tmp_path, extra)
    for k in ref:
        assert abs(ours[k] - ref[k]) <= 1e-10 * ref[k]
    for suffix in ("3.dg", ".dg"):
        for key in ("state", "mean"):
            _, _, a = dg.read_state(str(tmp_path / f"ours_{suffix}"), key)
            _, _, b = dg.read_state(str(tmp_path / f"ref_{suffix}"), key)
            assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12, (suffix, key)


def test_dgb_prandtl_option(tmp_path):
    """-prandtl turns the optional heat flux on (the bump channel's no-slip
    wall and turbulent state have temperature gradients); -prandtl 0 is the
    default physics, bit for bit."""
    _run(DGB, "plain_", tmp_path)
    _run(DGB, "zero_", tmp_path, ["-prandtl", "0"])
    _run(DGB, "heat_", tmp_path, ["-prandtl", "0.71"])
    plain, zero, heat = (dg.read_state(str(tmp_path / f"{k}_.dg"))[2] for k in ("plain", "zero", "heat"))
    assert np.array_equal(plain, zero)
    assert np.linalg.norm(heat - plain) > 1e-12 * np.linalg.norm(plain)
    out = subprocess.run([DGB] + ARGS + ["-prandtl", "-1", "-ofile", "bad_"], cwd=tmp_path, capture_output=True,
                         text=True, timeout=300)
    assert out.returncode != 0


def test_dgb_isothermal_wall_option(tmp_path):
    """An isothermal_wall side with -twall: the wall temperature changes the
    run; the option without such a side changes nothing."""
    iso = ["-bpy", "isothermal_wall"]
    base = [a for a in ARGS]
    i = base.index("-bpy")
    del base[i:i + 2]

    def run(prefix, extra):
        out = subprocess.run([DGB] + base + extra + ["-ofile", prefix], cwd=tmp_path, capture_output=True,
                             text=True, timeout=300)
        assert out.returncode == 0, out.stderr
        return dg.read_state(str(tmp_path / f"{prefix}.dg"))[2]

    a = run("a_", iso + ["-prandtl", "0.71", "-twall", "0.003"])
    b = run("b_", iso + ["-prandtl", "0.71", "-twall", "0.004"])
    assert np.linalg.norm(a - b) > 1e-12 * np.linalg.norm(a)
    c = run("c_", ["-bpy", "inviscid_wall", "-twall", "0.003"])
    d = run("d_", ["-bpy", "inviscid_wall"])
    assert np.array_equal(c, d)


def test_dgb_checkpoint_index_inside_a_short_restart(tmp_path):
    """A checkpoint index can fall inside a run shorter than -chkint: the
    reference checkpoints before every step with (tstep + 1) % chkint == 0,
    counting from the step the input file resumes at (cudg.cu:112-130).
    Restarting after step 3 for 4 steps with -chkint 7 writes the checkpoint
    before step 6, like the reference driver, with the same state."""
    if not os.path.exists(REF):
        pytest.skip("reference driver not built here")
    _run(DGB, "full_", tmp_path)
    args = ["-niter", "4", "-chkint", "7", "-dt", "1e-3", "-mu", "1e-2", "-u", "0.3", "-scheme", "RK4",
            "-ifile", "full_3"]
    for exe, prefix in ((DGB, "ours_"), (REF, "ref_")):
        out = subprocess.run([exe] + args + ["-ofile", prefix], cwd=tmp_path, capture_output=True, text=True,
                             timeout=300)
        assert out.returncode == 0, out.stderr
    for suffix in ("6.dg", ".dg"):
        ta, _, a = dg.read_state(str(tmp_path / f"ours_{suffix}"))
        tb, _, b = dg.read_state(str(tmp_path / f"ref_{suffix}"))
        assert ta == tb and np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12, suffix

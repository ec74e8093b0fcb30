"""The drop-in `vhci` command (vhci_b200/bin/vhci) against the reference program's CLI contract:
argument handling and messages (src/Input_Reader.cpp:17-168, exit status 0 on handled errors),
and on the GPU the output file and log lines of a full run against the reference's own output."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, levels_of, load_golden

BIN = os.path.join(ROOT, "vhci_b200", "bin", "vhci")


def run(args, cwd=None, timeout=600):
    return subprocess.run([BIN] + args, capture_output=True, text=True, cwd=cwd, timeout=timeout)


@pytest.fixture(scope="module", autouse=True)
def built():
    if not os.path.exists(BIN):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "vhci_b200", "csrc")], check=True)


def test_missing_arguments():
    r = run([])
    assert r.returncode == 0
    assert "Missing arguments..." in r.stdout
    assert "Usage: vhci -n Ncpus -i Modes.inp -o Freqs.dat -c Checkpoint.txt" in r.stdout


def test_wrong_number_of_arguments():
    r = run(["-n", "1", "-i"])
    assert r.returncode == 0
    assert "Wrong number of arguments..." in r.stdout


def test_help():
    r = run(["-h"])
    assert r.returncode == 0
    assert "Command line arguments:" in r.stdout and "-c    Checkpoint file" in r.stdout


def test_unreadable_input_and_strict_status(tmp_path):
    out = str(tmp_path / "f.dat")
    r = run(["-n", "1", "-i", str(tmp_path / "missing.inp"), "-o", out])
    assert r.returncode == 0
    assert " Error: Could not open input file." in r.stdout
    r = run(["-n", "1", "-i", str(tmp_path / "missing.inp"), "-o", out, "--strict"])
    assert r.returncode == 1


def test_thread_count_warnings(tmp_path):
    g = load_golden("clo2_vhci")
    r = run(["-n", "0", "-i", g["input"], "-o", str(tmp_path / "f.dat")])
    assert "Warning: Calculations cannot run with 0 CPUs." in r.stdout


def _parse_assign(s):
    # components "c (q w m+...)" -> multiset of (rounded coefficient, assignment)
    return sorted(re.findall(r"([0-9.]+) \(([^)]*)\)", s))


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["clo2_vhci_pt2", "syn_m6_pt2", "clo2_vci", "syn_m8_sextic_pt2",
                                  "syn_m5_cubic_pt2"])
def test_cli_run_matches_reference_output(tmp_path, case):
    g = load_golden(case)
    out = str(tmp_path / "freqs.dat")
    r = run(["-n", "2", "-i", g["input"], "-o", out], cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout[-2000:]
    assert "Done." in r.stdout
    lines = open(out).read().splitlines()
    ref_lines = open(os.path.join(g["dir"], "freqs.dat")).read().splitlines()
    assert len(lines) == len(ref_lines)
    got = np.array([float(l.split()[0]) for l in lines])
    ref = np.array(g["levels"])
    tol = 1e-3 if g["log"]["n_pert"] else 1e-4
    assert np.abs(got - ref).max() <= tol
    # assignments: same components (order within a line may differ, as between reference runs)
    for a, b in zip(lines, ref_lines):
        assert _parse_assign(a.split("   ", 1)[1]) == _parse_assign(b.split("   ", 1)[1])
    # the reference's log numbers: basis size per iteration, perturber count
    sizes = [int(x) for x in re.findall(r"Basis size after iteration \d+ is: (\d+)", r.stdout)]
    assert sizes == g["log"]["sizes"]
    # "% sparse" counts the reference's stored pattern, structural zeros included
    sparse = [float(x) for x in re.findall(r"The Hamiltonian is ([0-9.]+)% sparse", r.stdout)]
    assert sparse == g["log"]["sparse_percent"]
    if g["log"]["n_pert"]:
        assert f"Perturbative space contains {g['log']['n_pert']} states." in r.stdout
    assert not os.path.exists(os.path.join(str(tmp_path), "none"))

"""The ctb command-line tool's option handling (Ct/main.cpp:53-234), on the host.

Only paths that end before any device work run here: help, the argument
errors the reference reports, the device list and weight parsing (no device
is valid without a GPU, so the selection message appears and loading fails).
"""
import os
import subprocess

import pytest

from ct_b200 import build

pytestmark = pytest.mark.skipif(not os.path.exists(build.CLI), reason="ctb tool not built")


def run(*args):
    r = subprocess.run([build.CLI, *args], capture_output=True, text=True, timeout=120)
    return r.returncode, r.stdout + r.stderr


def test_help():
    rc, out = run("-h")
    assert rc == 0
    assert "Usage:" in out and "--cudadevices" in out and "--weights" in out


def test_input_and_output_required():
    rc, out = run("-i", "scan.csv")
    assert rc == 1
    assert "You must provide a file path to the config file as input as well as a file path for the output." in out


def test_weights_need_two_coefficients():
    rc, out = run("-i", "a.csv", "-o", "b.raw", "-w", "1")
    assert rc == 1
    assert "When using the flag -w you have to specify exactly two coefficients." in out


def test_unknown_parameter():
    rc, out = run("-i", "a.csv", "-o", "b.raw", "--bogus")
    assert rc == 1
    assert "Unknown or misplaced parameter --bogus." in out


def test_cpu_reconstruction_refused():
    rc, out = run("-i", "a.csv", "-o", "b.raw", "-n")
    assert rc == 1
    assert "remove -n" in out


def test_device_list_and_weights_parse(tmp_path):
    missing = str(tmp_path / "missing.csv")
    rc, out = run("-i", missing, "-o", str(tmp_path / "v.raw"), "-d", "0,1", "-w", "1.5,0.5")
    assert rc == 1
    assert "Beginning reconstruction." in out
    assert "load:" in out

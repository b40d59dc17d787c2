"""The C++ drop-in headers (include/aperture/...) compile against the C ABI,
and a lab written with them runs on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = "/usr/local/cuda"


def _build(tmp_path, lab="box_lab"):
    exe = str(tmp_path / lab)
    libdir = os.path.join(ROOT, "aperture3_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
           "-I", f"{CUDA}/include", os.path.join(ROOT, "tests", "cpp", lab + ".cpp"),
           "-o", exe, "-L", libdir, "-laperture_b200", f"-Wl,-rpath,{libdir}",
           "-L", f"{CUDA}/lib64", "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


def test_dropin_headers_compile(tmp_path):
    _build(tmp_path)
    _build(tmp_path, "pulsar_lab")
    _build(tmp_path, "gap_lab")
    _build(tmp_path, "gr_lab")


@pytest.mark.gpu
def test_dropin_box_lab_runs(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe, "12"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "box_lab ok" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_dropin_pulsar_lab_runs(tmp_path):
    exe = _build(tmp_path, "pulsar_lab")
    r = subprocess.run([exe, "12"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "pulsar_lab ok" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_dropin_gap_lab_runs(tmp_path):
    exe = _build(tmp_path, "gap_lab")
    r = subprocess.run([exe, "12"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "gap_lab ok" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_dropin_gr_lab_runs(tmp_path):
    exe = _build(tmp_path, "gr_lab")
    r = subprocess.run([exe, "12"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "gr_lab ok" in r.stdout, r.stdout + r.stderr

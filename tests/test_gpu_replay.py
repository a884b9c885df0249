"""Caller call patterns (apollo-stft frames, apollo-czt Bluestein workspace,
apollo-nufft oversampled grid, apollo-dctdst 2N-point DCT/DST, apollo-dht,
apollo-hilbert analytic signal) replayed by a C++ program through the C ABI
and checked against the oracle or the definitions; see
tests/replay/callers.cpp."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "replay", "callers.cpp")
OUT_DIR = os.path.join(ROOT, "tests", "replay", "_build")
EXE = os.path.join(OUT_DIR, "callers")


def build_replay():
    from apollofft_b200 import build as B
    from oracle import oracle as O
    lib = B.build()
    O.build()
    os.makedirs(OUT_DIR, exist_ok=True)
    libdir = os.path.dirname(lib)
    odir = os.path.join(ROOT, "oracle", "_build")
    cmd = ["/usr/bin/g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), SRC, "-o", EXE,
           "-L", libdir, "-lapollofft_cuda", "-L", odir, "-lapollo_oracle",
           f"-Wl,-rpath,{libdir}", f"-Wl,-rpath,{odir}"]
    subprocess.run(cmd, check=True)
    return EXE


def test_replay_harness_builds():
    assert os.path.exists(build_replay())


@pytest.mark.gpu
def test_replay_callers_match_oracle():
    exe = build_replay()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failure(s)" in r.stdout

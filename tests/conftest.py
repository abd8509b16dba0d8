"""Test configuration: the `gpu` marker, shared systems and settings.

`-m "not gpu"` tests run on any machine (oracle vs. the reference's golden
vectors, host logic, the C ABI surface); `-m gpu` tests call the CUDA library
through its C ABI and compare with the FP64 oracle.
"""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
REF_BUILD = os.path.join(ROOT, "oracle", "_ref")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU and libamoeba_gpu.so")


def golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def ref_fixture(*parts):
    """Input file from the reference's own tests, copied next to the
    compiled reference (oracle/_ref/testFiles) by oracle/ref.mk."""
    p = os.path.join(REF_BUILD, "testFiles", *parts)
    if not os.path.exists(p):
        pytest.skip("reference build (oracle/_ref) not present")
    return p


def last_structure(xyz, key, tmpdir):
    """The last structure of a concatenated Tinker .xyz (the reference's
    analyze processes every structure; its goldens hold the last one),
    written to tmpdir with a copy of the keyfile whose parameter path is
    made absolute.  Returns (xyz, key) paths."""
    def is_box_line(line):
        f = line.split()
        try:
            return len(f) == 6 and all(float(v) == float(v) for v in f)
        except ValueError:
            return False

    lines = open(xyz).read().splitlines()
    frames, i = [], 0
    while i < len(lines) and lines[i].strip():
        n = int(lines[i].split()[0])
        end = i + 1 + n + (1 if i + 1 < len(lines) and is_box_line(lines[i + 1]) else 0)
        frames.append((i, end))
        i = end
    s, end = frames[-1]
    out_xyz = os.path.join(tmpdir, "last.xyz")
    with open(out_xyz, "w") as f:
        f.write("\n".join(lines[s:end]) + "\n")
    out_key = os.path.join(tmpdir, "last.key")
    with open(out_key, "w") as f:
        for line in open(key):
            w = line.split()
            if w and w[0].lower() == "parameters":
                line = f"parameters {os.path.normpath(os.path.join(os.path.dirname(key), w[1]))}\n"
            f.write(line)
    return out_xyz, out_key


def ref_dump(xyz, key=None):
    """Runs the compiled reference on a Tinker .xyz (+ .key) and returns its
    globals (oracle/ref_dump.cpp)."""
    import subprocess
    import tempfile
    exe = os.path.join(REF_BUILD, "ref_dump")
    if not os.path.exists(exe):
        pytest.skip("reference build (oracle/_ref) not present")
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "d.json")
        args = [exe, "--out", out] + (["-k", key] if key else []) + [xyz]
        subprocess.check_call(args, cwd=os.path.dirname(xyz), stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        return json.load(open(out))

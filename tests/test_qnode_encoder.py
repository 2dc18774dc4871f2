"""The node encoder every tree build shares (nodebleed_b200/csrc/qnode.h,
host and device): tests/qnode_check.cpp compiled with g++ and run over
random nodes with extreme scales, infinite bounds, empty and NaN children.
It checks conservative planes, stored exponents and a slot for every child;
an encoder that never ends fails by the timeout.  tests/slots_warp_check.cpp
restates the warp form of the slot assignment (one CTA TLAS build) with 32
emulated lanes and compares it with the sequential one."""

import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(tmp_path, src, count):
    exe = tmp_path / src.replace(".cpp", "")
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-Wall",
                        "-I", os.path.join(ROOT, "nodebleed_b200", "csrc"),
                        os.path.join(ROOT, "tests", src),
                        "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe), str(count)], capture_output=True,
                       text=True, timeout=240)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout


@pytest.mark.timeout(300)
def test_qnode_encoder_random_and_extreme_nodes(tmp_path):
    _run(tmp_path, "qnode_check.cpp", 200000)


@pytest.mark.timeout(300)
def test_warp_slot_assignment_matches_sequential(tmp_path):
    _run(tmp_path, "slots_warp_check.cpp", 300000)

"""The device DFA builder's algorithm, restated on the CPU, against the host regex compiler.

`tests/c/dfa_subset_emulation.cpp` runs the steps of k_dfa_build (dfa_build.cu) one
(state, value) pair at a time over the NFA tables the host exports for the device
(mkre::nfa_tables): frontiers, chunks of 4096 pairs looked up against the states found so far,
new sets numbered in (state, value) order.  For every pattern of the device test's corpus, at
the default state limit and at limits around and below each DFA's size, its status, error
text, state count and table bytes must equal mk_regex_compile's.  This pins the tables and the
numbering without a GPU; `test_gpu_dfa_device.py` checks the kernel itself."""
import os
import shutil
import subprocess

import pytest

import meikey_b200 as mk
import test_gpu_dfa_device

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not installed")
def test_emulated_subset_construction_equals_host(tmp_path):
    exe = tmp_path / "dfa_subset_emulation"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "dfa_subset_emulation.cpp"),
                    os.path.join(ROOT, "meikey_b200", "csrc", "regex.cpp"), "-o", str(exe)], check=True)
    lines = []
    for pattern, cs in test_gpu_dfa_device._corpus():
        lines.append(f"{1 if cs else 0} 16384 {pattern}")
        try:
            states = mk.Needle.regex(pattern, cs).states
        except mk.GpuError:
            continue
        for limit in (states - 1, states, 2 + states // 2):
            if limit >= 2:
                lines.append(f"{1 if cs else 0} {limit} {pattern}")
    lines.append("1 16384 " + "a.{9}b.{2}[0-9]")  # 3457 states: frontiers of several chunks
    out = subprocess.run([str(exe)], input="\n".join(lines) + "\n", capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-3000:]
    last = out.stdout.strip().splitlines()[-1]
    n, built = int(last.split()[0]), int(last.split()[2])
    assert n == len(lines) and built > 300, last

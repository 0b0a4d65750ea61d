"""The header compiles as C and the library links and answers from a C program (gcc), for
the entry points that need no device."""
import json
import os
import shutil
import subprocess

import pytest

from conftest import GOLDEN, ROOT


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not installed")
def test_c_program_against_header(tmp_path):
    lib_dir = os.path.join(ROOT, "meikey_b200")
    exe = tmp_path / "abi_host"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "abi_host.c"), "-o", str(exe), "-L", lib_dir, "-lmeikey_b200",
                    "-lm", f"-Wl,-rpath,{lib_dir}"], check=True)
    vec = json.load(open(os.path.join(GOLDEN, "rfc8032.json")))
    pk = [v for v in vec if v["name"] in ("1", "TEST 1")][0]["public"] if any(
        v["name"] in ("1", "TEST 1") for v in vec) else vec[0]["public"]
    out = subprocess.run([str(exe), pk], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.count("ok ") == 8


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not installed")
def test_hit_order_radix_sort(tmp_path):
    """The library's host-side ordering of candidate hits (radix sort on index, then needle)
    equals a comparison sort on random, duplicate, constant, wide and nearly sorted sets."""
    exe = tmp_path / "hitsort_check"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "hitsort_check.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.count("ok ") == 11

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


@pytest.mark.gpu
@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not installed")
def test_c_program_drives_a_gpu_job(tmp_path, golden, oracle):
    """A C program (tests/c/abi_gpu.c) runs mk_ctx_create -> mk_job_prepare -> mk_job_launch ->
    mk_job_hits -> mk_job_first_matches with every golden text needle in one job: each
    needle's candidates over indices 0..65535 are the golden set (the reference matcher's),
    and each first match is the lowest candidate whose full key matches, with the oracle's key."""
    lib_dir = os.path.join(ROOT, "meikey_b200")
    exe = tmp_path / "abi_gpu"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-O1", "-D_POSIX_C_SOURCE=200809L", "-I",
                    os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "c", "abi_gpu.c"), "-o", str(exe),
                    "-L", lib_dir, "-lmeikey_b200", f"-Wl,-rpath,{lib_dir}"], check=True)
    cases = [c for c in golden["search"] if c["mode"] != 2]
    args = [f"{c['needle']}:{int(c['fold'])}:{c['mode']}" for c in cases]
    out = subprocess.run([str(exe), golden["chacha_key"]] + args, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = out.stdout.split("\n")
    hits = {int(ln.split()[1]): [int(x) for x in ln.split()[2:]] for ln in lines if ln.startswith("hits ")}
    firsts = {int(ln.split()[1]): ln.split()[2:] for ln in lines if ln.startswith("first ")}
    key = bytes.fromhex(golden["chacha_key"])
    for k, c in enumerate(cases):
        assert hits[k] == c["hits"], c["needle"]
        status, index, pk = int(firsts[k][0]), int(firsts[k][1]), bytes.fromhex(firsts[k][2])
        nb = c["needle"].lower().encode() if c["fold"] else c["needle"].encode()  # folded needles are lowercase
        lowest = next((i for i in c["hits"] if oracle.match(oracle.derive(key, 0, i, 1, threads=1), nb, len(nb),
                                                            c["fold"], c["mode"], False)), None)
        if lowest is not None:  # the lowest confirmed candidate of the golden range
            assert status == 0 and index == lowest and pk == oracle.derive(key, 0, index, 1), c["needle"]

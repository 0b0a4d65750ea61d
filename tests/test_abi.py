"""The C-ABI library loads and exports every entry point that include/meikey_b200.h
declares; argument checks and the no-device path return status codes (no GPU needed)."""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "meikey_b200.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^MK_API\s+[\w\s\*]+?\b(mk_\w+)\(", text, re.M)))


def test_header_declares_the_engine_surface():
    names = declared()
    for must in ["mk_ctx_create", "mk_ctx_destroy", "mk_job_prepare", "mk_job_launch", "mk_job_hits",
                 "mk_keys_per_iter", "mk_derive", "mk_last_error"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    from meikey_b200 import _lib
    lib = _lib.load()
    raw = ctypes.CDLL(_lib.LIB_PATH)
    bound = {n for n, _, _ in _lib.SIGNATURES}
    for name in declared():
        assert hasattr(raw, name), f"{name} declared but not exported"
        assert name in bound, f"{name} not bound in meikey_b200/_lib.py"
    assert lib.mk_abi_version() == 2


STRUCTS = {"Options": "mk_options", "NeedleC": "mk_needle", "HitC": "mk_hit", "InfoC": "mk_info",
           "TuneEntryC": "mk_tune_entry", "SearchConfigC": "mk_search_config", "OutcomeC": "mk_outcome",
           "ServerOptionsC": "mk_server_options", "JobResultC": "mk_job_result"}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not installed")
def test_struct_layouts_match_header(tmp_path):
    """Every ctypes mirror has the size and field offsets the C compiler gives the header's struct."""
    from meikey_b200 import _lib
    src = ['#include <stddef.h>', '#include <stdio.h>', '#include "meikey_b200.h"', 'int main(void) {']
    for py, c in STRUCTS.items():
        src.append(f'    printf("{py} size %zu\\n", sizeof({c}));')
        for f, _ in getattr(_lib, py)._fields_:
            src.append(f'    printf("{py} {f} %zu\\n", offsetof({c}, {f}));')
    src.append("    return 0;\n}")
    (tmp_path / "layout.c").write_text("\n".join(src))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(tmp_path / "layout.c"), "-o", str(exe)],
                   check=True)
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        py, field, value = line.split()
        cls = getattr(_lib, py)
        got = ctypes.sizeof(cls) if field == "size" else getattr(cls, field).offset
        assert got == int(value), (py, field)


def test_bad_arguments_return_status():
    from meikey_b200 import _lib
    lib = _lib.load()
    assert lib.mk_ctx_create(0, None, None) == _lib.ERR_BAD_ARG
    assert lib.mk_ctx_info(None, None) == _lib.ERR_BAD_ARG
    assert lib.mk_job_launch(None, 0, 1, None, None) == _lib.ERR_BAD_ARG
    assert lib.mk_job_hits(None, None, 0, None, None) == _lib.ERR_BAD_ARG
    assert lib.mk_ctx_sync(None) == _lib.ERR_BAD_ARG
    assert lib.mk_keys_per_iter(None) == 0
    buf = ctypes.create_string_buffer(8)
    assert lib.mk_last_error(None, buf, 8) == _lib.OK and buf.value == b""


def test_no_device_path_reports_an_error():
    from meikey_b200 import _lib
    import meikey_b200 as mk
    lib = _lib.load()
    if lib.mk_device_count() > 0:
        pytest.skip("a CUDA device is present")
    ptr = ctypes.c_void_p()
    st = lib.mk_ctx_create(0, None, ctypes.byref(ptr))
    assert st in (_lib.ERR_NO_DEVICE, _lib.ERR_DRIVER_NOT_FOUND)
    assert not ptr
    with pytest.raises(mk.GpuError) as e:
        mk.Context()
    assert e.value.status in (_lib.ERR_NO_DEVICE, _lib.ERR_DRIVER_NOT_FOUND)


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    """There is no CPU fallback: without the CUDA build the package refuses to run."""
    from meikey_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    with pytest.raises(OSError):
        _lib.load()


def test_tune_space_candidates_are_context_options():
    """Every candidate of the tuner's space is a valid keyword set of Context (so that
    Context(**best) works), hashing warps appear only with block 512 and 8 or 16 keys per
    thread, and never together with the rotating inversion."""
    import inspect
    from meikey_b200.engine import Context, tune_space
    params = set(inspect.signature(Context.__init__).parameters)
    space = tune_space(rows=(11, 12), hash_warps=(0, 4), inverter_rotates=(0, 1))
    assert space and all(set(c) <= params for c in space)
    assert all(c["block"] == 512 and c["keys_per_thread"] in (8, 16) for c in space if c["hash_warps"])
    assert not any(c["hash_warps"] and c["inverter_rotates"] for c in space)
    assert {(c["hash_warps"], c["inverter_rotates"]) for c in space} == {(0, 0), (0, 1), (4, 0)}

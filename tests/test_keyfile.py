"""OpenSSH output (mk_openssh_public / mk_openssh_private), no device needed: the public line
of RFC 8032 TEST 1 as the reference's own test states it (src/model/key.rs:165-176), the
private file byte for byte against a restatement of the openssh-key-v1 layout from
OpenSSH's PROTOCOL.key, and both read back by Python `cryptography`."""
import base64
import json
import os
import struct

import pytest

import meikey_b200 as mk
from meikey_b200.engine import openssh_private, openssh_public
from conftest import GOLDEN


def _test1():
    vec = json.load(open(os.path.join(GOLDEN, "rfc8032.json")))
    v = [x for x in vec if x["name"] in ("1", "TEST 1")] or vec[:1]
    return bytes.fromhex(v[0]["secret"]), bytes.fromhex(v[0]["public"])


def test_public_line_rfc8032_test1():
    _, pk = _test1()
    want = "ssh-ed25519 AAAAC3NzaC1lZDI1NTE5AAAAINdamAGCsQq31Uv+08lkBzoO4XLz2qYjJa8CGmj3B1Ea"
    assert openssh_public(pk) == want
    assert openssh_public(pk, "wakokara") == want + " wakokara"


def _string(b):
    return struct.pack(">I", len(b)) + b


def _spec_private(seed, pk, comment, checkint):
    blob = _string(b"ssh-ed25519") + _string(pk)
    priv = struct.pack(">II", checkint, checkint) + _string(b"ssh-ed25519") + _string(pk) + _string(seed + pk)
    priv += _string(comment.encode())
    priv += bytes(range(1, 1 + (-len(priv)) % 8))
    body = b"openssh-key-v1\0" + _string(b"none") + _string(b"none") + _string(b"") + struct.pack(">I", 1)
    body += _string(blob) + _string(priv)
    b64 = base64.b64encode(body).decode()
    lines = [b64[i:i + 70] for i in range(0, len(b64), 70)]
    return "-----BEGIN OPENSSH PRIVATE KEY-----\n" + "\n".join(lines) + "\n-----END OPENSSH PRIVATE KEY-----\n"


@pytest.mark.parametrize("comment,checkint", [("", 0), ("wakokara@example", 0x01020304), ("和光から", 0xdeadbeef)])
def test_private_file_layout(comment, checkint):
    seed, pk = _test1()
    assert openssh_private(seed, comment, checkint) == _spec_private(seed, pk, comment, checkint)


def test_files_load_in_cryptography(oracle):
    from cryptography.hazmat.primitives import serialization
    seed = oracle.seed(bytes(range(32)), 0, 77)
    pk = oracle.pubkey(seed)
    key = serialization.load_ssh_private_key(openssh_private(seed, "c", 7).encode(), password=None)
    raw = key.private_bytes(serialization.Encoding.Raw, serialization.PrivateFormat.Raw,
                            serialization.NoEncryption())
    assert raw == seed
    pub = serialization.load_ssh_public_key(openssh_public(pk, "c").encode())
    assert pub.public_bytes(serialization.Encoding.Raw, serialization.PublicFormat.Raw) == pk


@pytest.mark.parametrize("bad", ["a\nb", "a\rb"])
def test_comment_with_line_break_rejected(bad):
    _, pk = _test1()
    with pytest.raises(mk.GpuError):
        openssh_public(pk, bad)

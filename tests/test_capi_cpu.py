"""CPU checks of the C ABI: the library loads, exports every function declared in
include/*.h, and rejects bad arguments on the host (no GPU calls are made)."""
import ctypes
import glob
import os
import re

import pytest

from ever_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(ever_\w+)\s*\(", src))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = N.load()
    declared = _declared()
    assert len(declared) >= 9
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) <= set(N.SIGNATURES), set(declared) - set(N.SIGNATURES)


def test_abi_version_and_workspace_sizes():
    lib = N.load()
    assert lib.ever_abi_version() == 2
    a = lib.ever_scene_workspace_bytes(1000, 1)
    b = lib.ever_scene_workspace_bytes(1000, 16)
    assert 0 < a < b
    assert lib.ever_scene_workspace_bytes(-1, 1) == 0
    assert lib.ever_backward_workspace_bytes(1000, 16) >= 1000 * (16 + 48) * 4


def test_host_validation_errors():
    lib = N.load()
    sc = N.EverScene()
    rc = lib.ever_scene_build(None, None, None, None, None, 10, 1, None, 0, ctypes.byref(sc), None)
    assert rc == 1 and b"null" in lib.ever_last_error()
    rc = lib.ever_scene_build(None, None, None, None, None, 10, 17, None, 0, ctypes.byref(sc), None)
    assert rc == 1 and b"sh_coeffs" in lib.ever_last_error()
    rc = lib.ever_scene_build(None, None, None, None, None, -5, 1, None, 0, ctypes.byref(sc), None)
    assert rc == 1
    args = N.EverTraceArgs()
    args.max_iters, args.sh_degree = 10, 5
    out = N.EverForwardOut()
    sc.num_prims, sc.sh_coeffs = 0, 16
    rc = lib.ever_trace_forward(ctypes.byref(sc), None, None, 0, ctypes.byref(args), None, None, ctypes.byref(out),
                                None)
    assert rc == 1 and b"sh_degree" in lib.ever_last_error()
    rc = lib.ever_trace_forward(ctypes.byref(sc), None, None, 4, ctypes.byref(args), None, None, ctypes.byref(out),
                                None)
    assert rc == 1


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from ever_b200 import build as B
    monkeypatch.setattr(B, "LIB", str(tmp_path / "nope.so"))
    monkeypatch.setattr(B, "up_to_date", lambda: False)
    monkeypatch.setattr(B, "build", lambda *a, **k: (_ for _ in ()).throw(RuntimeError("no nvcc")))
    monkeypatch.setattr(N, "_lib", None)
    with pytest.raises(RuntimeError, match="missing"):
        N.load()
    monkeypatch.setattr(N, "_lib", None)

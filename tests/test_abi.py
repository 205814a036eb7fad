"""The C ABI library: loads, exports every declared symbol, reports errors."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(awsem_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(gpu_lib):
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(gpu_lib, n)]
    assert not missing, missing


def test_parse_errors_carry_reference_messages(gpu_lib, tmp_path):
    from awsemmd_b200 import engine

    h = C.c_void_p()
    rc = gpu_lib.awsem_create_from_files(str(tmp_path).encode(), b"data", b"nope.coeff", b"seq", b"2 3.5 3.5", b"",
                                         0, 0, C.byref(h))
    assert rc == -2
    assert b"Coefficient file was not found" in gpu_lib.awsem_last_error()
    assert not h.value
    rc = gpu_lib.awsem_create_from_files(str(tmp_path).encode(), b"data", b"c", b"s", b"2 3.5 3.5", b"", 7, 0,
                                         C.byref(h))
    assert rc == -1
    with pytest.raises(engine.AwsemError):
        engine.AwsemSystem({"workdir": str(tmp_path), "data": "d", "coeff": "missing", "seq": "s",
                            "pair_style": "2 3.5 3.5"})


def test_unsupported_sections_are_rejected(gpu_lib, tmp_path):
    (tmp_path / "c").write_text("[Chain]\n1 1 1\n2 2 2\n\n[Excluded]\n5.0 3.0\n5.0 4.0\n")
    h = C.c_void_p()
    rc = gpu_lib.awsem_create_from_files(str(tmp_path).encode(), b"d", b"c", b"s", b"2 3.5 3.5", b"", 0, 0,
                                         C.byref(h))
    assert rc == -2
    assert b"[Excluded]" in gpu_lib.awsem_last_error()


def test_disabled_sections_are_ignored(gpu_lib, tmp_path):
    """A trailing '-' disables a section (it no longer matches), as in the reference."""
    (tmp_path / "c").write_text("[AMH-Go]-\n1.0\n1\n8.0\n0\n")
    h = C.c_void_p()
    rc = gpu_lib.awsem_create_from_files(str(tmp_path).encode(), b"d", b"c", b"missing.seq", b"2 3.5 3.5", b"", 0,
                                         0, C.byref(h))
    assert rc == -2
    assert b"Sequence file was not found" in gpu_lib.awsem_last_error()

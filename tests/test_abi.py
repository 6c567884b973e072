"""The C ABI library loads and exports every entry point that
include/*.h declares (no compute calls: this runs without a GPU)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^\s*(?:int32_t|int64_t|void|const char\s*\*)\s*\**\s*(\w+)\s*\(", text, flags=re.M)
    return names


def test_header_declares_the_entry_points():
    names = declared()
    for n in ["mdrtNbCreate", "mdrtNbBuild", "mdrtNbForce", "mdrtPmeSetup", "mdrtNbEnergies",
              "mdrtCudaFFTForward3DF32", "mdrtCudaFFTBackward3DF32", "mdrtNbGroupsBuffer"]:
        assert n in names


def test_library_exports_every_declared_symbol():
    from mdir_b200 import _lib
    lib = ctypes.CDLL(str(_lib.LIBRARY))
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python loader binds a signature for each of them
    assert set(declared()) <= set(_lib.SIGNATURES)


def test_version_and_status_strings_need_no_device():
    from mdir_b200 import _lib
    lib = _lib.lib()
    assert lib.mdrtNbVersion() == 1
    assert b"reach" in lib.mdrtNbStatusString(_lib.INVALID_BOX)


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    from mdir_b200 import _lib
    monkeypatch.setattr(_lib, "LIBRARY", tmp_path / "absent.so")
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(ImportError):
        _lib.lib()

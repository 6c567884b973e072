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
    assert lib.mdrtNbVersion() == 2
    assert b"reach" in lib.mdrtNbStatusString(_lib.INVALID_BOX)


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    from mdir_b200 import _lib
    monkeypatch.setattr(_lib, "LIBRARY", tmp_path / "absent.so")
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(ImportError):
        _lib.lib()


def header_constants():
    """name -> value of every enum constant that include/mdrt_nb.h defines."""
    text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "mdrt_nb.h").read_text(), flags=re.S)
    out = {}
    for body in re.findall(r"enum\s+\w+\s*\{(.*?)\}", text, flags=re.S):
        for name, value in re.findall(r"(MDRT_NB_\w+)\s*=\s*(\d+)u?", body):
            out[name] = int(value)
    return out


def test_python_constants_are_the_header_values():
    """The loader's status codes, flags and slots carry the header's values."""
    from mdir_b200 import _lib as L
    h = header_constants()
    pairs = {
        "OK": "MDRT_NB_OK", "GROW": "MDRT_NB_GROW", "NAN_POSITION": "MDRT_NB_NAN_POSITION",
        "INVALID_BOX": "MDRT_NB_INVALID_BOX", "CUDA_ERROR": "MDRT_NB_CUDA_ERROR", "TIMEOUT": "MDRT_NB_TIMEOUT",
        "INVALID_ARGUMENT": "MDRT_NB_INVALID_ARGUMENT", "UNSUPPORTED": "MDRT_NB_UNSUPPORTED",
        "OVERFLOW": "MDRT_NB_OVERFLOW", "NOT_BUILT": "MDRT_NB_NOT_BUILT",
        "ENERGY": "MDRT_NB_ENERGY", "ACCUMULATE": "MDRT_NB_ACCUMULATE", "POTENTIAL": "MDRT_NB_POTENTIAL",
        "NO_PAIRS": "MDRT_NB_NO_PAIRS", "NO_PME": "MDRT_NB_NO_PME", "NO_EXCLUDED": "MDRT_NB_NO_EXCLUDED",
        "GRAPH": "MDRT_NB_GRAPH",
        "E_LJ": "MDRT_NB_E_LJ", "E_COULOMB": "MDRT_NB_E_COULOMB", "E_EXCLUDED": "MDRT_NB_E_EXCLUDED",
        "E_RECIPROCAL": "MDRT_NB_E_RECIPROCAL", "W_PAIR": "MDRT_NB_W_PAIR",
        "W_RECIPROCAL": "MDRT_NB_W_RECIPROCAL", "E_COUNT": "MDRT_NB_E_COUNT",
        "SIZE_PLACES": "MDRT_NB_SIZE_PLACES", "SIZE_LONGEST": "MDRT_NB_SIZE_LONGEST",
        "SIZE_UNITS": "MDRT_NB_SIZE_UNITS", "SIZE_EXCL_WIDE": "MDRT_NB_SIZE_EXCL_WIDE",
        "SIZE_NAN": "MDRT_NB_SIZE_NAN", "SIZE_OVERFLOW": "MDRT_NB_SIZE_OVERFLOW",
        "SIZE_GROUPS": "MDRT_NB_SIZE_GROUPS", "SIZE_ENTRIES": "MDRT_NB_SIZE_ENTRIES",
        "SIZE_COUNT": "MDRT_NB_SIZE_COUNT",
        "SLOT_ORDER": "MDRT_NB_GROUPS_ORDER", "SLOT_COUNTS": "MDRT_NB_GROUPS_COUNTS",
        "SLOT_ENTRIES": "MDRT_NB_GROUPS_ENTRIES", "SLOT_UNITS": "MDRT_NB_GROUPS_UNITS",
        "SLOT_SHIFTS": "MDRT_NB_GROUPS_SHIFTS", "SLOT_INNER_ENTRIES": "MDRT_NB_GROUPS_INNER_ENTRIES",
        "SLOT_INNER_COUNTS": "MDRT_NB_GROUPS_INNER_COUNTS", "SLOT_PLACED": "MDRT_NB_GROUPS_PLACED",
        "SLOT_PLACE_OF": "MDRT_NB_GROUPS_PLACE_OF",
        "TUNE_PAIR_BLOCKS_PER_SM": "MDRT_NB_TUNE_PAIR_BLOCKS_PER_SM",
        "TUNE_SEARCH_WARPS": "MDRT_NB_TUNE_SEARCH_WARPS", "TUNE_PAIR_SMS": "MDRT_NB_TUNE_PAIR_SMS",
        "GRAD_PRODUCT": "MDRT_NB_GRAD_PRODUCT", "GRAD_ENERGY": "MDRT_NB_GRAD_ENERGY",
    }
    for py, c in pairs.items():
        assert c in h, c
        assert getattr(L, py) == h[c], (py, getattr(L, py), c, h[c])

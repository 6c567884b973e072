"""Loads libmdrt_nb.so (include/mdrt_nb.h) with ctypes.

The library is built in-tree by `python __graft_entry__.py` (build()) or
`make -C mdir_b200/csrc`.  There is no fallback: a missing library raises."""

import ctypes
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "libmdrt_nb.so"

# Status codes, flags and slots (include/mdrt_nb.h).
OK, GROW, NAN_POSITION, INVALID_BOX, CUDA_ERROR, TIMEOUT, INVALID_ARGUMENT, UNSUPPORTED, \
    OVERFLOW, NOT_BUILT = range(10)
ENERGY, ACCUMULATE, POTENTIAL, NO_PAIRS, NO_PME, NO_EXCLUDED, GRAPH, PRUNE = 1, 2, 4, 8, 16, 32, 64, 128
TUNE_PAIR_BLOCKS_PER_SM, TUNE_SEARCH_WARPS, TUNE_PAIR_SMS, TUNE_FUSED_PRUNE, TUNE_STAGING_DEPTH = 0, 1, 2, 3, 4
TUNE_PME_FFT = 5
TUNE_PME_SPREAD = 6
TUNE_FRAME_GRAPHS = 7
E_LJ, E_COULOMB, E_EXCLUDED, E_RECIPROCAL, W_PAIR, W_RECIPROCAL, E_COUNT = 0, 1, 2, 3, 4, 10, 16
SIZE_PLACES, SIZE_LONGEST, SIZE_UNITS, SIZE_EXCL_WIDE, SIZE_NAN, SIZE_OVERFLOW, SIZE_GROUPS, \
    SIZE_ENTRIES, SIZE_COUNT = range(9)
SLOT_ORDER, SLOT_COUNTS, SLOT_ENTRIES, SLOT_UNITS, SLOT_SHIFTS, SLOT_PLACED, SLOT_PLACE_OF = \
    0, 1, 2, 4, 6, 15, 16
SLOT_INNER_ENTRIES, SLOT_INNER_COUNTS = 7, 9
GRAD_PRODUCT, GRAD_ENERGY = 0, 1
LEAP_FROG, VELOCITY_VERLET = 0, 1

_lib = None

# name -> (restype, argtypes); every symbol that include/mdrt_nb.h declares
_i32, _i64, _u32, _d, _p = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32, ctypes.c_double, ctypes.c_void_p
SIGNATURES = {
    "mdrtNbVersion": (_i32, []),
    "mdrtNbStatusString": (ctypes.c_char_p, [_i32]),
    "mdrtNbCreate": (_i32, [ctypes.POINTER(_p), _i32, _i64]),
    "mdrtNbDestroy": (_i32, [_p]),
    "mdrtNbSetParticles": (_i32, [_p, _p, _p, _i32, _p, _p]),
    "mdrtNbSetExclusions": (_i32, [_p, _p, _p]),
    "mdrtNbSetInteraction": (_i32, [_p, _d, _d, _d, _d, _i32, _i32, _d]),
    "mdrtNbSetDeterministic": (_i32, [_p, _i32]),
    "mdrtNbSetPrunedReach": (_i32, [_p, _d]),
    "mdrtNbSetTuning": (_i32, [_p, _i32, _i32]),
    "mdrtNbPrune": (_i32, [_p, _p, _p, _p]),
    "mdrtPmeSetup": (_i32, [_p, _i32, _i32, _i32, _i32]),
    "mdrtNbBuild": (_i32, [_p, _p, _i64, _p, _d, _p, _p]),
    "mdrtNbForce": (_i32, [_p, _p, _p, _u32, _p, _p]),
    "mdrtNbBuildTriclinic": (_i32, [_p, _p, _i64, _p, _d, _p, _p]),
    "mdrtNbForceTriclinic": (_i32, [_p, _p, _p, _u32, _p, _p]),
    "mdrtNbEnergies": (_i32, [_p, _p, _p]),
    "mdrtNbConstants": (_i32, [_p, _p, _i32, _p]),
    "mdrtPmePotential": (_i32, [_p, _p, _p]),
    "mdrtNbDisplacement": (_i32, [_p, _p, _i64, _p, _p, _p]),
    "mdrtNbDisplacementStart": (_i32, [_p, _p, _i64, _p, _p]),
    "mdrtNbDisplacementResult": (_i32, [_p, _p]),
    "mdrtNbParameterGradient": (_i32, [_p, _p, _p, _p, _i32, _p, _p, _p]),
    "mdrtNbParameterGradientPotential": (_i32, [_p, _p, _p, _p, _i32, _p, _p, _p, _p]),
    "mdrtPmePotentialGrid": (_i32, [_p, _p, _p]),
    "mdrtNbForceFrames": (_i32, [_p, _p, _i64, _i64, _p, _u32, _p, _i64, _p, _i64, _p]),
    "mdrtNbParameterGradientFrames": (_i32, [_p, _p, _i64, _i64, _p, _p, _i64, _i32, _p, _i64, _p, _p, _p]),
    "mdrtNbGroupsBuffer": (_i32, [_p, _i32, ctypes.POINTER(_p), ctypes.POINTER(_i64)]),
    "mdrtNbGroupsInfo": (_i32, [_p, ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    "mdrtNbFrameGraphInfo": (_i32, [_p, ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    "mdrtNbStatus": (_i32, [_p, _p, _i32, ctypes.POINTER(_i32)]),
    "mdrtNbTimeKernels": (_i32, [_p, _p, _p, _i32, _p, _p]),
    "mdrtMdCreate": (_i32, [ctypes.POINTER(_p), _p, _p, _i64, _p, _d, _d]),
    "mdrtMdDestroy": (_i32, [_p]),
    "mdrtMdSetThermostat": (_i32, [_p, _d, _d, ctypes.c_uint64]),
    "mdrtMdSetLookahead": (_i32, [_p, _d]),
    "mdrtMdSetIntegrator": (_i32, [_p, _i32]),
    "mdrtMdBuild": (_i32, [_p, _p, _p, _p]),
    "mdrtMdRefresh": (_i32, [_p, _p, _p, _p, _p]),
    "mdrtMdRun": (_i32, [_p, _p, _p, _p, _d, _i64, _i32, _p]),
    "mdrtMdThermo": (_i32, [_p, _p, _p]),
    "mdrtMdForces": (_i32, [_p, ctypes.POINTER(_p)]),
    "mdrtNbExcludedNoAlloc": (_i32, [_p, _p, _p, _i64, _p, _d, _d, _p, _p, _p]),
    "mdrtNbBatchCreate": (_i32, [ctypes.POINTER(_p), _i32, _i32, _p]),
    "mdrtNbBatchDestroy": (_i32, [_p]),
    "mdrtNbBatchSetParticles": (_i32, [_p, _p, _p, _i32, _p, _p]),
    "mdrtNbBatchSetExclusions": (_i32, [_p, _p, _p]),
    "mdrtNbBatchSetInteraction": (_i32, [_p, _d, _d, _d, _d]),
    "mdrtNbBatchPmeSetup": (_i32, [_p, _p, _i32]),
    "mdrtNbBatchSetTuning": (_i32, [_p, _i32, _i32]),
    "mdrtNbBatchBuild": (_i32, [_p, _p, _p, _p, _p]),
    "mdrtNbBatchForce": (_i32, [_p, _p, _u32, _p, _p]),
    "mdrtNbBatchEnergies": (_i32, [_p, _p, _p]),
    "mdrtNbBatchConstants": (_i32, [_p, _p]),
    "mdrtNbBatchAutotune": (_i32, [_p, _p, _p, _p, _p]),
    "mdrtCudaFFTForward3DF32": (_i32, [_p, _p, _i64, _i64, _i64, _p]),
    "mdrtCudaFFTBackward3DF32": (_i32, [_p, _p, _i64, _i64, _i64, _p]),
    # MDIR's own names (memref descriptors by pointer)
    "mdrtGroupsCreate": (_i64, [_i64, _i64]),
    "_mlir_ciface_mdrtGroupsBuffer": (None, [_p, _i64, _i64]),
    "mdrtGroupsGrow": (None, [_i64, _i64, _i64]),
    "mdrtGroupsBuilt": (_i64, [_i64]),
    "mdrtGroupsReserveBlockOf": (None, [_i64, _i64]),
    "_mlir_ciface_mdrtGroupsPlaced": (None, [_p, _i64]),
    "mdrtGroupsDestroy": (_i32, [_i64]),
    "mdrtGroupsLastStatus": (_i32, []),
    "mdrtNbGroupsExport": (_i32, [_p, _i64, _p]),
    "mdrtNbSetAbiStream": (_i32, [_p]),
    "_mlir_ciface_mdrtCudaFFTForward3DF32": (None, [_p, _p, _i64, _i64, _i64]),
    "_mlir_ciface_mdrtCudaFFTBackward3DF32": (None, [_p, _p, _i64, _i64, _i64]),
    "_mlir_ciface_mdrtCudaFFTGaussianBackwardF32": (None, [_p, _p, _p, _i64, _i64, _i64]),
}


class MemRef1D(ctypes.Structure):
    """MLIR's descriptor of a buffer of rank 1 (mdrtMemRef1D)."""
    _fields_ = [("allocated", _p), ("aligned", _p), ("offset", _i64), ("size", _i64), ("stride", _i64)]


class MemRef2D(ctypes.Structure):
    """MLIR's descriptor of a buffer of rank 2 (mdrtMemRef2D)."""
    _fields_ = [("allocated", _p), ("aligned", _p), ("offset", _i64), ("sizes", _i64 * 2), ("strides", _i64 * 2)]


# MDIR's slot table of a groups registry (mdrtGroupsSlot)
GROUPS_ORDER, GROUPS_COUNTS, GROUPS_ENTRIES, GROUPS_MASKS, GROUPS_UNIT_GROUPS, GROUPS_UNIT_ORDINALS, \
    GROUPS_SHIFTS, GROUPS_INNER_ENTRIES, GROUPS_INNER_MASKS, GROUPS_INNER_COUNTS, GROUPS_BLOCK_OF, \
    GROUPS_ACTIVE_UNITS, GROUPS_ACTIVE_COUNT = range(13)
GROUPS_PLACED, GROUPS_BUFFERS = 15, 24


class NativeError(RuntimeError):
    """A status code other than OK from the native library."""

    def __init__(self, status, call):
        self.status = status
        msg = lib().mdrtNbStatusString(status).decode() if _lib else str(status)
        super().__init__(f"{call}: {msg} (status {status})")


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            raise ImportError(f"{LIBRARY} is missing: build it with `python __graft_entry__.py` or "
                              "`make -C mdir_b200/csrc` (there is no CPU fallback)")
        handle = ctypes.CDLL(str(LIBRARY))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(status, call):
    if status != OK:
        raise NativeError(status, call)
    return status

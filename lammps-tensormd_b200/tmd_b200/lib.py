"""ctypes binding of libtmd_b200.so (declarations mirror include/tmd_b200.h)."""
from __future__ import annotations

import ctypes
from pathlib import Path

_PKG = Path(__file__).resolve().parent.parent
_LIB = None

TMD_OK = 0
ERRORS = {
    -1: "invalid argument", -2: "CUDA error", -3: "bad potential file",
    -4: "capacity exceeded", -5: "non-finite energy or force", -6: "I/O error",
    -7: "call order", -8: "timeout",
}

# (name, restype, argtypes) for every entry point of include/tmd_b200.h
_c_int, _c_long, _c_double, _vp = ctypes.c_int, ctypes.c_long, ctypes.c_double, ctypes.c_void_p
_pd = ctypes.POINTER(ctypes.c_double)
_pi = ctypes.POINTER(ctypes.c_int)
_pl = ctypes.POINTER(ctypes.c_long)
SIGNATURES = [
    ("tmd_model_load", _c_int, [ctypes.c_char_p, _c_int, ctypes.POINTER(_vp)]),
    ("tmd_model_free", None, [_vp]),
    ("tmd_model_info", _c_int, [_vp, _pd, _pi, _pi, _pi, _pi, _pi]),
    ("tmd_model_type_map", _c_int, [_vp, _pi, _pd]),
    ("tmd_system_create", _c_int, [_vp, _c_int, _c_double, ctypes.POINTER(_vp)]),
    ("tmd_system_free", None, [_vp]),
    ("tmd_system_set_box", _c_int, [_vp, _pd, _pi]),
    ("tmd_system_set_atoms", _c_int, [_vp, _c_int, _pd, _pi, _pd]),
    ("tmd_system_set_positions", _c_int, [_vp, _pd]),
    ("tmd_system_set_atoms_ghost", _c_int, [_vp, _c_int, _c_int, _pd, _pi]),
    ("tmd_system_get", _c_int, [_vp, _pd, _pd, _pd, _pi]),
    ("tmd_compute", _c_int, [_vp, _c_int, _c_int, _c_double, _pd, _pd, _pd, _pd, _pd]),
    ("tmd_nve_run", _c_int, [_vp, _c_int, _c_double, _c_int, _pd]),
    ("tmd_nvt_run", _c_int, [_vp, _c_int, _c_double, _c_double, _c_double, _c_double, _c_int,
                             _pd]),
    ("tmd_nvt_energy", _c_int, [_vp, _pd]),
    ("tmd_neighbor_list", _c_int, [_vp, _c_double, _pi, _pi, _c_long, _pl]),
    ("tmd_get_descriptors", _c_int, [_vp, _pd]),
    ("tmd_system_set_variant", _c_int, [_vp, _c_int, _c_int]),
    ("tmd_system_get_variant", _c_int, [_vp, _c_int, _pi]),
    ("tmd_system_autotune", _c_int, [_vp, _c_int, _c_int, _pd]),
    ("tmd_system_stream", _c_int, [_vp, ctypes.POINTER(_vp)]),
    ("tmd_system_launches", _c_long, [_vp]),
    ("tmd_system_rebuilds", _c_int, [_vp, _pl]),
    ("tmd_system_set_wait_probe", _c_int, [_vp, ctypes.c_longlong]),
    ("tmd_system_set_etemp", _c_int, [_vp, _c_double]),
    ("tmd_system_tdnp_energies", _c_int, [_vp, _pd, _pd]),
    ("tmd_fp32_peak", _c_int, [_c_int, _c_int, _pd]),
    ("tmd_profile_enable", _c_int, [_vp, _c_int]),
    ("tmd_profile_read", _c_int, [_vp, _pl, _pd, _c_int]),
    ("tmd_last_error", _c_int, [ctypes.c_char_p, _c_int]),
    ("tmd_batch_create", _c_int, [_vp, _c_int, _pi, _c_double, ctypes.POINTER(_vp)]),
    ("tmd_batch_free", None, [_vp]),
    ("tmd_batch_system", _c_int, [_vp, ctypes.POINTER(_vp)]),
    ("tmd_batch_set_cells", _c_int, [_vp, _pd, _pi]),
    ("tmd_batch_set_atoms", _c_int, [_vp, _pd, _pi, _pd]),
    ("tmd_batch_get", _c_int, [_vp, _pd, _pd, _pd, _pi]),
    ("tmd_batch_compute", _c_int, [_vp, _pd, _pd, _pd]),
    ("tmd_batch_nve_run", _c_int, [_vp, _c_int, _c_double, _c_int, _pd]),
    ("tmd_batch_nvt_run", _c_int, [_vp, _c_int, _c_double, _pd, _pd, _c_double, _c_int, _pd]),
    ("tmd_server_create", _c_int, [_vp, _c_int, _c_int, _c_double, _c_int,
                                   ctypes.POINTER(_vp)]),
    ("tmd_server_free", None, [_vp]),
    ("tmd_server_submit", _c_int, [_vp, _c_int, _c_int, _pd, _pi, _pd, _pd, _pi, _c_int,
                                   _c_double, _c_double, _pl]),
    ("tmd_server_wait", _c_int, [_vp, _c_long, _c_double, _pd, _pd, _pd, _pd, _pd, _pi, _pd]),
    ("tmd_server_stats", _c_int, [_vp, _pl, _pl, _pl, _pd, _pd]),
    ("tmd_server_timing", _c_int, [_vp, _pd]),
    ("tmd_server_create_bytes", _c_int, [_vp, ctypes.c_size_t, _c_double, _c_int, _c_double,
                                         _c_int, ctypes.POINTER(_vp)]),
    ("tmd_server_footprint", _c_int, [_vp, ctypes.POINTER(ctypes.c_size_t), _pi, _pi]),
    ("tmd_neighbor_list_noalloc", _c_int, [_vp, _c_int, _pd, _pi, _c_double, _c_int, _vp,
                                           _vp, _vp]),
]


class TmdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, 'error')} ({code}): {msg}")
        self.code = code


def library_path() -> Path:
    return _PKG / "libtmd_b200.so"


def load_library():
    """Load libtmd_b200.so; raises if it is missing (no fallback path)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    p = library_path()
    if not p.exists():
        raise ImportError(f"{p} is missing: run `python lammps-tensormd_b200/build.py`")
    lib = ctypes.CDLL(str(p))
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def check(rc: int):
    if rc != TMD_OK:
        buf = ctypes.create_string_buffer(1024)
        _LIB.tmd_last_error(buf, 1024)
        raise TmdError(rc, buf.value.decode(errors="replace"))

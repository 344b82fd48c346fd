"""ctypes binding of the C ABI in include/cellato_b200.h.

The shared library is built in-tree (``make -C 2026-cellato-smpt-journal_b200``)
into ``lib/libcellato_b200.so``.  There is no fallback: if the library is
missing, ``load()`` raises.
"""
from __future__ import annotations

import ctypes
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libcellato_b200.so")

OK, EINVAL, EINVAL_DIMS, ESMEM, ECUDA, ETIMEDOUT, ENOMEM, EUNSUPPORTED = range(8)
STATUS_NAMES = {0: "OK", 1: "EINVAL", 2: "EINVAL_DIMS", 3: "ESMEM", 4: "ECUDA", 5: "ETIMEDOUT",
                6: "ENOMEM", 7: "EUNSUPPORTED"}

LAYOUT_BIT_PLANES = 0
LAYOUT_TILED_BIT_PLANES = 1
LAYOUTS = {"bit_planes": LAYOUT_BIT_PLANES, "tiled_bit_planes": LAYOUT_TILED_BIT_PLANES}

# Every symbol include/cellato_b200.h declares (checked by the CPU tests).
EXPORTED = [
    "cellato_version", "cellato_last_error", "cellato_rule_from_name", "cellato_rule_name",
    "cellato_rule_planes", "cellato_rule_states", "cellato_rule_count", "cellato_rule_register",
    "cellato_plane_bytes", "cellato_check_dims",
    "cellato_planes_alloc", "cellato_planes_free", "cellato_planes_upload", "cellato_planes_download",
    "cellato_pack_cells", "cellato_unpack_cells",
    "cellato_run_simple", "cellato_run_temporal", "cellato_temporal_max_tile_rows",
    "cellato_device_wait_timeouts",
    "cellato_batch_create", "cellato_batch_launch", "cellato_batch_result_in_b", "cellato_batch_info",
    "cellato_batch_destroy", "cellato_batch_run_noalloc",
    "cellato_checksum", "cellato_rule_state_value", "cellato_fill_random", "cellato_diff_cells",
    "cellato_bit_array_bytes", "cellato_bit_array_to_planes", "cellato_planes_to_bit_array",
    "cellato_server_create", "cellato_server_submit_random", "cellato_server_submit_planes",
    "cellato_server_iterate", "cellato_server_poll", "cellato_server_planes", "cellato_server_release",
    "cellato_server_stats_get", "cellato_server_destroy", "cellato_server_submit_resume",
    "cellato_server_snapshot", "cellato_server_cancel",
]


class CellatoError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


BUILTIN_RULES = 10
MAX_RULES = 256


class Tune(ctypes.Structure):
    """cellato_tune: per-call kernel choices (0 = the library's choice)."""
    _fields_ = [("simple_kernel", ctypes.c_int), ("row_loop", ctypes.c_int), ("words_per_lane", ctypes.c_int),
                ("tile_rows", ctypes.c_int)]


class BatchGrid(ctypes.Structure):
    _fields_ = [("rule", ctypes.c_int), ("x_cells", ctypes.c_int), ("y_cells", ctypes.c_int),
                ("steps", ctypes.c_int), ("planes_a", ctypes.c_void_p * 8), ("planes_b", ctypes.c_void_p * 8)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("layout", ctypes.c_int), ("word_bits", ctypes.c_int), ("hbm_cap_bytes", ctypes.c_ulonglong),
                ("tile_budget", ctypes.c_int), ("chunk_rounds", ctypes.c_int), ("max_inflight", ctypes.c_int),
                ("k_per_rule", ctypes.POINTER(ctypes.c_int)), ("n_k_per_rule", ctypes.c_int)]


class ServerResult(ctypes.Structure):
    _fields_ = [("id", ctypes.c_longlong), ("rule", ctypes.c_int), ("x_cells", ctypes.c_int),
                ("y_cells", ctypes.c_int), ("steps", ctypes.c_int), ("result_in_b", ctypes.c_int),
                ("checksum", ctypes.c_ulonglong * 16), ("submit_s", ctypes.c_double), ("done_s", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    _fields_ = [("waiting", ctypes.c_longlong), ("running", ctypes.c_longlong), ("active", ctypes.c_longlong),
                ("completed_unpolled", ctypes.c_longlong), ("resident_bytes", ctypes.c_ulonglong),
                ("hbm_cap_bytes", ctypes.c_ulonglong), ("iterations", ctypes.c_longlong),
                ("kernel_launches", ctypes.c_longlong), ("cell_steps", ctypes.c_double),
                ("pool_trims", ctypes.c_longlong), ("memory_waits", ctypes.c_longlong)]


_lib = None
_vp = ctypes.c_void_p
_PP = ctypes.POINTER(ctypes.c_void_p)


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built; run `make -C {PKG_DIR}`")
    lib = ctypes.CDLL(path)
    lib.cellato_version.restype = ctypes.c_char_p
    lib.cellato_last_error.restype = ctypes.c_char_p
    lib.cellato_rule_from_name.argtypes = [ctypes.c_char_p]
    lib.cellato_rule_name.restype = ctypes.c_char_p
    lib.cellato_plane_bytes.restype = ctypes.c_size_t
    lib.cellato_plane_bytes.argtypes = [ctypes.c_int, ctypes.c_int]
    lib.cellato_planes_alloc.argtypes = [ctypes.c_int, ctypes.c_size_t, _PP]
    lib.cellato_planes_free.argtypes = [ctypes.c_int, _PP]
    lib.cellato_planes_upload.argtypes = [ctypes.c_int, _PP, _PP, ctypes.c_size_t, _vp]
    lib.cellato_planes_download.argtypes = [ctypes.c_int, _PP, _PP, ctypes.c_size_t, _vp]
    i = ctypes.c_int
    TP = ctypes.POINTER(Tune)
    lib.cellato_run_simple.argtypes = [i, i, i, _PP, _PP, i, i, i, i, TP, _vp, ctypes.POINTER(i)]
    lib.cellato_run_temporal.argtypes = [i, i, i, _PP, _PP, i, i, i, i, i, TP, _vp, ctypes.POINTER(i)]
    lib.cellato_temporal_max_tile_rows.argtypes = [i, i, i, i]
    lib.cellato_rule_register.argtypes = [_vp, ctypes.POINTER(i)]
    lib.cellato_batch_create.argtypes = [i, i, ctypes.POINTER(BatchGrid), i, ctypes.POINTER(ctypes.c_int), i,
                                         ctypes.POINTER(ctypes.c_void_p)]
    lib.cellato_batch_launch.argtypes = [_vp, _vp]
    lib.cellato_batch_result_in_b.argtypes = [_vp, i, ctypes.POINTER(i)]
    lib.cellato_batch_info.argtypes = [_vp, ctypes.POINTER(i), ctypes.POINTER(ctypes.c_longlong)]
    lib.cellato_batch_destroy.argtypes = [_vp]
    lib.cellato_batch_run_noalloc.argtypes = [i, i, ctypes.POINTER(BatchGrid), i, ctypes.POINTER(ctypes.c_int), i,
                                              _vp, ctypes.POINTER(ctypes.c_int)]
    lib.cellato_pack_cells.argtypes = [i, i, i, _vp, i, i, _PP, _vp]
    lib.cellato_unpack_cells.argtypes = [i, i, i, _PP, i, i, _vp, _vp]
    u32p = ctypes.POINTER(ctypes.c_uint32)
    ll = ctypes.c_longlong
    lib.cellato_checksum.argtypes = [i, i, i, _PP, i, i, _vp, _vp]
    lib.cellato_diff_cells.argtypes = [i, _PP, _PP, ctypes.c_size_t, _vp, _vp]
    lib.cellato_bit_array_bytes.argtypes = [i, i, i, i]
    lib.cellato_bit_array_bytes.restype = ctypes.c_size_t
    lib.cellato_bit_array_to_planes.argtypes = [i, i, _vp, i, i, i, i, _PP, _vp]
    lib.cellato_planes_to_bit_array.argtypes = [i, i, i, _PP, i, i, i, _vp, _vp]
    lib.cellato_rule_state_value.argtypes = [i, i, ctypes.POINTER(ll)]
    lib.cellato_fill_random.argtypes = [i, i, i, _PP, i, i, ctypes.c_ulonglong, u32p, i, _vp]
    lib.cellato_server_create.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(_vp)]
    lib.cellato_server_submit_random.argtypes = [_vp, i, i, i, i, ctypes.c_ulonglong, u32p, i, i,
                                                 ctypes.POINTER(ll)]
    lib.cellato_server_submit_planes.argtypes = [_vp, i, i, i, i, _PP, i, ctypes.POINTER(ll)]
    lib.cellato_server_iterate.argtypes = [_vp, ctypes.POINTER(i)]
    lib.cellato_server_poll.argtypes = [_vp, ctypes.POINTER(ServerResult), i, ctypes.POINTER(i)]
    lib.cellato_server_planes.argtypes = [_vp, ll, _PP]
    lib.cellato_server_release.argtypes = [_vp, ll]
    lib.cellato_server_stats_get.argtypes = [_vp, ctypes.POINTER(ServerStats)]
    lib.cellato_server_destroy.argtypes = [_vp]
    lib.cellato_server_submit_resume.argtypes = [_vp, i, i, i, i, i, _PP, i, ctypes.POINTER(ll)]
    lib.cellato_server_snapshot.argtypes = [_vp, ll, _PP, ctypes.POINTER(i), ctypes.POINTER(i)]
    lib.cellato_server_cancel.argtypes = [_vp, ll]
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != OK:
        raise CellatoError(status, load().cellato_last_error().decode())


def ptr_array(ptrs) -> ctypes.Array:
    arr = (ctypes.c_void_p * max(1, len(ptrs)))()
    for i, p in enumerate(ptrs):
        arr[i] = p
    return arr


def rule_id(name_or_id) -> int:
    if isinstance(name_or_id, int):
        return name_or_id
    r = load().cellato_rule_from_name(name_or_id.encode())
    if r < 0:
        raise ValueError(f"unknown automaton {name_or_id!r}")
    return r


def rule_planes(rule) -> int:
    return load().cellato_rule_planes(rule_id(rule))


def rule_states(rule) -> int:
    return load().cellato_rule_states(rule_id(rule))


def rule_name(rule) -> str:
    return load().cellato_rule_name(rule_id(rule)).decode()


def tune(simple_kernel: int = 0, row_loop: int = 0, words_per_lane: int = 0, tile_rows: int = 0) -> Tune:
    return Tune(simple_kernel, row_loop, words_per_lane, tile_rows)


def run_simple(rule, layout: int, word_bits: int, planes_a, planes_b, X: int, Y: int, t0: int, steps: int,
               stream: int = 0, simple_kernel: int = 0, words_per_lane: int = 0) -> int:
    """Returns 1 when the result ended in planes_b, else 0.  simple_kernel as
    cellato_tune (0 automatic, 1 register bands, 2 bulk-copy streaming, 3
    TMA-fed shared-memory tiles); words_per_lane: the TMA kernel's (0 its
    default)."""
    out = ctypes.c_int(0)
    t = tune(simple_kernel=simple_kernel, words_per_lane=words_per_lane)
    check(load().cellato_run_simple(rule_id(rule), layout, word_bits, ptr_array(planes_a), ptr_array(planes_b),
                                    X, Y, t0, steps, ctypes.byref(t), stream, ctypes.byref(out)))
    return out.value


def rule_count() -> int:
    return load().cellato_rule_count()


def rule_register(ops_ptr: int) -> int:
    """Registers a rule table (the address a custom_rule_ops<Config>() call
    returned in a caller-built library) and returns its rule id."""
    out = ctypes.c_int(-1)
    check(load().cellato_rule_register(ops_ptr, ctypes.byref(out)))
    return out.value


def temporal_max_tile_rows(rule, layout: int, word_bits: int, words_per_lane: int = 0) -> int:
    v = load().cellato_temporal_max_tile_rows(rule_id(rule), layout, word_bits, words_per_lane)
    if v < 0:
        check(-v)
    return v


def pack_cells(layout: int, word_bits: int, nb: int, cells_ptr: int, X: int, Y: int, planes, stream: int = 0) -> None:
    """Device uint8 cells (row-major) -> nb device planes."""
    check(load().cellato_pack_cells(layout, word_bits, nb, cells_ptr, X, Y, ptr_array(planes), stream))


def unpack_cells(layout: int, word_bits: int, nb: int, planes, X: int, Y: int, cells_ptr: int, stream: int = 0) -> None:
    """nb device planes -> device uint8 cells (row-major)."""
    check(load().cellato_unpack_cells(layout, word_bits, nb, ptr_array(planes), X, Y, cells_ptr, stream))


def device_wait_timeouts() -> int:
    """Bounded device waits that gave up since the last call (0 when healthy)."""
    c = ctypes.c_uint(0)
    rc = load().cellato_device_wait_timeouts(ctypes.byref(c))
    if rc not in (OK, ETIMEDOUT):
        check(rc)
    return c.value


def run_temporal(rule, layout: int, word_bits: int, planes_a, planes_b, X: int, Y: int, t0: int, steps: int,
                 k: int, tile_rows: int = 0, stream: int = 0, row_loop: int = 0, words_per_lane: int = 0) -> int:
    """k fused steps per launch; tile_rows, row_loop and words_per_lane as
    cellato_tune (0 = the library's choice).  Returns 1 when the result ended
    in planes_b, else 0."""
    out = ctypes.c_int(0)
    t = tune(row_loop=row_loop, words_per_lane=words_per_lane, tile_rows=tile_rows)
    check(load().cellato_run_temporal(rule_id(rule), layout, word_bits, ptr_array(planes_a), ptr_array(planes_b),
                                      X, Y, t0, steps, k, ctypes.byref(t), stream, ctypes.byref(out)))
    return out.value


def checksum(rule, layout: int, word_bits: int, planes, X: int, Y: int, sums_ptr: int, stream: int = 0) -> None:
    """4 x 4 tile sums of the state values into 16 uint64 of device memory at sums_ptr."""
    check(load().cellato_checksum(rule_id(rule), layout, word_bits, ptr_array(planes), X, Y, sums_ptr, stream))


def state_value(rule, index: int) -> int:
    v = ctypes.c_longlong()
    check(load().cellato_rule_state_value(rule_id(rule), index, ctypes.byref(v)))
    return v.value


def fill_random(layout: int, word_bits: int, nb: int, planes, X: int, Y: int, seed: int, thresholds,
                stream: int = 0) -> None:
    """Seeded i.i.d. initial state straight into nb device planes (see cellato_fill_random)."""
    th = (ctypes.c_uint32 * max(1, len(thresholds)))(*thresholds)
    check(load().cellato_fill_random(layout, word_bits, nb, ptr_array(planes), X, Y, seed, th, len(thresholds),
                                     stream))


def checksum_string(sums) -> str:
    """The reference's printed form of the 16 tile sums."""
    return "-".join(str(int(v)) for v in sums)


def download_planes(nb: int, dev_ptrs, plane_bytes: int, stream: int = 0):
    """Copy nb device planes into a new (nb, plane_bytes) uint8 host array (synchronous)."""
    import numpy as np
    out = np.empty((nb, plane_bytes), dtype=np.uint8)
    host = ptr_array([out[p].ctypes.data for p in range(nb)])
    check(load().cellato_planes_download(nb, host, ptr_array(dev_ptrs), plane_bytes, stream))
    return out


def diff_cells(nb: int, planes_a, planes_b, plane_bytes: int, count_ptr: int, stream: int = 0) -> None:
    """Number of differing cells between two grids of the same layout, into one
    uint64 of device memory at count_ptr."""
    check(load().cellato_diff_cells(nb, ptr_array(planes_a), ptr_array(planes_b), plane_bytes, count_ptr, stream))


def bit_array_to_planes(nb: int, array_word_bits: int, array_ptr: int, X: int, Y: int, layout: int, word_bits: int,
                        planes, stream: int = 0) -> None:
    """Device bit_array words -> device planes (the reference's bit_array layout)."""
    check(load().cellato_bit_array_to_planes(nb, array_word_bits, array_ptr, X, Y, layout, word_bits,
                                             ptr_array(planes), stream))


def planes_to_bit_array(nb: int, layout: int, word_bits: int, planes, X: int, Y: int, array_word_bits: int,
                        array_ptr: int, stream: int = 0) -> None:
    check(load().cellato_planes_to_bit_array(nb, layout, word_bits, ptr_array(planes), X, Y, array_word_bits,
                                             array_ptr, stream))


def k_array(k_per_rule):
    """A k-per-rule-id argument ({rule: k} or a sequence) as (ctypes int array
    or None, entry count)."""
    if k_per_rule is None:
        return None, 0
    if isinstance(k_per_rule, dict):
        n = max((rule_id(r) for r in k_per_rule), default=-1) + 1
        vals = [0] * n
        for r, k in k_per_rule.items():
            vals[rule_id(r)] = int(k)
    else:
        vals = [int(k) for k in k_per_rule]
    return (ctypes.c_int * max(1, len(vals)))(*vals), len(vals)

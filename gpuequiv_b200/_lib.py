"""ctypes binding of libgeq.so (include/geq.h).

The library is built in-tree (``python gpuequiv_b200/build.py``).  There is
no fallback: if the shared library is missing the import fails loudly, and
without a CUDA device the solver calls raise ``GeqError(NO_DEVICE)``.

Set ``GEQ_CHECKED=1`` to load the bounds-checked build instead.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))


class geq_energy_conf(C.Structure):
    _fields_ = [("elements", C.c_uint32), ("max", C.c_uint32)]


class geq_game_graph(C.Structure):
    _fields_ = [("conf", geq_energy_conf), ("n_vertices", C.c_uint32),
                ("row_offsets", C.POINTER(C.c_uint32)), ("column_indices", C.POINTER(C.c_uint32)),
                ("weights", C.POINTER(C.c_uint32)), ("attacker_pos", C.POINTER(C.c_uint8))]


class geq_energy_lists(C.Structure):
    _fields_ = [("n_vertices", C.c_uint32), ("energy_size", C.c_uint32),
                ("offsets", C.POINTER(C.c_uint64)), ("data", C.POINTER(C.c_uint32))]


class geq_solve_stats(C.Structure):
    _fields_ = [("rounds", C.c_uint64), ("positions_computed", C.c_uint64), ("edges_relaxed", C.c_uint64),
                ("algorithmic_bytes", C.c_uint64), ("arena_compactions", C.c_uint64),
                ("kernel_launches", C.c_uint64), ("device_ms", C.c_double),
                ("round_kernel_ms", C.c_double), ("round_kernel_launches", C.c_uint64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class geq_tuning(C.Structure):
    _fields_ = [("blocks_per_sm", C.c_uint32), ("rounds_per_graph", C.c_uint32),
                ("small_limit", C.c_uint32), ("flags", C.c_uint32), ("lane_limits", C.c_uint32)]


class geq_server_config(C.Structure):
    _fields_ = [("n_pipelines", C.c_uint32), ("max_batch_games", C.c_uint32), ("max_wait_us", C.c_uint32),
                ("max_game_positions", C.c_uint32), ("hbm_budget_bytes", C.c_uint64), ("max_queued", C.c_uint64)]


class geq_server_stats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("batches", C.c_uint64), ("queued", C.c_uint64), ("running", C.c_uint64),
                ("games_in_batches", C.c_uint64), ("max_batch_footprint", C.c_uint64), ("admit_ms", C.c_double), ("step_ms", C.c_double),
                ("retire_ms", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class geq_game_batch_info(C.Structure):
    _fields_ = [("positions", C.c_uint64), ("edges", C.c_uint64), ("levels", C.c_uint32),
                ("kernel_launches", C.c_uint32), ("attempts", C.c_uint32), ("upload_ms", C.c_double),
                ("build_ms", C.c_double), ("download_ms", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class geq_position(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("p", C.c_uint32), ("q", C.POINTER(C.c_uint32)), ("n_q", C.c_uint32),
                ("qx", C.POINTER(C.c_uint32)), ("n_qx", C.c_uint32)]


TUNE_FORCE_GENERIC = 1
TUNE_FORCE_LARGE = 2
TUNE_NO_GRAPH = 4
TUNE_PROFILE = 8
TUNE_NO_THREAD_PATH = 16
TUNE_NO_SPLIT = 32
TUNE_BUILD_WARP_ALL = 64
TUNE_FORCE_WIDE = 128
TUNE_READY = 256
TUNE_NO_EDGE_PAIRS = 512

STATUS = {0: "OK", 1: "NO_DEVICE", 2: "OUT_OF_MEMORY", 3: "INVALID_INPUT", 4: "TIMEOUT",
          5: "UNSUPPORTED", 6: "CUDA", 7: "IO", 8: "PARSE", 9: "BUSY", 10: "INTERNAL"}


class GeqError(Exception):
    """Error returned by libgeq (mirrors gpuequiv::Error / CSVError)."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.name = STATUS.get(status, str(status))
        super().__init__(f"{self.name}: {message}")


u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)
u64p = C.POINTER(C.c_uint64)
u8p = C.POINTER(C.c_uint8)
vp = C.c_void_p

_SIGS = {
    "geq_status_string": ([C.c_int], C.c_char_p),
    "geq_last_error": ([], C.c_char_p),
    "geq_abi_version": ([], C.c_int),
    "geq_conf_energy_bits": ([geq_energy_conf], C.c_uint32),
    "geq_conf_energy_size": ([geq_energy_conf], C.c_uint32),
    "geq_conf_energy_mask": ([geq_energy_conf], C.c_uint32),
    "geq_conf_update_bits": ([geq_energy_conf], C.c_uint32),
    "geq_conf_update_size": ([geq_energy_conf], C.c_uint32),
    "geq_conf_update_mask": ([geq_energy_conf], C.c_uint32),
    "geq_conf_supported": ([geq_energy_conf], C.c_int),
    "geq_conf_solvable": ([geq_energy_conf], C.c_int),
    "geq_energy_pack": ([geq_energy_conf, u32p, C.c_uint32, u32p], C.c_int),
    "geq_energy_unpack": ([geq_energy_conf, u32p, u32p], None),
    "geq_update_pack": ([geq_energy_conf, i32p, C.c_uint32, u32p], C.c_int),
    "geq_update_unpack": ([geq_energy_conf, u32p, i32p], None),
    "geq_test_equivalence": ([geq_energy_conf, u32p, C.c_uint64, u32p], C.c_int),
    "geq_standard_reach": ([C.POINTER(geq_game_graph), u32p], C.c_uint32),
    "geq_context_create": ([C.c_int, C.POINTER(vp)], C.c_int),
    "geq_context_destroy": ([vp], None),
    "geq_context_info": ([vp, C.c_char_p, C.c_size_t, C.POINTER(C.c_int), u64p], C.c_int),
    "geq_context_set_tuning": ([vp, C.POINTER(geq_tuning)], C.c_int),
    "geq_context_get_tuning": ([vp, C.POINTER(geq_tuning)], None),
    "geq_solution_n_games": ([vp], C.c_uint32),
    "geq_solution_lists": ([vp, C.c_uint32, C.POINTER(geq_energy_lists)], C.c_int),
    "geq_solution_flat": ([vp, C.POINTER(u64p), C.POINTER(C.c_uint64), C.POINTER(u32p), C.POINTER(C.c_uint64)],
                          C.c_int),
    "geq_solution_stats": ([vp, C.POINTER(geq_solve_stats)], None),
    "geq_solution_free": ([vp], None),
    "geq_energy_game_run": ([vp, C.POINTER(geq_game_graph), C.POINTER(geq_energy_lists), u32p, C.c_uint32,
                             C.POINTER(vp)], C.c_int),
    "geq_energy_game_run_static": ([vp, C.POINTER(geq_game_graph), u32p, C.c_uint32, u64p, u32p, C.c_uint64, u64p,
                                    C.POINTER(geq_solve_stats)], C.c_int),
    "geq_energy_game_run_batch": ([vp, C.c_uint32, C.POINTER(geq_game_graph),
                                   C.POINTER(C.POINTER(geq_energy_lists)), C.POINTER(u32p), u32p,
                                   C.POINTER(vp)], C.c_int),
    "geq_device_games_create": ([vp, C.c_uint32, C.POINTER(geq_game_graph),
                                 C.POINTER(C.POINTER(geq_energy_lists)), C.POINTER(u32p), u32p,
                                 C.POINTER(vp)], C.c_int),
    "geq_device_games_solve": ([vp, vp, C.POINTER(geq_solve_stats)], C.c_int),
    "geq_device_games_download": ([vp, vp, C.POINTER(vp)], C.c_int),
    "geq_device_games_free": ([vp], None),
    "geq_server_create": ([vp, C.POINTER(geq_server_config), C.POINTER(vp)], C.c_int),
    "geq_server_submit": ([vp, C.POINTER(geq_game_graph), C.POINTER(C.c_uint64)], C.c_int),
    "geq_server_submit_compare": ([vp, vp, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint64)], C.c_int),
    "geq_server_poll": ([vp, C.c_uint64, C.c_int32, C.POINTER(vp)], C.c_int),
    "geq_server_poll_any": ([vp, C.c_int32, C.POINTER(C.c_uint64), C.POINTER(vp)], C.c_int),
    "geq_server_get_stats": ([vp, C.POINTER(geq_server_stats)], None),
    "geq_server_destroy": ([vp], None),
    "geq_lts_from_edges": ([C.c_uint64, u32p, u32p, i32p, C.POINTER(vp)], C.c_int),
    "geq_lts_from_adjacency": ([C.c_uint32, C.c_uint64, u32p, u32p, i32p, C.POINTER(vp)], C.c_int),
    "geq_lts_from_csv_file": ([C.c_char_p, C.POINTER(vp)], C.c_int),
    "geq_lts_n_vertices": ([vp], C.c_uint32),
    "geq_lts_n_transitions": ([vp], C.c_uint64),
    "geq_lts_transitions": ([vp, u64p, u32p, i32p], None),
    "geq_lts_signature_refinement": ([vp, u64p, u64p], C.c_int),
    "geq_lts_bisimilar_minimize": ([vp, C.POINTER(vp), u64p], C.c_int),
    "geq_lts_signature_refinement_batch": ([vp, C.c_uint32, C.POINTER(vp), u64p, u64p], C.c_int),
    "geq_lts_free": ([vp], None),
    "geq_game_build_compare": ([vp, C.c_uint32, C.c_uint32, C.POINTER(vp)], C.c_int),
    "geq_game_build_compare_all": ([vp, C.POINTER(vp)], C.c_int),
    "geq_game_build_compare_bounded": ([vp, C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(vp)], C.c_int),
    "geq_game_build_compare_multiple": ([vp, u32p, C.c_uint32, C.POINTER(vp)], C.c_int),
    "geq_game_build_graph": ([vp, C.POINTER(geq_game_graph)], None),
    "geq_game_build_n_starting_points": ([vp], C.c_uint32),
    "geq_game_build_position": ([vp, C.c_uint32, C.POINTER(geq_position)], C.c_int),
    "geq_game_build_free": ([vp], None),
    "geq_game_build_compare_batch": ([vp, C.c_uint32, C.POINTER(vp), u32p, u32p, C.c_uint64, C.POINTER(vp)],
                                     C.c_int),
    "geq_game_build_starts_batch": ([vp, C.c_uint32, C.POINTER(vp), u32p, u32p, u32p, C.c_uint64, C.POINTER(vp)],
                                    C.c_int),
    "geq_game_batch_n_jobs": ([vp], C.c_uint32),
    "geq_game_batch_n_starting_points": ([vp, C.c_uint32], C.c_uint32),
    "geq_game_batch_graph": ([vp, C.c_uint32, C.POINTER(geq_game_graph)], C.c_int),
    "geq_game_batch_stats": ([vp, C.POINTER(geq_game_batch_info)], None),
    "geq_game_batch_free": ([vp], None),
    "geq_compare": ([vp, vp, C.c_uint32, C.c_uint32, C.c_int, C.POINTER(vp)], C.c_int),
    "geq_compare_batch": ([vp, C.c_uint32, C.POINTER(vp), u32p, u32p, C.c_int, C.POINTER(vp)], C.c_int),
    "geq_equivalences": ([vp, vp, C.c_int, C.POINTER(vp)], C.c_int),
    "geq_equivalence_energies": ([vp, C.c_uint32, C.c_uint32, C.POINTER(u32p), u64p], C.c_int),
    "geq_equivalence_preorder": ([vp, C.c_uint32, C.c_uint32, u32p], C.c_int),
    "geq_equivalence_equiv": ([vp, C.c_uint32, C.c_uint32, u32p], C.c_int),
    "geq_equivalence_relation": ([vp, u32p, u32p, u32p], C.c_int),
    "geq_equivalence_n_processes": ([vp], C.c_uint32),
    "geq_equivalence_n_starting_points": ([vp], C.c_uint32),
    "geq_equivalence_free": ([vp], None),
}


def library_path() -> str:
    """$GEQ_LIBRARY if set (another build of the same ABI), else the in-tree
    libgeq.so, or libgeq_checked.so when GEQ_CHECKED=1."""
    if os.environ.get("GEQ_LIBRARY"):
        return os.path.abspath(os.environ["GEQ_LIBRARY"])
    name = "libgeq_checked.so" if os.environ.get("GEQ_CHECKED") == "1" else "libgeq.so"
    return os.path.join(HERE, name)


def _load():
    path = library_path()
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python gpuequiv_b200/build.py`")
    L = C.CDLL(path)
    for name, (args, res) in _SIGS.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    return L


lib = _load()
EXPORTED = tuple(_SIGS)


def check(status: int) -> None:
    if status != 0:
        raise GeqError(status, lib.geq_last_error().decode(errors="replace"))

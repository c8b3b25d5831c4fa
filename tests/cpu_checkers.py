"""ctypes access to the CPU checkers of the VELO chain (test infrastructure only).

``load("oracle")`` -> oracle/_build/libvelo_oracle.so, the plain-C restatement;
``load("ref")``    -> oracle/_ref/libvelo_ref.so, the reference's VELO kernels
                      compiled as CPU C++ (present only where it was built).
Both export the interface of oracle/velo_cpu_api.h.  ``run`` returns every buffer
of the chain, keyed by its Allen argument name, as a numpy array.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBS = {
    "oracle": (os.path.join(REPO, "oracle", "_build", "libvelo_oracle.so"), "velo_oracle"),
    "ref": (os.path.join(REPO, "oracle", "_ref", "libvelo_ref.so"), "velo_ref"),
}

# dtype of each named buffer (everything else is u32)
DTYPES = {
    "dev_velo_cluster_container": np.uint8,
    "dev_sorted_velo_cluster_container": np.uint8,
    "dev_velo_track_hits": np.uint8,
    "dev_tracks": np.uint8,
    "dev_three_hit_tracks": np.uint16,
    "dev_three_hit_tracks_output": np.uint16,
    "dev_tracklets": np.uint16,
    "dev_hit_used": np.uint8,
    "dev_rel_indices": np.uint16,
    "dev_accepted_velo_tracks": np.uint8,
    "dev_is_backward": np.uint8,
    "dev_velo_kalman_beamline_states": np.uint8,
    "dev_velo_kalman_endvelo_states": np.uint8,
}


class VeloCpuInput(C.Structure):
    _fields_ = [
        ("raw", C.c_void_p), ("raw_offsets", C.c_void_p), ("raw_sizes", C.c_void_p),
        ("raw_types", C.c_void_p), ("event_start", C.c_uint), ("n_events", C.c_uint),
        ("bank_version", C.c_int), ("geometry", C.c_void_p), ("geometry_size", C.c_size_t),
        ("phi_tolerance", C.c_float), ("max_scatter", C.c_float),
        ("max_skipped_modules", C.c_uint), ("max_chi2", C.c_float),
        ("beamline_x", C.c_float), ("beamline_y", C.c_float), ("retina_decoding", C.c_int),
        ("mep_layout", C.c_int),
    ]


def available(kind: str) -> bool:
    return os.path.exists(LIBS[kind][0])


class Checker:
    def __init__(self, kind: str):
        path, prefix = LIBS[kind]
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C oracle {'ref' if kind == 'ref' else 'oracle'})")
        self.kind = kind
        self.lib = C.CDLL(path)
        self._run = getattr(self.lib, prefix + "_run")
        self._run.restype = C.c_void_p
        self._run.argtypes = [C.POINTER(VeloCpuInput)]
        self._get = getattr(self.lib, prefix + "_get")
        self._get.restype = C.c_void_p
        self._get.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_size_t)]
        self._free = getattr(self.lib, prefix + "_free")
        self._free.argtypes = [C.c_void_p]
        self._time = getattr(self.lib, prefix + "_time")
        self._time.restype = C.c_double
        self._time.argtypes = [C.POINTER(VeloCpuInput), C.c_uint, C.c_uint, C.c_uint]

    @staticmethod
    def make_input(s, geometry: bytes, event_start=0, n_events=None, phi_tolerance=0.045,
                   max_scatter=0.08, max_skipped_modules=1, max_chi2=20.0, beamline=(0.0, 0.0), retina=None):
        keep = (np.ascontiguousarray(s.raw), np.ascontiguousarray(s.offsets),
                np.ascontiguousarray(s.sizes), np.ascontiguousarray(s.types),
                np.frombuffer(geometry, dtype=np.uint8))
        inp = VeloCpuInput(
            keep[0].ctypes.data, keep[1].ctypes.data, keep[2].ctypes.data, keep[3].ctypes.data,
            event_start, s.n_events - event_start if n_events is None else n_events,
            s.bank_version, keep[4].ctypes.data, len(geometry),
            phi_tolerance, max_scatter, max_skipped_modules, max_chi2, beamline[0], beamline[1],
            int(retina if retina is not None else getattr(s, "retina", False)), int(getattr(s, "mep", False)))
        return inp, keep

    def run(self, s, geometry: bytes, **kw) -> dict:
        inp, keep = self.make_input(s, geometry, **kw)
        h = self._run(C.byref(inp))
        if not h:
            raise ValueError(f"{self.kind} checker refused the input (MEP layout?)")
        try:
            out = {}
            for name in list(DTYPES) + U32_BUFFERS:
                n = C.c_size_t(0)
                p = self._get(h, name.encode(), C.byref(n))
                if not p:
                    continue
                dt = np.dtype(DTYPES.get(name, np.uint32))
                buf = (C.c_char * n.value).from_address(p) if n.value else b""
                out[name] = np.frombuffer(bytes(buf), dtype=np.uint8).view(dt).copy() \
                    if n.value % dt.itemsize == 0 else np.frombuffer(bytes(buf), dtype=np.uint8).copy()
            return out
        finally:
            self._free(h)
            del keep

    def time(self, s, geometry: bytes, slice_size: int, n_slices: int, n_threads: int) -> float:
        inp, keep = self.make_input(s, geometry)
        return float(self._time(C.byref(inp), slice_size, n_slices, n_threads))


U32_BUFFERS = [
    "dev_each_sensor_pair_size", "dev_retina_bank_index", "dev_offsets_each_sensor_pair_size",
    "dev_hit_permutations",
    "dev_number_of_candidates", "dev_velo_bank_index", "dev_candidates_offsets",
    "dev_estimated_input_size", "dev_module_candidate_num", "dev_cluster_candidates",
    "dev_offsets_estimated_input_size", "dev_module_cluster_num", "dev_hit_permutation",
    "dev_tracks_to_follow", "dev_atomics_velo", "dev_number_of_velo_tracks",
    "dev_offsets_velo_tracks", "dev_number_of_three_hit_tracks_output",
    "dev_offsets_number_of_three_hit_tracks_filtered", "dev_velo_track_hit_number",
    "dev_offsets_all_velo_tracks", "host_number_of_reconstructed_velo_tracks",
    "dev_offsets_velo_track_hit_number",
]


def load(kind: str) -> Checker:
    return Checker(kind)


def ref_transpose_vp(stream: bytes, max_events: int, check_checksum: bool = False) -> dict:
    """The reference's own MDF reader + transpose (oracle/ref_transpose.cpp) on ``stream``:
    the VP slice it writes, as numpy arrays sized by what it wrote."""
    path = LIBS["ref"][0]
    lib = C.CDLL(path)
    f = lib.ref_transpose_vp
    f.restype = C.c_int
    f.argtypes = [C.c_char_p, C.c_size_t, C.c_uint, C.c_int, C.c_void_p, C.c_size_t, C.c_void_p,
                  C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.POINTER(C.c_uint), C.POINTER(C.c_uint),
                  C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)]
    cap = len(stream) + 4096 * (max_events + 1)
    raw = np.zeros(cap, dtype=np.uint8)
    offsets = np.zeros(max_events + 1, dtype=np.uint32)
    words = (len(stream) // 8) + 4 * (max_events + 1)
    sizes = np.zeros(words, dtype=np.uint32)
    types = np.zeros(words, dtype=np.uint32)
    n_ev, n_off, ver, by_src, secs = C.c_uint(0), C.c_uint(0), C.c_int(0), C.c_int(0), C.c_double(0)
    rc = f(stream, len(stream), max_events, int(check_checksum), raw.ctypes.data, cap, offsets.ctypes.data,
           sizes.ctypes.data, words, types.ctypes.data, words, C.byref(n_ev), C.byref(n_off), C.byref(ver),
           C.byref(by_src), C.byref(secs))
    n = n_ev.value
    out = {"status": rc, "n_events": n, "n_offsets": n_off.value, "bank_version": ver.value,
           "by_source_id": bool(by_src.value), "transpose_seconds": secs.value}
    if rc != 0:
        return out
    n_slice = n_off.value - 1  # events the slice holds
    out["offsets"] = offsets[:n_slice + 1].copy()
    out["raw"] = raw[:int(offsets[n_slice])].copy()
    size_words = (4 * (n + 1) + 2 * (int(sizes[n_slice]) - 2 * (n + 1)) + 3) // 4
    type_words = (4 * (n + 1) + (int(types[n_slice]) - 4 * (n + 1)) + 3) // 4
    out["sizes"] = sizes[:size_words].copy()
    out["types"] = types[:type_words].copy()
    return out

"""Python front end of the C ABI in include/velo_b200.h (ctypes).

Device memory and streams come from torch (plumbing only); every computation runs in
libvelo_b200.so.  There is no CPU fallback: without an sm_100 device the constructor
raises.

    chain = VeloChain()                       # geometry from allen_b200/data
    chain.reserve(max_events, max_super_pixels)
    dev = upload(raw_slice)                   # RawSlice -> device copy (torch tensors)
    chain.run(dev)                            # whole chain, one stream, no host sync
    totals = chain.synchronize()
    out = chain.outputs_to_host(totals)       # numpy arrays keyed by Allen argument name
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native
from .rawbanks import RawSlice, super_pixels_per_event

ELEMENT_SIZE = 18
TRACK_HITS_BYTES = 54
TRACKLET_BYTES = 6
N_MODULE_PAIRS = 26

STATUS = {0: "ok", 1: "argument", 2: "cuda", 3: "capacity", 4: "device flags", 5: "no device"}
DEVICE_FLAGS = {
    1: "cluster capacity", 2: "track capacity", 4: "tracks-to-follow overflow", 8: "bad sensor",
    16: "bulk copy timeout", 32: "output capacity", 64: "input capacity", 128: "hits per event",
}


class VeloError(RuntimeError):
    def __init__(self, status, message, flags=0):
        super().__init__(f"velo_b200: {STATUS.get(status, status)}: {message}")
        self.status = status
        self.flags = flags


class Properties(C.Structure):
    _fields_ = [("phi_tolerance", C.c_float), ("max_scatter", C.c_float),
                ("max_skipped_modules", C.c_uint), ("max_chi2", C.c_float)]


class DeviceSliceC(C.Structure):
    _fields_ = [("raw", C.c_void_p), ("offsets", C.c_void_p), ("sizes", C.c_void_p), ("types", C.c_void_p),
                ("event_start", C.c_uint), ("n_events", C.c_uint), ("bank_version", C.c_int),
                ("mep_layout", C.c_int)]


class HostSliceC(C.Structure):
    _fields_ = [("raw", C.c_void_p), ("raw_bytes", C.c_size_t), ("offsets", C.c_void_p),
                ("sizes", C.c_void_p), ("sizes_bytes", C.c_size_t), ("types", C.c_void_p),
                ("types_bytes", C.c_size_t), ("n_events", C.c_uint), ("bank_version", C.c_int)]


OUTPUT_FIELDS = [
    "dev_number_of_candidates", "dev_estimated_input_size", "dev_module_candidate_num",
    "dev_offsets_estimated_input_size", "dev_module_cluster_num", "dev_sorted_velo_cluster_container",
    "dev_tracks", "dev_three_hit_tracks", "dev_hit_used", "dev_atomics_velo", "dev_number_of_velo_tracks",
    "dev_offsets_velo_tracks", "dev_three_hit_tracks_output", "dev_number_of_three_hit_tracks_output",
    "dev_offsets_number_of_three_hit_tracks_filtered", "dev_offsets_all_velo_tracks",
    "dev_velo_track_hit_number", "dev_offsets_velo_track_hit_number", "dev_velo_track_hits",
    "dev_accepted_velo_tracks", "dev_seed_stats", "dev_is_backward", "dev_velo_kalman_beamline_states",
    "dev_velo_kalman_endvelo_states", "dev_each_sensor_pair_size", "dev_offsets_each_sensor_pair_size",
    "dev_retina_bank_index", "dev_seed_gate", "dev_gate_stats",
]


class OutputsC(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in OUTPUT_FIELDS]


class SeedModelC(C.Structure):
    """VeloSeedModel of velo_b200.h."""
    _fields_ = [("w1", (C.c_float * 12) * 32), ("b1", C.c_float * 32), ("w2", (C.c_float * 32) * 32),
                ("b2", C.c_float * 32), ("w3", C.c_float * 32), ("b3", C.c_float), ("mean", C.c_float * 12),
                ("inv_std", C.c_float * 12), ("threshold_logit", C.c_float), ("kept_lo", C.c_float),
                ("kept_hi", C.c_float)]


SEED_PARAMS = 32 * 12 + 32 + 32 * 32 + 32 + 32 + 1


class LaunchConfigC(C.Structure):
    _fields_ = [(f, C.c_uint) for f in (
        "search_threads", "search_lanes_per_seed", "search_hit_capacity", "cluster_stage_capacity",
        "cluster_blob_bytes", "estimate_blob_bytes", "persistent", "events_per_claim", "search_ring_global",
        "cluster_threads", "retina_order_capacity", "kalman_warp_hits", "seed_window")]


class TotalsC(C.Structure):
    _fields_ = [(f, C.c_uint) for f in (
        "n_events", "host_total_number_of_velo_clusters", "host_number_of_cluster_candidates",
        "host_number_of_velo_tracks_at_least_four_hits", "host_number_of_three_hit_tracks_filtered",
        "host_number_of_reconstructed_velo_tracks", "host_accumulated_number_of_hits_in_velo_tracks",
        "track_container_size", "device_flags")]


class SizesC(C.Structure):
    _fields_ = [(f, C.c_ulonglong) for f in (
        "offsets_estimated_input_size", "module_cluster_num", "sorted_velo_cluster_container_bytes",
        "offsets_all_velo_tracks", "velo_track_hit_number", "offsets_velo_track_hit_number",
        "velo_track_hits_bytes", "accepted_velo_tracks", "max_reconstructed_tracks", "workspace_bytes")]


class OutputBuffersC(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in (
        "dev_offsets_estimated_input_size", "dev_module_cluster_num", "dev_sorted_velo_cluster_container",
        "dev_offsets_all_velo_tracks", "dev_velo_track_hit_number", "dev_offsets_velo_track_hit_number",
        "dev_velo_track_hits", "dev_accepted_velo_tracks")]


COORDINATES_FP32, COORDINATES_FP16 = 0, 1
# view sizes (Allen::Views::Velo::Consolidated::{Hits, Track, Tracks, MultiEventTracks})
VIEW_BYTES = {"dev_velo_hits_view": 24, "dev_velo_track_view": 24, "dev_velo_tracks_view": 16,
              "dev_velo_multi_event_tracks_view": 24, "dev_imec_velo_tracks": 8}


def _lib():
    lib = _native.load_chain()
    if getattr(lib, "_typed", False):
        return lib
    lib.velo_last_error_string.restype = C.c_char_p
    lib.velo_device_check.restype = C.c_int
    lib.velo_default_properties.argtypes = [C.POINTER(Properties)]
    lib.velo_chain_create.restype = C.c_int
    lib.velo_chain_create.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(Properties), C.POINTER(C.c_void_p)]
    lib.velo_chain_reserve.restype = C.c_int
    lib.velo_chain_reserve.argtypes = [C.c_void_p, C.c_uint, C.c_ulonglong, C.c_ulonglong]
    lib.velo_chain_run.restype = C.c_int
    lib.velo_chain_run.argtypes = [C.c_void_p, C.POINTER(DeviceSliceC), C.c_void_p, C.c_int]
    lib.velo_chain_run_host.restype = C.c_int
    lib.velo_chain_run_host.argtypes = [C.c_void_p, C.POINTER(HostSliceC), C.c_void_p,
                                        C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t,
                                        C.POINTER(TotalsC), C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]
    lib.velo_chain_synchronize.restype = C.c_int
    lib.velo_chain_synchronize.argtypes = [C.c_void_p, C.POINTER(TotalsC)]
    lib.velo_chain_outputs.restype = C.c_int
    lib.velo_chain_outputs.argtypes = [C.c_void_p, C.POINTER(OutputsC)]
    lib.velo_check_contracts.restype = C.c_int
    lib.velo_check_contracts.argtypes = [C.POINTER(OutputsC), C.POINTER(TotalsC), C.c_void_p, C.c_void_p]
    lib.velo_chain_destroy.argtypes = [C.c_void_p]
    lib.velo_chain_sizes.restype = C.c_int
    lib.velo_chain_sizes.argtypes = [C.c_void_p, C.c_uint, C.c_ulonglong, C.c_int, C.POINTER(SizesC)]
    lib.velo_chain_bind.restype = C.c_int
    lib.velo_chain_bind.argtypes = [C.c_void_p, C.c_void_p, C.c_ulonglong, C.c_uint, C.c_ulonglong, C.c_int,
                                    C.POINTER(OutputBuffersC)]
    lib.velo_create_velo_views.restype = C.c_int
    lib.velo_create_velo_views.argtypes = [C.c_uint, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_uint, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.velo_copy_to_host.restype = C.c_int
    lib.velo_copy_to_host.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
    lib.velo_copy_to_host_async.restype = C.c_int
    lib.velo_copy_to_host_async.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]
    lib.velo_copy_to_device.restype = C.c_int
    lib.velo_copy_to_device.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
    lib.velo_chain_configure.restype = C.c_int
    lib.velo_chain_configure.argtypes = [C.c_void_p, C.POINTER(LaunchConfigC)]
    lib.velo_chain_get_config.restype = C.c_int
    lib.velo_chain_get_config.argtypes = [C.c_void_p, C.POINTER(LaunchConfigC)]
    lib.velo_chain_set_timing.restype = C.c_int
    lib.velo_chain_set_timing.argtypes = [C.c_void_p, C.c_int]
    lib.velo_chain_kernel_count.restype = C.c_uint
    lib.velo_chain_kernel_name.restype = C.c_char_p
    lib.velo_chain_kernel_name.argtypes = [C.c_uint]
    lib.velo_chain_kernel_times.restype = C.c_int
    lib.velo_chain_kernel_times.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_uint)]
    lib.velo_chain_set_front_end.restype = C.c_int
    lib.velo_chain_set_front_end.argtypes = [C.c_void_p, C.c_int]
    lib.velo_chain_set_kalman.restype = C.c_int
    lib.velo_chain_set_kalman.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_float]
    lib.velo_run_kalman_filter.restype = C.c_int
    lib.velo_run_kalman_filter.argtypes = [C.c_uint, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint, C.c_float, C.c_float,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.velo_chain_set_seed_model.restype = C.c_int
    lib.velo_chain_set_seed_model.argtypes = [C.c_void_p, C.POINTER(SeedModelC)]
    lib.velo_chain_record_seeds.restype = C.c_int
    lib.velo_chain_record_seeds.argtypes = [C.c_void_p, C.c_void_p, C.c_uint, C.c_uint, C.c_void_p]
    lib.velo_seed_trainer_create.restype = C.c_int
    lib.velo_seed_trainer_create.argtypes = [C.POINTER(SeedModelC), C.c_float, C.c_float, C.POINTER(C.c_void_p)]
    lib.velo_seed_trainer_step.restype = C.c_int
    lib.velo_seed_trainer_step.argtypes = [C.c_void_p, C.c_void_p, C.c_ulonglong, C.c_uint, C.c_void_p,
                                           C.POINTER(C.c_float)]
    lib.velo_seed_trainer_gradients.restype = C.c_int
    lib.velo_seed_trainer_gradients.argtypes = [C.c_void_p, C.c_void_p, C.c_ulonglong, C.c_uint, C.c_void_p,
                                                C.POINTER(C.c_float), C.POINTER(C.c_float)]
    lib.velo_seed_trainer_score.restype = C.c_int
    lib.velo_seed_trainer_score.argtypes = [C.c_void_p, C.c_void_p, C.c_ulonglong, C.c_void_p, C.c_void_p]
    lib.velo_seed_trainer_model.restype = C.c_int
    lib.velo_seed_trainer_model.argtypes = [C.c_void_p, C.POINTER(SeedModelC)]
    lib.velo_seed_trainer_destroy.argtypes = [C.c_void_p]
    lib._typed = True
    return lib


CONTRACTS = ["cluster_outside", "unsorted", "track_size", "repeated_hit", "zero_id", "id_type", "offsets"]


def check_contracts(outputs: dict, totals: dict, stream=None) -> dict:
    """The reference's contracts on a run's outputs, counted on the device
    (velo_check_contracts): outputs maps Allen output names to device pointers (FP32 layout),
    totals holds the run's host totals (VeloChainTotals fields).  Returns violations per
    contract (all zero for a correct run)."""
    import torch
    lib = _lib()
    o = OutputsC(**{f: outputs.get(f) for f in OUTPUT_FIELDS})
    t = TotalsC(**{f: int(totals.get(f, 0)) for f, _ in TotalsC._fields_})
    counts = torch.zeros(len(CONTRACTS), dtype=torch.int32, device="cuda")
    _check(lib, lib.velo_check_contracts(C.byref(o), C.byref(t), stream if stream is not None else _current_stream(),
                                         C.c_void_p(counts.data_ptr())))
    return dict(zip(CONTRACTS, (int(v) for v in counts.cpu().tolist())))


def _check(lib, status, flags=0):
    if status != 0:
        raise VeloError(status, lib.velo_last_error_string().decode(), flags)


def _current_stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


@dataclass
class DeviceSlice:
    """A RawSlice resident on the GPU (torch tensors keep the memory alive)."""
    raw: object
    offsets: object
    sizes: object
    types: object
    n_events: int
    bank_version: int
    event_start: int = 0
    retina: bool = False  # retina-cluster banks (type 73)
    mep: bool = False     # MEP layout

    def c_struct(self) -> DeviceSliceC:
        return DeviceSliceC(self.raw.data_ptr(), self.offsets.data_ptr(), self.sizes.data_ptr(),
                            self.types.data_ptr(), self.event_start, self.n_events, self.bank_version, int(self.mep))

    def sub(self, event_start: int, n_events: int) -> "DeviceSlice":
        return DeviceSlice(self.raw, self.offsets, self.sizes, self.types, n_events, self.bank_version,
                           event_start, self.retina, self.mep)


def upload(s: RawSlice, device="cuda") -> DeviceSlice:
    import torch
    raw = np.ascontiguousarray(s.raw)
    pad = (-raw.size) % 16
    if pad:
        raw = np.concatenate([raw, np.zeros(pad, np.uint8)])
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
    return DeviceSlice(t(raw), t(s.offsets.view(np.int32)), t(s.sizes.view(np.int32)),
                       t(s.types.view(np.int32)), s.n_events, s.bank_version, 0, s.retina, s.mep)


class VeloChain:
    def __init__(self, geometry: bytes | None = None, phi_tolerance=0.045, max_scatter=0.08,
                 max_skipped_modules=1, max_chi2=20.0, use_tuned: bool = True):
        self.lib = _lib()
        self.geometry = geometry if geometry is not None else _native.default_geometry()
        props = Properties(phi_tolerance, max_scatter, max_skipped_modules, max_chi2)
        h = C.c_void_p()
        _check(self.lib, self.lib.velo_chain_create(self.geometry, len(self.geometry), C.byref(props), C.byref(h)))
        self.handle = h
        self.max_events = 0
        self.max_super_pixels = 0
        if use_tuned:
            tuned = _native.tuned_launch_config()
            if tuned:
                self.configure(**tuned)

    def close(self):
        if getattr(self, "handle", None):
            self.lib.velo_chain_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reserve(self, max_events: int, max_super_pixels: int, max_raw_bytes: int = 0):
        _check(self.lib, self.lib.velo_chain_reserve(self.handle, max_events, max_super_pixels, max_raw_bytes))
        self.max_events, self.max_super_pixels = max_events, max_super_pixels

    def sizes(self, max_events: int, max_super_pixels: int, layout: int = COORDINATES_FP32) -> dict:
        """Element counts of the outputs and the scratch bytes for caller-owned memory."""
        out = SizesC()
        _check(self.lib, self.lib.velo_chain_sizes(self.handle, max_events, max_super_pixels, layout, C.byref(out)))
        return {f: getattr(out, f) for f, _ in SizesC._fields_}

    def bind(self, workspace_ptr: int, workspace_bytes: int, max_events: int, max_super_pixels: int,
             outputs: dict, layout: int = COORDINATES_FP32):
        """Runs into caller memory from now on: ``outputs`` maps each OutputBuffersC field to a
        device pointer (sized by sizes()); the chain allocates nothing more."""
        o = OutputBuffersC(*[outputs[f] for f, _ in OutputBuffersC._fields_])
        _check(self.lib, self.lib.velo_chain_bind(self.handle, workspace_ptr, workspace_bytes, max_events,
                                                  max_super_pixels, layout, C.byref(o)))
        self.max_events, self.max_super_pixels = max_events, max_super_pixels

    def reserve_for(self, s: RawSlice, margin: float = 1.0):
        n_sp = int(super_pixels_per_event(s).sum())
        self.reserve(s.n_events, int(n_sp * margin) + 64, s.raw.nbytes + 64)

    def set_front_end(self, retina: bool):
        """Decoding front end: super-pixel banks (False) or retina-cluster banks (True)."""
        _check(self.lib, self.lib.velo_chain_set_front_end(self.handle, int(retina)))
        self.retina = bool(retina)

    def run(self, d: DeviceSlice, stream=None, use_graph: bool = False):
        if bool(getattr(d, "retina", False)) != getattr(self, "retina", False):
            self.set_front_end(d.retina)
        st = d.c_struct()
        self.last_bank_version = d.bank_version
        _check(self.lib, self.lib.velo_chain_run(self.handle, C.byref(st),
                                                 stream if stream is not None else _current_stream(),
                                                 int(use_graph)))

    def synchronize(self, check: bool = True) -> dict:
        t = TotalsC()
        status = self.lib.velo_chain_synchronize(self.handle, C.byref(t))
        totals = {f: getattr(t, f) for f, _ in TotalsC._fields_}
        if check:
            _check(self.lib, status, totals["device_flags"])
        return totals

    def configure(self, **cfg):
        """Sets launch parameters (search_threads, search_lanes_per_seed, search_hit_capacity,
        cluster_stage_capacity, cluster_blob_bytes, estimate_blob_bytes); others keep their value."""
        cur = self.get_config()
        cur.update(cfg)
        c = LaunchConfigC(*[cur[f] for f, _ in LaunchConfigC._fields_])
        _check(self.lib, self.lib.velo_chain_configure(self.handle, C.byref(c)))

    def get_config(self) -> dict:
        c = LaunchConfigC()
        _check(self.lib, self.lib.velo_chain_get_config(self.handle, C.byref(c)))
        return {f: getattr(c, f) for f, _ in LaunchConfigC._fields_}

    def set_timing(self, enable: bool):
        _check(self.lib, self.lib.velo_chain_set_timing(self.handle, int(enable)))

    def kernel_times(self) -> tuple[dict, int]:
        """Per kernel: summed duration (ms) of the last execution of every cached graph."""
        n = self.lib.velo_chain_kernel_count()
        ms = (C.c_float * n)()
        runs = C.c_uint()
        _check(self.lib, self.lib.velo_chain_kernel_times(self.handle, ms, C.byref(runs)))
        return {self.lib.velo_chain_kernel_name(i).decode(): float(ms[i]) for i in range(n)}, runs.value

    def set_kalman(self, enable: bool = True, beamline=(0.0, 0.0)):
        """Appends velo_kalman_filter to the chain (states in the outputs)."""
        _check(self.lib, self.lib.velo_chain_set_kalman(self.handle, int(enable), beamline[0], beamline[1]))
        self.kalman = enable

    def kalman_outputs(self, totals: dict) -> dict:
        """dev_is_backward and the two state containers of the last run (host copies)."""
        p = self.device_outputs()
        reco = totals["host_number_of_reconstructed_velo_tracks"]
        return {"dev_is_backward": self._fetch(p["dev_is_backward"], reco, np.uint8),
                "dev_velo_kalman_beamline_states": self._fetch(p["dev_velo_kalman_beamline_states"], 56 * reco, np.uint8),
                "dev_velo_kalman_endvelo_states": self._fetch(p["dev_velo_kalman_endvelo_states"], 56 * reco, np.uint8)}

    def set_seed_model(self, model):
        """model: a SeedModelC (learned search) or None (plain search)."""
        _check(self.lib, self.lib.velo_chain_set_seed_model(self.handle, C.byref(model) if model is not None else None))

    def record_seeds(self, records, count, every: int = 1):
        """records: device uint8 tensor of 64-byte VeloSeedRecord entries, count: device
        int32 tensor of one element (zeroed by the caller); None stops the recording."""
        if records is None:
            _check(self.lib, self.lib.velo_chain_record_seeds(self.handle, None, 0, 1, None))
        else:
            _check(self.lib, self.lib.velo_chain_record_seeds(self.handle, records.data_ptr(), records.numel() // 64,
                                                              every, count.data_ptr()))

    def seed_stats(self, n_events: int) -> np.ndarray:
        """[n_events, 3]: seed candidates met unused, candidates searched, search mode (0 plain,
        1 learned, 2 gate out of its bounds: plain) of the last run."""
        p = self.device_outputs()["dev_seed_stats"]
        return self._fetch(p, 12 * n_events, np.uint8).view(np.uint32).reshape(n_events, 3)

    def gate_stats(self, n_events: int) -> np.ndarray:
        """[n_events, 2] of the last learned run: seed candidates, candidates the gate kept."""
        p = self.device_outputs()["dev_gate_stats"]
        return self._fetch(p, 8 * n_events, np.uint8).view(np.uint32).reshape(n_events, 2)

    def device_outputs(self) -> dict:
        o = OutputsC()
        _check(self.lib, self.lib.velo_chain_outputs(self.handle, C.byref(o)))
        return {f: getattr(o, f) for f in OUTPUT_FIELDS}

    def _fetch(self, ptr, nbytes, dtype):
        out = np.empty(nbytes, dtype=np.uint8)
        if nbytes:
            _check(self.lib, self.lib.velo_copy_to_host(out.ctypes.data, ptr, nbytes))
        return out.view(dtype) if nbytes % np.dtype(dtype).itemsize == 0 else out

    def outputs_to_host(self, totals: dict) -> dict:
        """Every output buffer, sized like the reference's set_arguments_size does."""
        n = totals["n_events"]
        T = totals["host_total_number_of_velo_clusters"]
        tcs = totals["track_container_size"]
        reco = totals["host_number_of_reconstructed_velo_tracks"]
        three = totals["host_number_of_three_hit_tracks_filtered"]
        TH = totals["host_accumulated_number_of_hits_in_velo_tracks"]
        p = self.device_outputs()
        u4 = np.uint32
        sizes = {
            "dev_number_of_candidates": (4 * n, u4), "dev_estimated_input_size": (4 * 26 * n, u4),
            "dev_module_candidate_num": (4 * n, u4), "dev_offsets_estimated_input_size": (4 * (26 * n + 1), u4),
            "dev_module_cluster_num": (4 * 26 * n, u4),
            "dev_sorted_velo_cluster_container": (ELEMENT_SIZE * T, np.uint8),
            "dev_tracks": (TRACK_HITS_BYTES * tcs, np.uint8), "dev_three_hit_tracks": (TRACKLET_BYTES * tcs, np.uint16),
            "dev_hit_used": (T, np.uint8), "dev_atomics_velo": (4 * 3 * n, u4),
            "dev_number_of_velo_tracks": (4 * n, u4), "dev_offsets_velo_tracks": (4 * (n + 1), u4),
            "dev_three_hit_tracks_output": (TRACKLET_BYTES * tcs, np.uint16),
            "dev_number_of_three_hit_tracks_output": (4 * n, u4),
            "dev_offsets_number_of_three_hit_tracks_filtered": (4 * (n + 1), u4),
            "dev_offsets_all_velo_tracks": (4 * (n + 1), u4), "dev_velo_track_hit_number": (4 * reco, u4),
            "dev_offsets_velo_track_hit_number": (4 * (reco + 1), u4),
            "dev_velo_track_hits": (ELEMENT_SIZE * TH, np.uint8),
            "dev_accepted_velo_tracks": (reco + three, np.uint8),
        }
        if getattr(self, "retina", False):
            for k in ("dev_number_of_candidates", "dev_estimated_input_size", "dev_module_candidate_num"):
                del sizes[k]
            per_event = 208 if self.last_bank_version in (2, 3) else 104
            sizes.update({"dev_each_sensor_pair_size": (4 * per_event * n, u4),
                          "dev_offsets_each_sensor_pair_size": (4 * (per_event * n + 1), u4),
                          "dev_retina_bank_index": (4 * per_event, u4)})
        return {k: self._fetch(p[k], nb, dt) for k, (nb, dt) in sizes.items()}

    def run_host(self, s: RawSlice, stream=None) -> tuple[dict, dict, int, int]:
        """End-to-end from host buffers; returns (totals, consolidated outputs, h2d bytes, d2h bytes)."""
        raw = np.ascontiguousarray(s.raw)
        hs = HostSliceC(raw.ctypes.data, raw.nbytes, s.offsets.ctypes.data, s.sizes.ctypes.data, s.sizes.nbytes,
                        s.types.ctypes.data, s.types.nbytes, s.n_events, s.bank_version)
        cap_tracks = 2 * self.max_super_pixels + 64
        off_all = np.empty(s.n_events + 1, np.uint32)
        off_hn = np.empty(cap_tracks + 1, np.uint32)
        hits = np.empty(ELEMENT_SIZE * cap_tracks, np.uint8)
        t = TotalsC()
        up, down = C.c_ulonglong(), C.c_ulonglong()
        status = self.lib.velo_chain_run_host(
            self.handle, C.byref(hs), stream if stream is not None else _current_stream(),
            off_all.ctypes.data, off_all.nbytes, off_hn.ctypes.data, off_hn.nbytes, hits.ctypes.data, hits.nbytes,
            C.byref(t), C.byref(up), C.byref(down))
        totals = {f: getattr(t, f) for f, _ in TotalsC._fields_}
        _check(self.lib, status, totals["device_flags"])
        reco = totals["host_number_of_reconstructed_velo_tracks"]
        TH = totals["host_accumulated_number_of_hits_in_velo_tracks"]
        out = {"dev_offsets_all_velo_tracks": off_all,
               "dev_offsets_velo_track_hit_number": off_hn[:reco + 1],
               "dev_velo_track_hits": hits[:ELEMENT_SIZE * TH]}
        return totals, out, up.value, down.value


def pin_slice(s: RawSlice) -> RawSlice:
    """A copy of ``s`` in page-locked host memory (numpy views of pinned torch tensors), as
    HostPipeline.run takes its slices."""
    import torch

    def pinned(a):
        t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
        v = t.numpy()
        v[:] = np.ascontiguousarray(a).view(np.uint8).reshape(-1)
        return v.view(a.dtype), t

    raw, t0 = pinned(s.raw)
    off, t1 = pinned(s.offsets)
    siz, t2 = pinned(s.sizes)
    typ, t3 = pinned(s.types)
    r = RawSlice(raw, off, siz, typ, s.bank_version, getattr(s, "mep", False))
    r._keep = (t0, t1, t2, t3)
    return r


class HostPipeline:
    """End-to-end processing of slices held in page-locked host memory, through the C ABI.

    Three chains (by default) take the slices in turn, each on its own CUDA stream; the copies
    run on two more streams, one per direction, so that a slice's input going in, another's
    tracks coming out and a third one's kernels all overlap (PCIe is full duplex).  A chain's
    next slice waits, through CUDA events, for its input copy and for the copy-out of the
    chain's previous results.  Per slice the host receives dev_offsets_all_velo_tracks,
    dev_offsets_velo_track_hit_number and the id + xyz columns of dev_velo_track_hits
    (16 bytes per track hit; the phi column is never written by the reference).
    """

    def __init__(self, geometry: bytes | None = None, n_chains: int = 3, **props):
        import torch
        self.torch = torch
        self.chains = [VeloChain(geometry, **props) for _ in range(n_chains)]
        self.streams = [torch.cuda.Stream() for _ in range(n_chains)]
        self.h2d_stream = torch.cuda.Stream()
        self.d2h_stream = torch.cuda.Stream()
        self.dev_in = [None] * n_chains
        self.host_out = []
        self.h2d_bytes = 0
        self.d2h_bytes = 0

    def reserve(self, max_events: int, max_super_pixels: int, max_raw_bytes: int, max_sizes_words: int,
                max_types_words: int):
        torch = self.torch
        for i, c in enumerate(self.chains):
            c.reserve(max_events, max_super_pixels)
            self.dev_in[i] = (torch.empty(max_raw_bytes + 16, dtype=torch.uint8, device="cuda"),
                              torch.empty(max_events + 1, dtype=torch.int32, device="cuda"),
                              torch.empty(max_sizes_words, dtype=torch.int32, device="cuda"),
                              torch.empty(max_types_words, dtype=torch.int32, device="cuda"))
        self.max_super_pixels = max_super_pixels
        self.max_events = max_events
        self._out_buffers(2 * len(self.chains) - 1)  # page-locked now, not inside a timed run

    def _out_buffers(self, k):
        torch = self.torch
        while len(self.host_out) <= k:
            cap = 2 * self.max_super_pixels + 64
            self.host_out.append((torch.empty(self.max_events + 1, dtype=torch.int32, pin_memory=True),
                                  torch.empty(cap + 1, dtype=torch.int32, pin_memory=True),
                                  torch.empty(16 * cap, dtype=torch.uint8, pin_memory=True)))
        return self.host_out[k]

    def run(self, host_slices, keep_outputs: int = 0):
        """host_slices: RawSlice objects whose arrays are page-locked.  Returns the totals per
        slice; the outputs of the first `keep_outputs` slices are returned as numpy arrays too."""
        torch = self.torch
        n_c = len(self.chains)
        pending = [None] * n_c   # (slice index, out buffers) whose results are still on the device
        copied_out = [None] * n_c  # event: the chain's previous results are on the host
        totals_all, outputs = {}, {}

        def drain(ci):
            """Waits for chain ci's last run and queues the copy of its results to the host."""
            if pending[ci] is None:
                return
            k, bufs = pending[ci]
            chain = self.chains[ci]
            t = chain.synchronize()
            p = chain.device_outputs()
            n = t["n_events"]
            tracks = t["host_number_of_reconstructed_velo_tracks"]
            TH = t["host_accumulated_number_of_hits_in_velo_tracks"]
            stream = C.c_void_p(self.d2h_stream.cuda_stream)
            sizes = ((bufs[0], p["dev_offsets_all_velo_tracks"], 4 * (n + 1)),
                     (bufs[1], p["dev_offsets_velo_track_hit_number"], 4 * (tracks + 1)),
                     (bufs[2], p["dev_velo_track_hits"], 16 * TH))
            for host, dev, nbytes in sizes:
                _check(chain.lib, chain.lib.velo_copy_to_host_async(host.data_ptr(), dev, nbytes, stream))
                self.d2h_bytes += nbytes
            ev = torch.cuda.Event()
            ev.record(self.d2h_stream)
            copied_out[ci] = ev
            totals_all[k] = t
            if k < keep_outputs:  # copied now: the host buffers are reused every 2 n_c slices
                ev.synchronize()
                outputs[k] = {"dev_offsets_all_velo_tracks": bufs[0][:n + 1].numpy().view(np.uint32).copy(),
                              "dev_offsets_velo_track_hit_number":
                                  bufs[1][:tracks + 1].numpy().view(np.uint32).copy(),
                              "dev_velo_track_hits_id_xyz": bufs[2][:16 * TH].numpy().copy()}
            pending[ci] = None

        for k, s in enumerate(host_slices):
            if getattr(s, "mep", False):
                raise ValueError("HostPipeline takes Allen-layout slices (upload MEPs with chain.upload)")
            ci = k % n_c
            drain(ci)  # the chain's previous slice: finished (host waits), its results queued out
            raw_t, off_t, siz_t, typ_t = self.dev_in[ci]
            with torch.cuda.stream(self.h2d_stream):
                for dst, src in ((raw_t, s.raw.view(np.uint8)), (off_t, s.offsets.view(np.int32)),
                                 (siz_t, s.sizes.view(np.int32)), (typ_t, s.types.view(np.int32))):
                    dst[:src.size].copy_(torch.from_numpy(src), non_blocking=True)
                    self.h2d_bytes += src.nbytes
            copied_in = torch.cuda.Event()
            copied_in.record(self.h2d_stream)
            stream = self.streams[ci]
            stream.wait_event(copied_in)
            if copied_out[ci] is not None:
                stream.wait_event(copied_out[ci])  # the chain's outputs are about to be overwritten
            d = DeviceSlice(raw_t, off_t, siz_t, typ_t, s.n_events, s.bank_version, 0, s.retina)
            self.chains[ci].run(d, stream=C.c_void_p(stream.cuda_stream), use_graph=True)
            pending[ci] = (k, self._out_buffers(k % (2 * n_c)))
        for ci in range(n_c):
            drain(ci)
        self.d2h_stream.synchronize()
        for st in self.streams:
            st.synchronize()
        return [totals_all[k] for k in sorted(totals_all)], [outputs[k] for k in sorted(outputs)]

    def close(self):
        for c in self.chains:
            c.close()

"""Python access to the seeded synthetic event generator (include/velo_generator.h)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native
from .rawbanks import RawSlice


class VeloGenConfig(C.Structure):
    _fields_ = [
        ("mean_pileup", C.c_double), ("pileup_min", C.c_double), ("pileup_max", C.c_double),
        ("tracks_per_pv", C.c_double), ("eta_min", C.c_double), ("eta_max", C.c_double),
        ("beam_sigma_xy", C.c_double), ("beam_sigma_z", C.c_double),
        ("hit_efficiency", C.c_double), ("scatter_sigma", C.c_double),
        ("noise_rate", C.c_double), ("share_fraction", C.c_double),
        ("drop_corner_fraction", C.c_double), ("bank_version", C.c_int), ("sp_order", C.c_int),
        ("raw_format", C.c_int),
    ]


class VeloGenSizes(C.Structure):
    _fields_ = [("n_events", C.c_uint64), ("raw_bytes", C.c_uint64), ("sizes_words", C.c_uint64),
                ("types_words", C.c_uint64), ("n_truth_pixels", C.c_uint64), ("n_particles", C.c_uint64)]


TRUTH_DTYPE = np.dtype([("lhcb_id", np.uint32), ("particle", np.uint32)])
PARTICLE_DTYPE = np.dtype([("pv", np.uint32), ("eta", np.float32), ("phi", np.float32),
                           ("n_hits", np.uint32), ("n_modules", np.uint32)])


@dataclass
class Generated:
    raw: RawSlice
    truth_pixels: np.ndarray
    truth_offsets: np.ndarray
    particles: np.ndarray
    particle_offsets: np.ndarray
    config: dict = field(default_factory=dict)


def _lib():
    lib = _native.load_generator()
    if not getattr(lib, "_typed", False):
        lib.velo_gen_default_config.argtypes = [C.POINTER(VeloGenConfig)]
        lib.velo_gen_create.restype = C.c_void_p
        lib.velo_gen_create.argtypes = [C.POINTER(VeloGenConfig), C.c_char_p, C.c_size_t, C.c_uint64,
                                        C.c_uint, C.c_uint, C.c_uint]
        lib.velo_gen_sizes.argtypes = [C.c_void_p, C.POINTER(VeloGenSizes)]
        lib.velo_gen_copy.argtypes = [C.c_void_p] + [C.c_void_p] * 8
        lib.velo_gen_destroy.argtypes = [C.c_void_p]
        lib._typed = True
    return lib


def default_config() -> dict:
    cfg = VeloGenConfig()
    _lib().velo_gen_default_config(C.byref(cfg))
    return {k: getattr(cfg, k) for k, _ in VeloGenConfig._fields_}


def generate(n_events: int, seed: int = 1, first_event: int = 0, geometry: bytes | None = None,
             n_threads: int = 0, pinned_alloc=None, **overrides) -> Generated:
    """Generates ``n_events`` events of stream ``seed``.

    ``overrides`` set VeloGenConfig fields (mean_pileup, pileup_min/max, noise_rate,
    hit_efficiency, bank_version, ...).  ``pinned_alloc(nbytes) -> uint8 array`` may
    supply the raw-byte buffer (e.g. page-locked host memory).
    """
    lib = _lib()
    cfg = VeloGenConfig()
    lib.velo_gen_default_config(C.byref(cfg))
    for k, v in overrides.items():
        if not hasattr(cfg, k):
            raise KeyError(f"unknown generator setting {k}")
        setattr(cfg, k, v)
    geo = geometry if geometry is not None else _native.default_geometry()
    h = lib.velo_gen_create(C.byref(cfg), geo, len(geo), seed, first_event, n_events, n_threads)
    if not h:
        raise ValueError("generator rejected the geometry blob or the bank version")
    try:
        sz = VeloGenSizes()
        lib.velo_gen_sizes(h, C.byref(sz))
        raw = pinned_alloc(sz.raw_bytes) if pinned_alloc else np.empty(sz.raw_bytes, dtype=np.uint8)
        offsets = np.empty(n_events + 1, dtype=np.uint32)
        sizes = np.zeros(sz.sizes_words, dtype=np.uint32)
        types = np.zeros(sz.types_words, dtype=np.uint32)
        truth = np.empty(sz.n_truth_pixels, dtype=TRUTH_DTYPE)
        truth_off = np.empty(n_events + 1, dtype=np.uint32)
        parts = np.empty(sz.n_particles, dtype=PARTICLE_DTYPE)
        part_off = np.empty(n_events + 1, dtype=np.uint32)
        lib.velo_gen_copy(h, raw.ctypes.data, offsets.ctypes.data, sizes.ctypes.data, types.ctypes.data,
                          truth.ctypes.data, truth_off.ctypes.data, parts.ctypes.data, part_off.ctypes.data)
    finally:
        lib.velo_gen_destroy(h)
    cfgd = {k: getattr(cfg, k) for k, _ in VeloGenConfig._fields_}
    return Generated(RawSlice(raw, offsets, sizes, types, cfg.bank_version), truth, truth_off,
                     parts, part_off, cfgd)

"""Locates (and if needed builds) the native libraries of the package.

* ``_lib/libvelo_b200.so`` - the sm_100a CUDA kernels behind the C ABI of
  include/velo_b200.h.  There is no CPU fallback: when this library cannot be
  loaded every GPU entry point raises.
* ``_lib/libvelo_gen.so``  - the host-only synthetic event generator.
* ``_lib/libvelo_io.so``   - the host-only MDF index and VELO transpose of include/velo_io.h.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(PKG, "_lib")
CHAIN_LIB = os.path.join(LIB_DIR, "libvelo_b200.so")
GEN_LIB = os.path.join(LIB_DIR, "libvelo_gen.so")
IO_LIB = os.path.join(LIB_DIR, "libvelo_io.so")
GEOMETRY = os.path.join(PKG, "data", "velo_geometry.bin")

_lock = threading.Lock()
_loaded = {}


def _load(path: str, builder):
    with _lock:
        if path in _loaded:
            return _loaded[path]
        if not os.path.exists(path):
            builder()
        if not os.path.exists(path):
            raise RuntimeError(f"native library {path} is missing and could not be built")
        lib = C.CDLL(path)
        _loaded[path] = lib
        return lib


def load_chain():
    from . import build
    return _load(CHAIN_LIB, build.build_chain)


def load_generator():
    from . import build
    return _load(GEN_LIB, build.build_generator)


def load_io():
    from . import build
    return _load(IO_LIB, build.build_io)


TUNED_CONFIG = os.path.join(PKG, "data", "launch_config.json")


def tuned_launch_config() -> dict | None:
    """The launch configuration picked by allen_b200.autotune, if one was saved."""
    import json
    try:
        with open(TUNED_CONFIG) as f:
            return json.load(f).get("config")
    except (OSError, ValueError):
        return None


def default_geometry() -> bytes:
    with open(GEOMETRY, "rb") as f:
        return f.read()

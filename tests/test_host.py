"""Host-side logic: raw-bank layout, generator, C-ABI library exports (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np

from allen_b200 import _native, generator, rawbanks

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_rawbank_roundtrip():
    g = generator.generate(5, seed=2)
    s = g.raw
    banks = [rawbanks.banks_of_event(s, e) for e in range(s.n_events)]
    s2 = rawbanks.build_slice(banks, s.bank_version)
    assert np.array_equal(s.raw, s2.raw)
    assert np.array_equal(s.offsets, s2.offsets)
    assert np.array_equal(s.sizes.view(np.uint8)[:s2.sizes.nbytes], s2.sizes.view(np.uint8)[:s.sizes.nbytes])


def test_generator_deterministic_and_thread_independent():
    a = generator.generate(12, seed=4, n_threads=1)
    b = generator.generate(12, seed=4, n_threads=5)
    assert np.array_equal(a.raw.raw, b.raw.raw)
    c = generator.generate(6, seed=4, first_event=6)
    assert np.array_equal(a.raw.raw[a.raw.offsets[6]:], c.raw.raw)


def test_generator_occupancy():
    g = generator.generate(50, seed=1)
    sp = rawbanks.super_pixels_per_event(g.raw)
    assert 1500 < sp.mean() < 4500
    assert g.particles.size > 50 * 100


def test_isolated_flag_is_exact():
    g = generator.generate(3, seed=8)
    for e in range(3):
        for (_, sensor, payload) in rawbanks.banks_of_event(g.raw, e):
            w = np.frombuffer(payload, np.uint32)[1:]
            w = [int(x) for x in w]
            addr = {((x >> 14) & 0x1FF, (x >> 8) & 0x3F) for x in w}
            for x in w:
                c, r = (x >> 14) & 0x1FF, (x >> 8) & 0x3F
                neigh = any((c + dc, r + dr) in addr for dc in (-1, 0, 1) for dr in (-1, 0, 1) if dc or dr)
                assert bool(x >> 31) == (not neigh)


def test_chain_library_exports_every_declared_symbol():
    from allen_b200 import build
    path = build.build_chain()
    lib = C.CDLL(path)
    header = open(os.path.join(REPO, "include", "velo_b200.h")).read()
    names = re.findall(r"^\s*(?:VeloStatus|void|const char\*)\s+(velo_\w+)\s*\(", header, re.M)
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n


def test_generator_library_exports():
    lib = C.CDLL(_native.GEN_LIB)
    header = open(os.path.join(REPO, "include", "velo_generator.h")).read()
    for n in re.findall(r"(velo_gen_\w+)\s*\(", header):
        assert hasattr(lib, n), n

"""Raw input path on the host: MDF record index and VELO transpose (libvelo_io.so), checked
against the reference's own MDF reader and transpose compiled as CPU C++ (oracle/_ref) and
against the committed fixture it produced (no GPU needed)."""
import ctypes as C
import os
import re
import struct
import sys

import numpy as np
import pytest

import cpu_checkers
import mdf_streams
from allen_b200 import _native, generator, mdf, rawbanks

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, "oracle"))
import build_checkers  # noqa: E402

_REF_ROOT = build_checkers.reference_root()
REF_MDF = os.path.join(_REF_ROOT or "", "input", "minbias", "mdf",
                       "MiniBrunel_2018_MinBias_FTv4_DIGI_retinacluster_v1.mdf")
FIXTURE = os.path.join(REPO, "tests", "golden", "mdf_synthetic_8ev.npz")

needs_ref = pytest.mark.skipif(not cpu_checkers.available("ref"), reason="reference CPU build absent")
needs_ref_mdf = pytest.mark.skipif(not os.path.exists(REF_MDF), reason="reference MDF sample absent")


def slice_bytes(s: rawbanks.RawSlice) -> dict:
    return {"raw": np.asarray(s.raw).view(np.uint8), "offsets": s.offsets.view(np.uint8),
            "sizes": s.sizes.view(np.uint8), "types": s.types.view(np.uint8)}


def assert_same_slice(ours: rawbanks.RawSlice, ref: dict):
    got = slice_bytes(ours)
    for k in ("raw", "offsets", "sizes", "types"):
        assert np.array_equal(got[k], ref[k].view(np.uint8)), k
    assert ours.bank_version == ref["bank_version"]


def test_io_library_exports_every_declared_symbol():
    lib = C.CDLL(_native.load_io()._name)
    header = open(os.path.join(REPO, "include", "velo_io.h")).read()
    names = re.findall(r"^\s*(?:VeloIoStatus|int|const char\*)\s+(velo_\w+)\s*\(", header, re.M)
    assert set(names) == {"velo_mdf_scan", "velo_mdf_select_by_source_id", "velo_transpose_vp", "velo_io_last_error"}
    for n in names:
        assert hasattr(lib, n), n


def test_checksum_of_written_records_verifies():
    g = generator.generate(3, seed=21)
    stream = mdf_streams.synthetic_stream(g.raw, seed=1)
    ev = mdf.scan(stream, check_checksum=True)
    assert ev.size == 3
    assert np.all(ev["record_bytes"] == ev["banks_bytes"] + 48)
    bad = bytearray(stream)
    bad[int(ev[1]["banks_offset"]) + 100] ^= 0x40
    with pytest.raises(mdf.MdfError) as e:
        mdf.scan(bytes(bad), check_checksum=True)
    assert e.value.status == mdf.ERR_CHECKSUM
    assert mdf.scan(bytes(bad)).size == 3  # not checked


@pytest.mark.parametrize("header_version", [0, 1, 2, 3])
def test_header_versions(header_version):
    g = generator.generate(2, seed=3)
    stream = mdf_streams.synthetic_stream(g.raw, seed=2, header_version=header_version)
    ev = mdf.scan(stream, check_checksum=True)
    hdr = {0: 40, 1: 48, 2: 20, 3: 48}[header_version]
    assert np.all(ev["banks_offset"] - ev["record_offset"] == hdr)
    s = mdf.transpose_vp(stream, ev)
    assert np.array_equal(s.raw, g.raw.raw) and np.array_equal(s.offsets, g.raw.offsets)


def test_scan_stops_before_an_incomplete_record_and_rejects_bad_headers():
    g = generator.generate(3, seed=5)
    stream = mdf_streams.synthetic_stream(g.raw, seed=3)
    full = mdf.scan(stream)
    cut = stream[:int(full[2]["record_offset"]) + 100]
    part = mdf.scan(cut)
    assert part.size == 2 and np.array_equal(part, full[:2])
    assert mdf.scan(stream, max_events=1).size == 1
    assert mdf.scan(b"").size == 0
    # indexed in batches of one record per library call, resuming each time: the same index
    assert np.array_equal(mdf.scan(stream, batch=1), full)
    assert np.array_equal(mdf.scan(stream, batch=2, max_events=3), full)
    compressed = bytearray(stream)
    compressed[int(full[1]["record_offset"]) + 16] = 0x12  # zlib-style compression code
    with pytest.raises(mdf.MdfError) as e:
        mdf.scan(bytes(compressed))
    assert e.value.status == mdf.ERR_UNSUPPORTED
    bad_version = bytearray(stream)
    bad_version[17] = 0x77
    with pytest.raises(mdf.MdfError) as e:
        mdf.scan(bytes(bad_version))
    assert e.value.status == mdf.ERR_FORMAT


def test_transpose_restores_the_generated_slice_in_both_selection_modes():
    g = generator.generate(25, seed=11)
    for by_source_id in (False, True):
        stream = mdf_streams.synthetic_stream(g.raw, seed=4, by_source_id=by_source_id)
        ev = mdf.scan(stream)
        assert mdf.select_by_source_id(stream, ev[0]) == by_source_id
        s = mdf.transpose_vp(stream, ev)
        banks = [rawbanks.banks_of_event(s, e) for e in range(s.n_events)]
        want = [[(t, mdf_streams.velo_source(src, by_source_id), p) for (t, src, p) in rawbanks.banks_of_event(g.raw, e)]
                for e in range(g.raw.n_events)]
        assert banks == want
        if not by_source_id:
            assert np.array_equal(s.raw, g.raw.raw)
            assert np.array_equal(s.sizes.view(np.uint8), g.raw.sizes.view(np.uint8)[:s.sizes.nbytes])


def test_transpose_is_independent_of_thread_count_and_sizes_itself():
    g = generator.generate(300, seed=12)
    stream = mdf_streams.synthetic_stream(g.raw, seed=5, extra_velo=True)
    ev = mdf.scan(stream)
    one = mdf.transpose_vp(stream, ev, n_threads=1)
    for t in (2, 3, 7, 0):
        many = mdf.transpose_vp(stream, ev, n_threads=t)
        for k, v in slice_bytes(one).items():
            assert np.array_equal(v, slice_bytes(many)[k]), (t, k)
    # a buffer one byte short is refused, nothing written
    lib = _native.load_io()
    info = mdf.TransposeInfoC()
    raw = np.zeros(one.raw.size - 1, np.uint8)
    off = np.zeros(ev.size + 1, np.uint32)
    sz = np.zeros(one.sizes.size, np.uint32)
    ty = np.zeros(one.types.size, np.uint32)
    buf = np.frombuffer(stream, np.uint8)
    st = lib.velo_transpose_vp(buf.ctypes.data, ev.ctypes.data, ev.size, 0, 0, raw.ctypes.data, raw.size, off.ctypes.data,
                               sz.ctypes.data, sz.nbytes, ty.ctypes.data, ty.nbytes, C.byref(info))
    assert st == mdf.ERR_CAPACITY and info.raw_bytes == one.raw.size
    assert not raw.any() and not off.any()


def test_event_without_velo_banks_is_written_empty():
    g = generator.generate(4, seed=13)
    stream = mdf_streams.synthetic_stream(g.raw, seed=6, drop_velo_events=(2,))
    s = mdf.transpose_vp(stream, mdf.scan(stream))
    assert s.n_events == 4
    assert rawbanks.banks_of_event(s, 2) == []
    for e in (0, 1, 3):
        assert rawbanks.banks_of_event(s, e) == rawbanks.banks_of_event(g.raw, e)


def test_malformed_bank_is_an_error():
    g = generator.generate(2, seed=14)
    stream = bytearray(mdf_streams.synthetic_stream(g.raw, seed=7))
    ev = mdf.scan(bytes(stream))
    p = int(ev[1]["banks_offset"])
    stream[p:p + 2] = struct.pack("<H", 0xABCD)
    with pytest.raises(mdf.MdfError) as e:
        mdf.transpose_vp(bytes(stream), ev, by_source_id=False)
    assert e.value.status == mdf.ERR_FORMAT and "event 1" in str(e.value)


def test_transpose_matches_the_committed_reference_fixture():
    """The fixture holds synthetic MDF streams and the VP slices the reference's own reader
    and transpose wrote for them (tests/golden/make_fixtures.py)."""
    z = np.load(FIXTURE)
    for mode in ("by_type", "by_source"):
        stream = z[mode + "__stream"].tobytes()
        ev = mdf.scan(stream, check_checksum=True)
        s = mdf.transpose_vp(stream, ev)
        ref = {k: z[mode + "__" + k] for k in ("raw", "offsets", "sizes", "types")}
        ref["bank_version"] = int(z[mode + "__bank_version"][0])
        assert_same_slice(s, ref)


@needs_ref
@pytest.mark.parametrize("by_source_id", [False, True])
def test_transpose_matches_reference_build(by_source_id):
    g = generator.generate(40, seed=15, mean_pileup=5.0)
    stream = mdf_streams.synthetic_stream(g.raw, seed=8, by_source_id=by_source_id, extra_velo=True)
    ref = cpu_checkers.ref_transpose_vp(stream, 40, check_checksum=True)
    assert ref["status"] == 0 and ref["by_source_id"] == by_source_id
    s = mdf.transpose_vp(stream, mdf.scan(stream, check_checksum=True))
    assert_same_slice(s, ref)


@needs_ref
@needs_ref_mdf
def test_real_sample_matches_reference_build():
    """The 2018 minbias MDF (VP and VPRetinaCluster banks in one VELO slice, version 2)."""
    stream = open(REF_MDF, "rb").read()
    ev = mdf.scan(stream, check_checksum=True)
    assert ev.size == 10 and not mdf.select_by_source_id(stream, ev[0])
    ref = cpu_checkers.ref_transpose_vp(stream, 10, check_checksum=True)
    s = mdf.transpose_vp(stream, ev)
    assert_same_slice(s, ref)
    assert s.n_events == 10 and int(s.sizes[1]) - int(s.sizes[0]) == 416

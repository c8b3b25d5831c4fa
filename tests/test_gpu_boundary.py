"""The drop-in boundary on the GPU: caller-owned memory (velo_chain_sizes / velo_chain_bind) in
both coordinate layouts, the consolidated track views (velo_create_velo_views), and the Allen
adaptor (integration/VeloB200Chain.cu) run through the reference's own ArgumentReferences with
the reference's own velo_kalman_filter reading its outputs (tests/allen_harness)."""
import ctypes as C
import os

import numpy as np
import pytest

import parity
from allen_b200 import generator
from allen_b200.chain import COORDINATES_FP16, COORDINATES_FP32, OutputBuffersC, VeloChain, _current_stream, upload
from allen_b200.rawbanks import super_pixels_per_event

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(REPO, "tests", "allen_harness", "_build", "libvelo_allen_harness.so")


def _caller_memory(chain, n, sp, layout):
    import torch
    s = chain.sizes(n, sp, layout)
    ws = torch.zeros(s["workspace_bytes"] + 256, dtype=torch.uint8, device="cuda")
    ws_ptr = (ws.data_ptr() + 255) & ~255
    counts = {
        "dev_offsets_estimated_input_size": 4 * s["offsets_estimated_input_size"],
        "dev_module_cluster_num": 4 * s["module_cluster_num"],
        "dev_sorted_velo_cluster_container": s["sorted_velo_cluster_container_bytes"],
        "dev_offsets_all_velo_tracks": 4 * s["offsets_all_velo_tracks"],
        "dev_velo_track_hit_number": 4 * s["velo_track_hit_number"],
        "dev_offsets_velo_track_hit_number": 4 * s["offsets_velo_track_hit_number"],
        "dev_velo_track_hits": s["velo_track_hits_bytes"],
        "dev_accepted_velo_tracks": s["accepted_velo_tracks"],
    }
    bufs = {k: torch.zeros(v + 16, dtype=torch.uint8, device="cuda") for k, v in counts.items()}
    return s, ws, ws_ptr, bufs


def _half_fields(buf, T):
    b = buf[:12 * T]
    return b[:4 * T].view(np.uint32), b[4 * T:10 * T].view(np.float16).reshape(T, 3), b[10 * T:12 * T].view(np.int16)


@pytest.mark.parametrize("layout", [COORDINATES_FP32, COORDINATES_FP16])
def test_caller_owned_memory(geometry, oracle, layout):
    """A chain bound to caller memory computes the oracle's outputs into the caller's buffers
    (FP32: bit for bit; FP16: the oracle's coordinates rounded to nearest half, ids and phi
    exact), allocates no device memory while it runs, and re-binding the same memory is free."""
    import torch
    slices = [generator.generate(50, seed=300 + i, pileup_min=1.0, pileup_max=15.0).raw for i in range(2)]
    n = max(s.n_events for s in slices)
    sp = max(int(super_pixels_per_event(s).sum()) for s in slices) + 64
    chain = VeloChain(geometry)
    try:
        s, ws, ws_ptr, bufs = _caller_memory(chain, n, sp, layout)
        assert s["workspace_bytes"] > 0
        outputs = {f: bufs[f].data_ptr() for f, _ in OutputBuffersC._fields_}
        for i, raw in enumerate(slices * 2):
            d = upload(raw)
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            chain.bind(ws_ptr, s["workspace_bytes"], n, sp, outputs, layout)
            chain.run(d)
            totals = chain.synchronize()
            torch.cuda.synchronize()
            if i > 0:
                assert free_before - torch.cuda.mem_get_info()[0] < (2 << 20)
            ref = oracle.run(raw, geometry)
            host = {k: v.cpu().numpy() for k, v in bufs.items()}
            N = raw.n_events
            assert np.array_equal(host["dev_offsets_estimated_input_size"][:4 * (26 * N + 1)].view(np.uint32),
                                  ref["dev_offsets_estimated_input_size"])
            assert np.array_equal(host["dev_module_cluster_num"][:4 * 26 * N].view(np.uint32),
                                  ref["dev_module_cluster_num"])
            assert np.array_equal(host["dev_offsets_all_velo_tracks"][:4 * (N + 1)].view(np.uint32),
                                  ref["dev_offsets_all_velo_tracks"])
            reco = int(ref["dev_offsets_all_velo_tracks"][-1])
            assert totals["host_number_of_reconstructed_velo_tracks"] == reco
            assert np.array_equal(host["dev_offsets_velo_track_hit_number"][:4 * (reco + 1)].view(np.uint32),
                                  ref["dev_offsets_velo_track_hit_number"])
            assert np.array_equal(host["dev_velo_track_hit_number"][:4 * reco].view(np.uint32),
                                  ref["dev_velo_track_hit_number"])
            assert np.array_equal(host["dev_accepted_velo_tracks"][:ref["dev_accepted_velo_tracks"].size],
                                  ref["dev_accepted_velo_tracks"])
            T = int(ref["dev_offsets_estimated_input_size"][-1])
            TH = int(ref["dev_offsets_velo_track_hit_number"][-1])
            mask = parity.sorted_container_mask(ref["dev_offsets_estimated_input_size"], ref["dev_module_cluster_num"], T)
            rid, rxyz, rphi = parity.container_fields(ref["dev_sorted_velo_cluster_container"], T)
            tid, txyz, _ = parity.container_fields(ref["dev_velo_track_hits"], TH)
            if layout == COORDINATES_FP32:
                gid, gxyz, gphi = parity.container_fields(host["dev_sorted_velo_cluster_container"][:18 * T], T)
                assert np.array_equal(parity._u8(gxyz[mask]), parity._u8(rxyz[mask]))
                hid, hxyz, _ = parity.container_fields(host["dev_velo_track_hits"][:18 * TH], TH)
                assert np.array_equal(parity._u8(hxyz), parity._u8(txyz))
            else:
                gid, gxyz, gphi = _half_fields(host["dev_sorted_velo_cluster_container"], T)
                assert np.array_equal(gxyz[mask].view(np.uint16), rxyz[mask].astype(np.float16).view(np.uint16))
                hid, hxyz, _ = _half_fields(host["dev_velo_track_hits"], TH)
                assert np.array_equal(hxyz.view(np.uint16), txyz.astype(np.float16).view(np.uint16))
            assert np.array_equal(gid[mask], rid[mask]) and np.array_equal(gphi[mask], rphi[mask])
            assert np.array_equal(hid, tid)
        with pytest.raises(Exception):
            chain.bind(ws_ptr, s["workspace_bytes"] - 256, n, sp, outputs, layout)
    finally:
        chain.close()


def test_velo_views(chain, geometry):
    """velo_create_velo_views writes each view field as the reference's constructors compute it
    (VeloConsolidated.cuh:68-80, 217-230, 278-281; MultiEventContainer.cuh:48-50)."""
    import torch
    g = generator.generate(40, seed=310)
    chain.reserve_for(g.raw)
    chain.run(upload(g.raw))
    totals = chain.synchronize()
    out = chain.outputs_to_host(totals)
    p = chain.device_outputs()
    n = g.raw.n_events
    reco = totals["host_number_of_reconstructed_velo_tracks"]
    hits_v = torch.zeros(24 * n, dtype=torch.uint8, device="cuda")
    track_v = torch.zeros(24 * reco, dtype=torch.uint8, device="cuda")
    tracks_v = torch.zeros(16 * n, dtype=torch.uint8, device="cuda")
    multi_v = torch.zeros(24, dtype=torch.uint8, device="cuda")
    imec = torch.zeros(8, dtype=torch.uint8, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = chain.lib.velo_create_velo_views(n, p["dev_velo_track_hits"], p["dev_offsets_all_velo_tracks"],
                                          p["dev_offsets_velo_track_hit_number"], hits_v.data_ptr(), track_v.data_ptr(),
                                          reco, tracks_v.data_ptr(), multi_v.data_ptr(), imec.data_ptr(),
                                          status.data_ptr(), _current_stream())
    assert st == 0
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    offs = out["dev_offsets_all_velo_tracks"].astype(np.int64)
    hn = out["dev_offsets_velo_track_hit_number"].astype(np.int64)
    hv = hits_v.cpu().numpy()
    for e in range(n):
        rec = hv[24 * e:24 * e + 24]
        assert int(rec[:8].view(np.uint64)[0]) == p["dev_velo_track_hits"]
        assert list(rec[8:20].view(np.uint32)) == [hn[offs[e]], hn[offs[e + 1]] - hn[offs[e]], hn[offs[n]]]
    tv = track_v.cpu().numpy().reshape(reco, 24)
    for e in range(n):
        for t in range(offs[e + 1] - offs[e]):
            rec = tv[offs[e] + t]
            assert int(rec[:8].view(np.uint64)[0]) == hits_v.data_ptr() + 24 * e
            first = offs[e] + t
            assert list(rec[8:24].view(np.uint32)) == [t, offs[e], hn[first] - hn[offs[e]], hn[first + 1] - hn[first]]
    tsv = tracks_v.cpu().numpy().reshape(n, 16)
    for e in range(n):
        assert int(tsv[e, :8].view(np.uint64)[0]) == track_v.data_ptr() + 24 * int(offs[e])
        assert list(tsv[e, 8:16].view(np.uint32)) == [offs[e + 1] - offs[e], offs[e]]
    m = multi_v.cpu().numpy()
    assert int(m[:4].view(np.int32)[0]) == 1
    assert int(m[8:16].view(np.uint64)[0]) == tracks_v.data_ptr() and int(m[16:20].view(np.uint32)[0]) == n
    assert int(imec.cpu().numpy().view(np.uint64)[0]) == multi_v.data_ptr()
    # too small a track-view capacity: flagged, nothing written
    status.zero_()
    track_v.zero_()
    chain.lib.velo_create_velo_views(n, p["dev_velo_track_hits"], p["dev_offsets_all_velo_tracks"],
                                     p["dev_offsets_velo_track_hit_number"], hits_v.data_ptr(), track_v.data_ptr(),
                                     reco - 1, tracks_v.data_ptr(), multi_v.data_ptr(), imec.data_ptr(),
                                     status.data_ptr(), _current_stream())
    torch.cuda.synchronize()
    assert int(status.item()) != 0 and int(track_v.sum().item()) == 0


class HarnessInput(C.Structure):
    _fields_ = [("raw", C.c_void_p), ("offsets", C.c_void_p), ("sizes", C.c_void_p), ("types", C.c_void_p),
                ("raw_bytes", C.c_size_t), ("sizes_words", C.c_size_t), ("types_words", C.c_size_t),
                ("event_start", C.c_uint), ("n_events", C.c_uint), ("n_slice", C.c_uint), ("bank_version", C.c_int),
                ("geometry", C.c_char_p), ("geometry_size", C.c_size_t), ("beamline_x", C.c_float),
                ("beamline_y", C.c_float)]


def _harness():
    if not os.path.exists(HARNESS):
        pytest.skip("Allen harness not built (it needs the reference tree: make -C tests/allen_harness)")
    lib = C.CDLL(HARNESS)
    lib.allen_harness_run.restype = C.c_void_p
    lib.allen_harness_run.argtypes = [C.POINTER(HarnessInput)]
    lib.allen_harness_error.restype = C.c_char_p
    lib.allen_harness_buffer.restype = C.c_int
    lib.allen_harness_buffer.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t),
                                         C.POINTER(C.c_int)]
    lib.allen_harness_names.restype = C.c_char_p
    lib.allen_harness_names.argtypes = [C.c_void_p]
    lib.allen_harness_free.argtypes = [C.c_void_p]
    return lib


def _buffer(chain, lib, h, name):
    ptr, nbytes, dev = C.c_void_p(), C.c_size_t(), C.c_int()
    assert lib.allen_harness_buffer(h, name.encode(), C.byref(ptr), C.byref(nbytes), C.byref(dev)), name
    if not dev.value:
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint8)), shape=(nbytes.value,)).copy()
    return chain._fetch(ptr.value, nbytes.value, np.uint8)


@pytest.mark.parametrize("beamline", [(0.0, 0.0), (0.2, -0.1)])
def test_allen_adaptor_with_reference_kalman(chain, oracle, geometry, beamline):
    """velo_b200_chain_t run as Allen runs an algorithm (ArgumentReferences, set_arguments_size,
    arena-style memory, operator()) in the reference's CUDA-build layout (half coordinates):
    its outputs are the oracle's; the reference's own view types walk its views to the
    consolidated hits; and the reference's own velo_kalman_filter, bound to its
    dev_velo_tracks_view and dev_offsets_all_velo_tracks, gives the states this library's
    Kalman filter computes on the same hits."""
    import torch
    lib = _harness()
    g = generator.generate(40, seed=320, pileup_min=1.0, pileup_max=15.0)
    d = upload(g.raw)
    n = g.raw.n_events
    hin = HarnessInput(d.raw.data_ptr(), d.offsets.data_ptr(), d.sizes.data_ptr(), d.types.data_ptr(),
                       d.raw.numel(), d.sizes.numel(), d.types.numel(), 0, n, n, g.raw.bank_version,
                       geometry, len(geometry), beamline[0], beamline[1])
    h = lib.allen_harness_run(C.byref(hin))
    assert h, lib.allen_harness_error().decode()
    try:
        get = lambda name: _buffer(chain, lib, h, name)  # noqa: E731
        ref = oracle.run(g.raw, geometry, beamline=beamline)
        reco = int(ref["dev_offsets_all_velo_tracks"][-1])
        T = int(ref["dev_offsets_estimated_input_size"][-1])
        TH = int(ref["dev_offsets_velo_track_hit_number"][-1])
        assert int(get("host_number_of_reconstructed_velo_tracks_t").view(np.uint32)[0]) == reco
        assert int(get("host_total_number_of_velo_clusters_t").view(np.uint32)[0]) == T
        assert int(get("host_accumulated_number_of_hits_in_velo_tracks_t").view(np.uint32)[0]) == TH
        for k in ("dev_offsets_estimated_input_size", "dev_module_cluster_num", "dev_offsets_all_velo_tracks",
                  "dev_velo_track_hit_number", "dev_offsets_velo_track_hit_number", "dev_accepted_velo_tracks"):
            assert np.array_equal(get(k + "_t"), parity._u8(ref[k])), k
        # containers in the CUDA build's layout (half coordinates), reduced to their exact sizes
        sorted_half = get("dev_sorted_velo_cluster_container_t")
        hits_half = get("dev_velo_track_hits_t")
        assert sorted_half.size == 12 * T and hits_half.size == 12 * TH
        tid, txyz, _ = parity.container_fields(ref["dev_velo_track_hits"], TH)
        hid, hxyz, _ = _half_fields(hits_half, TH)
        assert np.array_equal(hid, tid)
        assert np.array_equal(hxyz.view(np.uint16), txyz.astype(np.float16).view(np.uint16))
        # the views, walked with the reference's types
        counts = get("walked_counts").view(np.uint32)
        assert list(counts) == [n, reco, TH]
        walked = get("walked_hits").view(np.uint32).reshape(TH, 4)
        assert np.array_equal(walked[:, 0], tid)
        assert np.array_equal(walked[:, 1:].view(np.float32), hxyz.astype(np.float32))
        # the reference's Kalman filter on those views = this library's on the same (half) hits
        rebuilt = np.concatenate([tid.view(np.uint8), hxyz.astype(np.float32).reshape(-1).view(np.uint8),
                                  np.zeros(2 * TH, np.uint8)])
        t_hits = torch.from_numpy(rebuilt).cuda()
        t_offs = torch.from_numpy(ref["dev_offsets_all_velo_tracks"].view(np.int32).copy()).cuda()
        t_hn = torch.from_numpy(ref["dev_offsets_velo_track_hit_number"].view(np.int32).copy()).cuda()
        back = torch.zeros(reco + 1, dtype=torch.uint8, device="cuda")
        beam = torch.zeros(56 * reco + 8, dtype=torch.uint8, device="cuda")
        end = torch.zeros(56 * reco + 8, dtype=torch.uint8, device="cuda")
        st = chain.lib.velo_run_kalman_filter(n, t_offs.data_ptr(), t_hn.data_ptr(), t_hits.data_ptr(), reco,
                                              beamline[0], beamline[1], back.data_ptr(), beam.data_ptr(),
                                              end.data_ptr(), None, _current_stream())
        assert st == 0
        torch.cuda.synchronize()
        assert np.array_equal(get("ref_kalman_is_backward"), back.cpu().numpy()[:reco])
        w = parity.kalman_written_words(reco)
        for name, ours in (("ref_kalman_beamline_states", beam), ("ref_kalman_endvelo_states", end)):
            theirs = get(name)[:56 * reco].view(np.uint32)
            assert np.array_equal(theirs[w], ours.cpu().numpy()[:56 * reco].view(np.uint32)[w]), name
    finally:
        lib.allen_harness_free(h)

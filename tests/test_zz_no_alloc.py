"""The allocation-free decoding entry point, velo_decode_noalloc(), through the C ABI.

Callers that run inside a pre-reserved memory arena (an Allen sequence, whose scheduler
owns every device buffer) cannot call cudaMalloc; this entry point keeps its scratch in
static device memory instead.  Its outputs must equal those of the chain's own decoding
(velo_chain_run) bit for bit, on two calls in a row: the second call reuses the scratch
the first one left behind.  The file name keeps this test last in collection order.
"""
import ctypes as C

import numpy as np
import pytest

import parity

pytestmark = pytest.mark.gpu


def _noalloc_lib():
    from allen_b200 import chain as ch
    lib = ch._lib()
    lib.velo_decode_noalloc.restype = C.c_int
    lib.velo_decode_noalloc.argtypes = [
        C.c_char_p, C.c_size_t, C.POINTER(ch.DeviceSliceC), C.c_ulonglong, C.c_void_p,
        C.c_void_p, C.c_void_p, C.c_void_p, C.c_ulonglong, C.c_void_p]
    lib.velo_noalloc_max_events.restype = C.c_uint
    lib.velo_noalloc_max_clusters.restype = C.c_uint
    lib.velo_noalloc_last_error_string.restype = C.c_char_p
    return lib


# Calls in a row: two of the same size, then a smaller slice of v4 banks after a larger one
# (the scratch still holds the larger call's contents), then a v3 slice.
CALLS = [(40, 21, {}), (40, 22, {}), (44, 23, dict(pileup_min=1.0, pileup_max=15.0)),
         (25, 24, dict(bank_version=4)), (30, 25, dict(bank_version=3))]


def test_decode_noalloc_matches_chain_on_two_calls(geometry):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from allen_b200 import generator
    from allen_b200.chain import VeloChain, upload, _current_stream
    from allen_b200.rawbanks import super_pixels_per_event

    lib = _noalloc_lib()
    assert lib.velo_noalloc_max_events() >= max(n for n, _, _ in CALLS)
    chain = VeloChain(geometry)
    try:
        for n_events, seed, cfg in CALLS:
            g = generator.generate(n_events, seed=seed, **cfg)
            n = g.raw.n_events
            sp = int(super_pixels_per_event(g.raw).sum())
            assert 2 * sp <= lib.velo_noalloc_max_clusters()
            d = upload(g.raw)
            off = torch.full((26 * n + 1,), -1, dtype=torch.int32, device="cuda")
            num = torch.full((26 * n,), -1, dtype=torch.int32, device="cuda")
            cont = torch.zeros(18 * 2 * sp, dtype=torch.uint8, device="cuda")
            status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
            st = lib.velo_decode_noalloc(
                geometry, len(geometry), C.byref(d.c_struct()), sp, _current_stream(),
                off.data_ptr(), num.data_ptr(), cont.data_ptr(), cont.numel(), status.data_ptr())
            assert st == 0, lib.velo_noalloc_last_error_string().decode()
            torch.cuda.synchronize()

            chain.reserve_for(g.raw)
            chain.run(d)
            totals = chain.synchronize()
            ref = chain.outputs_to_host(totals)

            got_off = off.cpu().numpy().view(np.uint32)
            got_num = num.cpu().numpy().view(np.uint32)
            assert int(status.item()) == 0
            assert np.array_equal(got_off, ref["dev_offsets_estimated_input_size"])
            assert np.array_equal(got_num, ref["dev_module_cluster_num"])
            T = int(got_off[-1])
            mask = parity.sorted_container_mask(got_off, got_num, T)
            got = parity.container_fields(cont.cpu().numpy()[:18 * T], T)
            exp = parity.container_fields(ref["dev_sorted_velo_cluster_container"], T)
            for a, b in zip(got, exp):
                assert np.array_equal(parity._u8(a[mask]), parity._u8(b[mask]))
    finally:
        chain.close()


def test_decode_noalloc_rejects_oversized_slices(geometry):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from allen_b200 import generator
    from allen_b200.chain import upload, _current_stream

    lib = _noalloc_lib()
    g = generator.generate(4, seed=3)
    d = upload(g.raw)
    dummy = torch.zeros(64, dtype=torch.uint8, device="cuda")
    too_many = lib.velo_noalloc_max_clusters()  # 2 x super pixels above the limit
    st = lib.velo_decode_noalloc(geometry, len(geometry), C.byref(d.c_struct()), too_many, _current_stream(),
                                 dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), 64, None)
    assert st == 3  # VELO_ERR_CAPACITY, nothing queued


def test_decode_noalloc_understated_super_pixels(geometry):
    """A caller that states fewer super pixels than its banks hold: the estimate needs more
    clusters than 2 x the stated count, so the clustering writes nothing and dev_status
    receives err_input_capacity (bit 6); the call itself is accepted."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from allen_b200 import generator
    from allen_b200.chain import upload, _current_stream
    from allen_b200.rawbanks import super_pixels_per_event

    lib = _noalloc_lib()
    g = generator.generate(20, seed=26)
    n = g.raw.n_events
    sp = int(super_pixels_per_event(g.raw).sum())
    stated = sp // 4
    d = upload(g.raw)
    off = torch.full((26 * n + 1,), -1, dtype=torch.int32, device="cuda")
    num = torch.full((26 * n,), -1, dtype=torch.int32, device="cuda")
    cont = torch.full((18 * 2 * stated,), 0xAB, dtype=torch.uint8, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = lib.velo_decode_noalloc(geometry, len(geometry), C.byref(d.c_struct()), stated, _current_stream(),
                                 off.data_ptr(), num.data_ptr(), cont.data_ptr(), cont.numel(), status.data_ptr())
    assert st == 0, lib.velo_noalloc_last_error_string().decode()
    torch.cuda.synchronize()
    assert int(status.item()) & (1 << 6)
    assert bool((off == -1).all()) and bool((num == -1).all()) and bool((cont == 0xAB).all())

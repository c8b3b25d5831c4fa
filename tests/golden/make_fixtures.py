"""Builds the committed fixtures from the reference checkout (run here, not on the GPU box).

Outputs:
  allen_b200/data/velo_geometry.bin
      the detector description the reference ships as
      input/detector_configuration/velo_geometry.bin (written by
      Dumpers/BinaryDumpers/src/DumpVPGeometry.cpp:82-90), copied byte for byte;
  tests/golden/minbias_vp_10ev.npz
      the VP super-pixel banks (type 63, version 2) of the 10 events of
      input/minbias/mdf/MiniBrunel_2018_MinBias_FTv4_DIGI_retinacluster_v1.mdf, in
      Allen's raw-bank layout, plus the reference's own outputs for them;
  tests/golden/synthetic_seed7_20ev.npz
      20 generated events (nu = 7.6, seed 7, super pixels in column order) plus the
      reference's outputs for them;
  tests/golden/minbias_retina_10ev.npz
      the VPRetinaCluster banks (type 73, version 3) of the same 10 events, plus the
      reference's outputs through its retina-cluster decoding and the VELO Kalman filter;
  tests/golden/minbias_mdf_10ev.npz
      the VELO slice the reference's own MDF reader and transpose (main/src/Transpose.cpp)
      write for the same file: its VP and VPRetinaCluster banks together, bank version 2,
      as Allen's MDF provider hands them to the VELO decoding, plus the reference's outputs
      through the retina-cluster decoding (Allen's default front end) of that slice;
  tests/golden/mdf_synthetic_8ev.npz
      two synthetic MDF streams (8 generated events with other subdetectors' banks in
      shuffled order; source IDs without and with subdetector bits, tests/mdf_streams.py)
      and the VELO slices the reference's reader and transpose write for them.

The reference outputs come from oracle/_ref/libvelo_ref.so, the reference's VELO
kernels compiled as CPU C++ (oracle/Makefile).  Usage:
    python tests/golden/make_fixtures.py [/path/to/reference] [fixture names...]
"""
from __future__ import annotations

import os
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "tests"))

from allen_b200 import rawbanks  # noqa: E402

# Buffers whose contents do not depend on the order atomics are served in.
GOLDEN_BUFFERS = [
    "dev_number_of_candidates", "dev_candidates_offsets", "dev_estimated_input_size",
    "dev_offsets_estimated_input_size", "dev_module_candidate_num", "dev_module_cluster_num",
    "dev_number_of_velo_tracks", "dev_offsets_velo_tracks", "dev_number_of_three_hit_tracks_output",
    "dev_offsets_number_of_three_hit_tracks_filtered", "dev_offsets_all_velo_tracks",
    "dev_velo_track_hit_number", "dev_offsets_velo_track_hit_number", "dev_velo_track_hits",
    "dev_sorted_velo_cluster_container", "dev_cluster_candidates", "dev_three_hit_tracks_output",
    "dev_hit_used", "dev_atomics_velo",
]


RETINA_BUFFERS = [
    "dev_each_sensor_pair_size", "dev_offsets_each_sensor_pair_size", "dev_offsets_estimated_input_size",
    "dev_module_cluster_num", "dev_sorted_velo_cluster_container", "dev_number_of_velo_tracks",
    "dev_offsets_velo_tracks", "dev_number_of_three_hit_tracks_output",
    "dev_offsets_number_of_three_hit_tracks_filtered", "dev_offsets_all_velo_tracks", "dev_velo_track_hit_number",
    "dev_offsets_velo_track_hit_number", "dev_velo_track_hits", "dev_three_hit_tracks_output", "dev_hit_used",
    "dev_atomics_velo", "dev_is_backward", "dev_velo_kalman_beamline_states", "dev_velo_kalman_endvelo_states",
]


def read_mdf_vp_events(path, bank_type=rawbanks.BANK_TYPE_VP, version=2):
    data = open(path, "rb").read()
    p, events = 0, []
    while p + 20 <= len(data):
        size0 = struct.unpack_from("<I", data, p)[0]
        hdr = data[p + 17]
        sub = (hdr & 0x0F) * 4
        q, end = p + 20 + sub, p + size0
        banks = []
        while q < end:
            magic, size, btype, bank_version, src = struct.unpack_from("<HHBBH", data, q)
            assert magic == 0xCBCB
            if btype == bank_type:
                assert bank_version == version
                banks.append((btype, src, data[q + 8:q + size]))
            q += (size + 3) // 4 * 4
        events.append(banks)
        p = end
    return events


def main(ref_root, only=()):
    geo_src = os.path.join(ref_root, "input/detector_configuration/velo_geometry.bin")
    geometry = open(geo_src, "rb").read()
    os.makedirs(os.path.join(REPO, "allen_b200/data"), exist_ok=True)
    with open(os.path.join(REPO, "allen_b200/data/velo_geometry.bin"), "wb") as f:
        f.write(geometry)

    import cpu_checkers  # noqa: E402
    ref = cpu_checkers.load("ref")

    mdf = os.path.join(ref_root, "input/minbias/mdf/MiniBrunel_2018_MinBias_FTv4_DIGI_retinacluster_v1.mdf")
    real = rawbanks.build_slice(read_mdf_vp_events(mdf), bank_version=2)

    from allen_b200 import generator  # noqa: E402
    synth = generator.generate(20, seed=7, geometry=geometry, sp_order=0).raw
    retina = rawbanks.build_slice(read_mdf_vp_events(mdf, rawbanks.BANK_TYPE_VP_RETINA, 3), bank_version=3)

    stream = open(mdf, "rb").read()
    t = cpu_checkers.ref_transpose_vp(stream, 10, check_checksum=True)
    assert t["status"] == 0, t
    provider = rawbanks.RawSlice(t["raw"], t["offsets"], t["sizes"], t["types"], t["bank_version"])

    for name, s in (("minbias_vp_10ev", real), ("synthetic_seed7_20ev", synth), ("minbias_retina_10ev", retina),
                    ("minbias_mdf_10ev", provider)):
        if only and name not in only:
            continue
        out = ref.run(s, geometry)
        arrays = {"raw": s.raw, "offsets": s.offsets, "sizes": s.sizes, "types": s.types,
                  "bank_version": np.array([s.bank_version])}
        for b in (RETINA_BUFFERS if s.retina else GOLDEN_BUFFERS):
            arrays["ref__" + b] = out[b]
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
        print(name, s.n_events, "events;",
              int(out["dev_offsets_all_velo_tracks"][-1]), "tracks;",
              int(out["dev_module_cluster_num"].sum()), "clusters")

    if not only or "mdf_synthetic_8ev" in only:
        import mdf_streams  # noqa: E402
        arrays = {}
        g = generator.generate(8, seed=17, geometry=geometry)
        for mode, by_source in (("by_type", False), ("by_source", True)):
            st = mdf_streams.synthetic_stream(g.raw, seed=9, by_source_id=by_source, n_other=30, extra_velo=True)
            t = cpu_checkers.ref_transpose_vp(st, 8, check_checksum=True)
            assert t["status"] == 0 and t["by_source_id"] == by_source, t
            arrays[mode + "__stream"] = np.frombuffer(st, dtype=np.uint8)
            for k in ("raw", "offsets", "sizes", "types"):
                arrays[mode + "__" + k] = t[k]
            arrays[mode + "__bank_version"] = np.array([t["bank_version"]])
        np.savez_compressed(os.path.join(HERE, "mdf_synthetic_8ev.npz"), **arrays)
        print("mdf_synthetic_8ev", {k: v.size for k, v in arrays.items()})


if __name__ == "__main__":
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import build_checkers as oracle_build  # noqa: E402
    root = sys.argv[1] if len(sys.argv) > 1 else oracle_build.reference_root()
    if root is None:
        sys.exit("the reference tree was not found: pass its path or set ALLEN_REFERENCE_ROOT")
    main(root, tuple(sys.argv[2:]))

"""Loads the committed golden fixtures (tests/golden/*.npz)."""
import os

import numpy as np

from allen_b200.rawbanks import RawSlice

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = ["minbias_vp_10ev", "synthetic_seed7_20ev", "minbias_retina_10ev", "minbias_mdf_10ev"]


def load(name):
    z = np.load(os.path.join(HERE, name + ".npz"))
    s = RawSlice(z["raw"], z["offsets"], z["sizes"], z["types"], int(z["bank_version"][0]))
    ref = {k[len("ref__"):]: z[k] for k in z.files if k.startswith("ref__")}
    return s, ref

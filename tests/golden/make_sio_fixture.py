"""Writes muon_depos_head.npz: the first 300 depos of the reference's
sample depo file (test/data/muon-depos.npz in the reference tree), in the
file's own layout (depo_data_0 float32 [7][N], depo_info_0 int32 [4][N]).
Run where the reference tree is present, giving its root (or set
WCT_REFERENCE):
    python tests/golden/make_sio_fixture.py <reference tree>
"""

import os
import sys

import numpy as np

ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("WCT_REFERENCE")
if not ref:
    raise SystemExit("usage: make_sio_fixture.py <reference tree> (or set WCT_REFERENCE)")
z = np.load(os.path.join(ref, "test", "data", "muon-depos.npz"))
out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "muon_depos_head.npz")
np.savez(out, depo_data_0=z["depo_data_0"][:, :300], depo_info_0=z["depo_info_0"][:, :300])
print("wrote", out)

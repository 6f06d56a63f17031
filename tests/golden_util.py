"""Loading of the committed golden fixtures (tests/golden/*.npz, made by
tests/golden/make_golden.py from runs of the reference itself)."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# eddy-viscosity LES cases (WALE and Smagorinsky SGS flux)
LES_CASES = ["hex_wale_p3_n3_jit", "hex_smag_p2_n3", "quad_wale_p3_n6_jit"]
# Roe common flux (2-D)
ROE_CASES = ["quad_vortex_roe_p3_n6_jit", "quad_ns_roe_p2_n5"]
# boundary conditions (every Euler/Navier-Stokes boundary type of the reference)
BC_CASES = ["quad_bc_euler_p3", "quad_bc_euler2_p2", "quad_bc_roe_p3", "quad_ns_bc_p3", "hex_channel_p2",
            "hex_channel_char_p3"]
CASES = ["quad_vortex_p3_n6", "quad_vortex_p2_n5_jit", "quad_vortex_p3_n20", "hex_tgv_p3_n3",
         "hex_tgv_p2_n3_jit", "hex_tgv_p4_n2", "hex_euler_p3_n3", "quad_vortex_p1_n8_jit", "quad_vortex_p5_n4",
         "hex_tgv_p1_n4_jit"] + LES_CASES + ROE_CASES


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    arrs = {k: np.asfortranarray(z[k]) for k in z.files if k != "meta"}
    return meta, arrs


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))

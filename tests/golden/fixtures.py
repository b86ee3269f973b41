"""Loaders for the committed golden fixtures (see make_golden.py for their provenance)."""
import os

import numpy as np

from geaxdock_gpu_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))


def load_ref(name="1a07C1"):
    """Returns (fixture dict, ComplexArrays, EnePara) for a reference-pinned complex."""
    z = dict(np.load(os.path.join(HERE, "ref_%s.npz" % name)))
    temp = np.frombuffer(z["temp"].tobytes(), dtype=abi.TEMP_DTYPE).copy()
    cx = abi.ComplexArrays(
        lig_x=z["lig_x"], lig_y=z["lig_y"], lig_z=z["lig_z"], lig_center=z["lig_center"],
        lig_t=z["lig_t"], lig_c=z["lig_c"], lig_n=z["lig_n"],
        prt_x=z["prt_x"], prt_y=z["prt_y"], prt_z=z["prt_z"], prt_t=z["prt_t"], prt_c=z["prt_c"],
        prt_ele=z["prt_ele"], prt_seq3r=z["prt_seq3r"], prt_hflag=z["prt_hflag"],
        prt_hpp=z["prt_hpp"], pocket_center=z["pocket_center"], psp=z["psp"],
        kde_x=z["kde_x"], kde_y=z["kde_y"], kde_z=z["kde_z"], kde_t=z["kde_t"],
        mcs_x=z["mcs_x"], mcs_y=z["mcs_y"], mcs_z=z["mcs_z"], mcs_tcc=z["mcs_tcc"], temp=temp)
    ff = abi.enepara_from_array(z["enepara"])
    return z, cx, ff


def load_trajectory():
    """The reference's sample trajectory of 1a07C1 (see make_trajectory.py): float64 rows of
    PrtIdx, LigIdx, the six move-vector entries, cms and the weighted total energy."""
    return np.load(os.path.join(HERE, "trajectory_1a07C1.npz"))["rows"]


def load_trajectory_trace():
    """(rows, picked row indices, placed atoms [picked, lna, 3] in A) of the reference's trace
    program on every 13th trajectory row (see make_trajectory.py)."""
    z = np.load(os.path.join(HERE, "trajectory_1a07C1.npz"))
    return z["rows"], z["trace_rows"], z["trace_xyz"].astype(np.float64) * 1e-4

"""Ligand-record dumps: the reference's per-dump output files, and the records as the
post-processing sees them.

The reference writes, after every dump window, the LigRecord array of all replicas to
`<dir>/<name>_%04d.h5` (src/kernel_cuda_lancher_multigpu.cu:38, DumpLigRecord
src/hdf5io.C:11-28): one compound dataset "dset" of n_rep LigRecord elements whose in-memory
type is the C struct (src/hdf5_datastruct_ligrecord_create.h:42-84). No HDF5 library is
available to this package, so a dump is written as the bytes of that same struct array, one
file per dump, `<dir>/<name>_%04d.bin`; reading it back gives the array the HDF5 dataset
holds. `replica_records` is the reference's multi_reps_records map (src/dock.C:187-190): for
each replica the filled steps of the dump.
"""
from __future__ import annotations

import os
from typing import Dict

import numpy as np

from . import abi

LIG_RECORD_DTYPE = np.dtype([("step", abi.RECORD_DTYPE, (abi.STEPS_PER_DUMP + 1,)),
                             ("next_ptr", np.int32)])
assert LIG_RECORD_DTYPE.itemsize == abi.C.sizeof(abi.LigRecord)


def dump_path(directory: str, name: str, dump_index: int) -> str:
    return os.path.join(directory, "%s_%04d.bin" % (name, dump_index))


def write_dump(engine, directory: str, name: str, dump_index: int) -> str:
    """Writes every replica's LigRecord (the context's record window) to the dump file of
    `dump_index` (s1 / steps_per_dump in the reference) and returns its path."""
    os.makedirs(directory, exist_ok=True)
    path = dump_path(directory, name, dump_index)
    data = engine.lig_records()
    with open(path, "wb") as f:
        f.write(data)
    return path


def read_dump(path: str) -> np.ndarray:
    """A dump file as a LIG_RECORD_DTYPE array [n_rep]."""
    raw = np.fromfile(path, dtype=np.uint8)
    if raw.size % LIG_RECORD_DTYPE.itemsize:
        raise ValueError("%s: %d bytes is not a whole number of LigRecord (%d bytes)" %
                         (path, raw.size, LIG_RECORD_DTYPE.itemsize))
    return raw.view(LIG_RECORD_DTYPE)


def replica_records(lig_records: np.ndarray) -> Dict[int, np.ndarray]:
    """replica index -> its filled steps (RECORD_DTYPE), as multi_reps_records holds them."""
    return {i: lig_records[i]["step"][:int(lig_records[i]["next_ptr"])].copy()
            for i in range(lig_records.shape[0])}

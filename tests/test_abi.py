"""The C ABI library: loads, exports what include/geauxdock_b200.h declares, keeps the
reference's byte layouts, and its host-only entry points work without a GPU."""
import copy
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from geaxdock_gpu_b200 import abi, engine
from tests.conftest import have_gpu
from tests.golden.fixtures import load_ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "geauxdock_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|void|const char \*)\s*(gd_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = engine.lib()
    names = declared_symbols()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", engine.LIB_PATH], capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r" T (gd_\w+)", out))
    assert set(names) <= exported, set(names) - exported


def test_layouts_match_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text("""
#include <stdio.h>
#include <stddef.h>
#include "geauxdock_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(gd_energy), sizeof(gd_replica),
         sizeof(gd_record_step), sizeof(gd_lig_record), sizeof(gd_temp), sizeof(gd_enepara),
         sizeof(gd_enepara_raw), sizeof(gd_complex_desc), sizeof(gd_mc_params),
         sizeof(gd_replica_state), offsetof(gd_record_step, step));
  return 0;
}
""")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    want = [C.sizeof(abi.Energy), C.sizeof(abi.Replica), C.sizeof(abi.RecordStep),
            C.sizeof(abi.LigRecord), C.sizeof(abi.Temp), C.sizeof(abi.EnePara),
            C.sizeof(abi.EneParaRaw), C.sizeof(abi.ComplexDesc), C.sizeof(abi.McParams),
            C.sizeof(abi.ReplicaState), abi.RecordStep.step.offset]
    assert got == want
    # reference sizes: Energy 48, Replica 16, LigRecordSingleStep 92, LigRecord 2001*92+4
    assert got[:5] == [48, 16, 92, 2001 * 92 + 4, 12]


def test_fold_enepara_in_library_matches_reference():
    z, cx, ff = load_ref("1a07C1")
    raw = abi.enepara_raw_from_array(z["enepara_raw"])
    got = abi.struct_to_array(engine.fold_enepara(raw))
    assert np.array_equal(got.view(np.uint32), z["enepara"].view(np.uint32))


def test_set_temperature_in_library_matches_reference():
    z, cx, ff = load_ref("1a07C1")
    want = np.frombuffer(z["temp"].tobytes(), dtype=abi.TEMP_DTYPE)
    got = engine.set_temperature(4, 0.5, 2.0)
    assert np.array_equal(got["minus_beta"].view(np.uint32), want["minus_beta"].view(np.uint32))


def test_set_replica_flat_index():
    lib = engine.lib()
    n_prt, n_tmp, n_lig = 3, 4, 5
    rep = (abi.Replica * (n_prt * n_tmp * n_lig))()
    assert lib.gd_set_replica(n_prt, n_tmp, n_lig, rep) == 0
    a = np.frombuffer(bytes(rep), dtype=abi.REPLICA_DTYPE)
    f = np.arange(a.size)
    assert np.array_equal(a["idx_rep"], f)
    assert np.array_equal(a["idx_prt"], f // (n_tmp * n_lig))
    assert np.array_equal(a["idx_tmp"], (f // n_lig) % n_tmp)
    assert np.array_equal(a["idx_lig"], f % n_lig)


def test_invalid_arguments_are_rejected_with_a_message():
    lib = engine.lib()
    assert lib.gd_set_temperature(0, 0.3, 3.0, None) == abi.GD_ERR_INVALID
    assert b"gd_set_temperature" in lib.gd_last_error_string()
    z, cx, ff = load_ref("1a07C1")
    params = abi.mc_params()
    bad = cx.subset()
    bad.mcs_x = bad.mcs_x[:0]
    d = cx.desc()
    d.pos = 0
    h = C.c_void_p()
    rc = lib.gd_create(C.byref(ff), C.byref(d), 1, C.byref(params), 0, C.byref(h))
    assert rc == abi.GD_ERR_CAPACITY
    assert b"log(0/0)" in lib.gd_last_error_string()
    # a protein point off the number line: no cell grid can hold it (checked before any device
    # work, so this runs without a GPU)
    nan = copy.deepcopy(cx)
    nan.prt_y[0, 7] = np.nan
    d = nan.desc()
    rc = lib.gd_create(C.byref(ff), C.byref(d), 1, C.byref(params), 0, C.byref(h))
    assert rc == abi.GD_ERR_INVALID
    assert b"non-finite" in lib.gd_last_error_string()
    # so is a pocket centre off the number line (the points are ordered by distance from it)
    off = copy.deepcopy(cx)
    off.pocket_center = np.array([0.0, np.inf, 0.0], np.float32)
    d = off.desc()
    rc = lib.gd_create(C.byref(ff), C.byref(d), 1, C.byref(params), 0, C.byref(h))
    assert rc == abi.GD_ERR_INVALID
    assert b"pocket centre" in lib.gd_last_error_string()
    assert lib.gd_release_memory(-1) == abi.GD_ERR_INVALID


@pytest.mark.skipif(have_gpu(), reason="checks the no-device path")
def test_no_device_fails_loudly():
    z, cx, ff = load_ref("1a07C1")
    with pytest.raises(engine.GDError) as e:
        engine.Engine(ff, [cx], abi.mc_params())
    assert e.value.code in (abi.GD_ERR_NODEVICE, abi.GD_ERR_CUDA)

"""Ligand placement on the GPU (gd_place_ligand) and the `trace` tool end to end: the placed
atoms equal the FP32 oracle's bit for bit (both apply the same rotation and fused
multiply-adds) and the FP64 restatement of PlaceLigand (src/util.C:457-502) within 1e-5; the
tool's SDF files equal replaceLigandCoords of the oracle's atoms."""
import numpy as np
import pytest

from geaxdock_gpu_b200 import abi, engine, loaders
from geaxdock_gpu_b200 import trace as tr
from oracle import pyoracle as po
from tests.conftest import have_gpu
from tests.golden.fixtures import load_ref, load_trajectory
from tests.inputs import write_complex, write_paras

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a B200")]


def _oracle(cx, lc, mm, f64=False):
    xyz, _ = (po.place_f64 if f64 else po.place_f32)(cx, lc, mm)
    return xyz.T


def test_place_ligand_matches_oracle():
    z, cx, ff = load_ref("1a07C1")
    rows = load_trajectory()
    rng = np.random.default_rng(8)
    with engine.Engine(ff, [cx], abi.mc_params()) as e:
        mm = rows[:, 2:8].astype(np.float32)
        got = e.place_ligand(0, 0, mm)
        assert got.shape == (rows.shape[0], cx.lna, 3)
        for i in range(0, rows.shape[0], 37):
            assert np.array_equal(got[i], _oracle(cx, 0, mm[i]))
            ref = _oracle(cx, 0, mm[i], f64=True)
            assert np.max(np.abs(got[i] - ref)) <= 1e-5 * max(1.0, np.max(np.abs(ref)))
        for lc in (1, cx.n_lig - 1):
            mm = np.concatenate([rng.uniform(-2, 2, (5, 3)), rng.uniform(-7, 7, (5, 3))],
                                1).astype(np.float32)
            got = e.place_ligand(0, lc, mm)
            for i in range(5):
                assert np.array_equal(got[i], _oracle(cx, lc, mm[i]))
        assert e.place_ligand(0, 0, np.zeros((0, 6), np.float32)).shape == (0, cx.lna, 3)
        with pytest.raises(engine.GDError):
            e.place_ligand(0, cx.n_lig, mm)


def test_trace_tool_writes_the_placed_ligands(tmp_path, capsys):
    write_complex(tmp_path, np.random.default_rng(2))
    z, _, _ = load_ref("1a07C1")
    write_paras(tmp_path / "paras", abi.enepara_raw_from_array(z["enepara_raw"]))
    rng = np.random.default_rng(3)
    rows = []
    for k in range(7):
        mm = list(rng.uniform(-1, 1, 3)) + list(rng.uniform(-3.1, 3.1, 3))
        rows.append("0 %d " % (k % 4) + " ".join("%f" % v for v in mm) + " 0.5 -1.25")
    (tmp_path / "t.out").write_text("PrtIdx LigIdx v1 v2 v3 v4 v5 v6 cms ener\n"
                                    + "\n".join(rows) + "\n")
    args = ["-p", str(tmp_path / "p.pdb"), "-l", str(tmp_path / "l.sdf"),
            "-s", str(tmp_path / "p.ff"), "-para", str(tmp_path / "paras"), "-id", "synth",
            "-tr", str(tmp_path / "t.out"), "-lc", str(tmp_path / "pose")]
    assert tr.main(args) == 0
    out = capsys.readouterr().out
    assert out.count("write the new ligand conformation to") == 7
    cx, _, _ = loaders.load_complex(str(tmp_path / "p.pdb"), str(tmp_path / "l.sdf"),
                                    str(tmp_path / "p.ff"), str(tmp_path / "paras"), "synth",
                                    1, 0.3, 0.3)
    template = tr.sdf_lines(str(tmp_path / "l.sdf"))
    for k, r in enumerate(tr.read_trace(str(tmp_path / "t.out"))):
        want = tr.replace_ligand_coords(template, _oracle(cx, int(r[1]),
                                                          np.float32(r[2:8])))
        got = (tmp_path / ("pose_%d.sdf" % k)).read_text()
        assert got == "\n".join(want) + "\n", k


def test_place_ligand_is_the_reference_trace():
    """The library's placement against the reference's trace program on every 13th row of its
    sample trajectory (fixture from tests/golden/make_trajectory.py): every atom within the SDF
    lines' printed precision (5e-5 rounding, 1.5e-4 allowed)."""
    from tests.golden.fixtures import load_trajectory_trace
    rows, pick, ref = load_trajectory_trace()
    z, cx, ff = load_ref("1a07C1")
    with engine.Engine(ff, [cx], abi.mc_params()) as e:
        for lc in np.unique(rows[pick, 1]).astype(int):
            sel = np.nonzero(rows[pick, 1] == lc)[0]
            got = e.place_ligand(0, int(lc), rows[pick[sel], 2:8].astype(np.float32))
            assert np.max(np.abs(got.astype(np.float64) - ref[sel])) <= 1.5e-4, lc

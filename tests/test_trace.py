"""Host side of the `trace` tool (geaxdock_gpu_b200/trace.py, src/trace.C:18-136): the hand
parser, read2D's row rule, replaceLigandCoords' line format and the error paths that end
before any GPU work."""
import numpy as np

from geaxdock_gpu_b200 import abi
from geaxdock_gpu_b200 import trace as tr
from tests.golden.fixtures import load_ref
from tests.inputs import write_complex, write_paras


def test_parse_takes_the_next_word_and_the_last_occurrence():
    a = tr.parse(["-p", "a.pdb", "-l", "x.sdf", "-nc", "5", "junk", "-l", "y.sdf", "-s"])
    assert a["-p"] == "a.pdb" and a["-l"] == "y.sdf"
    assert "-s" not in a  # a flag without a following word is ignored
    assert a["-para"] == "gpudocksm.ff" and a["-lc"] == ""


def test_read_trace_rows_start_with_a_digit(tmp_path, capsys):
    p = tmp_path / "t.out"
    p.write_text("PrtIdx LigIdx v1 v2 v3 v4 v5 v6 cms ener\n"
                 "0 1 0.5 -0.25 1 2 3 4 0.1 -2.5\n"
                 "\n"
                 "# comment\n"
                 "-1 0 0 0 0 0 0 0\n"
                 "2 0 1.5 2.5 x 9\n")
    rows = tr.read_trace(str(p))
    assert rows == [[0, 1, 0.5, -0.25, 1, 2, 3, 4, np.float32(0.1), -2.5], [2, 0, 1.5, 2.5]]
    assert "reading near native traces" in capsys.readouterr().out
    assert tr.read_trace(str(tmp_path / "missing")) == []
    assert "Error opening file" in capsys.readouterr().out


def test_replace_ligand_coords_format():
    lines = ["name", "prog", "", "  2  1  0", "%10.4f%10.4f%10.4f C   0  0" % (1, 2, 3),
             "%10.4f%10.4f%10.4f N   0  0" % (4, 5, 6), "  1  2  1  0", "M  END"]
    xyz = np.array([[-12.34567, 0.00004, 100.5], [1.0, -2.0, 3.25]], np.float32)
    out = tr.replace_ligand_coords(lines, xyz)
    assert out[:4] == lines[:4] and out[6:] == lines[6:]
    assert out[4] == "%10.4f%10.4f%10.4f" % tuple(float(v) for v in xyz[0]) + " C   0  0"
    assert out[4][:30] == "  -12.3457    0.0000  100.5000"
    assert out[5] == "    1.0000   -2.0000    3.2500 N   0  0"


def test_replace_rejects_a_short_atom_line():
    import pytest
    with pytest.raises(tr.TraceError):
        tr.replace_ligand_coords(["a", "b", "", "  1  0", "  1.0  2.0"], np.zeros((1, 3)))


def test_sdf_lines_keep_carriage_returns(tmp_path):
    p = tmp_path / "l.sdf"
    p.write_bytes(b"a\r\nb\r\n\r\nc\n")
    assert tr.sdf_lines(str(p)) == ["a\r", "b\r", "\r", "c"]


def test_missing_inputs_print_the_reference_message(capsys):
    assert tr.main(["-l", "x.sdf", "-s", "x.ff"]) == 1
    assert "Provide target protein structure" in capsys.readouterr().out
    assert tr.main(["-p", "x.pdb", "-s", "x.ff"]) == 1
    assert "Provide compound library in SD format" in capsys.readouterr().out
    assert tr.main(["-p", "x.pdb", "-l", "x.sdf"]) == 1
    assert "Provide LHM potentials" in capsys.readouterr().out


def _files(tmp_path):
    write_complex(tmp_path, np.random.default_rng(2))
    z, _, _ = load_ref("1a07C1")
    write_paras(tmp_path / "paras", abi.enepara_raw_from_array(z["enepara_raw"]))
    return ["-p", str(tmp_path / "p.pdb"), "-l", str(tmp_path / "l.sdf"),
            "-s", str(tmp_path / "p.ff"), "-para", str(tmp_path / "paras"), "-id", "synth",
            "-lc", str(tmp_path / "pose")]


def test_bad_rows_are_reported_before_any_placement(tmp_path, capsys):
    args = _files(tmp_path)
    (tmp_path / "short.out").write_text("0 0 0.1 0.2 0.3\n")
    assert tr.main(args + ["-tr", str(tmp_path / "short.out")]) == 1
    assert "8 needed" in capsys.readouterr().err
    (tmp_path / "far.out").write_text("0 9 0 0 0 0 0 0 0 0\n")
    assert tr.main(args + ["-tr", str(tmp_path / "far.out")]) == 1
    assert "ligand conformer 9" in capsys.readouterr().err
    assert not list(tmp_path.glob("pose_*.sdf"))


def test_unreadable_trajectory_writes_nothing(tmp_path, capsys):
    args = _files(tmp_path)
    assert tr.main(args + ["-tr", str(tmp_path / "none.out")]) == 0
    assert "Error opening file" in capsys.readouterr().out
    assert not list(tmp_path.glob("pose_*.sdf"))

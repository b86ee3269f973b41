"""The `dock` command line (geaxdock_gpu_b200/dock.py) end to end on the GPU, on input files
written here in the reference's formats: load, Monte Carlo dump windows until the records
reach steps_per_dump x n_rep (or the dump cap), post_mc clustering, the trajectory table."""
import numpy as np
import pytest

from geaxdock_gpu_b200 import abi, dock, records
from tests.conftest import have_gpu
from tests.golden.fixtures import load_ref
from tests.inputs import write_complex, write_paras

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a B200")]


def test_dock_command_line(tmp_path, capsys):
    rng = np.random.default_rng(4)
    write_complex(tmp_path, rng)
    z, _, _ = load_ref("1a07C1")
    write_paras(tmp_path / "paras", abi.enepara_raw_from_array(z["enepara_raw"]))
    out = tmp_path / "out.csv"
    rc = dock.main(["-p", str(tmp_path / "p.pdb"), "-l", str(tmp_path / "l.sdf"),
                    "-s", str(tmp_path / "p.ff"), "--para", str(tmp_path / "paras"),
                    "-i", "synth", "-o", str(out), "--nt", "3", "--floor_temp", "0.3",
                    "--ceiling_temp", "0.9", "--seed", "5", "--max-dumps", "2",
                    "--dump-dir", str(tmp_path / "dumps")])
    assert rc == 0
    text = capsys.readouterr().out
    assert "# points" in text and "Final output" in text
    lines = out.read_text().splitlines()
    assert lines[0].startswith("lig prt cms rmsd mv1")
    body = np.array([[float(v) for v in l.split()] for l in lines[1:]])
    assert 1 <= body.shape[0] <= 500 and body.shape[1] == 20
    assert np.all(np.isfinite(body))
    assert np.all(np.diff(body[:, -1]) >= 0)  # sorted by total energy
    d0 = records.read_dump(str(tmp_path / "dumps" / "synth_0000.bin"))
    assert d0.shape[0] == 4 * 2 * 3 and d0["next_ptr"].max() > 0


def test_dock_command_line_with_surrogate(tmp_path, capsys):
    rng = np.random.default_rng(6)
    write_complex(tmp_path, rng)
    z, _, _ = load_ref("1a07C1")
    write_paras(tmp_path / "paras", abi.enepara_raw_from_array(z["enepara_raw"]))
    out = tmp_path / "out.csv"
    rc = dock.main(["-p", str(tmp_path / "p.pdb"), "-l", str(tmp_path / "l.sdf"),
                    "-s", str(tmp_path / "p.ff"), "--para", str(tmp_path / "paras"),
                    "-i", "synth", "-o", str(out), "--nt", "2", "--seed", "7",
                    "--max-dumps", "2", "--gaussian", "--surrogate", "--train-iterations", "20"])
    assert rc == 0
    text = capsys.readouterr().out
    assert "surrogate" in text and "proposed" in text
    body = np.array([[float(v) for v in l.split()] for l in out.read_text().splitlines()[1:]])
    assert body.shape[0] >= 1 and np.all(np.isfinite(body))

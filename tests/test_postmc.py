"""Post-processing on CPU: the k-means shuffle of the library equals the oracle's restatement,
the oracle's k-means on a known answer, the record dump layout, the trajectory table format."""
import ctypes as C

import numpy as np
import pytest

from geaxdock_gpu_b200 import abi, postmc, records
from oracle import kmeans as ok


@pytest.mark.parametrize("n", [0, 1, 2, 3, 50, 51, 1000, 2001])
def test_permutation_is_the_oracles(n):
    for seed, seg in ((0, 0), (42, 3), (2 ** 40 + 7, 6819)):
        a = postmc.permutation(seed, seg, n)
        assert sorted(a.tolist()) == list(range(n))
        assert np.array_equal(a, ok.permutation(seed, seg, n))


def test_permutation_depends_on_seed_and_segment():
    a = postmc.permutation(1, 0, 500)
    assert not np.array_equal(a, postmc.permutation(2, 0, 500))
    assert not np.array_equal(a, postmc.permutation(1, 1, 500))


def test_oracle_kmeans_known_answer():
    rng = np.random.default_rng(0)
    centres = np.eye(9, dtype=np.float32) * 50.0
    pts = np.concatenate([c + rng.normal(0, 0.5, (40, 9)) for c in centres[:3]]).astype(np.float32)
    mem, rep, size, passes = ok.cluster_by_kmeans(pts, 3, seed=7, seg=0)
    assert sorted(size.tolist()) == [40, 40, 40]
    for g in range(3):  # the three blobs are the three clusters
        assert len(set(mem[g * 40:(g + 1) * 40].tolist())) == 1
    assert all(mem[rep[c]] == c for c in range(3))
    assert 1 <= passes <= 501


def test_oracle_fewer_records_than_clusters():
    pts = np.arange(27, dtype=np.float32).reshape(3, 9)
    mem, rep, size, passes = ok.cluster_by_kmeans(pts, 50, seed=0, seg=0)
    assert mem.tolist() == [0, 1, 2] and rep.tolist() == [0, 1, 2] and passes == 0


def test_lig_record_dump_layout(tmp_path):
    assert records.LIG_RECORD_DTYPE.itemsize == C.sizeof(abi.LigRecord)
    buf = (abi.LigRecord * 3)()
    for i in range(3):
        buf[i].next_ptr = i + 1
        for s in range(i + 1):
            buf[i].step[s].step = 100 * i + s
            buf[i].step[s].energy.e[9] = -float(s)
            buf[i].step[s].replica.idx_rep = i
    p = tmp_path / "d_0000.bin"
    p.write_bytes(bytes(buf))
    arr = records.read_dump(str(p))
    assert arr.shape == (3,) and arr["next_ptr"].tolist() == [1, 2, 3]
    rr = records.replica_records(arr)
    assert [r.shape[0] for r in rr.values()] == [1, 2, 3]
    assert rr[2]["step"].tolist() == [200, 201, 202]
    assert rr[1]["energy"]["e"][:, 9].tolist() == [0.0, -1.0]
    assert records.dump_path("out", "run", 7).endswith("run_0007.bin")


def test_write_states_format(tmp_path):
    r = np.zeros(2, abi.RECORD_DTYPE)
    r["replica"]["idx_lig"] = [3, 4]
    r["replica"]["idx_prt"] = [1, 0]
    r["energy"]["cms"] = [0.5, 0.25]
    r["energy"]["rmsd"] = [1.23456, 2.0]
    r["movematrix"][0] = [0.1, 0.2, 0.3, 0.4, 0.5, 0.6]
    r["energy"]["e"][0] = np.arange(10) - 5.0
    p = tmp_path / "t.csv"
    postmc.write_states(r, str(p))
    lines = p.read_text().splitlines()
    assert lines[0] == ("lig prt cms rmsd mv1 mv2 mv3 mv4 mv5 mv6 "
                        "vdw ele pmf psp hdb hpc kde lhm edst ener")
    f = lines[1].split(" ")
    assert f[:4] == ["3", "1", "0.5000", "1.2346"] and len(f) == 20 and f[-1] == "4.0000"


def _kmeans_ref():
    import os
    return np.load(os.path.join(os.path.dirname(__file__), "golden", "kmeans_ref.npz"))


@pytest.mark.parametrize("name", ["edge100", "color100", "texture100"])
def test_oracle_seq_kmeans_is_the_references(name):
    """The oracle's seq_kmeans against the reference's own (src/seq_kmeans.c, run as
    src/cluster_test.C:23-66 runs it: 10 clusters, threshold 0.001, on the k-means module's
    sample data; fixtures from tests/golden/make_golden.py): the same membership, the same
    centres bit for bit, the same number of passes."""
    z = _kmeans_ref()
    obj, cen = z[name + "_objects"], z[name + "_centres"]
    mem, c, passes = ok.seq_kmeans(obj, cen.shape[0], 0.001)
    assert np.array_equal(np.asarray(mem), z[name + "_membership"])
    assert np.array_equal(np.asarray(c, np.float32).view(np.uint32), cen.view(np.uint32))
    assert passes == int(z[name + "_loops"][0])


@pytest.mark.parametrize("seed", [0, 5, 2 ** 33 + 1])
def test_oracle_shuffled_kmeans_reproduces_the_reference_order(seed):
    """Objects laid out so that the seeded shuffle puts them back in the file's order give
    clusterByKmeans the reference's seq_kmeans run on that order (membership and sizes)."""
    z = _kmeans_ref()
    obj, ref = z["color100_objects"], z["color100_membership"]
    perm = ok.permutation(seed, 0, obj.shape[0])
    objp = np.empty_like(obj)
    objp[perm] = obj
    mem, _, size, passes = ok.cluster_by_kmeans(objp, 10, seed, 0)
    assert np.array_equal(np.asarray(mem)[perm], ref)
    assert np.asarray(size).tolist() == np.bincount(ref, minlength=10).tolist()
    assert passes == int(z["color100_loops"][0])


def test_write_states_is_the_references_print_states(tmp_path):
    """The trajectory table against the reference's own printStates (src/util.C:1504-1545) on
    300 records with signed zeros, values rounding to zero from below and rounding ties
    (fixture from tests/golden/make_states.py): byte for byte."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "states_ref.npz"))
    rec = np.frombuffer(z["records"].tobytes(), abi.RECORD_DTYPE)
    p = tmp_path / "states.csv"
    postmc.write_states(rec, str(p))
    assert p.read_bytes() == z["table"].tobytes()

"""AERO-F's pre-partitioned mesh files: the C ABI reader (GeoSource's
format: connectivity, geometry and decomposition files behind
BinFileHandler headers) on files written by aerof_dev_b200.sower.write --
both byte orders, one and two clusters -- and the decomposition built from
them.  CPU only (the reader is host code)."""
import numpy as np
import pytest

from aerof_dev_b200 import decomposition as D
from aerof_dev_b200 import sower
from aerof_dev_b200 import workloads as W


@pytest.fixture(params=[(1, False), (2, True)], ids=["one-cluster-native", "two-clusters-swapped"])
def written(request, tmp_path):
    nclusters, swap = request.param
    m = W.make_lattice_mesh(7, jitter=0.2, codes="channel")
    m["codes"] = m["codes"].copy()
    m["codes"][:5] = 11                              # symmetry faces round-trip through file code 6
    part = sower.element_partition(m, 4)
    names = sower.write(str(tmp_path / "mesh"), m, part, nclusters=nclusters, swap=swap)
    return m, part, names, nclusters


def test_round_trip_global_mesh(written):
    m, part, names, nclusters = written
    gs = sower.GeoSource(names["con"], names["geo"], names["dec"])
    assert gs.num_subdomains == 4 and gs.num_clusters == nclusters
    g = gs.global_mesh()
    assert np.array_equal(g["X"], m["X"])
    assert np.array_equal(g["tets"], m["tets"])
    assert np.array_equal(g["faces"], m["faces"])
    assert np.array_equal(g["codes"], m["codes"])
    gs.close()


def test_subdomains_and_shared_nodes(written):
    m, part, names, _ = written
    gs = sower.GeoSource(names["con"], names["geo"], names["dec"])
    subs = [gs.read_subdomain(i) for i in range(gs.num_subdomains)]
    for i, s in enumerate(subs):
        # the subdomain's tets are exactly its partition, in local numbering
        assert np.array_equal(np.sort(s["elem_l2g"]), np.nonzero(part == i)[0])
        assert np.array_equal(s["node_l2g"][s["tets"]], m["tets"][s["elem_l2g"]])
        assert np.array_equal(s["X"], m["X"][s["node_l2g"]])
        # shared nodes pair up with the neighbour's list (same global order)
        for k, j in enumerate(s["neighb"]):
            mine = s["node_l2g"][s["shared"][s["shared_ptr"][k]: s["shared_ptr"][k + 1]]]
            t = subs[j]
            kk = list(t["neighb"]).index(i)
            theirs = t["node_l2g"][t["shared"][t["shared_ptr"][kk]: t["shared_ptr"][kk + 1]]]
            assert np.array_equal(mine, theirs) and mine.size > 0
    # owners: the lowest-numbered subdomain holding a node
    owner = gs.owners()
    for g in range(m["X"].shape[0]):
        holders = [i for i, s in enumerate(subs) if g in set(s["node_l2g"].tolist())]
        assert owner[g] == min(holders)
    # ghost-layer subdomains for several GPUs from the file's decomposition
    dsubs = D.decompose(gs.global_mesh(), owner)
    assert sum(s.n_owned for s in dsubs) == m["X"].shape[0]
    gs.close()


def test_reader_errors(tmp_path):
    bad = tmp_path / "x.con"
    bad.write_bytes(b"\x07\x00\x00\x00" + b"\x00" * 8)
    with pytest.raises(Exception):
        sower.GeoSource(str(bad), str(tmp_path / "g"), str(tmp_path / "d"))
    m = W.make_lattice_mesh(4)
    names = sower.write(str(tmp_path / "m"), m, sower.element_partition(m, 2))
    gs = sower.GeoSource(names["con"], names["geo"] + "missing", names["dec"])
    with pytest.raises(Exception) as e:
        gs.read_subdomain(0)
    assert "cannot open" in str(e.value)
    with pytest.raises(Exception):
        gs.read_subdomain(5)

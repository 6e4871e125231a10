"""The serving loop (mosp_server_*): resident graphs, change batches from
several client threads, coalesced per graph. Every response must equal the
oracle's combined tree of its graph after `version` batches applied one by
one, both when requests arrive together (mixed across graphs, coalesced)
and when each is submitted alone; the resident K trees must equal the
oracle's at the end."""
import threading

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import mosp_b200 as mb  # noqa: E402
import oracle as orc  # noqa: E402
from conftest import grid_graph, random_graph  # noqa: E402


@pytest.fixture(scope="module")
def scenario():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    K = 3
    graphs = [grid_graph(60, 50, K, 100, 0.2, 61), random_graph(3000, 9000, K, 1000, 62),
              grid_graph(90, 90, K, 50, 0.3, 63), random_graph(1500, 6000, K, 100, 64),
              grid_graph(40, 40, K, 100, 0.1, 65)]
    prefs = [None, [1, 2, 3], None, [1, 1, 2], None]
    rng = np.random.default_rng(66)
    modes = ["uniform", "targeted", "increase", "reweight"]
    batches = []
    for gi, g in enumerate(graphs):
        hg = mb.HostGraph.from_arrays(*g)
        seq = []
        for j in range(8):
            size = int(np.exp(rng.uniform(np.log(10), np.log(400))))
            mode = modes[(gi + j) % 4]
            try:
                b = mb.HostBatch.generate(hg, size, 50.0, mode, 0, False, 1000 * gi + j, 0, 1, 100)
            except mb.MospError:
                b = mb.HostBatch.generate(hg, size, 50.0, "uniform", 0, False, 1000 * gi + j, 0, 1, 100)
            ba = b.arrays()
            x = {k: ba[k] for k in ("ins_from", "ins_to", "ins_w", "del_from", "del_to")}
            if j % 2 == 1 and len(seq[-1]["ins_from"]):
                # delete some edges the previous batch inserted: a merged pass
                # must split here to stay equal to one-by-one application
                prev = seq[-1]
                x["del_from"] = np.concatenate([x["del_from"], prev["ins_from"][:5]]).astype(np.int32)
                x["del_to"] = np.concatenate([x["del_to"], prev["ins_to"][:5]]).astype(np.int32)
            seq.append(x)
        batches.append(seq)
    # oracle states after 0..len(seq) batches applied one by one
    states = []
    for gi, g in enumerate(graphs):
        row, col, w = g
        per = []
        for v in range(len(batches[gi]) + 1):
            if v > 0:
                b = batches[gi][v - 1]
                row, col, w, _ = orc.apply_batch(row, col, w, b["ins_from"], b["ins_to"], b["ins_w"],
                                                 b["del_from"], b["del_to"])
            n = len(row) - 1
            par = np.stack([orc.dijkstra(row, col, w, k, 0)[1] for k in range(K)])
            dist = np.stack([orc.dijkstra(row, col, w, k, 0)[0] for k in range(K)])
            crow, ccol, cw = orc.combined_graph(par, n, K, 0, prefs[gi])
            cd, cp = orc.dijkstra(crow, ccol, cw, 0, 0)
            per.append((dist, par, cd, cp))
        states.append(per)
    return K, graphs, prefs, batches, states


def serve(scenario, alone, workers=2):
    K, graphs, prefs, batches, states = scenario
    srv = mb.Server(workers=workers, reserve_bytes=0, max_coalesce=64)
    try:
        ids = [srv.add_graph(g, K, 0, p) for g, p in zip(graphs, prefs)]
        # version 0: the initial trees the server computed
        for gi, gid in enumerate(ids):
            v, d, p, cd, cp = srv.read_graph(gid)
            assert v == 0
            assert np.array_equal(d, states[gi][0][0]) and np.array_equal(p, states[gi][0][1])
            assert np.array_equal(cd, states[gi][0][2]) and np.array_equal(cp, states[gi][0][3])
        responses = []
        if alone:
            for gi, gid in enumerate(ids):
                for b in batches[gi]:
                    t = srv.submit(gid, b)
                    responses.append((gi, srv.wait(t, gid)))
        else:
            tickets = []
            lock = threading.Lock()

            def client(which):
                # each client submits its graphs' batches in order, interleaved
                for j in range(len(batches[0])):
                    for gi in which:
                        t = srv.submit(ids[gi], batches[gi][j])
                        with lock:
                            tickets.append((gi, t))

            threads = [threading.Thread(target=client, args=(w,)) for w in ([0, 3], [1, 4], [2])]
            for th in threads:
                th.start()
            for th in threads:
                th.join()
            for gi, t in tickets:
                responses.append((gi, srv.wait(t, ids[gi])))
        for gi, (cd, cp, info) in responses:
            assert info.status == 0 and 1 <= info.version <= len(batches[gi])
            exp = states[gi][info.version]
            assert np.array_equal(cd, exp[2]), (gi, info.version)
            assert np.array_equal(cp, exp[3]), (gi, info.version)
        for gi, gid in enumerate(ids):
            v, d, p, cd, cp = srv.read_graph(gid)
            assert v == len(batches[gi])
            assert np.array_equal(d, states[gi][-1][0]) and np.array_equal(p, states[gi][-1][1])
        return srv.stats()
    finally:
        srv.close()


def test_serving_mixed_requests(scenario):
    st = serve(scenario, alone=False, workers=2)
    assert st.requests == sum(len(b) for b in scenario[3])
    assert st.passes <= st.requests and st.passes <= st.applies


def test_serving_alone(scenario):
    st = serve(scenario, alone=True, workers=1)
    assert st.passes == st.requests and st.max_coalesced == 1


def test_serving_rejects_bad_requests(scenario):
    K, graphs, prefs, batches, states = scenario
    srv = mb.Server(workers=1, reserve_bytes=0)
    try:
        gid = srv.add_graph(graphs[0], K)
        with pytest.raises(mb.MospError):
            srv.submit(gid + 1, batches[0][0])
        bad = dict(batches[0][0])
        bad["del_to"] = np.full(len(bad["del_to"]), 10 ** 7, np.int32)
        if len(bad["del_to"]):
            with pytest.raises(mb.MospError):
                srv.submit(gid, bad)
        t = srv.submit(gid, batches[0][0])
        cd, cp, info = srv.wait(t, gid)
        assert info.version == 1 and np.array_equal(cd, states[0][1][2])
    finally:
        srv.close()


def test_serving_passes_share_the_device(scenario):
    """With several workers and overlap on, each worker's cooperative grids
    use its share of the SMs, so passes of different graphs run on the
    device at the same time; every response still equals the oracle (the
    checks of serve()). The same requests with overlap off are served one
    pass at a time and give the same results."""
    st = serve(scenario, alone=False, workers=4)
    assert st.passes <= st.requests
    assert st.overlapped >= 1, "no two passes' engine launches ran at the same time"
    K, graphs, prefs, batches, states = scenario
    srv = mb.Server(workers=2, reserve_bytes=0, overlap=False)
    try:
        gid = srv.add_graph(graphs[2], K, 0, prefs[2])
        for j, b in enumerate(batches[2]):
            cd, cp, info = srv.wait(srv.submit(gid, b), gid)
            assert np.array_equal(cd, states[2][info.version][2])
        assert srv.stats().overlapped == 0
    finally:
        srv.close()

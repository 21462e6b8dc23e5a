"""A batched search captured in a CUDA graph replays to the eager results.

The device-pointer entry point issues only stream work once its work areas
exist (memsets and kernel launches, no allocation or host synchronisation),
so after one eager call it can be captured and replayed; new queries are
copied into the captured input buffer between replays."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [1, 2, 4, 5, 6])
def test_graph_replay_equals_eager(golden, mode):
    import torch

    import liteqg_b200

    g = golden["mix128d64"]
    ix = liteqg_b200.Index("QG", "L2", g["n"], g["dim"], g["deg"])
    ix.load(g["path"])
    ix.set_tuning(mode=mode)
    rng = np.random.default_rng(mode)
    q_all = g["queries"]
    m, k, ef = len(q_all), 10, 100
    s = torch.cuda.Stream()
    q = torch.from_numpy(np.ascontiguousarray(q_all)).cuda()
    ids = torch.full((m, k), -1, dtype=torch.int32, device="cuda")
    with torch.cuda.stream(s):
        ix.search_device(q.data_ptr(), m, k, ids.data_ptr(), k, ef=ef, stream=s.cuda_stream)
    s.synchronize()
    eager = ids.cpu().numpy().view(np.uint32).copy()
    assert np.array_equal(eager, g["expected"][(100, 10)])
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        ix.search_device(q.data_ptr(), m, k, ids.data_ptr(), k, ef=ef, stream=s.cuda_stream)
    for rep in range(3):
        perm = rng.permutation(m)
        q.copy_(torch.from_numpy(np.ascontiguousarray(q_all[perm])))
        ids.fill_(-1)
        graph.replay()
        torch.cuda.synchronize()
        got = ids.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, eager[perm]), (mode, rep)
    del graph

"""Request sharding across devices, host side (no GPU): placement by budget and work,
and that processes placing the same stream agree (world size 2 over gloo)."""
import os

import pytest


def _stream(n=40):
    import bench
    from ausm import make_request
    cfg = dict(bench.SERVE, requests=n)
    return [make_request(sp["M"], sp["N"], naca4=sp["naca"], far_radius=20.0, first_spacing=1e-3, grid_iters=200,
                         residual_drop=4.0, max_steps=50000, mach=sp["mach"], aoa_deg=sp["aoa"], scheme=sp["scheme"])
            for sp in bench.serve_stream(cfg)]


def test_place_requests_balances_work():
    from ausm import place_requests, request_bytes
    from ausm.shard import request_work
    reqs = _stream()
    b = [request_bytes(r) for r in reqs]
    w = [request_work(r) for r in reqs]
    for n in (1, 2, 3, 8):
        dev = place_requests(b, w, n, 160e9)
        assert len(dev) == len(reqs) and set(dev) <= set(range(n))
        load = [sum(x for x, d in zip(w, dev) if d == k) for k in range(n)]
        # greedy least-loaded: no device exceeds another by more than the largest request
        assert max(load) - min(load) <= max(w) + 1e-9
        assert dev == place_requests(b, w, n, 160e9)  # deterministic
    with pytest.raises(ValueError):
        place_requests([2e9], [1.0], 2, 1e9)


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from ausm import place_requests, request_bytes
    from ausm.shard import request_work
    reqs = _stream()
    dev = place_requests([request_bytes(r) for r in reqs], [request_work(r) for r in reqs], world, 160e9)
    mine = torch.tensor([k for k, d in enumerate(dev) if d == rank] + [-1] * len(reqs))[:len(reqs)]
    allv = [torch.zeros_like(mine) for _ in range(world)]
    dist.all_gather(allv, mine)
    q.put((rank, [sorted(int(x) for x in v if x >= 0) for v in allv]))
    dist.destroy_process_group()


def test_ranks_agree_on_placement_gloo():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(180)
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res[0] == res[1]  # both ranks see the same partition
    a, b = res[0]
    assert not set(a) & set(b) and sorted(a + b) == list(range(40)) and a and b

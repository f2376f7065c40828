"""Multi-GPU routing logic on the CPU: the per-group cost model that
balances clip shards across ranks, and the request router that sends each
request to the device with the least outstanding work (fake engines stand in
for the per-device servers)."""

import numpy as np

from metalmom_b200.shard import Router, balanced_shards, clip_cost, frame_cost, frames_of


def test_cost_model_orders_groups_by_work():
    # per frame: a 4096-point frame costs more than a 1024-point one
    assert frame_cost(4096) > frame_cost(2048) > frame_cost(1024)
    # per clip: a 44.1 kHz clip has twice the frames of a 22.05 kHz clip of
    # the same duration at the same hop
    assert clip_cost(44100 * 10, n_fft=2048) > 1.9 * clip_cost(22050 * 10, n_fft=2048)
    assert clip_cost(1000, n_fft=2048) == frames_of(1000, 2048, 512) * frame_cost(2048)


def test_balanced_shards_mixed_groups_balance_cost():
    rng = np.random.default_rng(3)
    lengths, params = [], []
    for _ in range(200):
        n_fft = int(rng.choice([1024, 2048, 4096]))
        sr = int(rng.choice([22050, 44100]))
        params.append(dict(sr=sr, n_fft=n_fft, hop_length=n_fft // 4, n_mels=int(rng.choice([64, 128]))))
        lengths.append(int(rng.uniform(1, 120) * sr))
    for world in (2, 3, 8):
        shards = balanced_shards(lengths, world, params)
        assert sorted(i for s in shards for i in s) == list(range(len(lengths)))
        loads = [sum(clip_cost(lengths[i], **params[i]) for i in s) for s in shards]
        assert max(loads) <= 1.02 * min(loads) + max(clip_cost(L, **p) for L, p in zip(lengths, params))
        assert max(loads) / (sum(loads) / world) < 1.05


class _FakeServer:
    def __init__(self):
        self.reqs = {}

    def submit(self, y, **params):
        rid = len(self.reqs) + 1
        self.reqs[rid] = len(y)
        return rid

    def result(self, rid, timeout_ms=-1):
        return self.reqs.pop(rid)

    def close(self):
        pass


def test_router_sends_requests_to_the_least_loaded_device():
    with Router([0, 1, 2], make_server=lambda d: _FakeServer()) as r:
        g = dict(sr=22050, n_fft=2048, hop_length=512)
        long = r.submit(np.zeros(22050 * 60, np.float32), **g)  # one long clip
        short = [r.submit(np.zeros(22050, np.float32), **g) for _ in range(10)]
        # the long clip's device takes nothing else while the others have less work
        assert all(h[0] != long[0] for h in short)
        assert abs(r.load[short[0][0]] - r.load[short[1][0]]) <= clip_cost(22050, **g)
        assert r.result(long) == 22050 * 60
        assert r.load[long[0]] == 0.0
        for h in short:
            r.result(h)
        assert all(v == 0.0 for v in r.load)


def test_bench_uneven_batch_routed_over_ranks():
    """The bench's uneven mixed-group batch at N GPUs: every clip goes to
    exactly one rank, the ranks' device costs are within 1 % of each other,
    and one rank keeps the whole batch in workload order."""
    import bench
    work = bench.uneven_workload()
    assert bench.uneven_shard(work, 0, 1) == list(range(len(work)))
    for world in (2, 4, 8):
        shards = [bench.uneven_shard(work, r, world) for r in range(world)]
        assert sorted(i for s in shards for i in s) == list(range(len(work)))
        costs = [sum(clip_cost(work[i][2], **work[i][0]) for i in s) for s in shards]
        assert max(costs) <= 1.01 * (sum(costs) / world)

"""Clip sharding and request routing across GPUs.

Clips are independent -- the only intra-clip coupling, the top_db floor's
clip-global maximum, never leaves the GPU that owns the clip -- so multi-GPU
work is a partition of clips with no collective on the data path:

* ``balanced_shards``: one process per GPU (torchrun), each rank taking the
  clips of its shard, balanced by a per-parameter-group frame cost;
* ``Router``: one process driving several GPUs, one serving engine
  (``Server``) per device, each request sent to the device with the least
  outstanding cost.
"""

import heapq
import math


def frames_of(length, n_fft=2048, hop=512, center=True):
    """The reference's frame count (STFT.swift:241-254) for a power-of-two n_fft."""
    padded = length + (2 * (n_fft // 2) if center else 0)
    return 0 if padded < n_fft else 1 + (padded - n_fft) // hop


def frame_cost(n_fft=2048, n_mels=128, n_mfcc=20):
    """Relative device cost of one frame of a parameter group: the FFT-form
    flop count 2.5 N log2 N, plus the filterbank walk over N/2 + 1 bins and
    the DCT (2 n_mfcc n_mels)."""
    return 2.5 * n_fft * math.log2(max(n_fft, 2)) + 4.0 * (n_fft // 2 + 1) + 2.0 * min(n_mfcc, n_mels) * n_mels


def clip_cost(length, sr=22050, n_fft=2048, hop_length=None, n_mels=128, n_mfcc=20, center=True, **_):
    """Cost of one clip under its parameter group (frames x frame_cost)."""
    hop = hop_length if hop_length else n_fft // 4
    return frames_of(length, n_fft, hop, center) * frame_cost(n_fft, n_mels, n_mfcc)


def balanced_shards(lengths, world, params=None, **group):
    """Assign clip indices to `world` ranks, balancing device cost
    (longest-processing-time greedy; deterministic tie-break on rank).

    ``params``: one parameter dict per clip (its group), or None for one
    group given by the keyword arguments (n_fft, hop_length, n_mels, n_mfcc,
    center) for every clip."""
    if world < 1:
        raise ValueError("world must be >= 1")
    if params is not None and len(params) != len(lengths):
        raise ValueError("one parameter dict per clip")
    costs = [clip_cost(L, **(params[i] if params is not None else group)) for i, L in enumerate(lengths)]
    order = sorted(range(len(lengths)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    shards = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(s) for s in shards]


class Router:
    """Requests over several devices, one ``Server`` per device.

    ``submit`` sends a request to the device whose outstanding cost (the
    ``clip_cost`` of its requests not yet collected) is least, so long and
    short clips and different parameter groups spread by work rather than by
    count; ``result`` collects it.  ``make_server(device)`` builds a device's
    engine (default: ``Server`` created with that device current)."""

    def __init__(self, devices, make_server=None, **server_kw):
        self.devices = list(devices)
        if not self.devices:
            raise ValueError("no devices")
        if make_server is None:
            def make_server(dev):
                import torch
                from .serve import Server
                with torch.cuda.device(dev):
                    return Server(**server_kw)
        self.servers = [make_server(d) for d in self.devices]
        self.load = [0.0] * len(self.devices)
        self._cost = {}

    def pick(self, cost):
        """Index of the device that takes a request of this cost."""
        return min(range(len(self.devices)), key=lambda i: (self.load[i], i))

    def submit(self, y, **params):
        cost = clip_cost(len(y), **params)
        i = self.pick(cost)
        rid = self.servers[i].submit(y, **params)
        self.load[i] += cost
        self._cost[(i, rid)] = cost
        return (i, rid)

    def result(self, handle, timeout_ms=-1):
        i, rid = handle
        try:
            out = self.servers[i].result(rid, timeout_ms)
        except TimeoutError:
            raise  # still outstanding
        except Exception:
            self.load[i] -= self._cost.pop((i, rid), 0.0)
            raise
        self.load[i] -= self._cost.pop((i, rid), 0.0)
        return out

    def close(self):
        for s in self.servers:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def max_over_ranks(value, dist=None, device=None):
    """Max of a float over all ranks (elapsed-time reduction); identity without a group."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())

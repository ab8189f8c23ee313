"""Work over several GPUs (one process per GPU).

Two forms, both without any exchange of packets:

* replicas (one instance): every rank holds the whole grid and traces its own
  packets with a rank-specific seed; after the transport phase the ranks sum
  the intensity integrals J with one all-reduce over NCCL (NVLink / NVSwitch)
  and each solves the ionization balance for the combined packet count.  This
  is the replica form of the reference's MPI copy merge
  (testDensitySubGrid.cpp:3320-3379).
* shards (many independent instances): ``shard_instances`` gives every rank
  a subset of the instances, balanced by their work; ranks run their own
  instances and only the timing and counters are combined.

With one rank both reduce to TransportEngine.run_iterations.
"""
from __future__ import annotations

import numpy as np

_GOLDEN = 0x9E3779B97F4A7C15
_MASK64 = (1 << 64) - 1


def replica_seed(seed: int, rank: int) -> int:
    """Independent Philox key per rank (rank 0 keeps the plain seed)."""
    return (int(seed) + _GOLDEN * int(rank)) & _MASK64


def shard_instances(costs, world):
    """Assign independent instances to ``world`` ranks: longest first, each
    to the least-loaded rank (ties to the lower rank).  Returns one sorted
    list of instance indices per rank."""
    costs = [float(c) for c in costs]
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(o) for o in out]


class _CudaArray:
    """__cuda_array_interface__ view of device memory owned by the engine."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {
            "shape": (count,), "typestr": "<f8", "data": (ptr, False), "version": 3,
            "strides": None, "stream": None,
        }


def intensity_tensor(engine, instance=0):
    """Zero-copy torch view of the instance's J array on its GPU."""
    import torch
    ptr, count = engine.device_field(instance, "J")
    return torch.as_tensor(_CudaArray(ptr, count), device="cuda")


class ReplicaRunner:
    """Iterations of the plain method on one engine, summed over ranks."""

    def __init__(self, engine, group=None, instance=0, intensity=None, allreduce=None,
                 mode="replicas"):
        if mode not in ("replicas", "shards"):
            raise ValueError(f"mode must be 'replicas' or 'shards', not {mode!r}")
        self.eng = engine
        self.group = group
        self.mode = mode
        self.instance = instance
        self._intensity = intensity or (lambda: intensity_tensor(engine, instance))
        self._allreduce = allreduce
        self.iteration = 0
        self.launches = 0
        if group is not None:
            import torch.distributed as dist
            self.world = dist.get_world_size(group)
            self.rank = dist.get_rank(group)
        else:
            self.world, self.rank = 1, 0

    # ---- collectives (no-ops with one rank) ----
    def _reduce(self, t, op):
        import torch.distributed as dist
        if self._allreduce is not None:
            self._allreduce(t, op)
        else:
            dist.all_reduce(t, op=op, group=self.group)

    def barrier(self):
        if self.world > 1:
            import torch
            import torch.distributed as dist
            t = torch.zeros(1, device="cuda" if torch.cuda.is_available() else "cpu")
            self._reduce(t, dist.ReduceOp.SUM)

    def _scalar(self, v, op_name):
        if self.world == 1:
            return v
        import torch
        import torch.distributed as dist
        dev = "cuda" if torch.cuda.is_available() else "cpu"
        t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
        self._reduce(t, getattr(dist.ReduceOp, op_name))
        return t.item()

    def max_over_ranks(self, v):
        return self._scalar(v, "MAX")

    def sum_over_ranks(self, v):
        return self._scalar(v, "SUM")

    # ---- iterations ----
    def run(self, iterations, seed=42):
        """Returns one summed stats dict per iteration (this rank's packets).

        One rank without a custom all-reduce, or shards: the engine's own
        iterations.  Replicas: per iteration the engine's captured transport
        graph (cmi_shoot_packets), the all-reduce of J ordered on the engine's
        stream (the collective waits for the transport on the device, and the
        balance launched after it on the same stream waits for the collective),
        then the balance for the packets of all ranks."""
        if self.mode == "shards" or (self.world == 1 and self._allreduce is None):
            out = []
            for it in self.eng.run_iterations(iterations, seed):
                out.append(_sum_stats(it))
            self.launches = self.eng.last_launch_count()
            self.iteration += iterations
            return out
        import contextlib

        import torch
        import torch.distributed as dist
        grid = self.eng.grids[self.instance]
        lum = float(np.sum(np.asarray(grid.sources, dtype=np.float64).reshape(-1, 4)[:, 3]))
        engine_stream = None
        if torch.cuda.is_available() and hasattr(self.eng, "stream"):
            engine_stream = torch.cuda.ExternalStream(self.eng.stream())
        out = []
        launches = 0
        for _ in range(iterations):
            st = self.eng.shoot_packets(seed=replica_seed(seed, self.rank),
                                        iteration=self.iteration)
            launches += self.eng.last_launch_count()
            J = self._intensity()
            with (torch.cuda.stream(engine_stream) if engine_stream is not None
                  else contextlib.nullcontext()):
                self._reduce(J, dist.ReduceOp.SUM)
            dx = self.eng.compute_neutral_fraction(self.instance, lum,
                                                   int(grid.num_photon) * self.world)
            launches += 2
            s = _sum_stats(st)
            s["mean_abs_dx"] = dx
            out.append(s)
            self.iteration += 1
        self.launches = launches
        return out

    def close(self):
        pass


def _sum_stats(per_instance):
    out = dict(per_instance[0])
    for s in per_instance[1:]:
        for k in ("packets_emitted", "packets_absorbed", "packets_escaped", "cell_crossings",
                  "subgrid_transits"):
            out[k] += s[k]
        out["error_flags"] |= s["error_flags"]
        out["rounds"] = max(out["rounds"], s["rounds"])
    return out

"""Packet replicas over ranks (parallelcmacionize_b200/distributed.py), on CPU.

Two gloo ranks each trace their own packets (rank-specific Philox key), sum J
with one all-reduce and solve the balance for the combined packet count.  The
transport on each rank is the oracle (a CPU stand-in for the GPU engine, test
infrastructure only); the result must equal one process tracing both ranks'
packets.
"""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

PC = 3.086e16
BOX = (-5 * PC, -5 * PC, -5 * PC, 10 * PC, 10 * PC, 10 * PC)
NCELL, NSUB = (16, 16, 16), (4, 4, 4)
NPH = 3000


class OracleEngine:
    """CPU stand-in with the engine calls ReplicaRunner uses."""

    def __init__(self, rank):
        import oracle as O
        from parallelcmacionize_b200 import GridSpec
        self.O = O
        self.lat = O.LatticeGrid(BOX, NCELL, NSUB)
        self.grids = [GridSpec(box=BOX, ncell=NCELL, num_subgrid=NSUB,
                               sources=[(0.0, 0.0, 0.0, 4.26e49)], num_photon=NPH)]
        rng = np.random.default_rng(3)
        self.nH = np.exp(rng.normal(np.log(1e8) - 0.5, 1.0, 16 ** 3))
        self.xH = np.full(16 ** 3, 1e-3)
        self.J = np.zeros(16 ** 3)
        self.launches = 0

    def packets(self, seed, iteration):
        O = self.O
        dirs, tau = O.philox_packets(seed, iteration, 0, NPH)
        ph = np.zeros(NPH, O.PHOTON_DTYPE)
        ph["direction"] = dirs
        ph["tau"] = tau
        ph["sigma"] = 6.3e-22
        ph["weight"] = 1.0
        return ph

    def shoot_packets(self, seed, iteration):
        ph = self.packets(seed, iteration)
        start = np.full(NPH, self.lat.locate([0.0, 0.0, 0.0]), np.uint32)
        c = self.lat.transport(self.nH, self.xH, self.J, ph, start)
        return [dict(packets_emitted=NPH, packets_absorbed=c["absorbed"],
                     packets_escaped=c["escaped"], cell_crossings=c["crossings"],
                     subgrid_transits=c["transits"], mean_abs_dx=0.0, error_flags=0, rounds=1)]

    def last_launch_count(self):
        return 1

    def compute_neutral_fraction(self, instance, luminosity, num_photon):
        O = self.O
        x_old = self.xH.copy()
        jf = O.jfac(luminosity, num_photon, np.array(self.lat.subgrid_desc(0).inv_cell_size))
        O.compute_neutral_fraction(self.nH, self.xH, self.J, jf, 4e-19, form=1)
        return float(np.mean(np.abs(self.xH - x_old)))


def _rank(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    from parallelcmacionize_b200.distributed import ReplicaRunner
    eng = OracleEngine(rank)
    runner = ReplicaRunner(eng, group=dist.group.WORLD,
                           intensity=lambda: torch.from_numpy(eng.J))
    stats = runner.run(2, seed=42)
    total = runner.sum_over_ranks(stats[-1]["cell_crossings"])
    np.save(os.path.join(out_dir, f"x{rank}.npy"), eng.xH)
    np.save(os.path.join(out_dir, f"c{rank}.npy"), np.array([total]))
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_replicas_equal_one_process(tmp_path):
    mp.spawn(_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    x0, x1 = np.load(tmp_path / "x0.npy"), np.load(tmp_path / "x1.npy")
    assert np.array_equal(x0, x1)  # every rank holds the same balanced field

    from parallelcmacionize_b200.distributed import replica_seed
    ref = OracleEngine(0)
    crossings = 0
    for it in range(2):
        for r in range(2):
            st = ref.shoot_packets(replica_seed(42, r), it)
            crossings = st[0]["cell_crossings"] if r == 0 else crossings + st[0]["cell_crossings"]
        ref.compute_neutral_fraction(0, 4.26e49, 2 * NPH)
    # J summed in a different order: agree to rounding
    np.testing.assert_allclose(x0, ref.xH, rtol=1e-12, atol=1e-15)
    assert int(np.load(tmp_path / "c0.npy")[0]) == crossings


def test_replica_seeds_distinct():
    from parallelcmacionize_b200.distributed import replica_seed
    seeds = {replica_seed(42, r) for r in range(64)}
    assert len(seeds) == 64 and replica_seed(42, 0) == 42


def test_shard_instances_balances_and_covers():
    from parallelcmacionize_b200.distributed import shard_instances
    from parallelcmacionize_b200.problems import batch_configs
    cfgs = batch_configs(count=64, select=set())
    assert all(n is None for _, n in cfgs)
    costs = [g.num_photon * sum(g.ncell) for g, _ in cfgs]
    for world in (1, 2, 3, 8):
        parts = shard_instances(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(64))
        loads = [sum(costs[i] for i in p) for p in parts]
        # longest-processing-time bound: max load <= mean + largest item
        assert max(loads) <= sum(costs) / world + max(costs)
    assert shard_instances([5.0, 1.0, 1.0], 2) == [[0], [1, 2]]
    # the selected densities equal the full generation
    full = batch_configs(count=6)
    part = batch_configs(count=6, select={1, 4})
    for i in range(6):
        assert full[i][0] == part[i][0]
        if i in (1, 4):
            assert np.array_equal(full[i][1], part[i][1])
        else:
            assert part[i][1] is None


def test_runner_modes():
    from parallelcmacionize_b200.distributed import ReplicaRunner
    with pytest.raises(ValueError):
        ReplicaRunner(None, mode="bogus")

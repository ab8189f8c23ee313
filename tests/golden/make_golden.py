"""Generate the golden fixtures of tests/golden/ from the reference's own code.

Runs the reference harness (oracle/_ref/ref_harness_exact, built by
oracle/build_ref.sh from the reference headers, no fast-math) on seeded
inputs and stores inputs + reference outputs as compressed .npz files:

  directions.npz   get_output_direction / get_start_index / mirror /
                   compatibility answers (testDensitySubGridDirections.cpp
                   grid, swept over every face, edge and corner)
  rng.npz          RandomGenerator streams (ranlxd) for several seeds
  emission.npz     per-buffer photon streams (seed, copy-pick draw, packets)
  walk_<case>.npz  DensitySubGrid::interact on packet lists: final photons,
                   exit directions, accumulated J and per-packet cell tallies
  balance.npz      compute_neutral_fraction on a wide range of J / n_H
  transport.npz    interact + neighbour routing through a lattice of subgrids
  stromgren_ensemble.npz  64^3 Stromgren runs (reference code, 8 seeds):
                   radial x_H profiles and ionized radii
  stromgren_reemission_ensemble.npz  the same with do_reemission's
                   probability 0.364 (testDensitySubGrid_omp.cpp:675-702)
  lognormal_ensemble.npz  the 128^3 log-normal workload (8^3 subgrids of 16^3,
                   sigma_ln = 1, 4 sources, 1e7 packets x 20 iterations from
                   x_H = 1e-6; reference code, 8 seeds): x_H means over
                   blocks of 8^3 cells
  dust_walks.npz   DensitySubGrid::propagate and compute_optical_depth on the
                   packet lists of walk_interior16 / walk_entries8 /
                   walk_noncubic (propagate only where the target depth is > 0:
                   the reference asserts that)
  dust_image.npz   image.dat of the reference's dust driver
                   (oracle/_ref/testDensitySubGrid_omp_dust: forced first
                   scattering, peel-off image) for a unit-density sphere of
                   radius 1 in a [-1, 1]^3 box, albedo 0.5, 1e6 packets; the
                   second iteration's image (x_H = 1 after the first balance)
  outputs_random.npz  the same driver's files for its random density field
                   (10 cosine modes), one thread
  outputs.npz      the result files of the reference's own driver
                   (oracle/_ref/testDensitySubGrid_omp_files, -DMM_FILE
                   -DBIN_FILE): neutral_fractions.dat and .bin of a small
                   non-cubic run, one thread (files written in subgrid order)

Usage: python tests/golden/make_golden.py [--skip-ensemble | --only-ensembles]
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
PC = 3.086e16
SIGNS = [
    (0, 0, 0),
    (1, 1, 1), (1, 1, -1), (1, -1, 1), (1, -1, -1),
    (-1, 1, 1), (-1, 1, -1), (-1, -1, 1), (-1, -1, -1),
    (0, 1, 1), (0, 1, -1), (0, -1, 1), (0, -1, -1),
    (1, 0, 1), (1, 0, -1), (-1, 0, 1), (-1, 0, -1),
    (1, 1, 0), (1, -1, 0), (-1, 1, 0), (-1, -1, 0),
    (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
]


def save(name, **arrays):
    path = os.path.join(OUT, name)
    np.savez_compressed(path, **arrays)
    print(f"wrote {name}: {os.path.getsize(path) / 1024:.1f} KiB")


def gen_directions():
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "d.txt")
        O.ref_run(["directions", p])
        lines = open(p).read().splitlines()
    out, start, mirror, compat = [], [], [], []
    for ln in lines:
        f = ln.split()
        if f[0] == "output":
            out.append([int(v) for v in f[1:]])
        elif f[0] == "start":
            start.append([float(v) for v in f[1:]])
        elif f[0] == "mirror":
            mirror.append([int(v) for v in f[1:]])
        elif f[0] == "compat":
            compat.append([float(v) for v in f[1:]])
    save("directions.npz", output=np.array(out, np.int32), start=np.array(start),
         mirror=np.array(mirror, np.int32), compat=np.array(compat))


def gen_rng():
    seeds = np.array([0, 1, 42, 1234, 123456789, 2 ** 31 - 1], dtype=np.int64)
    streams = np.stack([O.ref_rng(int(s), 2500) for s in seeds])
    save("rng.npz", seeds=seeds, streams=streams)


def gen_emission():
    cases = [(42, 200, (0.0, 0.0, 0.0)), (7, 137, (1.5e16, -2.0e16, 3.0e15)),
             (2 ** 30, 200, (-4.9 * PC, 4.9 * PC, 0.1 * PC))]
    seeds = np.array([c[0] for c in cases])
    counts = np.array([c[1] for c in cases])
    src = np.array([c[2] for c in cases])
    photons = np.concatenate([O.ref_emit(s, n, p) for s, n, p in cases])
    save("emission.npz", seeds=seeds, counts=counts, sources=src, photons=photons)


def isotropic(rng, n):
    d = rng.normal(size=(n, 3))
    return d / np.linalg.norm(d, axis=1)[:, None]


def walk_case(name, box, ncell, nH, xH, photons, in_dirs):
    out, res, J, per = O.ref_walk(box, ncell, nH, xH, photons, in_dirs)
    offsets = np.cumsum([0] + [len(c) for c, _ in per]).astype(np.int64)
    cells = np.concatenate([c for c, _ in per]).astype(np.int32) if offsets[-1] else np.zeros(0, np.int32)
    vals = np.concatenate([v for _, v in per]) if offsets[-1] else np.zeros(0)
    save(f"walk_{name}.npz", box=np.asarray(box, float), ncell=np.asarray(ncell, np.int32),
         nH=nH, xH=xH, photons=photons, in_dirs=np.asarray(in_dirs, np.int32), out=out,
         result=res, J=J, offsets=offsets, cells=cells, values=vals)


def make_photons(pos, dirs, tau, sigma=6.3e-22, weight=1.0):
    n = len(pos)
    ph = np.zeros(n, O.PHOTON_DTYPE)
    ph["position"] = pos
    ph["direction"] = dirs
    ph["tau"] = tau
    ph["sigma"] = sigma
    ph["weight"] = weight
    return ph


def gen_walks():
    rng = np.random.default_rng(2024)
    # (a) 16^3 subgrid of the 128^3 workload, log-normal density, mixed x_H
    box = np.array([-1.25 * PC, 0.0, 2.5 * PC, 1.25 * PC, 1.25 * PC, 1.25 * PC])
    n3 = (16, 16, 16)
    C = 16 ** 3
    nH = np.exp(rng.normal(np.log(1e8) - 0.5, 1.0, C))
    xH = 10.0 ** rng.uniform(-6, 0, C)
    n = 400
    pos = box[:3] + rng.uniform(size=(n, 3)) * box[3:]
    walk_case("interior16", box, n3, nH, xH,
              make_photons(pos, isotropic(rng, n), rng.exponential(size=n)), np.zeros(n, int))

    # (b) 8^3 subgrid, nearly transparent: packets leave through every face,
    # edge and corner; entries from all 27 TravelDirections
    box = np.array([0.0, 0.0, 0.0, 0.625 * PC, 0.625 * PC, 0.625 * PC])
    n3 = (8, 8, 8)
    C = 512
    nH = np.full(C, 1.0e8)
    xH = np.full(C, 1.0e-6)
    pos, dirs, dirs_in = [], [], []
    for d in range(27):
        s = SIGNS[d]
        for _ in range(12):
            p = box[:3] + rng.uniform(0.02, 0.98, 3) * box[3:]
            v = rng.normal(size=3)
            for a in range(3):
                if s[a] != 0:
                    p[a] = box[a] if s[a] < 0 else box[a] + box[3 + a]
                    v[a] = abs(v[a]) * (-s[a])
            pos.append(p)
            dirs.append(v / np.linalg.norm(v))
            dirs_in.append(d)
    n = len(pos)
    walk_case("entries8", box, n3, nH, xH,
              make_photons(np.array(pos), np.array(dirs), rng.exponential(size=n) * 5.0),
              dirs_in)

    # (c) edge cases: source on the subgrid corner (the Stromgren source sits
    # on the corner of 8 subgrids), axis-aligned and diagonal rays with zero
    # components, positions on internal cell faces, tau = 0 and tiny tau
    box = np.array([0.0, 0.0, 0.0, 1.25 * PC, 1.25 * PC, 1.25 * PC])
    n3 = (16, 16, 16)
    C = 16 ** 3
    nH = np.full(C, 1.0e8)
    xH = np.where(rng.uniform(size=C) < 0.5, 1e-4, 1e-2)
    cs = box[3] / 16
    pos, dirs, taus = [], [], []
    special_dirs = [
        (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
        (1, 1, 0), (1, -1, 0), (0, 1, 1), (-1, 0, 1), (1, 1, 1), (-1, -1, -1), (1, -1, 1),
    ]
    for v in special_dirs:
        v = np.asarray(v, float)
        v /= np.linalg.norm(v)
        for p in (box[:3], box[:3] + np.array([5, 7, 3]) * cs, box[:3] + np.array([5.5, 7, 3.25]) * cs):
            pos.append(np.array(p, float))
            dirs.append(v)
            taus.append(3.0)
    for _ in range(40):  # corner source, isotropic
        pos.append(box[:3].copy())
        dirs.append(isotropic(rng, 1)[0])
        taus.append(rng.exponential())
    for t in (0.0, 1e-300, 1e-12, 50.0):
        pos.append(box[:3] + 0.5 * box[3:])
        dirs.append(isotropic(rng, 1)[0])
        taus.append(t)
    n = len(pos)
    walk_case("edges16", box, n3, nH, xH, make_photons(np.array(pos), np.array(dirs),
                                                      np.array(taus)), np.zeros(n, int))

    # (d) non-cubic cells and uneven cell counts, weights and cross sections
    box = np.array([-2.0e16, 1.0e16, -3.0e15, 3.0e16, 1.2e16, 2.0e16])
    n3 = (12, 5, 9)
    C = 12 * 5 * 9
    nH = 10.0 ** rng.uniform(6, 9, C)
    xH = 10.0 ** rng.uniform(-5, 0, C)
    n = 300
    pos = box[:3] + rng.uniform(size=(n, 3)) * box[3:]
    ph = make_photons(pos, isotropic(rng, n), rng.exponential(size=n),
                      sigma=rng.uniform(1e-22, 1e-21, n), weight=rng.uniform(0.5, 2.0, n))
    walk_case("noncubic", box, n3, nH, xH, ph, np.zeros(n, int))


def gen_balance():
    rng = np.random.default_rng(99)
    box = np.array([-5 * PC, -5 * PC, -5 * PC, 10 * PC, 10 * PC, 10 * PC])
    n3 = (8, 8, 8)
    C = 512
    nH = 10.0 ** rng.uniform(6, 10, C)
    J = 10.0 ** rng.uniform(-12, 6, C)
    J[rng.uniform(size=C) < 0.1] = 0.0
    L, N = 4.26e49, 1_000_000
    x, Jout = O.ref_balance(box, n3, nH, J, L, N)
    save("balance.npz", box=box, ncell=np.asarray(n3, np.int32), nH=nH, J=J, L=L, N=N, xH=x,
         J_after=Jout)


def gen_transport():
    rng = np.random.default_rng(5)
    box = np.array([-5 * PC, -5 * PC, -5 * PC, 10 * PC, 10 * PC, 10 * PC])
    ncell, nsub = (16, 16, 16), (4, 4, 4)
    lat = O.LatticeGrid(box, ncell, nsub)
    cube = np.exp(rng.normal(np.log(1e8) - 0.5, 1.0, ncell))
    from parallelcmacionize_b200.engine import cube_to_blocked
    nH = cube_to_blocked(cube, ncell, nsub)
    xH = cube_to_blocked(10.0 ** rng.uniform(-4, 0, ncell), ncell, nsub)
    n = 600
    srcs = [np.zeros(3), np.array([1.7 * PC, -3.1 * PC, 2.2 * PC])]
    pos = np.array([srcs[i % 2] for i in range(n)])
    start = np.array([lat.locate(p) for p in pos], np.uint32)
    ph = make_photons(pos, isotropic(rng, n), rng.exponential(size=n))
    J, fin, fate, tr = O.ref_transport(box, ncell, nsub, nH, xH, ph, start)
    save("transport.npz", box=box, ncell=np.asarray(ncell, np.int32),
         num_subgrid=np.asarray(nsub, np.int32), nH=nH, xH=xH, photons=ph, start=start, J=J,
         final=fin, fate=fate, transits=tr)


def gen_ensemble(seeds=8, packets=1_000_000, iterations=10):
    """64^3 Stromgren sphere with the reference code (all host threads).

    Member k draws buffer b of iteration i from ranlxd(seed_k + b + i * 5000):
    seeds 10^7 apart keep the members' streams disjoint."""
    box = np.array([-5 * PC, -5 * PC, -5 * PC, 10 * PC, 10 * PC, 10 * PC])
    ncell, nsub = (64, 64, 64), (8, 8, 8)
    cells = 64 ** 3
    nH = np.full(cells, 1e8)
    xH0 = np.full(cells, 1e-6)
    from parallelcmacionize_b200.engine import blocked_to_cube
    from parallelcmacionize_b200.problems import GridSpec, cell_radii, ionized_radius
    g = GridSpec(box=tuple(box), ncell=ncell, num_subgrid=nsub)
    r = cell_radii(g).reshape(-1)
    edges = np.linspace(0, 6.0 * PC, 49)
    which = np.digitize(r, edges) - 1
    profiles, radii = [], []
    for k in range(seeds):
        x, its = O.ref_iterations(box, ncell, nsub, nH, xH0, [0.0, 0.0, 0.0], [4.26e49],
                                  packets, iterations, seed=1000 + 10_000_000 * k,
                                  binary="ref_harness_exact")
        cube = blocked_to_cube(x, ncell, nsub).reshape(-1)
        prof = np.array([cube[which == b].mean() for b in range(len(edges) - 1)])
        profiles.append(prof)
        radii.append(ionized_radius(blocked_to_cube(x, ncell, nsub), g))
        print(f"  ensemble seed {k}: R_ion = {radii[-1] / PC:.4f} pc")
    save("stromgren_ensemble.npz", edges=edges, profiles=np.array(profiles),
         radii=np.array(radii), packets=packets, iterations=iterations)


def gen_ensemble_reemission(seeds=8, packets=1_000_000, iterations=10, probability=0.364):
    """gen_ensemble's Stromgren sphere with reemission: an absorbed packet is
    re-emitted in place with probability 0.364 (params.txt:12, the value the
    reference calls realistic), drawing from its buffer's generator."""
    box = np.array([-5 * PC, -5 * PC, -5 * PC, 10 * PC, 10 * PC, 10 * PC])
    ncell, nsub = (64, 64, 64), (8, 8, 8)
    cells = 64 ** 3
    nH = np.full(cells, 1e8)
    xH0 = np.full(cells, 1e-6)
    from parallelcmacionize_b200.engine import blocked_to_cube
    from parallelcmacionize_b200.problems import GridSpec, cell_radii, ionized_radius
    g = GridSpec(box=tuple(box), ncell=ncell, num_subgrid=nsub)
    r = cell_radii(g).reshape(-1)
    edges = np.linspace(0, 6.0 * PC, 49)
    which = np.digitize(r, edges) - 1
    profiles, radii = [], []
    for k in range(seeds):
        x, _ = O.ref_iterations(box, ncell, nsub, nH, xH0, [0.0, 0.0, 0.0], [4.26e49], packets,
                                iterations, seed=3000 + 10_000_000 * k,
                                binary="ref_harness_exact", reemission=probability)
        cube = blocked_to_cube(x, ncell, nsub).reshape(-1)
        profiles.append(np.array([cube[which == b].mean() for b in range(len(edges) - 1)]))
        radii.append(ionized_radius(blocked_to_cube(x, ncell, nsub), g))
        print(f"  reemission ensemble seed {k}: R_ion = {radii[-1] / PC:.4f} pc")
    save("stromgren_reemission_ensemble.npz", edges=edges, profiles=np.array(profiles),
         radii=np.array(radii), packets=packets, iterations=iterations,
         probability=probability)


def gen_ensemble_lognormal(seeds=8, packets=10_000_000, iterations=20, block=8):
    """The 128^3 log-normal workload with the reference code: member k draws
    buffer b of iteration i from ranlxd(2000 + 10^7 k + b + i * 50000)."""
    from parallelcmacionize_b200.engine import blocked_to_cube
    from parallelcmacionize_b200.problems import lognormal_config
    g, nH = lognormal_config(ncell=128, num_subgrid=8, num_photon=packets, num_sources=4,
                             sigma_ln=1.0, seed=42)
    src = np.asarray(g.sources, np.float64)
    m = 128 // block
    blocks = []
    for k in range(seeds):
        x, its = O.ref_iterations(g.box, g.ncell, g.num_subgrid, nH, np.full(nH.size, 1e-6),
                                  src[:, :3], src[:, 3], packets, iterations,
                                  seed=2000 + 10_000_000 * k, binary="ref_harness_exact")
        cube = blocked_to_cube(x, g.ncell, g.num_subgrid)
        blocks.append(cube.reshape(m, block, m, block, m, block).mean(axis=(1, 3, 5)))
        print(f"  log-normal ensemble seed {k}: mean x_H = {x.mean():.6f}, "
              f"{sum(r['seconds'] for r in its):.1f} s")
    save("lognormal_ensemble.npz", blocks=np.array(blocks), block=np.array(block),
         packets=np.array(packets), iterations=np.array(iterations))


DUST_CASES = ("interior16", "entries8", "noncubic")


def gen_dust_walks():
    arrays = {}
    for case in DUST_CASES:
        g = np.load(os.path.join(OUT, f"walk_{case}.npz"))
        ph, dirs = g["photons"], g["in_dirs"]
        keep = ph["tau"] > 0
        out, res = O.ref_dust_walk(g["box"], g["ncell"], g["nH"], g["xH"], ph[keep], dirs[keep])
        arrays[f"{case}_keep"] = keep
        arrays[f"{case}_prop_out"] = out
        arrays[f"{case}_prop_res"] = res
        out, res = O.ref_dust_walk(g["box"], g["ncell"], g["nH"], g["xH"], ph, dirs, depth=True)
        arrays[f"{case}_depth_out"] = out
        arrays[f"{case}_depth_res"] = res
    save("dust_walks.npz", **arrays)


DUST_IMAGE_CASE = {"ncell": 32, "num_subgrid": 4, "num_photon": 1000000, "albedo": 0.5,
                   "threads": 4}


def gen_dust_image():
    """Runs the reference's dust driver (params with the keys of
    params_single_uniform.txt; box in metres) and stores its image.dat."""
    import subprocess
    import tempfile
    b = O.ref_binary("testDensitySubGrid_omp_dust")
    if b is None:
        sys.exit("oracle/_ref/testDensitySubGrid_omp_dust missing: run oracle/build_ref.sh")
    c = DUST_IMAGE_CASE
    params = "\n".join([
        "box:", "  anchor: [-1. m, -1. m, -1. m]", "  sides: [2. m, 2. m, 2. m]",
        f"ncell: [{c['ncell']}, {c['ncell']}, {c['ncell']}]", f"num_photon: {c['num_photon']}",
        "number_of_iterations: 2", f"reemission_probability: {c['albedo']}",
        "number_of_sources: 1", "random_density: false",
        f"num_subgrid: [{c['num_subgrid']}, {c['num_subgrid']}, {c['num_subgrid']}]",
        "queue_size_per_thread: 1000", "memoryspace_size: 500000", "number_of_tasks: 5000000",
        "MPI_buffer_size: 1000", "cost_copy_factor: 10", "edge_copy_factor: 0.01",
        "general_queue_size: 100000", ""])
    with tempfile.TemporaryDirectory() as td:
        with open(os.path.join(td, "params.txt"), "w") as f:
            f.write(params)
        subprocess.run([b, "-p", "params.txt", "-t", str(c["threads"])], cwd=td, check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        img = np.fromfile(os.path.join(td, "image.dat"), dtype=np.float64).reshape(101, 101)
    save("dust_image.npz", image=img, **{k: np.array(v) for k, v in c.items()})


OUTPUT_CASE = {"ncell": (16, 16, 8), "num_subgrid": (2, 2, 1),
               "anchor_pc": (-5.0, -4.0, -3.0), "sides_pc": (10.0, 8.0, 6.0),
               "num_photon": 20000, "iterations": 2}


def _files_run(random_density=False, number_of_sources=1):
    """Runs the reference driver with its file output switched on in a
    temporary directory (params written here: the keys of
    params_single_uniform.txt), one thread; returns the .dat bytes, the .bin
    values and the params text."""
    import subprocess
    import tempfile
    b = O.ref_binary("testDensitySubGrid_omp_files")
    if b is None:
        sys.exit("oracle/_ref/testDensitySubGrid_omp_files missing: run oracle/build_ref.sh")
    c = OUTPUT_CASE
    v = lambda t: "[" + ", ".join(str(int(x)) for x in t) + "]"
    pcs = lambda t: "[" + ", ".join(f"{x} pc" for x in t) + "]"
    params = "\n".join([
        "box:", f"  anchor: {pcs(c['anchor_pc'])}", f"  sides: {pcs(c['sides_pc'])}",
        f"ncell: {v(c['ncell'])}", f"num_photon: {c['num_photon']}",
        f"number_of_iterations: {c['iterations']}", "reemission_probability: 0.",
        f"number_of_sources: {number_of_sources}",
        f"random_density: {'true' if random_density else 'false'}",
        f"num_subgrid: {v(c['num_subgrid'])}",
        "queue_size_per_thread: 100", "memoryspace_size: 50000", "number_of_tasks: 500000",
        "MPI_buffer_size: 1000", "cost_copy_factor: 10", "edge_copy_factor: 0.01",
        "general_queue_size: 100000", ""])
    with tempfile.TemporaryDirectory() as td:
        with open(os.path.join(td, "params.txt"), "w") as f:
            f.write(params)
        subprocess.run([b, "-p", "params.txt", "-t", "1"], cwd=td, check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        dat = np.fromfile(os.path.join(td, "neutral_fractions.dat"), dtype=np.uint8)
        binf = np.fromfile(os.path.join(td, "neutral_fractions.bin"), dtype=np.float64)
    return dat, binf, params


def gen_outputs():
    """outputs.npz: uniform density; outputs_random.npz: the driver's random
    density field (10 cosine modes), for the C++ surface's set-up of the same
    run (seeded 42 + threads).  One source each: with several sources whose
    packet counts are not multiples of 100, the driver does not finish (its
    last task of a source emits 200 - n % 200 packets instead of n % 200,
    testDensitySubGrid_omp.cpp:2266-2270, so the count of finished packets
    never equals num_photon, its stop test at :2390)."""
    c = OUTPUT_CASE
    geo = dict(ncell=np.array(c["ncell"]), num_subgrid=np.array(c["num_subgrid"]),
               anchor_pc=np.array(c["anchor_pc"]), sides_pc=np.array(c["sides_pc"]))
    dat, binf, _ = _files_run()
    save("outputs.npz", dat=dat, bin=binf, **geo)
    dat, binf, params = _files_run(random_density=True, number_of_sources=1)
    save("outputs_random.npz", dat=dat, bin=binf, params=np.array(params), threads=np.array(1),
         **geo)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--skip-ensemble", action="store_true")
    ap.add_argument("--only-ensembles", action="store_true",
                    help="regenerate the reemission and log-normal ensembles only")
    ap.add_argument("--only-outputs", action="store_true",
                    help="regenerate outputs.npz only")
    ap.add_argument("--only-dust", action="store_true",
                    help="regenerate dust_walks.npz only (from the walk fixtures)")
    args = ap.parse_args()
    if args.only_outputs:
        gen_outputs()
        return
    if args.only_ensembles:
        gen_ensemble_reemission()
        gen_ensemble_lognormal()
        return
    if args.only_dust:
        gen_dust_walks()
        gen_dust_image()
        return
    if O.ref_binary() is None:
        sys.exit("oracle/_ref/ref_harness_exact missing: run oracle/build_ref.sh first")
    gen_directions()
    gen_rng()
    gen_emission()
    gen_walks()
    gen_balance()
    gen_transport()
    gen_dust_walks()
    gen_dust_image()
    gen_outputs()
    if not args.skip_ensemble:
        gen_ensemble()
        gen_ensemble_reemission()
        gen_ensemble_lognormal()


if __name__ == "__main__":
    main()

"""Python host mirror of the reference's photoionization surface.

``TransportEngine`` wraps one library context (one or many grid instances).
Its methods follow the reference's calls for this path:

* ``trace_packet``      -- DensitySubGrid::interact (DensitySubGrid.hpp:1180)
* ``traverse_buffer``   -- do_photon_traversal (testDensitySubGrid_omp.cpp:607)
* ``compute_neutral_fraction`` -- DensitySubGrid::compute_neutral_fraction
  (DensitySubGrid.hpp:1628)
* ``run_iterations``    -- the driver's shoot/balance loop
  (testDensitySubGrid_omp.cpp:2213-2434)

Errors raise ``CMIError`` (the reference aborts via cmac_error/myassert).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import CMIError, PHOTON_DTYPE, check, ptr

PARSEC = 3.086e16  # m, UnitConverter.hpp:102

TRAVEL_DIRECTIONS = [
    "INSIDE",
    "CORNER_PPP", "CORNER_PPN", "CORNER_PNP", "CORNER_PNN",
    "CORNER_NPP", "CORNER_NPN", "CORNER_NNP", "CORNER_NNN",
    "EDGE_X_PP", "EDGE_X_PN", "EDGE_X_NP", "EDGE_X_NN",
    "EDGE_Y_PP", "EDGE_Y_PN", "EDGE_Y_NP", "EDGE_Y_NN",
    "EDGE_Z_PP", "EDGE_Z_PN", "EDGE_Z_NP", "EDGE_Z_NN",
    "FACE_X_P", "FACE_X_N", "FACE_Y_P", "FACE_Y_N", "FACE_Z_P", "FACE_Z_N",
]
TravelDirection = {name: i for i, name in enumerate(TRAVEL_DIRECTIONS)}

# transport precisions (cmi_precision): "fp64" the reference's walk operation for
# operation; "mixed" its FP64 geometry with FP32 opacity, optical depths and
# tallies; "fp32" the FP32 cell-unit walk
PRECISIONS = {"fp64": _lib.TRANSPORT_FP64, "fp32": _lib.TRANSPORT_FP32,
              "mixed": _lib.TRANSPORT_MIXED}

# shared-memory path-length tallies of the FP32 and mixed transports (cmi_tally)
TALLY_MODES = {"fp32": _lib.TALLY_FP32, "fp32_compensated": _lib.TALLY_FP32_COMPENSATED,
               "fixed64": _lib.TALLY_FIXED64, "fixed64_atomic64": _lib.TALLY_FIXED64_ATOMIC64}


@dataclass
class GridSpec:
    """One grid instance (box in m, cells and subgrids per axis)."""

    box: tuple
    ncell: tuple
    num_subgrid: tuple
    recombination_rate: float = 4.0e-19  # DensitySubGrid.hpp:1637
    cross_section: float = 6.3e-22       # testDensitySubGrid_omp.cpp:589
    sources: list = field(default_factory=list)  # [(x, y, z, L), ...]
    num_photon: int = 0
    reemission_probability: float = 0.0          # params.txt reemission_probability

    def desc(self) -> _lib.GridDesc:
        g = _lib.GridDesc()
        for i in range(6):
            g.box[i] = float(self.box[i])
        for i in range(3):
            g.ncell[i] = int(self.ncell[i])
            g.num_subgrid[i] = int(self.num_subgrid[i])
        g.recombination_rate = float(self.recombination_rate)
        g.cross_section = float(self.cross_section)
        return g

    @property
    def num_cells(self) -> int:
        return int(np.prod(self.ncell))

    @property
    def sub_ncell(self):
        return tuple(int(n) // int(s) for n, s in zip(self.ncell, self.num_subgrid))


def blocked_to_cube(a, ncell, num_subgrid):
    """Subgrid-blocked order (reference output order) -> (nx, ny, nz) cube."""
    sx, sy, sz = num_subgrid
    cx, cy, cz = (n // s for n, s in zip(ncell, num_subgrid))
    return (np.asarray(a).reshape(sx, sy, sz, cx, cy, cz)
            .transpose(0, 3, 1, 4, 2, 5).reshape(ncell[0], ncell[1], ncell[2]))


def cube_to_blocked(a, ncell, num_subgrid):
    sx, sy, sz = num_subgrid
    cx, cy, cz = (n // s for n, s in zip(ncell, num_subgrid))
    return (np.asarray(a).reshape(sx, cx, sy, cy, sz, cz)
            .transpose(0, 2, 4, 1, 3, 5).reshape(-1))


class TransportEngine:
    """A library context holding one or more grid instances on one GPU."""

    def __init__(self, grids, precision="mixed", balance="stable", rng="philox", device=0,
                 packets_per_chunk=0, tally="fixed64", use_graph=True, ctas_per_sm=0,
                 max_run_chunks=0, refill_lanes=0):
        if isinstance(grids, GridSpec):
            grids = [grids]
        self.grids = list(grids)
        self._L = _lib.load()
        opts = _lib.default_options(
            transport_precision=PRECISIONS[precision],
            balance_form={"reference": _lib.BALANCE_REFERENCE, "stable": _lib.BALANCE_STABLE}[balance],
            rng={"philox": _lib.RNG_PHILOX, "ranlux": _lib.RNG_RANLUX}[rng],
            device=device, packets_per_chunk=packets_per_chunk,
            tally_mode=TALLY_MODES[tally], use_graph=int(bool(use_graph)),
            ctas_per_sm=ctas_per_sm, max_run_chunks=max_run_chunks, refill_lanes=refill_lanes)
        descs = (_lib.GridDesc * len(self.grids))(*[g.desc() for g in self.grids])
        h = C.c_void_p()
        check(self._L.cmi_create(descs, len(self.grids), C.byref(opts), C.byref(h)))
        self._h = h
        self.precision = precision
        for i, g in enumerate(self.grids):
            if g.sources:
                s = np.asarray(g.sources, dtype=np.float64).reshape(-1, 4)
                self.set_sources(i, s[:, :3], s[:, 3])
            if g.num_photon:
                self.set_packet_budget(i, g.num_photon)
            if g.reemission_probability:
                self.set_reemission_probability(i, g.reemission_probability)

    # ---- lifetime ----
    def close(self):
        if getattr(self, "_h", None):
            self._L.cmi_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- state ----
    def set_fields(self, instance=0, number_density=None, neutral_fraction=None,
                   layout="blocked"):
        lay = {"blocked": _lib.LAYOUT_BLOCKED, "cube": _lib.LAYOUT_CUBE}[layout]
        n = None if number_density is None else np.ascontiguousarray(number_density, np.float64)
        x = None if neutral_fraction is None else np.ascontiguousarray(neutral_fraction, np.float64)
        for a in (n, x):
            if a is not None and a.size != self.grids[instance].num_cells:
                raise ValueError("field size does not match the grid")
        check(self._L.cmi_set_fields(self._h, instance, lay, _lib.MEMORY_HOST, ptr(n), ptr(x)))

    def prefetch_number_density(self, instance, number_density, layout="blocked"):
        """Start copying n_H (a pinned host array) on a side stream.  The array
        must stay unchanged until the next run_iterations, run_until_converged,
        shoot_packets, get_fields or synchronize returns."""
        lay = {"blocked": _lib.LAYOUT_BLOCKED, "cube": _lib.LAYOUT_CUBE}[layout]
        n = np.asarray(number_density)
        if n.dtype != np.float64 or not n.flags.c_contiguous or \
                n.size != self.grids[instance].num_cells:
            raise ValueError("n_H must be a contiguous float64 array of the grid's size")
        self._prefetched = getattr(self, "_prefetched", {})
        self._prefetched[instance] = n  # keep the array alive until it is consumed
        check(self._L.cmi_prefetch_number_density(self._h, instance, lay, ptr(n)))

    def set_fields_prefetched(self, instance, neutral_fraction=None):
        """n_H from the last prefetch of the instance, x_H from the host.  The
        copies run on the side stream and the next iteration waits for them
        after its emission; x_H (pinned or not) must stay unchanged until the
        next run_iterations, run_until_converged, shoot_packets, get_fields or
        synchronize returns."""
        x = None if neutral_fraction is None else np.ascontiguousarray(neutral_fraction,
                                                                       np.float64)
        if x is not None and x.size != self.grids[instance].num_cells:
            raise ValueError("field size does not match the grid")
        check(self._L.cmi_set_fields_prefetched(self._h, instance, _lib.MEMORY_HOST, ptr(x)))
        # both host arrays may still be read by the side stream
        self._in_flight = getattr(self, "_in_flight", [])
        self._in_flight.append(getattr(self, "_prefetched", {}).pop(instance, None))
        self._in_flight.append(x)

    def _settled(self):
        """The side stream's copies are complete: release their arrays."""
        self._in_flight = []

    def set_fields_device(self, instance, number_density_ptr=0, neutral_fraction_ptr=0,
                          layout="blocked"):
        lay = {"blocked": _lib.LAYOUT_BLOCKED, "cube": _lib.LAYOUT_CUBE}[layout]
        check(self._L.cmi_set_fields(self._h, instance, lay, _lib.MEMORY_DEVICE,
                                     number_density_ptr or None, neutral_fraction_ptr or None))

    def get_fields(self, instance=0, layout="blocked", neutral_fraction=True,
                   intensity=True, out_x=None, out_j=None):
        lay = {"blocked": _lib.LAYOUT_BLOCKED, "cube": _lib.LAYOUT_CUBE}[layout]
        n = self.grids[instance].num_cells
        x = (out_x if out_x is not None else np.empty(n)) if neutral_fraction else None
        j = (out_j if out_j is not None else np.empty(n)) if intensity else None
        check(self._L.cmi_get_fields(self._h, instance, lay, _lib.MEMORY_HOST, ptr(x), ptr(j)))
        self._settled()
        return x, j

    def set_intensity(self, instance, J, layout="blocked"):
        lay = {"blocked": _lib.LAYOUT_BLOCKED, "cube": _lib.LAYOUT_CUBE}[layout]
        a = np.ascontiguousarray(J, np.float64)
        check(self._L.cmi_set_intensity(self._h, instance, lay, _lib.MEMORY_HOST, ptr(a)))

    def set_sources(self, instance, positions, luminosities):
        p = np.ascontiguousarray(positions, np.float64).reshape(-1)
        l = np.ascontiguousarray(luminosities, np.float64).reshape(-1)
        if p.size != 3 * l.size:
            raise ValueError("3 coordinates per source")
        check(self._L.cmi_set_sources(self._h, instance, ptr(p), ptr(l), l.size))

    def set_reemission_probability(self, instance, probability):
        check(self._L.cmi_set_reemission_probability(self._h, instance, float(probability)))

    def set_packet_budget(self, instance, num_photon):
        check(self._L.cmi_set_packet_budget(self._h, instance, int(num_photon)))

    # ---- the hot path ----
    def run_iterations(self, iterations=1, seed=42):
        """Shoot + balance; returns stats[iteration][instance] dicts."""
        ninst = len(self.grids)
        st = (_lib.Stats * (iterations * ninst))()
        check(self._L.cmi_run_iterations(self._h, iterations, int(seed), st))
        self._settled()
        return [[st[it * ninst + i].as_dict() for i in range(ninst)] for it in range(iterations)]

    def run_until_converged(self, tolerance, max_iterations=100, min_iterations=2, seed=42):
        """Iterate until each instance's mean |delta x_H| < tolerance (then it
        is frozen for the rest of the call).  Returns (stats, converged_at):
        stats[iteration][instance] dicts and, per instance, the 1-based
        iteration after which it converged (0: not within max_iterations)."""
        ninst = len(self.grids)
        st = (_lib.Stats * (max_iterations * ninst))()
        done = C.c_int32(0)
        at = (C.c_int32 * ninst)()
        check(self._L.cmi_run_until_converged(self._h, int(max_iterations), int(min_iterations),
                                              float(tolerance), int(seed), st, C.byref(done),
                                              at))
        self._settled()
        stats = [[st[it * ninst + i].as_dict() for i in range(ninst)]
                 for it in range(done.value)]
        return stats, list(at)

    def walk_photons(self, instance, subgrid, photons, input_directions, depth=False):
        """DensitySubGrid::propagate (or, with depth, compute_optical_depth) of
        each photon (PHOTON_DTYPE records, copied) through one subgrid.
        Returns (photons out, output TravelDirections)."""
        ph = np.ascontiguousarray(photons, dtype=PHOTON_DTYPE).copy()
        dirs = np.ascontiguousarray(np.broadcast_to(input_directions, ph.shape), dtype=np.int32)
        out = np.zeros(ph.size, dtype=np.int32)
        mode = _lib.WALK_OPTICAL_DEPTH if depth else _lib.WALK_PROPAGATE
        check(self._L.cmi_walk_photons(self._h, int(instance), int(subgrid), mode,
                                       ph.ctypes.data, dirs.ctypes.data, ph.size,
                                       out.ctypes.data))
        return ph, out

    def dust_image(self, instance, num_photon, albedo, source=(0.0, 0.0, 0.0), npix=(101, 101),
                   seed=42, iteration=0):
        """The reference dust driver's photon loop on this instance's n_H and x_H
        (cmi_dust_run: forced first scattering, isotropic scattering with
        probability `albedo`, peel-off image along +z).  Returns (image
        [npix_x, npix_y] divided by num_photon, stats dict)."""
        img = np.zeros(int(npix[0]) * int(npix[1]))
        src = np.ascontiguousarray(source, dtype=np.float64)
        st = _lib.DustStats()
        check(self._L.cmi_dust_run(self._h, int(instance), int(num_photon), int(seed),
                                   int(iteration), float(albedo), src.ctypes.data,
                                   int(npix[0]), int(npix[1]), img.ctypes.data, C.byref(st)))
        return img.reshape(int(npix[0]), int(npix[1])), st.as_dict()

    def shoot_packets(self, seed=42, iteration=0):
        ninst = len(self.grids)
        st = (_lib.Stats * ninst)()
        check(self._L.cmi_shoot_packets(self._h, int(seed), int(iteration), st))
        self._settled()
        return [st[i].as_dict() for i in range(ninst)]

    def emit_photons(self, seed=42, iteration=0):
        """fill_buffer for every source: the photons an iteration with this seed
        and iteration index emits (PHOTON_DTYPE, instance, source, emission order)."""
        n = C.c_uint64(0)
        rc = self._L.cmi_emit_photons(self._h, int(seed), int(iteration), None, 0, C.byref(n))
        if rc not in (_lib.OK, _lib.ERR_CAPACITY):
            check(rc)
        out = np.zeros(n.value, PHOTON_DTYPE)
        if n.value:
            check(self._L.cmi_emit_photons(self._h, int(seed), int(iteration), ptr(out),
                                           out.size, C.byref(n)))
        return out

    def transport_packets(self, instance, photons, start_subgrid):
        ph = np.ascontiguousarray(photons, dtype=PHOTON_DTYPE)
        s = np.ascontiguousarray(start_subgrid, dtype=np.uint32)
        st = _lib.Stats()
        check(self._L.cmi_transport_packets(self._h, instance, ptr(ph), ptr(s), ph.size,
                                            C.byref(st)))
        return st.as_dict()

    def traverse_buffer(self, instance, subgrid, input_direction, photons, enabled=None):
        """do_photon_traversal: returns (grouped photons, counts[27], num_done)."""
        ph = np.ascontiguousarray(photons, dtype=PHOTON_DTYPE)
        out = np.zeros(max(ph.size, 1), dtype=PHOTON_DTYPE)
        counts = np.zeros(27, dtype=np.uint32)
        done = C.c_uint32(0)
        en = None if enabled is None else np.ascontiguousarray(enabled, dtype=np.uint8)
        check(self._L.cmi_traverse_buffer(self._h, instance, int(subgrid), int(input_direction),
                                          ptr(ph), ph.size, ptr(en), ptr(out), ptr(counts),
                                          C.byref(done)))
        return out[: int(counts.sum())], counts, int(done.value)

    def trace_packet(self, instance, subgrid, input_direction, photon, max_steps=4096):
        """interact() for one packet: (photon_out, out_direction, cells, lengths, nsteps)."""
        ph = np.array(photon, dtype=PHOTON_DTYPE).reshape(1).copy()
        cells = np.zeros(max(max_steps, 1), dtype=np.int32)
        lengths = np.zeros(max(max_steps, 1), dtype=np.float64)
        nsteps = C.c_int32(0)
        out_dir = C.c_int32(-1)
        check(self._L.cmi_trace_packet(self._h, instance, int(subgrid), int(input_direction),
                                       ptr(ph), int(max_steps), ptr(cells), ptr(lengths),
                                       C.byref(nsteps), C.byref(out_dir)))
        k = min(nsteps.value, max_steps)
        return ph[0], out_dir.value, cells[:k].copy(), lengths[:k].copy(), nsteps.value

    def compute_neutral_fraction(self, instance, luminosity, num_photon):
        dx = C.c_double(0.)
        check(self._L.cmi_compute_neutral_fraction(self._h, instance, float(luminosity),
                                                   int(num_photon), C.byref(dx)))
        return dx.value

    # ---- interop ----
    def device_field(self, instance, which="J"):
        w = {"J": 0, "x": 1, "n": 2}[which]
        p = C.POINTER(C.c_double)()
        n = C.c_uint64(0)
        check(self._L.cmi_device_field(self._h, instance, w, C.byref(p), C.byref(n)))
        return C.cast(p, C.c_void_p).value, int(n.value)

    def stream(self) -> int:
        s = C.c_void_p()
        check(self._L.cmi_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def synchronize(self):
        check(self._L.cmi_synchronize(self._h))
        self._settled()

    KERNEL_CLASSES = ("walk", "plan_scatter", "emission", "balance")

    def set_kernel_timing(self, enable=True):
        check(self._L.cmi_set_kernel_timing(self._h, int(bool(enable))))

    def kernel_timing(self):
        """{class: (milliseconds, launches)} since the last call (timing mode)."""
        ms = np.zeros(4, np.float64)
        n = np.zeros(4, np.uint64)
        check(self._L.cmi_kernel_timing(self._h, ptr(ms), ptr(n)))
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(self.KERNEL_CLASSES)}

    def last_launch_count(self) -> int:
        n = C.c_uint64(0)
        check(self._L.cmi_last_launch_count(self._h, C.byref(n)))
        return int(n.value)


__all__ = ["TransportEngine", "GridSpec", "CMIError", "PHOTON_DTYPE", "TravelDirection",
           "TRAVEL_DIRECTIONS", "PARSEC", "blocked_to_cube", "cube_to_blocked"]

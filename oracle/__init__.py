"""CPU oracle for the transport + ionization-balance path (test infrastructure).

ctypes binding of ``oracle/libcmi_oracle.so`` (the plain-C restatement of the
reference algorithm in ``cmi_oracle.c``) plus helpers to run the reference
harness built from the reference's own sources (``oracle/_ref``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcmi_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

INSIDE = 0
NUM_DIRECTIONS = 27
NEIGHBOUR_OUTSIDE = 0xFFFFFFFF

PHOTON_DTYPE = np.dtype(
    [
        ("position", "<f8", (3,)),
        ("direction", "<f8", (3,)),
        ("tau", "<f8"),
        ("sigma", "<f8"),
        ("weight", "<f8"),
        ("type", "<i4"),
        ("reserved", "<i4"),
    ]
)
assert PHOTON_DTYPE.itemsize == 80

PACKET32_DTYPE = np.dtype(
    [("pos", "<f4", (3,)), ("dir", "<f4", (3,)), ("tau", "<f4"), ("meta", "<u4")]
)
assert PACKET32_DTYPE.itemsize == 32

# mixed-precision packet (cmio_packetm): absolute FP64 position and direction,
# FP32 remaining optical depth
PACKETM_DTYPE = np.dtype(
    [("pos", "<f8", (3,)), ("dir", "<f8", (3,)), ("tau", "<f4"), ("meta", "<u4"),
     ("pad", "<u4", (2,))]
)
assert PACKETM_DTYPE.itemsize == 64

_DIRECTION_NAMES = [
    "INSIDE",
    "CORNER_PPP", "CORNER_PPN", "CORNER_PNP", "CORNER_PNN",
    "CORNER_NPP", "CORNER_NPN", "CORNER_NNP", "CORNER_NNN",
    "EDGE_X_PP", "EDGE_X_PN", "EDGE_X_NP", "EDGE_X_NN",
    "EDGE_Y_PP", "EDGE_Y_PN", "EDGE_Y_NP", "EDGE_Y_NN",
    "EDGE_Z_PP", "EDGE_Z_PN", "EDGE_Z_NP", "EDGE_Z_NN",
    "FACE_X_P", "FACE_X_N", "FACE_Y_P", "FACE_Y_N", "FACE_Z_P", "FACE_Z_N",
]
DIRECTION = {name: i for i, name in enumerate(_DIRECTION_NAMES)}


class Subgrid(C.Structure):
    _fields_ = [
        ("anchor", C.c_double * 3),
        ("cell_size", C.c_double * 3),
        ("inv_cell_size", C.c_double * 3),
        ("ncell", C.c_int32 * 4),
    ]


class Ranlux(C.Structure):
    _fields_ = [
        ("x", C.c_double * 12),
        ("carry", C.c_double),
        ("ir", C.c_uint32),
        ("jr", C.c_uint32),
        ("ir_old", C.c_uint32),
        ("pr", C.c_uint32),
    ]


class Lattice(C.Structure):
    _fields_ = [
        ("num_subgrid", C.c_int32 * 3),
        ("sub_ncell", C.c_int32 * 3),
        ("cells_per_subgrid", C.c_int64),
        ("nsub", C.c_int64),
        ("sub", C.POINTER(Subgrid)),
        ("ngb", C.POINTER(C.c_uint32)),
    ]


class Reemission(C.Structure):
    _fields_ = [
        ("probability", C.c_double),
        ("seed", C.c_uint64),
        ("instance", C.c_uint32),
        ("iteration", C.c_uint32),
    ]


class Counts(C.Structure):
    _fields_ = [
        ("absorbed", C.c_uint64),
        ("escaped", C.c_uint64),
        ("crossings", C.c_uint64),
        ("transits", C.c_uint64),
        ("reemitted", C.c_uint64),
    ]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class DustStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("emitted", "scatterings", "absorbed", "escaped",
                                          "cell_crossings", "subgrid_transits",
                                          "peeloffs_off_image")] + \
               [("generations", C.c_uint32), ("error_flags", C.c_uint32)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


_lib = None


def lib():
    """Load (building if needed) the oracle shared library."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        L = C.CDLL(LIB_PATH)
        d, i32, u32, i64, u64 = C.c_double, C.c_int32, C.c_uint32, C.c_int64, C.c_uint64
        pd, pi32, pu32, pf = C.POINTER(d), C.POINTER(i32), C.POINTER(u32), C.POINTER(C.c_float)
        L.cmio_output_to_input_direction.argtypes = [C.c_int]
        L.cmio_direction_from_mask.argtypes = [C.c_int]
        L.cmio_is_compatible_input_direction.argtypes = [pd, C.c_int]
        L.cmio_is_compatible_output_direction.argtypes = [pd, C.c_int]
        L.cmio_subgrid_init.argtypes = [C.POINTER(Subgrid), pd, pi32]
        L.cmio_get_start_index.argtypes = [C.POINTER(Subgrid), pd, C.c_int, pi32]
        L.cmio_get_output_direction.argtypes = [C.POINTER(Subgrid), pi32]
        L.cmio_interact.argtypes = [C.POINTER(Subgrid), pd, pd, pd, C.c_void_p, C.c_int,
                                    pi32, pd, i32, pi32]
        L.cmio_interact32.argtypes = [pi32, pf, pf, pf, pd, C.POINTER(u64), C.c_float,
                                      C.c_void_p, pi32, pf, i32, pi32]
        L.cmio_interact_mixed.argtypes = [C.POINTER(Subgrid), pf, pd, C.POINTER(u64),
                                          C.c_float, C.c_void_p, pi32, pd, i32, pi32]
        L.cmio_transportm_r.argtypes = [C.POINTER(Lattice), pf, pd, C.POINTER(u64),
                                        C.c_void_p, pu32, i64, C.POINTER(Counts), C.c_void_p]
        L.cmio_fixed_scale.argtypes = [C.POINTER(Subgrid)]
        L.cmio_fixed_scale.restype = C.c_float
        L.cmio_jfac.argtypes = [d, d, pd]
        L.cmio_jfac.restype = d
        L.cmio_compute_neutral_fraction.argtypes = [i64, pd, pd, pd, d, d, C.c_int]
        L.cmio_ranlux_seed.argtypes = [C.POINTER(Ranlux), i32]
        L.cmio_ranlux_uniform.argtypes = [C.POINTER(Ranlux)]
        L.cmio_ranlux_uniform.restype = d
        L.cmio_fill_buffer_stream.argtypes = [i32, pd, C.c_void_p, i32, d]
        L.cmio_fill_buffer_stream_cr.argtypes = [i32, pd, C.c_void_p, i32, d]
        L.cmio_cr_sincos.argtypes = [d, pd, pd]
        L.cmio_cr_neg_log.argtypes = [d]
        L.cmio_cr_neg_log.restype = d
        L.cmio_source_numbers.argtypes = [i32, pd, u32, pu32]
        L.cmio_distribute.argtypes = [i32, i32, C.POINTER(Ranlux), pu32]
        L.cmio_philox4x32.argtypes = [pu32, pu32, pu32]
        L.cmio_philox_packet.argtypes = [u64, u32, u64, pd, pd]
        L.cmio_lattice_init.argtypes = [C.POINTER(Lattice), pd, pi32, pi32]
        L.cmio_lattice_free.argtypes = [C.POINTER(Lattice)]
        L.cmio_lattice_locate.argtypes = [C.POINTER(Lattice), pd, pd]
        L.cmio_lattice_locate.restype = u32
        L.cmio_transport.argtypes = [C.POINTER(Lattice), pd, pd, pd, C.c_void_p, pu32, i64,
                                     C.POINTER(Counts)]
        L.cmio_transport32.argtypes = [C.POINTER(Lattice), pf, pd, C.POINTER(u64), C.c_void_p,
                                       pu32, i64, C.POINTER(Counts)]
        L.cmio_transport_r.argtypes = [C.POINTER(Lattice), pd, pd, pd, C.c_void_p, pu32, i64,
                                       C.POINTER(Counts), C.c_void_p]
        L.cmio_transport32_r.argtypes = [C.POINTER(Lattice), pf, pd, C.POINTER(u64),
                                         C.c_void_p, pu32, i64, C.POINTER(Counts), C.c_void_p]
        L.cmio_split_packets.argtypes = [i32, pd, u64, u64, u32, C.POINTER(u64)]
        L.cmio_kappa32.argtypes = [i64, pd, pd, d, pf]
        L.cmio_iteration_omp.argtypes = [C.POINTER(Lattice), pd, pd, pd, pd, i32, pd, pd, u64,
                                         u64, u32, d, d, C.c_int, C.c_int, C.POINTER(Counts)]
        L.cmio_propagate.argtypes = [C.POINTER(Subgrid), pd, pd, C.c_void_p, C.c_int, pi32]
        L.cmio_compute_optical_depth.argtypes = [C.POINTER(Subgrid), pd, pd, C.c_void_p,
                                                 C.c_int, pi32]
        L.cmio_dust_exp.argtypes = [d]
        L.cmio_dust_exp.restype = d
        L.cmio_dust_run.argtypes = [C.POINTER(Lattice), pd, pd, pd, u32, u64, u32, u32, d, pd,
                                    u32, i32, i32, pd, C.POINTER(DustStats)]
        _lib = L
    return _lib


# --------------------------------------------------------------------------
# thin numpy wrappers
# --------------------------------------------------------------------------
def output_to_input_direction(d: int) -> int:
    return lib().cmio_output_to_input_direction(d)


def direction_from_mask(mask: int) -> int:
    return lib().cmio_direction_from_mask(mask)


def subgrid(box, ncell) -> Subgrid:
    sg = Subgrid()
    b = np.ascontiguousarray(box, dtype=np.float64)
    n = np.ascontiguousarray(ncell, dtype=np.int32)
    lib().cmio_subgrid_init(C.byref(sg), _ptr(b, C.c_double), _ptr(n, C.c_int32))
    return sg


def get_start_index(sg: Subgrid, position, input_direction: int):
    p = np.ascontiguousarray(position, dtype=np.float64)
    out = np.zeros(3, dtype=np.int32)
    lib().cmio_get_start_index(C.byref(sg), _ptr(p, C.c_double), input_direction,
                               _ptr(out, C.c_int32))
    return tuple(int(v) for v in out)


def get_output_direction(sg: Subgrid, three_index) -> int:
    t = np.ascontiguousarray(three_index, dtype=np.int32)
    return lib().cmio_get_output_direction(C.byref(sg), _ptr(t, C.c_int32))


def is_compatible_input_direction(direction, d: int) -> bool:
    v = np.ascontiguousarray(direction, dtype=np.float64)
    return bool(lib().cmio_is_compatible_input_direction(_ptr(v, C.c_double), d))


def is_compatible_output_direction(direction, d: int) -> bool:
    v = np.ascontiguousarray(direction, dtype=np.float64)
    return bool(lib().cmio_is_compatible_output_direction(_ptr(v, C.c_double), d))


def interact(sg: Subgrid, nH, xH, J, photon, input_direction: int, max_steps: int = 0):
    """Walk one photon (a PHOTON_DTYPE record, modified in place).

    Returns (result_direction, trace_cells, trace_lengths)."""
    cells = np.zeros(max(max_steps, 1), dtype=np.int32)
    lengths = np.zeros(max(max_steps, 1), dtype=np.float64)
    nsteps = C.c_int32(0)
    res = lib().cmio_interact(
        C.byref(sg), _ptr(nH, C.c_double), _ptr(xH, C.c_double), _ptr(J, C.c_double),
        photon.ctypes.data, input_direction,
        _ptr(cells, C.c_int32) if max_steps else None,
        _ptr(lengths, C.c_double) if max_steps else None, max_steps, C.byref(nsteps))
    n = min(nsteps.value, max_steps)
    return res, cells[:n].copy(), lengths[:n].copy(), nsteps.value


def propagate(sg: Subgrid, nH, xH, photon, input_direction: int):
    """DensitySubGrid::propagate on one photon (modified in place): (result, steps)."""
    nsteps = C.c_int32(0)
    res = lib().cmio_propagate(C.byref(sg), _ptr(nH, C.c_double), _ptr(xH, C.c_double),
                               photon.ctypes.data, input_direction, C.byref(nsteps))
    return res, nsteps.value


def compute_optical_depth(sg: Subgrid, nH, xH, photon, input_direction: int):
    """DensitySubGrid::compute_optical_depth on one photon (in place): (result, steps)."""
    nsteps = C.c_int32(0)
    res = lib().cmio_compute_optical_depth(C.byref(sg), _ptr(nH, C.c_double),
                                           _ptr(xH, C.c_double), photon.ctypes.data,
                                           input_direction, C.byref(nsteps))
    return res, nsteps.value


def dust_exp(x: float) -> float:
    return lib().cmio_dust_exp(float(x))


def interact32(ncell, cell_size, kappa, tally, packet, max_steps: int = 0,
               inv_cell_size=None):
    """FP32 cell-unit walk; inv_cell_size defaults to float(1 / cell_size)."""
    n3 = np.ascontiguousarray(ncell, dtype=np.int32)
    cs = np.ascontiguousarray(cell_size, dtype=np.float32)
    if inv_cell_size is None:
        inv_cell_size = 1.0 / np.asarray(cell_size, dtype=np.float64)
    ics = np.ascontiguousarray(inv_cell_size, dtype=np.float32)
    cells = np.zeros(max(max_steps, 1), dtype=np.int32)
    lengths = np.zeros(max(max_steps, 1), dtype=np.float32)
    nsteps = C.c_int32(0)
    res = lib().cmio_interact32(
        _ptr(n3, C.c_int32), _ptr(cs, C.c_float), _ptr(ics, C.c_float), _ptr(kappa, C.c_float),
        _ptr(tally, C.c_double) if tally is not None else None, None, 1.0, packet.ctypes.data,
        _ptr(cells, C.c_int32) if max_steps else None,
        _ptr(lengths, C.c_float) if max_steps else None, max_steps, C.byref(nsteps))
    n = min(nsteps.value, max_steps)
    return res, cells[:n].copy(), lengths[:n].copy(), nsteps.value


def tau32(tau):
    """FP32 optical depth of the mixed walk: round to nearest, and a positive
    depth below the FP32 range becomes the smallest subnormal (not 0), so a
    packet the reference walks is walked."""
    t = np.asarray(tau, np.float64)
    f = t.astype(np.float32)
    tiny = np.frombuffer(np.uint32(1).tobytes(), np.float32)[0]
    return np.where((f == 0) & (t > 0), tiny, f).astype(np.float32)


def packets_mixed(photons, input_directions=None):
    """PACKETM_DTYPE records of PHOTON_DTYPE photons (tau as tau32)."""
    q = np.zeros(photons.size, PACKETM_DTYPE)
    q["pos"] = photons["position"]
    q["dir"] = photons["direction"]
    q["tau"] = tau32(photons["tau"])
    if input_directions is not None:
        q["meta"] = np.asarray(input_directions, np.uint32)
    return q


def interact_mixed(sg: Subgrid, kappa, packet, max_steps: int = 0, tally=None, fixed=None):
    """Mixed-precision walk of one PACKETM_DTYPE record (modified in place).

    Returns (result_direction, trace_cells, trace_lengths (FP64), steps)."""
    cells = np.zeros(max(max_steps, 1), dtype=np.int32)
    lengths = np.zeros(max(max_steps, 1), dtype=np.float64)
    nsteps = C.c_int32(0)
    res = lib().cmio_interact_mixed(
        C.byref(sg), _ptr(kappa, C.c_float),
        _ptr(tally, C.c_double) if tally is not None else None,
        _ptr(fixed, C.c_uint64) if fixed is not None else None,
        lib().cmio_fixed_scale(C.byref(sg)), packet.ctypes.data,
        _ptr(cells, C.c_int32) if max_steps else None,
        _ptr(lengths, C.c_double) if max_steps else None, max_steps, C.byref(nsteps))
    n = min(nsteps.value, max_steps)
    return res, cells[:n].copy(), lengths[:n].copy(), nsteps.value


def jfac(luminosity, num_photon, inv_cell_size):
    v = np.ascontiguousarray(inv_cell_size, dtype=np.float64)
    return lib().cmio_jfac(float(luminosity), float(num_photon), _ptr(v, C.c_double))


def compute_neutral_fraction(nH, xH, J, jfac_value, alpha_H=4e-19, form=0):
    lib().cmio_compute_neutral_fraction(nH.size, _ptr(nH, C.c_double), _ptr(xH, C.c_double),
                                        _ptr(J, C.c_double), jfac_value, alpha_H, form)


class RanluxGenerator:
    """RandomGenerator (RandomGenerator.hpp) restated."""

    def __init__(self, seed: int = 42):
        self.state = Ranlux()
        lib().cmio_ranlux_seed(C.byref(self.state), int(seed))

    def uniform(self, n: int | None = None):
        f = lib().cmio_ranlux_uniform
        if n is None:
            return f(C.byref(self.state))
        return np.array([f(C.byref(self.state)) for _ in range(n)])


def fill_buffer_stream(seed, source_position, n, cross_section=6.3e-22):
    out = np.zeros(n, dtype=PHOTON_DTYPE)
    p = np.ascontiguousarray(source_position, dtype=np.float64)
    lib().cmio_fill_buffer_stream(int(seed), _ptr(p, C.c_double), out.ctypes.data, n,
                                  cross_section)
    return out


def fill_buffer_stream_cr(seed, source_position, n, cross_section=6.3e-22):
    """fill_buffer_stream with correctly rounded sin, cos and log (the CUDA
    library's replay of the reference stream)."""
    out = np.zeros(n, dtype=PHOTON_DTYPE)
    p = np.ascontiguousarray(source_position, dtype=np.float64)
    lib().cmio_fill_buffer_stream_cr(int(seed), _ptr(p, C.c_double), out.ctypes.data, n,
                                     cross_section)
    return out


def cr_sincos(x):
    """Correctly rounded (sin x, cos x) for x in [0, 8)."""
    s, c = C.c_double(0.), C.c_double(0.)
    lib().cmio_cr_sincos(float(x), C.byref(s), C.byref(c))
    return s.value, c.value


def cr_neg_log(u):
    """Correctly rounded -ln(u) for u in [0, 1)."""
    return lib().cmio_cr_neg_log(float(u))


def philox4x32(counter, key):
    c = np.ascontiguousarray(counter, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib().cmio_philox4x32(_ptr(c, C.c_uint32), _ptr(k, C.c_uint32), _ptr(out, C.c_uint32))
    return out


def philox_packets(seed, stream, first, n):
    dirs = np.zeros((n, 3), dtype=np.float64)
    tau = np.zeros(n, dtype=np.float64)
    f = lib().cmio_philox_packet
    for i in range(n):
        f(seed, stream, first + i, _ptr(dirs[i], C.c_double),
          tau[i:].ctypes.data_as(C.POINTER(C.c_double)))
    return dirs, tau


def split_packets(luminosity, num_photon, seed, iteration):
    L = np.ascontiguousarray(luminosity, dtype=np.float64)
    out = np.zeros(L.size, dtype=np.uint64)
    lib().cmio_split_packets(L.size, _ptr(L, C.c_double), int(num_photon), int(seed),
                             int(iteration), _ptr(out, C.c_uint64))
    return out


def kappa32(nH, xH, sigma=6.3e-22):
    out = np.zeros(nH.size, dtype=np.float32)
    lib().cmio_kappa32(nH.size, _ptr(nH, C.c_double), _ptr(xH, C.c_double), sigma,
                       _ptr(out, C.c_float))
    return out


class LatticeGrid:
    """Lattice of subgrids with neighbour table (testDensitySubGrid_omp.cpp:1801-1877)."""

    def __init__(self, box, ncell, num_subgrid):
        self.box = np.ascontiguousarray(box, dtype=np.float64)
        self.ncell = np.ascontiguousarray(ncell, dtype=np.int32)
        self.num_subgrid = np.ascontiguousarray(num_subgrid, dtype=np.int32)
        self.lat = Lattice()
        rc = lib().cmio_lattice_init(C.byref(self.lat), _ptr(self.box, C.c_double),
                                     _ptr(self.ncell, C.c_int32),
                                     _ptr(self.num_subgrid, C.c_int32))
        if rc != 0:
            raise ValueError("ncell must be a multiple of num_subgrid")
        self.C = int(self.lat.cells_per_subgrid)
        self.nsub = int(self.lat.nsub)

    def __del__(self):
        try:
            lib().cmio_lattice_free(C.byref(self.lat))
        except Exception:
            pass

    def neighbours(self):
        return np.ctypeslib.as_array(self.lat.ngb, shape=(self.nsub * 27,)).reshape(
            self.nsub, 27).copy()

    def subgrid_desc(self, s):
        return self.lat.sub[s]

    def locate(self, position):
        p = np.ascontiguousarray(position, dtype=np.float64)
        return lib().cmio_lattice_locate(C.byref(self.lat), _ptr(self.box, C.c_double),
                                         _ptr(p, C.c_double))

    def transport(self, nH, xH, J, packets, start_subgrid, reemission=None):
        """FP64 transport; reemission = (probability, seed, instance, iteration)."""
        counts = Counts()
        s = np.ascontiguousarray(start_subgrid, dtype=np.uint32)
        r = Reemission(*reemission) if reemission else None
        lib().cmio_transport_r(C.byref(self.lat), _ptr(nH, C.c_double), _ptr(xH, C.c_double),
                               _ptr(J, C.c_double), packets.ctypes.data, _ptr(s, C.c_uint32),
                               packets.size, C.byref(counts), C.byref(r) if r else None)
        return counts.as_dict()

    def transport32(self, kappa, tally, packets, start_subgrid, fixed=None, reemission=None):
        """FP32 transport; tally: double sums of lmin, fixed: uint64 fixed-point sums."""
        counts = Counts()
        s = np.ascontiguousarray(start_subgrid, dtype=np.uint32)
        r = Reemission(*reemission) if reemission else None
        lib().cmio_transport32_r(C.byref(self.lat), _ptr(kappa, C.c_float),
                                 _ptr(tally, C.c_double) if tally is not None else None,
                                 _ptr(fixed, C.c_uint64) if fixed is not None else None,
                                 packets.ctypes.data, _ptr(s, C.c_uint32), packets.size,
                                 C.byref(counts), C.byref(r) if r else None)
        return counts.as_dict()

    def transport_mixed(self, kappa, tally, packets, start_subgrid, fixed=None,
                        reemission=None):
        """Mixed-precision transport (PACKETM_DTYPE packets, modified in place)."""
        counts = Counts()
        s = np.ascontiguousarray(start_subgrid, dtype=np.uint32)
        r = Reemission(*reemission) if reemission else None
        lib().cmio_transportm_r(C.byref(self.lat), _ptr(kappa, C.c_float),
                                _ptr(tally, C.c_double) if tally is not None else None,
                                _ptr(fixed, C.c_uint64) if fixed is not None else None,
                                packets.ctypes.data, _ptr(s, C.c_uint32), packets.size,
                                C.byref(counts), C.byref(r) if r else None)
        return counts.as_dict()

    def fixed_unit(self, s=0):
        """Metres per fixed-point tally unit of subgrid s (lref / 2^22)."""
        return float(max(np.float32(v) for v in self.lat.sub[s].cell_size)) / 4194304.0

    def dust_run(self, nH, xH, num_photon, seed, albedo, source, source_subgrid,
                 npix=(101, 101), instance=0, iteration=0):
        """Dust photon loop (cmio_dust_run): (image [npix_x, npix_y] / num_photon, stats)."""
        img = np.zeros(int(npix[0]) * int(npix[1]))
        src = np.ascontiguousarray(source, dtype=np.float64)
        nh = np.ascontiguousarray(nH, np.float64)
        xh = np.ascontiguousarray(xH, np.float64)
        st = DustStats()
        lib().cmio_dust_run(C.byref(self.lat), _ptr(self.box, C.c_double), _ptr(nh, C.c_double),
                            _ptr(xh, C.c_double), int(num_photon), int(seed), int(instance),
                            int(iteration), float(albedo), _ptr(src, C.c_double),
                            int(source_subgrid), int(npix[0]), int(npix[1]),
                            _ptr(img, C.c_double), C.byref(st))
        return img.reshape(int(npix[0]), int(npix[1])), st.as_dict()

    def iteration_omp(self, nH, xH, J, src_pos, src_lum, num_photon, seed, iteration,
                      alpha_H=4e-19, cross_section=6.3e-22, balance_form=1, threads=0):
        counts = Counts()
        sp = np.ascontiguousarray(src_pos, dtype=np.float64).reshape(-1)
        sl = np.ascontiguousarray(src_lum, dtype=np.float64)
        lib().cmio_iteration_omp(C.byref(self.lat), _ptr(self.box, C.c_double),
                                 _ptr(nH, C.c_double), _ptr(xH, C.c_double),
                                 _ptr(J, C.c_double), sl.size, _ptr(sp, C.c_double),
                                 _ptr(sl, C.c_double), int(num_photon), int(seed),
                                 int(iteration), alpha_H, cross_section, balance_form,
                                 threads, C.byref(counts))
        return counts.as_dict()


# --------------------------------------------------------------------------
# reference harness (the reference's own code, built by build_ref.sh)
# --------------------------------------------------------------------------
def ref_binary(name: str = "ref_harness_exact") -> str | None:
    p = os.path.join(REF_DIR, name)
    return p if os.path.exists(p) else None


def ref_run(args, binary: str = "ref_harness_exact", **kw):
    b = ref_binary(binary)
    if b is None:
        raise FileNotFoundError(f"{binary} not built (oracle/build_ref.sh)")
    return subprocess.run([b] + [str(a) for a in args], check=True, capture_output=True, **kw)


def ref_dust_walk(box, ncell, nH, xH, photons, in_dirs, depth=False):
    """Reference DensitySubGrid::propagate (depth=False) or compute_optical_depth
    on each photon, each on the same grid: (photons_out, results)."""
    with tempfile.TemporaryDirectory() as td:
        inp, out = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(inp, "wb") as f:
            f.write(np.asarray(box, "<f8").tobytes())
            f.write(np.asarray(ncell, "<i4").tobytes())
            f.write(np.zeros(1, "<i4").tobytes())
            f.write(np.asarray(nH, "<f8").tobytes())
            f.write(np.asarray(xH, "<f8").tobytes())
            f.write(np.asarray([photons.size], "<i8").tobytes())
            rec = np.zeros(photons.size, dtype=[("p", PHOTON_DTYPE), ("d", "<i4")])
            rec["p"] = photons
            rec["d"] = in_dirs
            f.write(rec.tobytes())
        ref_run(["depth" if depth else "propagate", inp, out])
        raw = open(out, "rb").read()
    rec_dt = np.dtype([("p", PHOTON_DTYPE), ("r", "<i4")])
    head = np.frombuffer(raw, dtype=rec_dt, count=photons.size)
    return head["p"].copy(), head["r"].copy()


def ref_walk(box, ncell, nH, xH, photons, in_dirs):
    """Reference DensitySubGrid::interact on each photon (in order).

    Returns (photons_out, results, J_total, per_packet[(cells, values)])."""
    C_ = int(np.prod(ncell))
    with tempfile.TemporaryDirectory() as td:
        inp, out = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(inp, "wb") as f:
            f.write(np.asarray(box, "<f8").tobytes())
            f.write(np.asarray(ncell, "<i4").tobytes())
            f.write(np.zeros(1, "<i4").tobytes())
            f.write(np.asarray(nH, "<f8").tobytes())
            f.write(np.asarray(xH, "<f8").tobytes())
            f.write(np.asarray([photons.size], "<i8").tobytes())
            rec = np.zeros(photons.size, dtype=[("p", PHOTON_DTYPE), ("d", "<i4")])
            rec["p"] = photons
            rec["d"] = in_dirs
            f.write(rec.tobytes())
        ref_run(["walk", inp, out])
        raw = open(out, "rb").read()
    n = photons.size
    rec_dt = np.dtype([("p", PHOTON_DTYPE), ("r", "<i4")])
    head = np.frombuffer(raw, dtype=rec_dt, count=n)
    off = rec_dt.itemsize * n
    J = np.frombuffer(raw, dtype="<f8", count=C_, offset=off).copy()
    off += 8 * C_
    per = []
    for _ in range(n):
        k = int(np.frombuffer(raw, "<i4", 1, off)[0])
        off += 4
        pair = np.frombuffer(raw, dtype=[("c", "<i4"), ("v", "<f8")], count=k, offset=off)
        off += 12 * k
        per.append((pair["c"].copy(), pair["v"].copy()))
    return head["p"].copy(), head["r"].copy(), J, per


def ref_rng(seed, n):
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "r.bin")
        ref_run(["rng", seed, n, out])
        return np.fromfile(out, dtype="<f8")


def ref_emit(seed, n, source):
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "e.bin")
        ref_run(["emit", seed, n, repr(float(source[0])), repr(float(source[1])),
                 repr(float(source[2])), out])
        return np.fromfile(out, dtype=PHOTON_DTYPE)


def ref_balance(box, ncell, nH, J, luminosity, num_photon):
    C_ = int(np.prod(ncell))
    with tempfile.TemporaryDirectory() as td:
        inp, out = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(inp, "wb") as f:
            f.write(np.asarray(box, "<f8").tobytes())
            f.write(np.asarray(ncell, "<i4").tobytes())
            f.write(np.zeros(1, "<i4").tobytes())
            f.write(np.asarray([luminosity], "<f8").tobytes())
            f.write(np.asarray([num_photon, 0], "<u4").tobytes())
            f.write(np.asarray(nH, "<f8").tobytes())
            f.write(np.asarray(J, "<f8").tobytes())
        ref_run(["balance", inp, out])
        raw = np.fromfile(out, dtype="<f8")
    return raw[:C_].copy(), raw[C_:].copy()


def ref_iterations(box, ncell, num_subgrid, nH_blocked, xH_blocked, src_pos, src_lum,
                   packets, iterations, threads=0, seed=42, count=False,
                   binary="ref_harness_fast", timeout=None, reemission=0.0):
    """Whole plain-method iterations with the reference code on the host cores
    (reemission: do_reemission's probability, testDensitySubGrid_omp.cpp:675-702).

    Returns (xH_final_blocked, per_iteration list of dicts)."""
    ncells = int(np.prod(ncell))
    with tempfile.TemporaryDirectory() as td:
        inp, out = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(inp, "wb") as f:
            f.write(np.asarray(box, "<f8").tobytes())
            f.write(np.asarray(ncell, "<i4").tobytes())
            f.write(np.asarray(num_subgrid, "<i4").tobytes())
            f.write(np.asarray([len(src_lum), 0], "<i4").tobytes())
            f.write(np.asarray(nH_blocked, "<f8").tobytes())
            f.write(np.asarray(xH_blocked, "<f8").tobytes())
            for p, L in zip(np.asarray(src_pos).reshape(-1, 3), src_lum):
                f.write(np.asarray(list(p) + [L], "<f8").tobytes())
        args = ["run", inp, out, int(packets), int(iterations), int(threads), int(seed),
                int(bool(count))]
        if reemission > 0.0:
            args.append(repr(float(reemission)))
        ref_run(args, binary=binary, timeout=timeout)
        raw = open(out, "rb").read()
    x = np.frombuffer(raw, "<f8", ncells).copy()
    it_dt = np.dtype([("t", "<f8"), ("cross", "<u8"), ("abs", "<u8"), ("esc", "<u8")])
    its = np.frombuffer(raw, it_dt, iterations, offset=8 * ncells)
    return x, [dict(seconds=float(r["t"]), crossings=int(r["cross"]), absorbed=int(r["abs"]),
                    escaped=int(r["esc"])) for r in its]


def ref_transport(box, ncell, num_subgrid, nH_blocked, xH_blocked, photons, start_subgrid):
    """Reference interact + neighbour routing over a lattice, packets in order.

    Returns (J_blocked, photons_final, fate (0 absorbed / 1 escaped), transits)."""
    cells = int(np.prod(ncell))
    n = photons.size
    with tempfile.TemporaryDirectory() as td:
        inp, out = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(inp, "wb") as f:
            f.write(np.asarray(box, "<f8").tobytes())
            f.write(np.asarray(ncell, "<i4").tobytes())
            f.write(np.asarray(num_subgrid, "<i4").tobytes())
            f.write(np.asarray([n], "<i8").tobytes())
            f.write(np.asarray(nH_blocked, "<f8").tobytes())
            f.write(np.asarray(xH_blocked, "<f8").tobytes())
            rec = np.zeros(n, dtype=[("p", PHOTON_DTYPE), ("s", "<u4"), ("pad", "<i4")])
            rec["p"] = photons
            rec["s"] = start_subgrid
            f.write(rec.tobytes())
        ref_run(["transport", inp, out])
        raw = open(out, "rb").read()
    J = np.frombuffer(raw, "<f8", cells).copy()
    tail = np.frombuffer(raw, [("p", PHOTON_DTYPE), ("fate", "<i4"), ("tr", "<i4")], n,
                         offset=8 * cells)
    return J, tail["p"].copy(), tail["fate"].copy(), tail["tr"].copy()

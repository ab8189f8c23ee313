"""ctypes binding of libcmacionize_b200.so (include/cmacionize_b200.h).

The library is built in-tree (``python -c "import __graft_entry__ as g; g.build()"``
or ``make -C parallelcmacionize_b200/csrc``).  Loading fails loudly when it is
missing: there is no CPU fallback for the transport.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcmacionize_b200.so")

OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_CUDA = 2
ERR_OUT_OF_MEMORY = 3
ERR_CAPACITY = 4
ERR_DEVICE_TIMEOUT = 5
ERR_INVARIANT = 6
ERR_NOT_SUPPORTED = 7

TRANSPORT_FP64 = 0
TRANSPORT_FP32 = 1
TRANSPORT_MIXED = 2
BALANCE_REFERENCE = 0
BALANCE_STABLE = 1
TALLY_FP32 = 0
TALLY_FP32_COMPENSATED = 1
TALLY_FIXED64 = 2
TALLY_FIXED64_ATOMIC64 = 3
RNG_PHILOX = 0
RNG_RANLUX = 1
LAYOUT_BLOCKED = 0
LAYOUT_CUBE = 1
MEMORY_HOST = 0
MEMORY_DEVICE = 1

NUM_DIRECTIONS = 27
NEIGHBOUR_OUTSIDE = 0xFFFFFFFF

# every symbol the header declares (checked by the CPU tests)
EXPORTED = [
    "cmi_default_options", "cmi_last_error_string", "cmi_abi_version", "cmi_create",
    "cmi_destroy", "cmi_set_fields", "cmi_get_fields", "cmi_set_intensity", "cmi_set_sources",
    "cmi_set_packet_budget", "cmi_set_reemission_probability", "cmi_run_iterations",
    "cmi_run_until_converged", "cmi_dust_run", "cmi_walk_photons",
    "cmi_prefetch_number_density", "cmi_set_fields_prefetched",
    "cmi_shoot_packets", "cmi_emit_photons",
    "cmi_transport_packets", "cmi_traverse_buffer", "cmi_trace_packet",
    "cmi_compute_neutral_fraction", "cmi_device_field", "cmi_get_stream", "cmi_synchronize",
    "cmi_last_launch_count", "cmi_set_kernel_timing", "cmi_kernel_timing",
    "cmi_compute_neutral_fraction_subgrids", "cmi_traverse_buffer_noalloc",
    # learned warm start
    "cmi_unet_default_config", "cmi_unet_last_error_string", "cmi_unet_create",
    "cmi_unet_destroy", "cmi_unet_num_params", "cmi_unet_get_params", "cmi_unet_set_params",
    "cmi_unet_forward", "cmi_unet_gradients", "cmi_unet_train_step", "cmi_unet_features",
    "cmi_unet_to_neutral_fraction", "cmi_unet_conv3", "cmi_unet_pack_weights",
    "cmi_unet_conv3_wgrad", "cmi_unet_block_mean", "cmi_unet_upsample_nearest",
    "cmi_unet_features_coarse_ratio", "cmi_unet_set_loss_weight",
]

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


class GridDesc(C.Structure):
    _fields_ = [
        ("box", C.c_double * 6),
        ("ncell", C.c_int32 * 3),
        ("num_subgrid", C.c_int32 * 3),
        ("recombination_rate", C.c_double),
        ("cross_section", C.c_double),
    ]


class Options(C.Structure):
    _fields_ = [
        ("transport_precision", C.c_int32),
        ("balance_form", C.c_int32),
        ("rng", C.c_int32),
        ("device", C.c_int32),
        ("threads_per_cta", C.c_int32),
        ("ctas_per_sm", C.c_int32),
        ("packets_per_chunk", C.c_int32),
        ("tally_mode", C.c_int32),
        ("use_graph", C.c_int32),
        ("max_run_chunks", C.c_int32),
        ("refill_lanes", C.c_int32),
        ("reserved", C.c_int32 * 5),
    ]


WALK_PROPAGATE, WALK_OPTICAL_DEPTH = 1, 2  # cmi_walk_photons modes


class Stats(C.Structure):
    _fields_ = [
        ("packets_emitted", C.c_uint64),
        ("packets_absorbed", C.c_uint64),
        ("packets_escaped", C.c_uint64),
        ("cell_crossings", C.c_uint64),
        ("subgrid_transits", C.c_uint64),
        ("mean_abs_dx", C.c_double),
        ("error_flags", C.c_uint32),
        ("rounds", C.c_uint32),
        ("packets_reemitted", C.c_uint64),
    ]

    def as_dict(self):
        return {k: (float(getattr(self, k)) if k == "mean_abs_dx" else int(getattr(self, k)))
                for k, _ in self._fields_}


class DustStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("emitted", "scatterings", "absorbed", "escaped",
                                          "cell_crossings", "subgrid_transits",
                                          "peeloffs_off_image")] + \
               [("generations", C.c_uint32), ("error_flags", C.c_uint32)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class UNetConfig(C.Structure):
    _fields_ = [
        ("channels", C.c_int32 * 3),
        ("leaky_slope", C.c_float),
        ("device", C.c_int32),
        ("reserved", C.c_int32 * 8),
    ]


class CMIError(RuntimeError):
    """A library call returned a non-zero status."""

    def __init__(self, code, message):
        super().__init__(f"[cmi status {code}] {message}")
        self.code = code


_lib = None


def load():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make -C parallelcmacionize_b200/csrc` "
            "(no CPU fallback exists for the transport)")
    L = C.CDLL(LIB_PATH)
    i32, u32, u64, d, vp = C.c_int32, C.c_uint32, C.c_uint64, C.c_double, C.c_void_p
    ctx = vp
    L.cmi_default_options.argtypes = [C.POINTER(Options)]
    L.cmi_default_options.restype = None
    L.cmi_last_error_string.restype = C.c_char_p
    L.cmi_abi_version.restype = C.c_int
    L.cmi_create.argtypes = [C.POINTER(GridDesc), i32, C.POINTER(Options), C.POINTER(vp)]
    L.cmi_destroy.argtypes = [ctx]
    L.cmi_set_fields.argtypes = [ctx, i32, i32, i32, vp, vp]
    L.cmi_get_fields.argtypes = [ctx, i32, i32, i32, vp, vp]
    L.cmi_set_intensity.argtypes = [ctx, i32, i32, i32, vp]
    L.cmi_set_sources.argtypes = [ctx, i32, vp, vp, i32]
    L.cmi_set_packet_budget.argtypes = [ctx, i32, u64]
    L.cmi_set_reemission_probability.argtypes = [ctx, i32, d]
    L.cmi_run_iterations.argtypes = [ctx, i32, u64, vp]
    L.cmi_run_until_converged.argtypes = [ctx, i32, i32, d, u64, vp, vp, vp]
    L.cmi_dust_run.argtypes = [ctx, i32, u64, u64, u32, d, vp, i32, i32, vp, vp]
    L.cmi_walk_photons.argtypes = [ctx, i32, u32, i32, vp, vp, u32, vp]
    L.cmi_prefetch_number_density.argtypes = [ctx, i32, i32, vp]
    L.cmi_set_fields_prefetched.argtypes = [ctx, i32, i32, vp]
    L.cmi_shoot_packets.argtypes = [ctx, u64, u32, vp]
    L.cmi_emit_photons.argtypes = [ctx, u64, u32, vp, u64, C.POINTER(u64)]
    L.cmi_transport_packets.argtypes = [ctx, i32, vp, vp, u64, vp]
    L.cmi_traverse_buffer.argtypes = [ctx, i32, u32, i32, vp, u32, vp, vp, vp, vp]
    L.cmi_trace_packet.argtypes = [ctx, i32, u32, i32, vp, i32, vp, vp, vp, vp]
    L.cmi_compute_neutral_fraction.argtypes = [ctx, i32, d, u64, vp]
    L.cmi_compute_neutral_fraction_subgrids.argtypes = [ctx, i32, u32, u32, d, u64, vp]
    L.cmi_device_field.argtypes = [ctx, i32, i32, C.POINTER(C.POINTER(C.c_double)),
                                   C.POINTER(u64)]
    L.cmi_get_stream.argtypes = [ctx, C.POINTER(vp)]
    L.cmi_synchronize.argtypes = [ctx]
    L.cmi_last_launch_count.argtypes = [ctx, C.POINTER(u64)]
    L.cmi_set_kernel_timing.argtypes = [ctx, i32]
    L.cmi_kernel_timing.argtypes = [ctx, vp, vp]
    f32, i64 = C.c_float, C.c_int64
    L.cmi_unet_default_config.argtypes = [C.POINTER(UNetConfig)]
    L.cmi_unet_default_config.restype = None
    L.cmi_unet_last_error_string.restype = C.c_char_p
    L.cmi_unet_create.argtypes = [C.POINTER(UNetConfig), C.POINTER(vp)]
    L.cmi_unet_destroy.argtypes = [vp]
    L.cmi_unet_num_params.argtypes = [vp, C.POINTER(i64)]
    L.cmi_unet_get_params.argtypes = [vp, vp]
    L.cmi_unet_set_params.argtypes = [vp, vp]
    L.cmi_unet_forward.argtypes = [vp, vp, vp, i32, vp]
    L.cmi_unet_gradients.argtypes = [vp, vp, vp, i32, vp, C.POINTER(f32), vp]
    L.cmi_unet_train_step.argtypes = [vp, vp, vp, i32, vp, f32, C.POINTER(f32)]
    L.cmi_unet_features.argtypes = [vp, vp, vp, vp, vp, i32, d, vp, vp]
    L.cmi_unet_to_neutral_fraction.argtypes = [vp, vp, vp, i64, f32]
    L.cmi_unet_conv3.argtypes = [vp, vp, i32, vp, vp, vp, i32, i32, i32, vp]
    L.cmi_unet_pack_weights.argtypes = [vp, vp, i32, i32, i32, vp]
    L.cmi_unet_conv3_wgrad.argtypes = [vp, vp, i32, vp, i32, i32, vp, vp]
    L.cmi_unet_block_mean.argtypes = [vp, vp, vp, i32, vp]
    L.cmi_unet_upsample_nearest.argtypes = [vp, vp, vp, i32, vp]
    L.cmi_unet_features_coarse_ratio.argtypes = [vp, vp, vp, vp, vp, i32, C.c_double, vp, i32,
                                                 vp]
    L.cmi_unet_set_loss_weight.argtypes = [vp, C.c_float]
    for name in EXPORTED:
        f = getattr(L, name)
        if f.restype is C.c_int and name not in ("cmi_abi_version",):
            f.restype = C.c_int
    _lib = L
    return L


def check(rc):
    if rc != OK:
        msg = load().cmi_last_error_string()
        raise CMIError(rc, msg.decode() if msg else "")
    return rc


def check_unet(rc):
    if rc != OK:
        msg = load().cmi_unet_last_error_string()
        raise CMIError(rc, msg.decode() if msg else "")
    return rc


def default_options(**kw) -> Options:
    o = Options()
    load().cmi_default_options(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k}")
        setattr(o, k, int(v))
    return o


def ptr(a):
    """Address of a C-contiguous numpy array (or None)."""
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data

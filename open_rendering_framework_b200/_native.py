"""ctypes binding of the C ABI in include/orf_b200.h (library: libpt_b200.so in this package).

This is the binding a Python caller of the reference-facing boundary uses; it is also what the
tests and the benchmark call.  There is no fallback: if the compiled library is missing the
import of any entry point raises ``NativeLibraryMissing``.
"""
import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpt_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(HERE), "include", "orf_b200.h")

P = ctypes.c_void_p
U32 = ctypes.c_uint32
U64 = ctypes.c_uint64
I32 = ctypes.c_int
F32 = ctypes.c_float
SZ = ctypes.c_size_t

STATUS_NAMES = {
    0: "PT_OK",
    1: "PT_INVALID_ARG",
    2: "PT_OOM",
    3: "PT_CUDA_ERROR",
    4: "PT_DEVICE_TIMEOUT",
    5: "PT_CAP_EXCEEDED",
    6: "PT_NOT_READY",
}


class NativeLibraryMissing(RuntimeError):
    pass


class PtError(RuntimeError):
    def __init__(self, status, where, message):
        self.status = status
        super().__init__("%s failed: %s (%s)" % (where, STATUS_NAMES.get(status, status), message))


# name -> (restype, argtypes).  Every function declared in include/orf_b200.h appears here; the
# CPU test suite checks both directions.
SIGNATURES = {
    "pt_last_error_message": (ctypes.c_char_p, []),
    "pt_version": (I32, []),
    "pt_kernel_launch_count": (U64, []),
    "pt_bsdf_queries": (I32, [P, P, U64, U64, U64, F32, P, P, P, P, P]),
    "pt_bsdf_queries_host": (I32, [P, P, U64, U64, U64, F32, P, P, P, P]),
    "pt_bsdf_queries_host_noalloc": (I32, [P, P, U64, U64, U64, F32, P, P, P, P]),
    "pt_c1_make_inputs": (I32, [U64, U64, P, P]),
    "pt_bssrdf_queries": (I32, [P, U32, P, U64, P, P]),
    "pt_microfacet_queries": (I32, [P, P, P, P, P, P, U64, P, P, P]),
    "pt_rng_streams": (I32, [I32, P, U64, U32, P, P]),
    "pt_context_create": (I32, [I32, P]),
    "pt_context_destroy": (I32, [P]),
    "pt_context_stream": (P, [P]),
    "pt_set_integrator": (I32, [P, U32, F32, P, U32]),
    "pt_set_camera": (I32, [P, P, P, P, P, U32, U32, P, P]),
    "pt_set_background_constant": (I32, [P, P]),
    "pt_set_envmap": (I32, [P, P, U32, U32]),
    "pt_set_envmap_hdr": (I32, [P, ctypes.c_char_p]),
    "pt_hdr_read": (I32, [ctypes.c_char_p, P, U64, P, P]),
    "pt_obj_read": (I32, [ctypes.c_char_p, P]),
    "pt_obj_get_info": (I32, [P, P]),
    "pt_obj_get_arrays": (I32, [P, P, P, P, P, P, P, P]),
    "pt_obj_get_group": (I32, [P, U32, P]),
    "pt_obj_free": (I32, [P]),
    "pt_set_accumulation": (I32, [P, P, U32]),
    "pt_get_envmap_tables": (I32, [P, P, P, P, P]),
    "pt_env_query": (I32, [P, P, U32, P, P, U32, P, P]),
    "pt_material_create": (I32, [P, U32, P, SZ, P]),
    "pt_material_update": (I32, [P, U32, P, SZ]),
    "pt_mesh_add": (I32, [P, P, U32, P, U32, P, U32, P, U32, P]),
    "pt_lights_upload": (I32, [P, P, U32, P, U32]),
    "pt_build": (I32, [P]),
    "pt_render_frames": (I32, [P, U32, U32]),
    "pt_readback": (I32, [P, P]),
    "pt_readback_device": (I32, [P, P]),
    "pt_sync": (I32, [P]),
    "pt_get_render_stats": (I32, [P, P]),
    "pt_set_max_paths_in_flight": (I32, [P, U64]),
    "pt_set_probe_count": (I32, [P, U32]),
    "pt_texture_create": (I32, [P, P, U32, U32, U32, P]),
    "pt_texture_bind": (I32, [P, U32, P]),
    "pt_texture_bind_grad": (I32, [P, U32, P]),
    "pt_material_set_texture": (I32, [P, U32, U32, P]),
    "pt_material_bind_sigma_grad": (I32, [P, U32, P]),
    "pt_render_adjoint": (I32, [P, U32, U32, P]),
    "pt_get_next_frame": (I32, [P, P]),
    "pt_batch_create": (I32, [ctypes.c_int, P]),
    "pt_batch_destroy": (I32, [P]),
    "pt_batch_stream": (P, [P]),
    "pt_batch_add": (I32, [P, P, U32]),
    "pt_batch_set_option": (I32, [P, ctypes.c_char_p, ctypes.c_int64]),
    "pt_batch_render": (I32, [P]),
    "pt_batch_render_sequential": (I32, [P]),
    "pt_batch_get_stats": (I32, [P, P]),
    "pt_batch_autotune": (I32, [P, U32, P]),
    "pt_get_probes": (I32, [P, P, U64, P]),
    "pt_get_scattering_properties": (I32, [P, U32, P]),
    "pt_set_profiling": (I32, [P, I32]),
    "pt_get_build_info": (I32, [P, P]),
    "pt_set_option": (I32, [P, ctypes.c_char_p, ctypes.c_int64]),
    "pt_trace_closest": (I32, [P, P, P, U32, P, P, P]),
    "pt_trace_any": (I32, [P, P, P, U32, P]),
}

_lib = None


def lib():
    """The loaded C-ABI library (raises NativeLibraryMissing if it was never built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise NativeLibraryMissing(
                "%s is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status, where):
    """Raise PtError unless status is PT_OK."""
    if status != 0:
        msg = lib().pt_last_error_message()
        raise PtError(status, where, msg.decode() if msg else "")
    return status


def call(name, *args):
    """Call an entry point by name and raise on a non-OK status."""
    return check(getattr(lib(), name)(*args), name)


def declared_functions():
    """Names of the functions declared in include/orf_b200.h."""
    text = open(HEADER_PATH).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pt_[a-z0-9_]+)\s*\(", text)))

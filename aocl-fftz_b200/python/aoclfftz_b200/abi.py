"""ctypes mirror of the aoclfftz.h C ABI.

The structures and prototypes are the same for this library and for the
reference library it replaces (AOCL-FFTZ 6.0.0, api/aoclfftz.h:60-507), so one
set of descriptors drives either shared object.
"""
import ctypes as C

AOCLFFTZ_SUCCESS = 0
AOCLFFTZ_EXECUTION_FAILURE = -1
AOCLFFTZ_SETUP_FAILURE = -2
AOCLFFTZ_INVALID_INPUT = -3
AOCLFFTZ_MEMORY_FAILURE = -4
AOCLFFTZ_TIME_OUT = -5


class Flags(C.Structure):
    """aoclfftz_flags_t (api/aoclfftz.h:86-102)."""
    _fields_ = [("fft_type", C.c_uint8), ("fft_direction", C.c_uint8), ("storage_order", C.c_uint8),
                ("fft_placement", C.c_uint8), ("transpose_mode", C.c_uint8), ("bit_reproducibility", C.c_uint8)]


class Dim(C.Structure):
    """aoclfftz_dim_t, LP64 (api/aoclfftz.h:108-113)."""
    _fields_ = [("n", C.c_int32), ("in_stride", C.c_int32), ("out_stride", C.c_int32)]


class Dim64(C.Structure):
    """aoclfftz_dim_t_64_, ILP64 (api/aoclfftz.h:119-124)."""
    _fields_ = [("n", C.c_ssize_t), ("in_stride", C.c_ssize_t), ("out_stride", C.c_ssize_t)]


class Smp(C.Structure):
    _fields_ = [("num_threads", C.c_int32), ("dynamic_load_model", C.c_uint32)]


class Cntrl(C.Structure):
    _fields_ = [("opt_level", C.c_int32), ("opt_off", C.c_int32), ("logger_mode", C.c_int),
                ("measure_stats", C.c_int32)]


def _desc(dimtype):
    class Desc(C.Structure):
        _fields_ = [("in_", C.c_void_p), ("out", C.c_void_p), ("vec_rank", C.c_int32), ("dim_rank", C.c_int32),
                    ("dims", C.POINTER(dimtype)), ("vecs", C.POINTER(dimtype)), ("flags", Flags),
                    ("pthr_fft", Smp), ("cntrl_params", Cntrl)]
    return Desc


DescLP64 = _desc(Dim)     # aoclfftz_prob_desc_f / _d
DescILP64 = _desc(Dim64)  # aoclfftz_prob_desc_f_64_ / _d_64_


class Hints(C.Structure):
    """aoclfftz_gpu_hints_t (include/aoclfftz_gpu.h)."""
    _fields_ = [("fourstep_n1", C.c_int64), ("tpc_col", C.c_int32), ("tpc_row", C.c_int32),
                ("batch_chunk", C.c_int64), ("algorithm", C.c_int32), ("kernel_family", C.c_int32),
                ("twiddles", C.c_int32), ("reserved", C.c_int32 * 5)]


def bind(lib):
    """Declares the aoclfftz.h prototypes on a loaded shared object."""
    for name, desc in (("aoclfftz_setup_f", DescLP64), ("aoclfftz_setup_d", DescLP64),
                       ("aoclfftz_setup_f_64_", DescILP64), ("aoclfftz_setup_d_64_", DescILP64)):
        fn = getattr(lib, name)
        fn.argtypes = [C.POINTER(desc)]
        fn.restype = C.c_void_p
    lib.aoclfftz_execute.argtypes = [C.c_void_p]
    lib.aoclfftz_execute.restype = C.c_int
    lib.aoclfftz_execute_io.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.aoclfftz_execute_io.restype = C.c_int
    lib.aoclfftz_destroy.argtypes = [C.c_void_p]
    lib.aoclfftz_destroy.restype = None
    lib.aoclfftz_version.argtypes = []
    lib.aoclfftz_version.restype = C.c_char_p
    return lib


def bind_gpu(lib):
    """Declares the aoclfftz_gpu.h extension prototypes."""
    bind(lib)
    lib.aoclfftz_gpu_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    lib.aoclfftz_gpu_set_stream.restype = C.c_int
    lib.aoclfftz_gpu_get_stream.argtypes = [C.c_void_p]
    lib.aoclfftz_gpu_get_stream.restype = C.c_void_p
    lib.aoclfftz_gpu_synchronize.argtypes = [C.c_void_p]
    lib.aoclfftz_gpu_synchronize.restype = C.c_int
    lib.aoclfftz_gpu_num_launches.argtypes = [C.c_void_p]
    lib.aoclfftz_gpu_num_launches.restype = C.c_int32
    lib.aoclfftz_gpu_describe.argtypes = [C.c_void_p, C.c_char_p, C.c_int32]
    lib.aoclfftz_gpu_describe.restype = C.c_int32
    lib.aoclfftz_gpu_device_bytes.argtypes = [C.c_void_p]
    lib.aoclfftz_gpu_device_bytes.restype = C.c_int64
    lib.aoclfftz_gpu_profile_begin.argtypes = [C.c_void_p, C.c_int32]
    lib.aoclfftz_gpu_profile_begin.restype = C.c_int
    lib.aoclfftz_gpu_profile_end.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.c_int32]
    lib.aoclfftz_gpu_profile_end.restype = C.c_int32
    lib.aoclfftz_gpu_pass_info.argtypes = [C.c_void_p, C.c_int32, C.c_char_p, C.c_int32, C.POINTER(C.c_int64),
                                           C.POINTER(C.c_int64)]
    lib.aoclfftz_gpu_pass_info.restype = C.c_int32
    lib.aoclfftz_gpu_set_hints.argtypes = [C.c_void_p]
    lib.aoclfftz_gpu_set_hints.restype = C.c_int
    lib.aoclfftz_gpu_ragged_setup.argtypes = [C.c_int32, C.c_int32, C.c_int64, C.POINTER(C.c_int64),
                                              C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.aoclfftz_gpu_ragged_setup.restype = C.c_void_p
    lib.aoclfftz_gpu_ragged_execute.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.aoclfftz_gpu_ragged_execute.restype = C.c_int
    fp = C.c_void_p
    lib.aoclfftz_gpu_mlp_nparams.argtypes = [C.c_int32]
    lib.aoclfftz_gpu_mlp_nparams.restype = C.c_int32
    lib.aoclfftz_gpu_mlp_forward.argtypes = [fp, C.c_int32, fp, C.c_int32, fp, fp, fp]
    lib.aoclfftz_gpu_mlp_forward.restype = C.c_int32
    lib.aoclfftz_gpu_mlp_grad.argtypes = [fp, C.c_int32, fp, fp, C.c_int32, fp, fp, fp, fp]
    lib.aoclfftz_gpu_mlp_grad.restype = C.c_int32
    lib.aoclfftz_gpu_mlp_adam.argtypes = [fp, fp, fp, fp, C.c_int32, C.c_float, C.c_int32, fp]
    lib.aoclfftz_gpu_mlp_adam.restype = C.c_int32
    lib.aoclfftz_gpu_last_error.argtypes = []
    lib.aoclfftz_gpu_last_error.restype = C.c_char_p
    lib.aoclfftz_gpu_inject_fault.argtypes = [C.c_int32, C.c_int64]
    lib.aoclfftz_gpu_inject_fault.restype = C.c_int32
    lib.aoclfftz_gpu_transpose.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p] + [C.c_int64] * 6 + \
        [C.c_void_p]
    lib.aoclfftz_gpu_transpose.restype = C.c_int
    return lib


# fault-injection kinds of aoclfftz_gpu_inject_fault (include/aoclfftz_gpu.h)
FAULT_NONE, FAULT_TMA_SHORT, FAULT_RAGGED_WAIT, FAULT_RAGGED_DEP, FAULT_ALLOC = 0, 1, 2, 3, 4


def make_desc(in_ptr, out_ptr, dims, vecs, fft_type=0, direction=0, placement=1, ilp64=False, logger_mode=0,
              opt_level=3, num_threads=1):
    """Builds a problem descriptor. dims/vecs are lists of (n, in_stride, out_stride),
    dims[0] innermost. Returns (desc, keepalive)."""
    dt = Dim64 if ilp64 else Dim
    D = DescILP64 if ilp64 else DescLP64
    darr = (dt * len(dims))(*[dt(*d) for d in dims])
    varr = (dt * len(vecs))(*[dt(*v) for v in vecs])
    d = D()
    d.in_ = in_ptr
    d.out = out_ptr
    d.vec_rank = len(vecs)
    d.dim_rank = len(dims)
    d.dims = C.cast(darr, C.POINTER(dt))
    d.vecs = C.cast(varr, C.POINTER(dt))
    d.flags = Flags(fft_type, direction, 0, placement, 0, 0)
    d.pthr_fft = Smp(num_threads, 1)
    d.cntrl_params = Cntrl(opt_level, 0, logger_mode, 0)
    return d, (darr, varr)


def setup(lib, desc, dtype, ilp64=False):
    """Calls the matching aoclfftz_setup_* entry point; returns the handle or None."""
    name = {("f32", False): "aoclfftz_setup_f", ("f64", False): "aoclfftz_setup_d",
            ("f32", True): "aoclfftz_setup_f_64_", ("f64", True): "aoclfftz_setup_d_64_"}[(dtype, ilp64)]
    h = getattr(lib, name)(C.byref(desc))
    return h

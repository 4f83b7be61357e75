"""Python mirror of the plfft.h C API over libplfft_b200.so (ctypes).

The names, argument meanings and status codes are those of PLFFT's public
interface (arm/perf-libs-fft include/plfft.h:212-532): create a config, set
its batch / type / alias, create a plan, execute, destroy.  Errors from the
create functions raise :class:`PlfftError` carrying the ``plfft_status_t``.

Execution takes raw pointers (``int``): device pointers (e.g.
``tensor.data_ptr()``) or host pointers (e.g. ``ndarray.ctypes.data``), the
same as the C call.  The library is required: importing this module on a
machine without ``lib/libplfft_b200.so`` raises, there is no fallback.
"""
import ctypes
import enum
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libplfft_b200.so")


class Status(enum.IntEnum):
    OK = 0
    NULL_ARGUMENT = 1
    INVALID_SIZE = 2
    UNSUPPORTED_BATCH = 3
    INVALID_TRANSFORM_KIND = 4
    INVALID_DATA_TYPE = 5
    INVALID_IO_ALIAS = 6
    PLAN_CREATION_FAILED = 7
    INVALID_SME_MODE = 8
    SME_NOT_ENABLED = 9
    SME_UNSUPPORTED_R2R = 10
    FP16_NOT_AVAILABLE = 11
    SME_NOT_AVAILABLE = 12
    SME_UNSUPPORTED_FIXED_POINT = 13
    INVALID_PLANNER_RIGOR = 14
    CUDA_ERROR = 100
    DEVICE_TIMEOUT = 101
    INVALID_ARGUMENT = 102


FORWARD = -1
BACKWARD = 1


class R2RKind(enum.IntEnum):
    DCT_1 = 0
    DCT_2 = 1
    DCT_3 = 2
    DCT_4 = 3
    DST_1 = 4
    DST_2 = 5
    DST_3 = 6
    DST_4 = 7
    DHT = 8
    R2HC = 9
    HC2R = 10


class DataType(enum.IntEnum):
    FP32 = 0
    FP64 = 1
    FP16 = 2
    Q7 = 3
    Q15 = 4


class IoAlias(enum.IntEnum):
    NO_ALIAS = 0
    MAY_ALIAS = 1


class SmeMode(enum.IntEnum):
    DISABLED = 0
    ENABLED = 1


class Rigor(enum.IntEnum):
    ESTIMATE = 0
    MEASURE = 1
    PATIENT = 2
    EXHAUSTIVE = 3


class Precision(enum.IntEnum):
    FP32 = 0
    SPLIT_BF16 = 1


class PlfftError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = Status(status) if status in Status._value2member_map_ else status
        super().__init__(f"{what}: {status_to_string(status)} ({int(status)})")


_lib = None

# (name, restype, argtypes)
_P = ctypes.c_void_p
_PP = ctypes.POINTER(ctypes.c_void_p)
_I64 = ctypes.c_int64
_INT = ctypes.c_int
_SIGS = [
    ("plfft_status_to_string", ctypes.c_char_p, [_INT]),
    ("plfft_config_create", _INT, [_PP, _I64, _INT]),
    ("plfft_config_create_r2c", _INT, [_PP, _I64]),
    ("plfft_config_create_c2r", _INT, [_PP, _I64]),
    ("plfft_config_create_r2r", _INT, [_PP, _I64, _INT]),
    ("plfft_config_destroy", None, [_P]),
    ("plfft_config_set_data_type", None, [_P, _INT]),
    ("plfft_config_get_data_type", _INT, [_P]),
    ("plfft_config_set_io_alias", None, [_P, _INT]),
    ("plfft_config_get_io_alias", _INT, [_P]),
    ("plfft_config_set_sme_mode", None, [_P, _INT]),
    ("plfft_config_get_sme_mode", _INT, [_P]),
    ("plfft_config_set_rigor", None, [_P, _INT]),
    ("plfft_config_get_rigor", _INT, [_P]),
    ("plfft_config_set_batch", None, [_P, _I64, _I64, _I64, _I64, _I64]),
    ("plfft_config_get_howmany", _I64, [_P]),
    ("plfft_config_get_istride", _I64, [_P]),
    ("plfft_config_get_idist", _I64, [_P]),
    ("plfft_config_get_ostride", _I64, [_P]),
    ("plfft_config_get_odist", _I64, [_P]),
    ("plfft_plan_create_from_config", _INT, [_PP, _P]),
    ("plfft_plan_destroy", None, [_P]),
    ("plfft_plan_execute", None, [_P, _P, _P]),
    ("plfft_cuda_config_set_scale", None, [_P, ctypes.c_double]),
    ("plfft_cuda_config_get_scale", ctypes.c_double, [_P]),
    ("plfft_cuda_config_set_precision", None, [_P, _INT]),
    ("plfft_cuda_config_get_precision", _INT, [_P]),
    ("plfft_cuda_get_last_status", _INT, []),
    ("plfft_cuda_plan_get_workspace_size", _INT, [_P, ctypes.POINTER(ctypes.c_size_t)]),
    ("plfft_cuda_plan_get_launch_count", _INT, [_P]),
    ("plfft_cuda_plan_describe", _INT, [_P, ctypes.c_char_p, ctypes.c_size_t]),
    ("plfft_cuda_execute_async", _INT, [_P, _P, _P, _P, _P]),
    ("plfft_cuda_plan_get_device_status", _INT, [_P, _P]),
    ("plfft_cuda_c2c_execute_noalloc", _INT, [_P, _P, _I64, _I64, _INT, _P]),
    ("plfft_cuda_execute_adjoint_async", _INT, [_P, _P, _P, _P, _P]),
    ("plfft_cuda_plan_get_adjoint_workspace_size", _INT, [_P, ctypes.POINTER(ctypes.c_size_t)]),
    ("plfft_cuda_group_create", _INT, [_PP, _I64, _P, _P, _P, _INT]),
    ("plfft_cuda_group_create_tuned", _INT, [_PP, _I64, _P, _P, _P, _INT, _INT]),
    ("plfft_cuda_group_execute_async", _INT, [_P, _P, _P, _P]),
    ("plfft_cuda_group_get_launch_count", _INT, [_P]),
    ("plfft_cuda_group_describe", _INT, [_P, ctypes.c_char_p, ctypes.c_size_t]),
    ("plfft_cuda_group_destroy", None, [_P]),
    ("plfft_cuda_wisdom_export", _INT, [ctypes.c_char_p]),
    ("plfft_cuda_wisdom_import", _INT, [ctypes.c_char_p]),
    ("plfft_cuda_wisdom_forget", None, []),
]

# symbols bound when the library exports them (added by later components)
_OPTIONAL_SIGS = []


def lib():
    """Load libplfft_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libplfft_b200.so not built: {LIB_PATH} (run make -C perf-libs-fft_b200)")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        for name, res, args in _OPTIONAL_SIGS:
            if hasattr(L, name):
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return [s[0] for s in _SIGS] + [s[0] for s in _OPTIONAL_SIGS]


def status_to_string(status):
    return lib().plfft_status_to_string(int(status)).decode()


def _check(status, what):
    if status != 0:
        raise PlfftError(status, what)


class Config:
    """plfft_config_t.  Use the classmethods to create one."""

    def __init__(self, handle):
        self.handle = handle

    @classmethod
    def c2c(cls, n, direction=FORWARD):
        h = ctypes.c_void_p()
        _check(lib().plfft_config_create(ctypes.byref(h), int(n), int(direction)), "plfft_config_create")
        return cls(h)

    @classmethod
    def r2c(cls, n):
        h = ctypes.c_void_p()
        _check(lib().plfft_config_create_r2c(ctypes.byref(h), int(n)), "plfft_config_create_r2c")
        return cls(h)

    @classmethod
    def c2r(cls, n):
        h = ctypes.c_void_p()
        _check(lib().plfft_config_create_c2r(ctypes.byref(h), int(n)), "plfft_config_create_c2r")
        return cls(h)

    @classmethod
    def r2r(cls, n, kind):
        h = ctypes.c_void_p()
        _check(lib().plfft_config_create_r2r(ctypes.byref(h), int(n), int(kind)), "plfft_config_create_r2r")
        return cls(h)

    def destroy(self):
        if self.handle is not None:
            lib().plfft_config_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def set_batch(self, howmany, istride, idist, ostride, odist):
        lib().plfft_config_set_batch(self.handle, howmany, istride, idist, ostride, odist)
        return self

    data_type = property(lambda s: DataType(lib().plfft_config_get_data_type(s.handle)),
                         lambda s, v: lib().plfft_config_set_data_type(s.handle, int(v)))
    io_alias = property(lambda s: lib().plfft_config_get_io_alias(s.handle),
                        lambda s, v: lib().plfft_config_set_io_alias(s.handle, int(v)))
    sme_mode = property(lambda s: lib().plfft_config_get_sme_mode(s.handle),
                        lambda s, v: lib().plfft_config_set_sme_mode(s.handle, int(v)))
    rigor = property(lambda s: lib().plfft_config_get_rigor(s.handle),
                     lambda s, v: lib().plfft_config_set_rigor(s.handle, int(v)))
    scale = property(lambda s: lib().plfft_cuda_config_get_scale(s.handle),
                     lambda s, v: lib().plfft_cuda_config_set_scale(s.handle, float(v)))
    precision = property(lambda s: lib().plfft_cuda_config_get_precision(s.handle),
                         lambda s, v: lib().plfft_cuda_config_set_precision(s.handle, int(v)))
    howmany = property(lambda s: lib().plfft_config_get_howmany(s.handle))
    istride = property(lambda s: lib().plfft_config_get_istride(s.handle))
    idist = property(lambda s: lib().plfft_config_get_idist(s.handle))
    ostride = property(lambda s: lib().plfft_config_get_ostride(s.handle))
    odist = property(lambda s: lib().plfft_config_get_odist(s.handle))


class Plan:
    """plfft_plan_t created from a Config (plfft_plan_create_from_config)."""

    def __init__(self, config):
        h = ctypes.c_void_p()
        st = lib().plfft_plan_create_from_config(ctypes.byref(h), config.handle if config else None)
        _check(st, "plfft_plan_create_from_config")
        self.handle = h

    def destroy(self):
        if self.handle is not None:
            lib().plfft_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def execute(self, inp, out):
        """plfft_plan_execute on raw (host or device) pointers; synchronous."""
        lib().plfft_plan_execute(self.handle, ctypes.c_void_p(int(inp)), ctypes.c_void_p(int(out)))
        st = lib().plfft_cuda_get_last_status()
        _check(st, "plfft_plan_execute")

    def execute_async(self, inp, out, workspace=0, stream=0):
        st = lib().plfft_cuda_execute_async(self.handle, ctypes.c_void_p(int(inp)), ctypes.c_void_p(int(out)),
                                            ctypes.c_void_p(int(workspace)) if workspace else None,
                                            ctypes.c_void_p(int(stream)) if stream else None)
        _check(st, "plfft_cuda_execute_async")

    def device_status(self, stream=0):
        """plfft_cuda_plan_get_device_status: drains `stream`, returns (and
        clears) the Status of device-side failures of earlier executions."""
        return Status(lib().plfft_cuda_plan_get_device_status(self.handle,
                                                              ctypes.c_void_p(int(stream)) if stream else None))

    def execute_adjoint(self, inp, out, workspace=0, stream=0):
        """Adjoint of this plan's transform (input = plan's output layout)."""
        st = lib().plfft_cuda_execute_adjoint_async(self.handle, ctypes.c_void_p(int(inp)),
                                                    ctypes.c_void_p(int(out)),
                                                    ctypes.c_void_p(int(workspace)) if workspace else None,
                                                    ctypes.c_void_p(int(stream)) if stream else None)
        _check(st, "plfft_cuda_execute_adjoint_async")

    def workspace_size(self):
        v = ctypes.c_size_t()
        _check(lib().plfft_cuda_plan_get_workspace_size(self.handle, ctypes.byref(v)), "workspace")
        return v.value

    def launch_count(self):
        return lib().plfft_cuda_plan_get_launch_count(self.handle)

    def describe(self):
        buf = ctypes.create_string_buffer(4096)
        _check(lib().plfft_cuda_plan_describe(self.handle, buf, 4096), "describe")
        return buf.value.decode()


def c2c_execute_noalloc(d_in, d_out, n, howmany, direction=FORWARD, stream=0):
    """plfft_cuda_c2c_execute_noalloc: four-step C2C with no device allocation
    (device pointers, contiguous batch).  Returns the plfft_status_t."""
    return Status(lib().plfft_cuda_c2c_execute_noalloc(
        ctypes.c_void_p(int(d_in)), ctypes.c_void_p(int(d_out)), int(n), int(howmany), int(direction),
        ctypes.c_void_p(int(stream)) if stream else None))


class Group:
    """plfft_cuda_group_t: many C2C transforms of different lengths in one grouped execution."""

    def __init__(self, lengths, in_offsets, out_offsets, direction=FORWARD, rigor=None):
        import numpy as np

        self._len = np.ascontiguousarray(lengths, dtype=np.int64)
        self._io = np.ascontiguousarray(in_offsets, dtype=np.int64)
        self._oo = np.ascontiguousarray(out_offsets, dtype=np.int64)
        h = ctypes.c_void_p()
        if rigor is None:
            st = lib().plfft_cuda_group_create(ctypes.byref(h), len(self._len), self._len.ctypes.data,
                                               self._io.ctypes.data, self._oo.ctypes.data, int(direction))
            _check(st, "plfft_cuda_group_create")
        else:
            st = lib().plfft_cuda_group_create_tuned(ctypes.byref(h), len(self._len), self._len.ctypes.data,
                                                     self._io.ctypes.data, self._oo.ctypes.data, int(direction),
                                                     int(rigor))
            _check(st, "plfft_cuda_group_create_tuned")
        self.handle = h

    def execute_async(self, d_in, d_out, stream=0):
        st = lib().plfft_cuda_group_execute_async(self.handle, ctypes.c_void_p(int(d_in)),
                                                  ctypes.c_void_p(int(d_out)),
                                                  ctypes.c_void_p(int(stream)) if stream else None)
        _check(st, "plfft_cuda_group_execute_async")

    def launch_count(self):
        return lib().plfft_cuda_group_get_launch_count(self.handle)

    def describe(self):
        buf = ctypes.create_string_buffer(4096)
        _check(lib().plfft_cuda_group_describe(self.handle, buf, 4096), "group describe")
        return buf.value.decode()

    def destroy(self):
        if self.handle is not None:
            lib().plfft_cuda_group_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def make_plan(kind, n, howmany=1, istride=1, idist=None, ostride=1, odist=None, direction=FORWARD,
              r2r_kind=None, data_type=DataType.FP32, alias=IoAlias.NO_ALIAS, scale=1.0,
              precision=Precision.FP32, rigor=Rigor.ESTIMATE):
    """Create config -> set options -> plan -> destroy config (the reference's usage order)."""
    if kind == "c2c":
        cfg = Config.c2c(n, direction)
    elif kind == "r2c":
        cfg = Config.r2c(n)
    elif kind == "c2r":
        cfg = Config.c2r(n)
    elif kind == "r2r":
        cfg = Config.r2r(n, r2r_kind)
    else:
        raise ValueError(kind)
    nin = n // 2 + 1 if kind == "c2r" else n
    nout = n // 2 + 1 if kind == "r2c" else n
    cfg.set_batch(howmany, istride, idist if idist is not None else nin, ostride,
                  odist if odist is not None else nout)
    cfg.data_type = data_type
    cfg.io_alias = alias
    cfg.scale = scale
    cfg.precision = precision
    cfg.rigor = rigor
    try:
        return Plan(cfg)
    finally:
        cfg.destroy()


# ---------------------------------------------------------------------------
# wisdom of the MEASURE / PATIENT / EXHAUSTIVE planners
# ---------------------------------------------------------------------------
def wisdom_export(path):
    _check(lib().plfft_cuda_wisdom_export(os.fsencode(path)), "wisdom_export")


def wisdom_import(path):
    _check(lib().plfft_cuda_wisdom_import(os.fsencode(path)), "wisdom_import")


def wisdom_forget():
    lib().plfft_cuda_wisdom_forget()


# ---------------------------------------------------------------------------
# multi-GPU: contiguous batch shards, no collective on the data path
# ---------------------------------------------------------------------------
def shard_range(howmany, world, rank):
    """First member and member count of `rank`'s contiguous share of a batch.

    Members of a batch are independent, so a batch spread over `world`
    processes (one per GPU) needs no exchange: rank r transforms members
    [first, first + count) with a plan of howmany = count whose input and
    output pointers are offset by first * idist and first * odist.
    """
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    first = howmany * rank // world
    return first, howmany * (rank + 1) // world - first

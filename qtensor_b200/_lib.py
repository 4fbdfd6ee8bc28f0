"""ctypes binding of ``libqtb.so`` (declared in ``include/qtb.h``).

Loading fails loudly when the library is missing: the product has no CPU
fallback.  Every non-zero status becomes a ``QtbError`` carrying the
library's last error message.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, 'libqtb.so')

QTB_OK, QTB_ERR_ARG, QTB_ERR_CUDA, QTB_ERR_UNSUPPORTED, QTB_ERR_DEVICE = range(5)
QTB_MAX_BUCKET_INPUTS = 16
QTB_MAX_BUCKET_VARS = 31

GATE_M, GATE_H, GATE_Z, GATE_X, GATE_Y, GATE_CX, GATE_CZ = range(7)
GATE_ZPHASE, GATE_XPHASE, GATE_YPHASE, GATE_ZZ, GATE_T = range(7, 12)

COMPOSER_DEFAULT, COMPOSER_ZZ, COMPOSER_CX = 0, 1, 2
SLICE_GREEDY, SLICE_TREE_TRIM, SLICE_LATE = 0, 1, 2

# Exported entry points, in the order of include/qtb.h.
EXPORTS = (
    'qtb_version', 'qtb_init', 'qtb_last_error', 'qtb_bucket_c64',
    'qtb_contract_outer_c64', 'qtb_contract_sum_scratch_bytes', 'qtb_contract_sum_c64',
    'qtb_plan_create', 'qtb_plan_destroy', 'qtb_plan_add_circuit',
    'qtb_plan_add_lightcone', 'qtb_plan_add_lightcones', 'qtb_plan_add_circuit_batch',
    'qtb_plan_set_max_width', 'qtb_plan_set_slicing',
    'qtb_plan_set_order_trials', 'qtb_plan_set_share_lightcones', 'qtb_plan_set_records',
    'qtb_plan_n_networks',
    'qtb_plan_network_info', 'qtb_plan_network_peo', 'qtb_plan_check_params',
    'qtb_plan_export', 'qtb_plan_table_elems', 'qtb_plan_upload',
    'qtb_plan_scratch_bytes', 'qtb_plan_run', 'qtb_plan_plain_scratch_bytes',
    'qtb_plan_run_plain', 'qtb_plan_set_autotune', 'qtb_plan_set_wave_ctas_per_sm',
    'qtb_plan_set_dynamic_claims',
    'qtb_plan_last_launch_config', 'qtb_plan_device_bytes', 'qtb_plan_device_status',
    'qtb_selftest_wait_timeout', 'qtb_host_device_pointer', 'qtb_copy_c',
    'qtb_plan_set_timing', 'qtb_plan_collect_timing', 'qtb_plan_run_noalloc',
)
NOALLOC_SCRATCH_BYTES = 64 << 20


class QtbError(RuntimeError):
    """A libqtb call returned a non-zero status."""

    def __init__(self, code, message):
        super().__init__('libqtb error {}: {}'.format(code, message))
        self.code = code


class BucketDesc(ctypes.Structure):
    _fields_ = [('n_inputs', ctypes.c_int32), ('n_vars', ctypes.c_int32),
                ('sum_first', ctypes.c_int32),
                ('masks', ctypes.c_uint32 * QTB_MAX_BUCKET_INPUTS)]


class Gate(ctypes.Structure):
    _fields_ = [('kind', ctypes.c_int32), ('q0', ctypes.c_int32), ('q1', ctypes.c_int32),
                ('param', ctypes.c_int32), ('coef', ctypes.c_double)]


GATE_DTYPE = np.dtype([('kind', '<i4'), ('q0', '<i4'), ('q1', '<i4'), ('param', '<i4'),
                       ('coef', '<f8')])


class NetworkInfo(ctypes.Structure):
    _fields_ = [('n_qubits', ctypes.c_int32), ('n_vars', ctypes.c_int32),
                ('treewidth', ctypes.c_int32), ('max_rank', ctypes.c_int32),
                ('n_ops', ctypes.c_int32), ('n_phases', ctypes.c_int32),
                ('arena_elems', ctypes.c_int32), ('angle_specific', ctypes.c_int32),
                ('alg_bytes', ctypes.c_double), ('alg_flops', ctypes.c_double),
                ('ref_flops', ctypes.c_double), ('n_slices', ctypes.c_int32),
                ('group', ctypes.c_int32)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


# numpy views of the exported plan arrays (plan.h)
NET_DTYPE = np.dtype([('op_begin', '<u4'), ('n_ops', '<u4'), ('phase_begin', '<u4'),
                      ('n_phases', '<u4'), ('arena_elems', '<u4'), ('result_src', '<u4'),
                      ('max_elems', '<u4'), ('pad', '<u4')])
OP_DTYPE = np.dtype([('u', 'u1'), ('sum', 'u1'), ('k', 'u1'), ('pad', 'u1'), ('dst', '<u4'),
                     ('elem_begin', '<u4'), ('in_begin', '<u4')])
IN_DTYPE = np.dtype([('mask', '<u4'), ('src', '<u4'), ('runs', '<u8')])
PHASE_DTYPE = np.dtype([('op_first', '<u4'), ('op_count', '<u4'), ('total_elems', '<u4'),
                        ('chunk_off', '<u4')])
ENTRY_DTYPE = np.dtype([('kind', '<i4'), ('expr_begin', '<i4'), ('expr_count', '<i4'),
                        ('off', '<u4'), ('rank_in', 'i1'), ('rank_out', 'i1'),
                        ('sliced_mask', 'u1'), ('perm', 'i1', (4,)), ('sliced_value', 'u1')])
TERM_DTYPE = np.dtype([('param', '<i4'), ('pad', '<i4'), ('coef', '<f8')])
RUN_DTYPE = np.dtype([('blob_off16', '<u4'), ('blob_bytes', '<u4'), ('n_phases', '<u4'),
                      ('ins_off', '<u4'), ('arena_elems', '<u4'), ('result_src', '<u4'),
                      ('max_elems', '<u4'), ('tail_start', '<u4'), ('rec_off', '<u4'),
                      ('rec_words', '<u4'), ('rec_format', '<u4'), ('pad1', '<u4')])
REC_WIDE = 1
REC_COMPACT = 2
SRC_TABLE = 0x80000000
STATUS_WAIT_TIMEOUT = 16

_lib = None


def _declare(lib):
    c = ctypes
    P = c.c_void_p
    sig = {
        'qtb_version': (c.c_char_p, []),
        'qtb_init': (c.c_int, [c.c_int]),
        'qtb_last_error': (c.c_int, [c.c_char_p, c.c_size_t]),
        'qtb_bucket_c64': (c.c_int, [c.POINTER(BucketDesc), c.POINTER(P), P, P]),
        'qtb_contract_outer_c64': (c.c_int, [P, P, P, c.c_int64, c.c_int64, c.c_int64, P]),
        'qtb_contract_sum_scratch_bytes': (c.c_int, [c.c_int64, c.c_int64, c.c_int64, c.c_int64, c.c_int32,
                                                     c.POINTER(c.c_size_t)]),
        'qtb_contract_sum_c64': (c.c_int, [P, P, P, c.c_int64, c.c_int64, c.c_int64, c.c_int64, c.c_int32,
                                           P, c.c_size_t, P]),
        'qtb_plan_create': (c.c_int, [c.c_int32, c.POINTER(P)]),
        'qtb_plan_destroy': (c.c_int, [P]),
        'qtb_plan_add_circuit': (c.c_int, [P, c.c_int32, P, c.c_int32, c.c_int32, P,
                                           c.POINTER(c.c_int32)]),
        'qtb_plan_add_circuit_batch': (c.c_int, [P, c.c_int32, P, c.c_int32, c.c_int32, P, c.c_int32,
                                                 c.POINTER(c.c_int32), c.POINTER(c.c_int32)]),
        'qtb_plan_add_lightcone': (c.c_int, [P, c.c_int32, P, P, c.c_int32, c.c_int32,
                                             c.c_int32, c.c_int32, P, c.POINTER(c.c_int32)]),
        'qtb_plan_add_lightcones': (c.c_int, [P, c.c_int32, P, P, P, c.c_int32, c.c_int32,
                                              c.c_int32, P, c.c_int32, c.POINTER(c.c_int32)]),
        'qtb_plan_set_max_width': (c.c_int, [P, c.c_int32, c.c_int32]),
        'qtb_plan_set_slicing': (c.c_int, [P, c.c_int32]),
        'qtb_plan_set_order_trials': (c.c_int, [P, c.c_int32]),
        'qtb_plan_set_share_lightcones': (c.c_int, [P, c.c_int32]),
        'qtb_plan_set_records': (c.c_int, [P, c.c_int32]),
        'qtb_plan_n_networks': (c.c_int, [P, c.POINTER(c.c_int32)]),
        'qtb_plan_network_info': (c.c_int, [P, c.c_int32, c.POINTER(NetworkInfo)]),
        'qtb_plan_network_peo': (c.c_int, [P, c.c_int32, P, c.c_int32, c.POINTER(c.c_int32)]),
        'qtb_plan_check_params': (c.c_int, [P, P, c.POINTER(c.c_int32)]),
        'qtb_plan_export': (c.c_int, [P, c.c_int32, P, c.c_size_t, c.POINTER(c.c_size_t)]),
        'qtb_plan_table_elems': (c.c_int, [P, c.POINTER(c.c_int64)]),
        'qtb_plan_upload': (c.c_int, [P]),
        'qtb_plan_scratch_bytes': (c.c_int, [P, c.c_int32, c.c_int32, c.POINTER(c.c_size_t)]),
        'qtb_plan_run': (c.c_int, [P, c.c_int32, c.c_int32, P, P, P, P, P]),
        'qtb_plan_set_autotune': (c.c_int, [P, c.c_int32]),
        'qtb_plan_set_wave_ctas_per_sm': (c.c_int, [P, c.c_int32]),
        'qtb_plan_set_dynamic_claims': (c.c_int, [P, c.c_int32]),
        'qtb_plan_last_launch_config': (c.c_int, [P, P, c.c_int32, c.POINTER(c.c_int32)]),
        'qtb_plan_device_bytes': (c.c_int, [P, c.POINTER(c.c_size_t)]),
        'qtb_plan_device_status': (c.c_int, [P, c.POINTER(c.c_int32)]),
        'qtb_selftest_wait_timeout': (c.c_int, [c.c_int32, c.POINTER(c.c_int32)]),
        'qtb_host_device_pointer': (c.c_int, [c.c_void_p, c.POINTER(c.c_void_p)]),
        'qtb_copy_c': (c.c_int, [c.c_void_p, c.c_void_p, c.c_size_t, c.c_void_p]),
        'qtb_plan_set_timing': (c.c_int, [P, c.c_int32]),
        'qtb_plan_collect_timing': (c.c_int, [P, c.POINTER(c.c_double), c.POINTER(c.c_int64)]),
        'qtb_plan_run_noalloc': (c.c_int, [P, c.c_int32, c.c_int32, P, P, P, P]),
        'qtb_plan_plain_scratch_bytes': (c.c_int, [P, c.c_int32, c.c_int32, c.POINTER(c.c_size_t)]),
        'qtb_plan_run_plain': (c.c_int, [P, c.c_int32, c.c_int32, P, P, P, P, c.c_size_t, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def lib():
    """The loaded library (raises if ``libqtb.so`` has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError('libqtb.so is missing; build it with `python -m qtensor_b200.build`')
        handle = ctypes.CDLL(LIB_PATH)
        _declare(handle)
        _lib = handle
    return _lib


def available_cpus():
    """CPUs this process may run on: its affinity mask, bounded by a cgroup
    CPU quota (cgroup v2 ``cpu.max`` or v1 ``cpu.cfs_quota_us``); in a
    container ``os.cpu_count()`` reports the host's."""
    try:
        n = len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        n = os.cpu_count() or 1
    quota = None
    try:
        with open('/sys/fs/cgroup/cpu.max') as f:
            q, period = f.read().split()[:2]
            if q != 'max':
                quota = float(q) / float(period)
    except (OSError, ValueError):
        try:
            with open('/sys/fs/cgroup/cpu/cpu.cfs_quota_us') as f:
                q = float(f.read())
            with open('/sys/fs/cgroup/cpu/cpu.cfs_period_us') as f:
                period = float(f.read())
            if q > 0 and period > 0:
                quota = q / period
        except (OSError, ValueError):
            pass
    if quota:
        n = min(n, max(1, int(-(-quota // 1))))
    return max(1, n)


def last_error():
    buf = ctypes.create_string_buffer(1024)
    lib().qtb_last_error(buf, len(buf))
    return buf.value.decode(errors='replace')


def check(code):
    if code != 0:
        raise QtbError(code, last_error())
    return code


def ptr(x):
    """Raw address of a torch tensor, numpy array or integer (None -> NULL)."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, 'data_ptr'):
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    raise TypeError('cannot take the address of {!r}'.format(type(x)))

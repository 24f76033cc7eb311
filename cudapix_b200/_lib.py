"""Loader for the CUDA library (cudapix_b200/lib/libcudapix_b200.so).

The library is built in-tree by `make -C cudapix_b200` (nvcc, sm_100a).  There
is no CPU fallback: if the shared object is missing, importing the compute
API raises ExtensionMissing.
"""
import ctypes
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libcudapix_b200.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "cpx.h")


class ExtensionMissing(RuntimeError):
    pass


class CpxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cpx error {code}: {msg}")
        self.code = code


CPX_OK, CPX_EINVAL, CPX_EOOM, CPX_ECUDA, CPX_ETIMEOUT, CPX_ERANGE, CPX_ESTATE = range(7)


class U128(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_uint64), ("hi", ctypes.c_uint64)]

    @classmethod
    def of(cls, v):
        v = int(v)
        if v < 0:
            v &= (1 << 128) - 1
        return cls(v & 0xFFFFFFFFFFFFFFFF, v >> 64)

    def value(self, signed=False):
        v = (self.hi << 64) | self.lo
        if signed and v >> 127:
            v -= 1 << 128
        return v


class Terms(ctypes.Structure):
    _fields_ = [
        ("P2", U128),
        ("ordinary", U128),
        ("trivial", U128),
        ("easy", U128),
        ("hard", U128),
        ("pi_y", U128),
        ("pi", U128),
        ("x_lo", ctypes.c_uint64),
        ("x_hi", ctypes.c_uint64),
        ("y", ctypes.c_uint64),
        ("z", ctypes.c_uint64),
        ("c", ctypes.c_uint32),
        ("pad", ctypes.c_uint32),
    ]

    def as_dict(self):
        d = {k: getattr(self, k).value(signed=True) for k in ("P2", "ordinary", "trivial", "easy", "hard", "pi_y", "pi")}
        d.update(x=(self.x_hi << 64) | self.x_lo, y=self.y, z=self.z, c=self.c)
        return d


class GourdonTerms(ctypes.Structure):
    _fields_ = [(k, U128) for k in ("A", "B", "C", "D", "phi0", "sigma", "pi")] + [
        ("x", ctypes.c_uint64), ("y", ctypes.c_uint64)]

    def as_dict(self):
        d = {k: getattr(self, k).value(signed=True) for k in ("A", "B", "C", "D", "phi0", "sigma", "pi")}
        d.update(x=self.x, y=self.y)
        return d


class BatchStats(ctypes.Structure):
    _fields_ = [
        ("roots_ms", ctypes.c_double),
        ("tables_ms", ctypes.c_double),
        ("plan_ms", ctypes.c_double),
        ("launch_ms", ctypes.c_double),
        ("wait_ms", ctypes.c_double),
        ("queries", ctypes.c_uint64),
        ("segments", ctypes.c_uint64),
        ("hard_jobs", ctypes.c_uint64),
        ("offload_min", ctypes.c_uint64),
        ("shared_groups", ctypes.c_uint64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class LeafCounts(ctypes.Structure):
    _fields_ = [("hard", ctypes.c_uint64), ("easy_composite", ctypes.c_uint64),
                ("easy_prime", ctypes.c_uint64), ("trivial", ctypes.c_uint64)]


class TuneEntry(ctypes.Structure):
    _fields_ = [("decade", ctypes.c_uint32), ("alpha_scale_milli", ctypes.c_uint32), ("log2_bits", ctypes.c_uint32),
                ("threads", ctypes.c_uint32), ("offload_min", ctypes.c_uint32), ("ms", ctypes.c_float)]


class HardLevel(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint64), ("msum", ctypes.c_int64), ("carry0", ctypes.c_uint64),
                ("anchored", ctypes.c_uint32), ("pad", ctypes.c_uint32)]


class Params(ctypes.Structure):
    _fields_ = [
        ("alpha_num", ctypes.c_uint32),
        ("alpha_den", ctypes.c_uint32),
        ("c", ctypes.c_uint16),
        ("flags", ctypes.c_uint16),
        ("hard_log2_bits", ctypes.c_uint32),
        ("hard_threads", ctypes.c_uint32),
    ]


class ServeConfig(ctypes.Structure):
    _fields_ = [
        ("lanes", ctypes.c_uint32),
        ("max_batch", ctypes.c_uint32),
        ("admit_fraction", ctypes.c_double),
        ("reserve_x", U128),
        ("params", Params),
        ("fill_target", ctypes.c_uint32),
        ("window_us", ctypes.c_uint32),
    ]


class ServeCounters(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_uint64),
        ("completed", ctypes.c_uint64),
        ("failed", ctypes.c_uint64),
        ("pending", ctypes.c_uint64),
        ("batches", ctypes.c_uint64),
        ("max_batch_seen", ctypes.c_uint64),
        ("table_growths", ctypes.c_uint64),
        ("busy_ms", ctypes.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


P = ctypes.c_void_p
PP = ctypes.POINTER(ctypes.c_void_p)
u16, u32, u64, i32, i64 = ctypes.c_uint16, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_int64
pu64, pi64, pu32 = ctypes.POINTER(u64), ctypes.POINTER(i64), ctypes.POINTER(u32)
pU = ctypes.POINTER(U128)

_SIGS = {
    "cpx_create": (ctypes.c_int, [ctypes.c_int, PP]),
    "cpx_destroy": (ctypes.c_int, [P]),
    "cpx_last_error": (ctypes.c_char_p, [P]),
    "cpx_version": (ctypes.c_char_p, []),
    "cpx_stream": (P, [P]),
    "cpx_launch_count": (u64, [P]),
    "cpx_sm_count": (ctypes.c_int, [P]),
    "cpx_free": (ctypes.c_int, [P]),
    "cpx_device_alloc": (ctypes.c_int, [ctypes.c_size_t, PP]),
    "cpx_copy_to_host": (ctypes.c_int, [P, P, ctypes.c_size_t]),
    "cpx_copy_to_device": (ctypes.c_int, [P, P, ctypes.c_size_t]),
    "cpx_device_count": (ctypes.c_int, []),
    "cpx_set_hard_params": (ctypes.c_int, [P, u32, u32]),
    "cpx_set_hard_offload": (ctypes.c_int, [P, u32]),
    "cpx_set_hard_shared": (ctypes.c_int, [P, u32]),
    "cpx_set_p2_window": (ctypes.c_int, [P, u64]),
    "cpx_S2_hard_layout": (ctypes.c_int, [P, U128, u64, u16, u32, pu64, pu32]),
    "cpx_S2_hard_part": (ctypes.c_int, [P, U128, u64, u16, u32, u64, u64, pU, ctypes.POINTER(HardLevel)]),
    "cpx_S2_hard_merge": (ctypes.c_int, [pU, ctypes.POINTER(HardLevel), u32, u32, pU]),
    "cpx_autotune": (ctypes.c_int, [P, u32, u32, ctypes.c_double]),
    "cpx_autotune_batch": (ctypes.c_int, [P, pU, ctypes.c_size_t]),
    "cpx_tune_save": (ctypes.c_int, [P, ctypes.c_char_p]),
    "cpx_tune_load": (ctypes.c_int, [P, ctypes.c_char_p]),
    "cpx_tune_get": (ctypes.c_int, [P, u32, ctypes.POINTER(TuneEntry)]),
    "cpx_tune_clear": (ctypes.c_int, [P]),
    "cpx_leaf_count": (ctypes.c_int, [P, U128, u64, u16, ctypes.POINTER(LeafCounts)]),
    "cpx_last_hard_stats": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)]),
    "cpx_last_kernel_span": (ctypes.c_int, [P, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                                            ctypes.POINTER(ctypes.c_float)]),
    "cpx_set_timing": (ctypes.c_int, [P, ctypes.c_int]),
    "cpx_last_batch_ms": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_float)]),
    "cpx_timer_start": (ctypes.c_int, [P]),
    "cpx_timer_stop": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_float)]),
    "cpx_flush_l2": (ctypes.c_int, [P]),
    "cpx_last_batch_io": (ctypes.c_int, [P, pu64, pu64]),
    "cpx_last_batch_stats": (ctypes.c_int, [P, ctypes.POINTER(BatchStats)]),
    "cpx_iroots": (ctypes.c_int, [U128, pu64, pu64, pu64]),
    "cpx_default_y": (ctypes.c_int, [U128, u32, u32, pu64]),
    "cpx_alpha_milli": (u32, [U128]),
    "cpx_P2_u64": (ctypes.c_int, [P, u64, u64, pu64]),
    "cpx_P2_u128": (ctypes.c_int, [P, U128, u64, pU]),
    "cpx_trivial_u64": (ctypes.c_int, [P, u64, u64, pu64]),
    "cpx_trivial_u128": (ctypes.c_int, [P, U128, u64, pU]),
    "cpx_ordinary_u64": (ctypes.c_int, [P, u64, u64, u16, pi64]),
    "cpx_ordinary_u128": (ctypes.c_int, [P, U128, u64, u16, pU]),
    "cpx_S2_easy_u64": (ctypes.c_int, [P, u64, u64, u16, pi64]),
    "cpx_S2_easy_u128": (ctypes.c_int, [P, U128, u64, u16, pU]),
    "cpx_S2_hard_u64": (ctypes.c_int, [P, u64, u64, u16, pi64]),
    "cpx_S2_hard_u128": (ctypes.c_int, [P, U128, u64, u16, pU]),
    "cpx_pi_u64": (ctypes.c_int, [P, u64, u64, u16, pu64, ctypes.POINTER(Terms)]),
    "cpx_gourdon_u64": (ctypes.c_int, [P, u64, u64, u16, ctypes.POINTER(GourdonTerms)]),
    "cpx_pi_u128": (ctypes.c_int, [P, U128, u64, u16, pU, ctypes.POINTER(Terms)]),
    "cpx_gen_d_mu": (ctypes.c_int, [P, u64, u64, PP]),
    "cpx_gen_d_lpf32": (ctypes.c_int, [P, u64, u64, PP]),
    "cpx_gen_d_lpf64": (ctypes.c_int, [P, u64, u64, PP]),
    "cpx_gen_d_mu_lpf": (ctypes.c_int, [P, u64, u64, P, P]),
    "cpx_gen_h_mu": (ctypes.c_int, [P, u64, u64, P]),
    "cpx_gen_h_lpf32": (ctypes.c_int, [P, u64, u64, P]),
    "cpx_mutest": (ctypes.c_int, [P, u64, pi64]),
    "cpx_mutest_noalloc": (ctypes.c_int, [P, u64, pi64]),
    "cpx_pitable": (ctypes.c_int, [P, u64, PP]),
    "cpx_pitable_window": (ctypes.c_int, [P, u64, u64, P, pu64]),
    "cpx_primes": (ctypes.c_int, [P, u64, u64, PP, pu64]),
    "cpx_count_primes": (ctypes.c_int, [P, u64, u64, pu64]),
    "cpx_phi": (ctypes.c_int, [P, u64, u32, pu64]),
    "cpx_phi_range": (ctypes.c_int, [P, u32, u32, PP]),
    "cpx_phisieve_create": (ctypes.c_int, [P, u32, u32, PP]),
    "cpx_phisieve_destroy": (ctypes.c_int, [P]),
    "cpx_phisieve_first": (ctypes.c_int, [P, u16]),
    "cpx_phisieve_mark_next": (ctypes.c_int, [P]),
    "cpx_phisieve_update": (ctypes.c_int, [P]),
    "cpx_phisieve_counts": (ctypes.c_int, [P, PP, pu32]),
    "cpx_phisieve_set_a": (ctypes.c_int, [P, ctypes.c_uint32]),
    "cpx_pi_batch": (ctypes.c_int, [P, pU, ctypes.c_size_t, ctypes.POINTER(Params), pU]),
    "cpx_terms_batch": (ctypes.c_int, [P, pU, pu64, ctypes.c_size_t, ctypes.POINTER(Params), ctypes.POINTER(Terms)]),
    "cpx_mem_info": (ctypes.c_int, [P, pu64, pu64]),
    "cpx_serve_create": (ctypes.c_int, [P, ctypes.POINTER(ServeConfig), PP]),
    "cpx_serve_destroy": (ctypes.c_int, [P]),
    "cpx_serve_submit": (ctypes.c_int, [P, U128, pu64]),
    "cpx_serve_wait": (ctypes.c_int, [P, u64, pU, ctypes.POINTER(ctypes.c_double)]),
    "cpx_serve_replay": (ctypes.c_int, [P, pU, ctypes.POINTER(ctypes.c_double), ctypes.c_size_t, pU,
                                        ctypes.POINTER(ctypes.c_double)]),
    "cpx_serve_stats": (ctypes.c_int, [P, ctypes.POINTER(ServeCounters)]),
    "cpx_serve_last_error": (ctypes.c_char_p, [P]),
}

_lib = None


def header_symbols(path=HEADER):
    """Every function name declared in include/cpx.h."""
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cpx_[a-z0-9_]+)\s*\(", txt)))


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ExtensionMissing(
            f"{LIB_PATH} is missing; build it with `make -C cudapix_b200` (nvcc, sm_100a). "
            "There is no CPU fallback."
        )
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L

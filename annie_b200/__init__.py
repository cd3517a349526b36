"""annie_b200: B200-native modular-squaring engine (PRP tests of large integers).

Python mirror of the reference's ``transform`` interface (galloty/annie,
src/transform.h:18-45) over the C ABI in include/annie_b200.h.  Integers are
Python ints; registers are ``Transform.Reg0/Reg1/Reg2``.  The CUDA library is
required: importing works without it, but creating a transform raises
``EngineUnavailable`` when libannie_b200.so is missing or no CUDA device is
present -- there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libannie_b200.so")

AB_OK = 0
AB_E_ARG = -1
AB_E_UNSUPPORTED = -2
AB_E_CUDA = -3
AB_E_INIT_FAILED = -4
AB_E_CHECKPOINT = -5
AB_E_CAPACITY = -6
AB_E_TIMEOUT = -7


class EngineUnavailable(RuntimeError):
    pass


class EngineError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("annie_b200 error %d: %s" % (code, msg))
        self.code = code


class Params(C.Structure):
    _fields_ = [("K", C.c_int), ("pck", C.c_int), ("ln", C.c_int), ("lbase", C.c_int)]

    def astuple(self):
        return (self.K, self.pck, self.ln, self.lbase)


class PrpOptions(C.Structure):
    _fields_ = [("euler", C.c_int), ("base", C.c_int32), ("device", C.c_int), ("gl_check_blocks", C.c_int),
                ("inject_iteration", C.c_int64), ("inject_word", C.c_uint32), ("checkpoint_path", C.c_char_p),
                ("checkpoint_seconds", C.c_double), ("verbose", C.c_int)]


class PrpResult(C.Structure):
    _fields_ = [("status", C.c_int), ("decided_early", C.c_int), ("is_prp", C.c_int), ("res64", C.c_uint64),
                ("base", C.c_int32), ("K", C.c_int), ("pck", C.c_int), ("ln", C.c_int), ("lbase", C.c_int),
                ("gl_block", C.c_int), ("squarings", C.c_int64), ("gl_checks", C.c_int), ("gl_failures", C.c_int),
                ("rollbacks", C.c_int), ("resumed", C.c_int), ("seconds", C.c_double), ("message", C.c_char * 256)]

    def asdict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_}
        d["message"] = self.message.decode(errors="replace")
        return d


class BenchRow(C.Structure):
    _fields_ = [("e", C.c_uint64), ("digits", C.c_int64), ("K", C.c_int), ("pck", C.c_int), ("ln", C.c_int),
                ("lbase", C.c_int), ("validated", C.c_int), ("squarings", C.c_int64), ("ms_per_bit", C.c_double),
                ("estimated_seconds", C.c_double)]

    def asdict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


# the sizes of the reference's benchmark table (src/annie.h:448): N = 3 2^e + 1
BENCH_TABLE_E = [33216, 83048, 166092, 332190, 664381, 1162672, 1660962, 3321924, 6643854, 16609638, 33219278,
                 66438557, 159200000]


class RunnerOptions(C.Structure):
    _fields_ = [("device", C.c_int), ("hbm_budget_bytes", C.c_size_t), ("max_slots_per_class", C.c_int), ("chunk", C.c_int),
                ("autotune", C.c_int), ("gl_check_blocks", C.c_int), ("inject_tag", C.c_uint64), ("inject_bit", C.c_int64),
                ("inject_word", C.c_uint32), ("latency_ln", C.c_int), ("epoch_us", C.c_int)]


class RunnerClass(C.Structure):
    _fields_ = [("cls", Params), ("slots", C.c_int), ("active", C.c_int), ("squarings", C.c_uint64), ("chunks", C.c_uint64)]


_u64p = C.POINTER(C.c_uint64)
_u32p = C.POINTER(C.c_uint32)
_u8p = C.POINTER(C.c_uint8)
_lib = None

# (name, argtypes, restype) of every exported symbol of include/annie_b200.h
ABI = [
    ("ab_probe", [_u64p, C.c_size_t, C.c_int32, C.POINTER(Params), C.POINTER(Params), C.POINTER(C.c_int)], C.c_int),
    ("ab_create", [_u64p, C.c_size_t, C.c_int32, C.c_int, C.POINTER(Params), C.POINTER(C.c_void_p)], C.c_int),
    ("ab_destroy", [C.c_void_p], None),
    ("ab_init_failed", [C.c_void_p], C.c_int),
    ("ab_get_factor", [C.c_void_p, _u64p, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
    ("ab_info", [C.c_void_p, C.POINTER(Params)], C.c_int),
    ("ab_set1", [C.c_void_p], C.c_int),
    ("ab_copy", [C.c_void_p, C.c_size_t, C.c_size_t], C.c_int),
    ("ab_square_mul", [C.c_void_p, C.c_int32], C.c_int),
    ("ab_mul", [C.c_void_p, C.c_size_t, C.c_size_t], C.c_int),
    ("ab_get", [C.c_void_p, C.c_size_t, _u64p, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
    ("ab_checkpoint_size", [C.c_void_p], C.c_size_t),
    ("ab_save_checkpoint", [C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
    ("ab_read_checkpoint", [C.c_void_p, C.c_void_p, C.c_size_t], C.c_int),
    ("ab_host_alloc", [C.c_size_t], C.c_void_p),
    ("ab_host_free", [C.c_void_p], None),
    ("ab_read_register", [C.c_void_p, C.c_size_t, _u32p, C.c_size_t], C.c_int),
    ("ab_write_register", [C.c_void_p, C.c_size_t, _u32p, C.c_size_t], C.c_int),
    ("ab_inject_word", [C.c_void_p, C.c_size_t, C.c_size_t, C.c_int32], C.c_int),
    ("ab_synchronize", [C.c_void_p], C.c_int),
    ("ab_square_mul_bits", [C.c_void_p, _u64p, C.c_size_t, C.c_int32], C.c_int),
    ("ab_set_geometry", [C.c_void_p, C.c_int], C.c_int),
    ("ab_get_geometry", [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    ("ab_set_overlap", [C.c_void_p, C.c_int], C.c_int),
    ("ab_timer_start", [C.c_void_p], C.c_int),
    ("ab_timer_stop", [C.c_void_p, C.POINTER(C.c_float)], C.c_int),
    ("ab_last_error", [], C.c_char_p),
    ("ab_launch_count", [C.c_void_p, C.POINTER(C.c_uint64)], C.c_int),
    ("ab_profile_square", [C.c_void_p, C.c_int32, C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_int)], C.c_int),
    ("ab_flush_l2", [C.c_void_p, C.c_size_t], C.c_int),
    ("ab_square_mul_noalloc", [C.c_void_p, C.c_void_p, C.c_int32], C.c_int),
    ("ab_prp_options_default", [C.POINTER(PrpOptions)], None),
    ("ab_prp_check", [_u64p, C.c_size_t, C.POINTER(PrpOptions), C.POINTER(PrpResult)], C.c_int),
    ("ab_prp_quit", [], None),
    ("ab_prp_reset_quit", [], None),
    ("ab_bench_table", [C.c_int, _u64p, C.c_int, C.c_double, C.POINTER(BenchRow)], C.c_int),
    ("ab_batch_slot_bytes", [C.POINTER(Params)], C.c_size_t),
    ("ab_batch_create", [C.c_int, C.POINTER(Params), C.c_int, C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    ("ab_batch_destroy", [C.c_void_p], None),
    ("ab_batch_load", [C.c_void_p, C.c_int, _u64p, C.c_size_t, C.c_int32, C.POINTER(C.c_int)], C.c_int),
    ("ab_batch_load_many", [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(_u64p), C.POINTER(C.c_size_t),
                            C.POINTER(C.c_int32), C.POINTER(C.c_int)], C.c_int),
    ("ab_batch_prepare", [_u64p, C.c_size_t, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(Params), C.POINTER(C.c_int)], C.c_int),
    ("ab_prepared_factor", [C.c_void_p, _u64p, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
    ("ab_prepared_bytes", [C.c_void_p], C.c_size_t),
    ("ab_prepared_destroy", [C.c_void_p], None),
    ("ab_batch_install", [C.c_void_p, C.c_int, C.c_void_p], C.c_int),
    ("ab_batch_slot", [C.c_void_p, C.c_int], C.c_void_p),
    ("ab_batch_clone", [C.c_void_p, C.c_int, C.c_int], C.c_int),
    ("ab_batch_release", [C.c_void_p, C.c_int], C.c_int),
    ("ab_batch_steps", [C.c_void_p, C.c_int, _u32p, _u8p], C.c_int),
    ("ab_batch_ready", [C.c_void_p], C.c_int),
    ("ab_batch_gl_mul", [C.c_void_p, C.c_int], C.c_int),
    ("ab_batch_set_geometry", [C.c_void_p, C.c_int], C.c_int),
    ("ab_batch_autotune", [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int)], C.c_int),
    ("ab_batch_synchronize", [C.c_void_p], C.c_int),
    ("ab_batch_launch_count", [C.c_void_p, C.POINTER(C.c_uint64)], C.c_int),
    ("ab_mixed_create", [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    ("ab_mixed_destroy", [C.c_void_p], None),
    ("ab_mixed_steps", [C.c_void_p, C.c_int, C.POINTER(_u32p), C.POINTER(_u8p)], C.c_int),
    ("ab_mixed_ready", [C.c_void_p], C.c_int),
    ("ab_mixed_synchronize", [C.c_void_p], C.c_int),
    ("ab_mixed_launch_count", [C.c_void_p, C.POINTER(C.c_uint64)], C.c_int),
    ("ab_runner_options_default", [C.POINTER(RunnerOptions)], None),
    ("ab_runner_create", [C.POINTER(RunnerOptions), C.POINTER(C.c_void_p)], C.c_int),
    ("ab_runner_destroy", [C.c_void_p], None),
    ("ab_runner_submit", [C.c_void_p, _u64p, C.c_size_t, C.c_int, C.c_int32, C.c_uint64], C.c_int),
    ("ab_runner_advance", [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    ("ab_runner_synchronize", [C.c_void_p], C.c_int),
    ("ab_runner_poll", [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(PrpResult)], C.c_int),
    ("ab_runner_stats", [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_int)], C.c_int),
    ("ab_runner_classes", [C.c_void_p, C.POINTER(RunnerClass), C.c_int, C.POINTER(C.c_int)], C.c_int),
    ("ab_runner_host_seconds", [C.c_void_p, C.POINTER(C.c_double)], C.c_int),
    ("ab_diag_forward", [C.c_void_p, C.c_int, _u32p, _u32p], C.c_int),
    ("ab_diag_product", [C.c_void_p, C.c_int, _u32p, _u32p, C.c_uint32, _u32p, C.c_int, _u32p], C.c_int),
]


def lib(build_if_missing=False):
    """The loaded C ABI library (built in-tree by annie_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            if build_if_missing:
                from . import build
                build.build()
            else:
                raise EngineUnavailable("CUDA engine not built: %s missing (run python -m annie_b200.build)" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, args, res in ABI:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def _check(rc):
    if rc != AB_OK:
        raise EngineError(rc, lib().ab_last_error().decode(errors="replace"))


def int_to_limbs(x):
    n = max(1, (x.bit_length() + 63) // 64)
    return np.frombuffer(x.to_bytes(n * 8, "little"), dtype=np.uint64).copy()


def limbs_to_int(a, count):
    return int.from_bytes(np.asarray(a[:count], dtype=np.uint64).tobytes(), "little")


def probe(N, a, forced=None, gcd=True):
    """(params tuple, init_failed) by the factory rule of transformGPU.h:822-857; no GPU
    needed.  gcd=False skips the gcd(N, R) test (init_failed is then None)."""
    limbs = int_to_limbs(N)
    out = Params()
    failed = C.c_int()
    fp = None if forced is None else C.byref(Params(*forced))
    _check(lib().ab_probe(limbs.ctypes.data_as(_u64p), len(limbs), a, fp, C.byref(out),
                          C.byref(failed) if gcd else None))
    return out.astuple(), (bool(failed.value) if gcd else None)


def prp_check(N, euler=False, base=0, device=0, gl_check_blocks=0, inject_iteration=-1, inject_word=0,
              checkpoint_path=None, checkpoint_seconds=600.0):
    """Full probable-prime test of N (the reference's annie::check, src/annie.h:217-430)
    with optional periodic Gerbicz-Li checks, rollback and fault injection.  Returns a dict."""
    L = lib()
    o = PrpOptions()
    L.ab_prp_options_default(C.byref(o))
    o.euler, o.base, o.device, o.gl_check_blocks = int(euler), base, device, gl_check_blocks
    o.inject_iteration, o.inject_word = inject_iteration, inject_word
    o.checkpoint_path = None if checkpoint_path is None else checkpoint_path.encode()
    o.checkpoint_seconds = checkpoint_seconds
    r = PrpResult()
    limbs = int_to_limbs(N)
    L.ab_prp_check(limbs.ctypes.data_as(_u64p), len(limbs), C.byref(o), C.byref(r))
    return r.asdict()


def bench_table(e_list=None, seconds=10.0, device=0):
    """The reference's benchmark mode (annie::bench, src/annie.h:432-556): one
    row per N = 3 2^e + 1 (dicts), stopping after a row that does not validate."""
    e_list = BENCH_TABLE_E if e_list is None else list(e_list)
    es = np.array(e_list, dtype=np.uint64)
    rows = (BenchRow * len(e_list))()
    done = lib().ab_bench_table(device, es.ctypes.data_as(_u64p), len(e_list), seconds, rows)
    if done < 0:
        raise EngineError(AB_E_CUDA, "ab_bench_table failed")
    return [rows[i].asdict() for i in range(done)]


class Transform:
    """The reference's transform register machine on one GPU (transform.h:18-45)."""

    Reg0, Reg1, Reg2 = 0, 1, 2

    def __init__(self, N, a, device=0, params=None):
        self.N, self.a = N, a
        L = lib()
        limbs = int_to_limbs(N)
        h = C.c_void_p()
        fp = None if params is None else C.byref(Params(*params))
        _check(L.ab_create(limbs.ctypes.data_as(_u64p), len(limbs), a, device, fp, C.byref(h)))
        self.h = h
        self.L = L
        info = Params()
        _check(L.ab_info(h, C.byref(info)))
        self.K, self.pck, self.ln, self.lbase = info.astuple()
        self.n = 1 << self.ln
        self._cap = len(limbs) + 2

    def close(self):
        if getattr(self, "h", None):
            self.L.ab_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- transform.h:26-34
    def init_failed(self):
        return bool(self.L.ab_init_failed(self.h))

    def get_factor(self):
        out = np.zeros(self._cap, dtype=np.uint64)
        cnt = C.c_size_t()
        _check(self.L.ab_get_factor(self.h, out.ctypes.data_as(_u64p), len(out), C.byref(cnt)))
        return limbs_to_int(out, cnt.value)

    def set1(self):
        _check(self.L.ab_set1(self.h))

    def copy(self, dst, src):
        _check(self.L.ab_copy(self.h, dst, src))

    def square_mul(self, a):
        _check(self.L.ab_square_mul(self.h, a))

    def square_mul_bits(self, bits, count, a):
        """count squarings; step i multiplies by a when bit i of `bits` (an int) is set."""
        bits &= (1 << count) - 1
        words = np.frombuffer(bits.to_bytes(max(8, (count + 63) // 64 * 8), "little"), dtype=np.uint64).copy()
        _check(self.L.ab_square_mul_bits(self.h, words.ctypes.data_as(_u64p), count, a))

    def set_geometry(self, row_levels):
        _check(self.L.ab_set_geometry(self.h, row_levels))

    def geometry(self):
        """(row levels, column levels) of the NTT split."""
        rl, cl = C.c_int(), C.c_int()
        _check(self.L.ab_get_geometry(self.h, C.byref(rl), C.byref(cl)))
        return rl.value, cl.value

    def set_overlap(self, on):
        """Q-domain chain on a second stream (True, default) or one stream for everything."""
        _check(self.L.ab_set_overlap(self.h, int(bool(on))))

    def mul(self, dst, src):
        _check(self.L.ab_mul(self.h, dst, src))

    def get(self, src):
        out = np.zeros(self._cap, dtype=np.uint64)
        cnt = C.c_size_t()
        _check(self.L.ab_get(self.h, src, out.ctypes.data_as(_u64p), len(out), C.byref(cnt)))
        return limbs_to_int(out, cnt.value)

    # -- checkpoint payload (transformGPU.h:608-641)
    def save_checkpoint(self):
        size = self.L.ab_checkpoint_size(self.h)
        buf = np.zeros(size, dtype=np.uint8)
        written = C.c_size_t()
        _check(self.L.ab_save_checkpoint(self.h, buf.ctypes.data_as(C.c_void_p), size, C.byref(written)))
        return buf.tobytes()

    def read_checkpoint(self, payload):
        buf = np.frombuffer(payload, dtype=np.uint8).copy()
        rc = self.L.ab_read_checkpoint(self.h, buf.ctypes.data_as(C.c_void_p), len(buf))
        if rc == AB_E_CHECKPOINT:
            return False
        _check(rc)
        return True

    def pinned(self, nbytes):
        """A page-locked host buffer (numpy uint8 view) and its pointer; free with free_pinned."""
        ptr = self.L.ab_host_alloc(nbytes)
        if not ptr:
            raise EngineError(AB_E_CUDA, "cudaMallocHost failed")
        arr = np.ctypeslib.as_array((C.c_uint8 * nbytes).from_address(ptr))
        return arr, ptr

    def free_pinned(self, ptr):
        self.L.ab_host_free(ptr)

    def save_checkpoint_into(self, ptr, cap):
        written = C.c_size_t()
        _check(self.L.ab_save_checkpoint(self.h, C.c_void_p(ptr), cap, C.byref(written)))
        return written.value

    def read_checkpoint_from(self, ptr, size):
        _check(self.L.ab_read_checkpoint(self.h, C.c_void_p(ptr), size))

    def read_register(self, reg):
        out = np.zeros(self.K * self.n, dtype=np.uint32)
        _check(self.L.ab_read_register(self.h, reg, out.ctypes.data_as(_u32p), len(out)))
        return out

    def write_register(self, reg, words):
        w = np.ascontiguousarray(words, dtype=np.uint32)
        _check(self.L.ab_write_register(self.h, reg, w.ctypes.data_as(_u32p), len(w)))

    def inject_word(self, reg, index, delta=-1):
        """Adds delta to one 32-bit word of the engine's copy of register reg (fault injection)."""
        _check(self.L.ab_inject_word(self.h, reg, index, delta))

    def synchronize(self):
        _check(self.L.ab_synchronize(self.h))

    def timer_start(self):
        _check(self.L.ab_timer_start(self.h))

    def timer_stop(self):
        ms = C.c_float()
        _check(self.L.ab_timer_stop(self.h, C.byref(ms)))
        return ms.value

    def launch_count(self):
        c = C.c_uint64()
        _check(self.L.ab_launch_count(self.h, C.byref(c)))
        return c.value

    def profile_square(self, a, cap=16):
        ms = (C.c_float * cap)()
        cnt = C.c_int()
        _check(self.L.ab_profile_square(self.h, a, ms, cap, C.byref(cnt)))
        return [ms[i] for i in range(cnt.value)]

    def flush_l2(self, nbytes=256 << 20):
        _check(self.L.ab_flush_l2(self.h, nbytes))

    def square_mul_noalloc(self, device_ptr, a):
        """square_mul on a caller-owned device register (K*n u32), no allocation."""
        _check(self.L.ab_square_mul_noalloc(self.h, C.c_void_p(device_ptr), a))

    # -- information strings (transformGPU.h:766-795)
    def get_info_short(self):
        return "%d-prime NTT of length %d, packed-base = 2^{%dx%d}" % (self.K + 1, self.n, self.pck, self.lbase)

    def get_info(self):
        return "Montgomery-McLaughlin-Gallot-Woltman reduction, " + self.get_info_short()

    # -- diagnostics
    def diag_forward(self, words, domain_q):
        """Forward NTT of a normal-form register over the engine's K+1 transform primes."""
        w = np.ascontiguousarray(words, dtype=np.uint32)
        out = np.zeros((self.K + 1) * self.n, dtype=np.uint32)
        _check(self.L.ab_diag_forward(self.h, int(domain_q), w.ctypes.data_as(_u32p), out.ctypes.data_as(_u32p)))
        return out

    def diag_product(self, words, domain_q, a, y=None, sub=None, lower_mode=0):
        """Product (square when y is None) of normal-form registers in one domain, then the carry."""
        w = np.ascontiguousarray(words, dtype=np.uint32)
        out = np.zeros_like(w)
        xpa = None if y is None else np.ascontiguousarray(y, dtype=np.uint32)
        sba = None if sub is None else np.ascontiguousarray(sub, dtype=np.uint32)
        _check(self.L.ab_diag_product(self.h, int(domain_q), w.ctypes.data_as(_u32p),
                                      None if xpa is None else xpa.ctypes.data_as(_u32p), a,
                                      None if sba is None else sba.ctypes.data_as(_u32p), lower_mode,
                                      out.ctypes.data_as(_u32p)))
        return out


class SlotView(Transform):
    """A batch slot used through the transform interface (owned by its Batch)."""

    def __init__(self, batch, slot, handle):
        self.N, self.a = batch.Ns[slot], batch.bases[slot]
        self.L = batch.L
        self.h = C.c_void_p(handle)
        info = Params()
        _check(self.L.ab_info(self.h, C.byref(info)))
        self.K, self.pck, self.ln, self.lbase = info.astuple()
        self.n = 1 << self.ln
        self._cap = len(int_to_limbs(self.N)) + 2

    def close(self):
        self.h = None


class Batch:
    """Size class (K, pck, ln) of `capacity` slots squared together (captured CUDA graph)."""

    def __init__(self, cls, capacity, max_steps=64, device=0):
        self.L = lib()
        self.cls = Params(*cls)
        self.capacity, self.max_steps = capacity, max_steps
        h = C.c_void_p()
        _check(self.L.ab_batch_create(device, C.byref(self.cls), capacity, max_steps, C.byref(h)))
        self.h = h
        self.Ns = [None] * capacity
        self.bases = [None] * capacity

    def close(self):
        if getattr(self, "h", None):
            self.L.ab_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load(self, slot, N, a):
        limbs = int_to_limbs(N)
        failed = C.c_int()
        _check(self.L.ab_batch_load(self.h, slot, limbs.ctypes.data_as(_u64p), len(limbs), a, C.byref(failed)))
        self.Ns[slot], self.bases[slot] = N, a
        return bool(failed.value)

    def load_many(self, items):
        """items: list of (slot, N, a); loads them together (host set-up on threads).
        Returns the init_failed flags."""
        cnt = len(items)
        limbs = [int_to_limbs(N) for _, N, _ in items]
        slots = (C.c_int * cnt)(*[s for s, _, _ in items])
        ptrs = (_u64p * cnt)(*[x.ctypes.data_as(_u64p) for x in limbs])
        nn = (C.c_size_t * cnt)(*[len(x) for x in limbs])
        aa = (C.c_int32 * cnt)(*[a for _, _, a in items])
        failed = (C.c_int * cnt)()
        _check(self.L.ab_batch_load_many(self.h, cnt, slots, ptrs, nn, aa, failed))
        for s, N, a in items:
            self.Ns[s], self.bases[s] = N, a
        return [bool(f) for f in failed]

    def slot(self, slot):
        hv = self.L.ab_batch_slot(self.h, slot)
        return None if not hv else SlotView(self, slot, hv)

    def release(self, slot):
        _check(self.L.ab_batch_release(self.h, slot))
        self.Ns[slot] = None

    def clone(self, dst, src):
        _check(self.L.ab_batch_clone(self.h, dst, src))
        self.Ns[dst], self.bases[dst] = self.Ns[src], self.bases[src]

    def steps(self, mult, snap=None):
        """mult: array [steps, capacity] of multipliers (0 = idle); snap: same shape, nonzero = keep Reg0."""
        m = np.ascontiguousarray(mult, dtype=np.uint32)
        s = None if snap is None else np.ascontiguousarray(snap, dtype=np.uint8)
        _check(self.L.ab_batch_steps(self.h, m.shape[0], m.ctypes.data_as(_u32p), None if s is None else s.ctypes.data_as(_u8p)))

    def gl_mul(self, slot):
        _check(self.L.ab_batch_gl_mul(self.h, slot))

    def set_geometry(self, lb):
        _check(self.L.ab_batch_set_geometry(self.h, lb))

    def autotune(self, src, steps):
        """Fastest row/column split for this class (times every split on copies of slot src)."""
        lb = C.c_int()
        _check(self.L.ab_batch_autotune(self.h, src, steps, C.byref(lb)))
        return lb.value

    def synchronize(self):
        _check(self.L.ab_batch_synchronize(self.h))

    def launch_count(self):
        c = C.c_uint64()
        _check(self.L.ab_batch_launch_count(self.h, C.byref(c)))
        return c.value


class Mixed:
    """A mixed-size group of batches (include/annie_b200_batch.h, ab_mixed_*):
    their squarings run together, one launch per pass for every class."""

    def __init__(self, batches, max_steps=64):
        self.L = lib()
        self.batches = list(batches)
        arr = (C.c_void_p * len(self.batches))(*[b.h.value for b in self.batches])
        h = C.c_void_p()
        _check(self.L.ab_mixed_create(arr, len(self.batches), max_steps, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.ab_mixed_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def steps(self, mults, snaps=None):
        """mults[i]: (steps, capacity_i) multipliers of batch i; snaps[i] the same
        shape of 0/1 flags (nullable)."""
        ms = [np.ascontiguousarray(m, dtype=np.uint32) for m in mults]
        steps = ms[0].shape[0]
        assert all(m.shape == (steps, b.capacity) for m, b in zip(ms, self.batches))
        mp = (_u32p * len(ms))(*[m.ctypes.data_as(_u32p) for m in ms])
        sp = None
        if snaps is not None:
            ss = [None if x is None else np.ascontiguousarray(x, dtype=np.uint8) for x in snaps]
            sp = (_u8p * len(ss))(*[_u8p() if x is None else x.ctypes.data_as(_u8p) for x in ss])
            self._keep = ss
        _check(self.L.ab_mixed_steps(self.h, steps, mp, sp))

    def ready(self):
        return self.L.ab_mixed_ready(self.h)

    def synchronize(self):
        _check(self.L.ab_mixed_synchronize(self.h))

    def launch_count(self):
        c = C.c_uint64()
        _check(self.L.ab_mixed_launch_count(self.h, C.byref(c)))
        return c.value


class Runner:
    """Continuous-batching PRP runner: submit tests, advance, poll results."""

    def __init__(self, device=0, hbm_budget_bytes=32 << 30, max_slots_per_class=256, chunk=64, autotune=True,
                 gl_check_blocks=0, inject_tag=0, inject_bit=-1, inject_word=0, latency_ln=0, epoch_us=20000):
        self.L = lib()
        o = RunnerOptions()
        self.L.ab_runner_options_default(C.byref(o))
        o.device, o.hbm_budget_bytes, o.max_slots_per_class, o.chunk = device, hbm_budget_bytes, max_slots_per_class, chunk
        o.autotune = int(bool(autotune))
        o.gl_check_blocks = gl_check_blocks
        o.inject_tag, o.inject_bit, o.inject_word = inject_tag, inject_bit, inject_word
        o.latency_ln, o.epoch_us = latency_ln, epoch_us
        h = C.c_void_p()
        _check(self.L.ab_runner_create(C.byref(o), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.ab_runner_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, N, euler=False, base=0, tag=0):
        limbs = int_to_limbs(N)
        _check(self.L.ab_runner_submit(self.h, limbs.ctypes.data_as(_u64p), len(limbs), int(euler), base, tag))

    def advance(self):
        a, q = C.c_int(), C.c_int()
        _check(self.L.ab_runner_advance(self.h, C.byref(a), C.byref(q)))
        return a.value, q.value

    def poll(self):
        tag = C.c_uint64()
        r = PrpResult()
        out = []
        while self.L.ab_runner_poll(self.h, C.byref(tag), C.byref(r)):
            out.append((tag.value, r.asdict()))
        return out

    def synchronize(self):
        _check(self.L.ab_runner_synchronize(self.h))

    def stats(self):
        s, l, b = C.c_uint64(), C.c_uint64(), C.c_int()
        _check(self.L.ab_runner_stats(self.h, C.byref(s), C.byref(l), C.byref(b)))
        return {"squarings": s.value, "launches": l.value, "batches": b.value}

    def classes(self):
        """Per size class: (K, pck, ln), slots, active tests, squarings, chunks."""
        cnt = C.c_int()
        _check(self.L.ab_runner_classes(self.h, None, 0, C.byref(cnt)))
        arr = (RunnerClass * max(1, cnt.value))()
        _check(self.L.ab_runner_classes(self.h, arr, cnt.value, C.byref(cnt)))
        return [{"class": [x.cls.K, x.cls.pck, x.cls.ln], "slots": x.slots, "active": x.active,
                 "squarings": x.squarings, "chunks": x.chunks} for x in arr[:cnt.value]]

    def host_seconds(self):
        """Host time inside advance(): admission, autotune, phase steps, sleeping."""
        out = (C.c_double * 4)()
        _check(self.L.ab_runner_host_seconds(self.h, out))
        return dict(zip(("admission", "autotune", "phase_steps", "sleep"), [round(x, 3) for x in out]))

"""TEST INFRASTRUCTURE ONLY: ctypes bindings for the two CPU checkers.

* ``Oracle``    -- this project's C restatement (annie_oracle.c, _ref/liboracle.so)
* ``RefTransform`` -- the reference's own transformCPU / transformGMP compiled
  from its sources (ref_shim.cpp, _ref/libannie_ref.so)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_u64p = C.POINTER(C.c_uint64)
_u32p = C.POINTER(C.c_uint32)


def build(ref_src=None):
    """Build _ref/liboracle.so, and _ref/libannie_ref.so when the reference's src
    folder is given (argument, or the ANNIE_REF_SRC environment variable)."""
    ref_src = ref_src or os.environ.get("ANNIE_REF_SRC", "")
    cmd = ["make", "-s", "-C", HERE]
    if ref_src:
        cmd.append("REF_SRC=" + ref_src)
    subprocess.run(cmd, check=True)


def int_to_limbs(x):
    n = max(1, (x.bit_length() + 63) // 64)
    return np.frombuffer(x.to_bytes(n * 8, "little"), dtype=np.uint64).copy()


def limbs_to_int(a, count):
    return int.from_bytes(np.asarray(a[:count], dtype=np.uint64).tobytes(), "little")


def _ptr64(a):
    return a.ctypes.data_as(_u64p)


def _ptr32(a):
    return a.ctypes.data_as(_u32p)


_lib_oracle = None
_lib_ref = None


def lib_oracle():
    global _lib_oracle
    if _lib_oracle is None:
        path = os.path.join(REF_DIR, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.or_select_params.argtypes = [_u64p, C.c_size_t, C.c_int32, C.c_int] + [C.POINTER(C.c_int)] * 4
        L.or_create.argtypes = [_u64p, C.c_size_t, C.c_int32, C.c_int, C.c_int, C.c_int]
        L.or_create.restype = C.c_void_p
        for name in ("or_destroy", "or_set1"):
            getattr(L, name).argtypes = [C.c_void_p]
        L.or_init_failed.argtypes = [C.c_void_p]
        L.or_copy.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t]
        L.or_square_mul.argtypes = [C.c_void_p, C.c_int32]
        L.or_mul.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t]
        L.or_read_reg.argtypes = [C.c_void_p, C.c_size_t, _u32p]
        L.or_write_reg.argtypes = [C.c_void_p, C.c_size_t, _u32p]
        L.or_read_roots.argtypes = [C.c_void_p, C.c_int, _u32p]
        L.or_fwd_full.argtypes = [C.c_void_p, C.c_int, _u32p]
        L.or_inv_full.argtypes = [C.c_void_p, C.c_int, _u32p]
        L.or_fwd_levels.argtypes = [C.c_void_p, C.c_int, _u32p, C.c_int, C.c_int]
        L.or_inv_levels.argtypes = [C.c_void_p, C.c_int, _u32p, C.c_int, C.c_int]
        L.or_pointwise.argtypes = [C.c_void_p, C.c_int, _u32p, _u32p]
        L.or_carry.argtypes = [C.c_void_p, _u32p, C.c_uint32, C.c_int, _u32p, C.c_int]
        L.or_get.argtypes = [C.c_void_p, C.c_size_t, _u64p, C.c_size_t]
        L.or_get.restype = C.c_long
        L.or_get_factor.argtypes = [C.c_void_p, _u64p, C.c_size_t, C.POINTER(C.c_size_t)]
        L.or_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 4
        _lib_oracle = L
    return _lib_oracle


def lib_ref():
    global _lib_ref
    if _lib_ref is None:
        path = os.path.join(REF_DIR, "libannie_ref.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.ref_create.argtypes = [_u64p, C.c_size_t, C.c_int32, C.c_int]
        L.ref_create.restype = C.c_void_p
        for name in ("ref_destroy", "ref_set1"):
            getattr(L, name).argtypes = [C.c_void_p]
        L.ref_init_failed.argtypes = [C.c_void_p]
        L.ref_copy.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t]
        L.ref_square_mul.argtypes = [C.c_void_p, C.c_int32]
        L.ref_square_mul_seq.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.c_size_t]
        L.ref_mul.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t]
        L.ref_get.argtypes = [C.c_void_p, C.c_size_t, _u64p, C.c_size_t]
        L.ref_get.restype = C.c_long
        L.ref_get_factor.argtypes = [C.c_void_p, _u64p, C.c_size_t, C.POINTER(C.c_size_t)]
        L.ref_info.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t]
        L.ref_save_checkpoint.argtypes = [C.c_void_p, C.c_char_p]
        L.ref_read_checkpoint.argtypes = [C.c_void_p, C.c_char_p]
        L.ref_cpu_get_n_base.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, C.c_double, C.c_double]
        L.ref_check.argtypes = [_u64p, C.c_size_t, C.c_int, C.c_int, C.c_char_p]
        L.ref_file_write_checkpoint.argtypes = [C.c_char_p, C.c_int, C.c_double, C.POINTER(C.c_uint8), C.c_size_t]
        L.ref_file_read_checkpoint.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                               C.POINTER(C.c_uint8), C.c_size_t]
        _lib_ref = L
    return _lib_ref


def ref_available():
    return os.path.exists(os.path.join(REF_DIR, "libannie_ref.so"))


def select_params(N, a, rule=0):
    """(K, pck, ln, lbase) by the reference's GPU factory rule (rule=0) or transformCPU's (rule=1)."""
    L = lib_oracle()
    limbs = int_to_limbs(N)
    out = [C.c_int() for _ in range(4)]
    L.or_select_params(_ptr64(limbs), len(limbs), a, rule, *[C.byref(o) for o in out])
    return tuple(o.value for o in out)


class Oracle:
    """C restatement of the MMGW transform; same register machine as ``transform``."""

    Reg0, Reg1, Reg2 = 0, 1, 2

    def __init__(self, N, a, params=None, rule=0):
        self.N, self.a = N, a
        K, pck, ln, lbase = params if params is not None else select_params(N, a, rule)
        self.K, self.pck, self.ln, self.lbase = K, pck, ln, lbase
        self.n = 1 << ln
        limbs = int_to_limbs(N)
        self.L = lib_oracle()
        self.h = self.L.or_create(_ptr64(limbs), len(limbs), a, K, ln, lbase)

    def close(self):
        if self.h:
            self.L.or_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_failed(self):
        return bool(self.L.or_init_failed(self.h))

    def get_factor(self):
        out = np.zeros(len(int_to_limbs(self.N)) + 2, dtype=np.uint64)
        cnt = C.c_size_t()
        self.L.or_get_factor(self.h, _ptr64(out), len(out), C.byref(cnt))
        return limbs_to_int(out, cnt.value)

    def set1(self):
        self.L.or_set1(self.h)

    def copy(self, dst, src):
        self.L.or_copy(self.h, dst, src)

    def square_mul(self, a):
        self.L.or_square_mul(self.h, a)

    def mul(self, dst, src):
        self.L.or_mul(self.h, dst, src)

    def get(self, src):
        out = np.zeros(len(int_to_limbs(self.N)) + 2, dtype=np.uint64)
        cnt = self.L.or_get(self.h, src, _ptr64(out), len(out))
        assert cnt >= 0
        return limbs_to_int(out, cnt)

    def read_reg(self, r):
        out = np.zeros(self.K * self.n, dtype=np.uint32)
        self.L.or_read_reg(self.h, r, _ptr32(out))
        return out

    def write_reg(self, r, words):
        w = np.ascontiguousarray(words, dtype=np.uint32)
        self.L.or_write_reg(self.h, r, _ptr32(w))

    def roots(self, domain_q):
        out = np.zeros(self.K * self.n, dtype=np.uint32)
        self.L.or_read_roots(self.h, int(domain_q), _ptr32(out))
        return out

    # kernel-level pieces (operate on a copy, return the result)
    def fwd_full(self, x, domain_q):
        y = np.ascontiguousarray(x, dtype=np.uint32).copy()
        self.L.or_fwd_full(self.h, int(domain_q), _ptr32(y))
        return y

    def inv_full(self, x, domain_q):
        y = np.ascontiguousarray(x, dtype=np.uint32).copy()
        self.L.or_inv_full(self.h, int(domain_q), _ptr32(y))
        return y

    def fwd_levels(self, x, domain_q, lv_from, lv_to):
        y = np.ascontiguousarray(x, dtype=np.uint32).copy()
        self.L.or_fwd_levels(self.h, int(domain_q), _ptr32(y), lv_from, lv_to)
        return y

    def inv_levels(self, x, domain_q, lv_from, lv_to):
        y = np.ascontiguousarray(x, dtype=np.uint32).copy()
        self.L.or_inv_levels(self.h, int(domain_q), _ptr32(y), lv_from, lv_to)
        return y

    def pointwise(self, x, domain_q, xp=None):
        y = np.ascontiguousarray(x, dtype=np.uint32).copy()
        p = None if xp is None else np.ascontiguousarray(xp, dtype=np.uint32)
        self.L.or_pointwise(self.h, int(domain_q), _ptr32(y), None if p is None else _ptr32(p))
        return y

    def carry(self, x, a, nega, y=None, lower_mode=0):
        z = np.ascontiguousarray(x, dtype=np.uint32).copy()
        yy = None if y is None else np.ascontiguousarray(y, dtype=np.uint32)
        self.L.or_carry(self.h, _ptr32(z), a, int(nega), None if yy is None else _ptr32(yy), lower_mode)
        return z


class RefTransform:
    """The reference's own transformCPU (kind=0) or transformGMP (kind=1)."""

    Reg0, Reg1, Reg2 = 0, 1, 2

    def __init__(self, N, a, kind=0):
        self.N, self.a = N, a
        self.L = lib_ref()
        limbs = int_to_limbs(N)
        self.h = self.L.ref_create(_ptr64(limbs), len(limbs), a, kind)
        assert self.h

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_failed(self):
        return bool(self.L.ref_init_failed(self.h))

    def get_factor(self):
        out = np.zeros(len(int_to_limbs(self.N)) + 2, dtype=np.uint64)
        cnt = C.c_size_t()
        self.L.ref_get_factor(self.h, _ptr64(out), len(out), C.byref(cnt))
        return limbs_to_int(out, cnt.value)

    def info(self):
        buf = C.create_string_buffer(256)
        self.L.ref_info(self.h, buf, 256)
        return buf.value.decode()

    def set1(self):
        self.L.ref_set1(self.h)

    def copy(self, dst, src):
        self.L.ref_copy(self.h, dst, src)

    def square_mul(self, a):
        self.L.ref_square_mul(self.h, a)

    def square_mul_seq(self, as_):
        arr = (C.c_int32 * len(as_))(*as_)
        self.L.ref_square_mul_seq(self.h, arr, len(as_))

    def mul(self, dst, src):
        self.L.ref_mul(self.h, dst, src)

    def get(self, src):
        out = np.zeros(len(int_to_limbs(self.N)) + 2, dtype=np.uint64)
        cnt = self.L.ref_get(self.h, src, _ptr64(out), len(out))
        assert cnt >= 0
        return limbs_to_int(out, cnt)

    def load_checkpoint_words(self, words, path):
        """Reg0 || Reg1 (plane-major, K*n words each) through the reference's own
        read_checkpoint (format of src/transformCPU.h:1475-1491)."""
        np.ascontiguousarray(words, dtype=np.uint32).tofile(path)
        assert self.L.ref_read_checkpoint(self.h, path.encode()) == 0

    def checkpoint_words(self, path):
        """Reg0 and Reg1 as saved by the reference (plane-major, K*n words each)."""
        assert self.L.ref_save_checkpoint(self.h, path.encode()) == 0
        return np.fromfile(path, dtype=np.uint32)


def ref_file_write_checkpoint(path, i, elapsed, payload):
    """A checkpoint file written by the reference's file class (src/file.h) in the
    layout of annie::save_checkpoint (src/annie.h:162-181)."""
    buf = np.frombuffer(payload, dtype=np.uint8).copy()
    return lib_ref().ref_file_write_checkpoint(path.encode(), i, elapsed, buf.ctypes.data_as(C.POINTER(C.c_uint8)), len(buf))


def ref_file_read_checkpoint(path, size):
    """(status, i, elapsed, payload bytes) read and seal-checked by the reference's file class."""
    buf = np.zeros(size, dtype=np.uint8)
    i, el = C.c_int(), C.c_double()
    st = lib_ref().ref_file_read_checkpoint(path.encode(), C.byref(i), C.byref(el), buf.ctypes.data_as(C.POINTER(C.c_uint8)), size)
    return st, i.value, el.value, buf.tobytes()

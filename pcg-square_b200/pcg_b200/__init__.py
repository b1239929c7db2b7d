"""ctypes shim over libpcg_b200.so, the B200 PCG-OLE expansion library.

The functions mirror the reference's pcg_cuda:: hooks
(GPU_baseline/common/dpf_gpu.h, leaf_convert_cuda.h, poly_mul_cuda.h,
aes_gpu.h): same names, same argument meaning, host numpy arrays in and out,
and a RuntimeError where the reference throws std::runtime_error.  The
native device-resident API (keyed DPF, fused expansion, batched NTT) is
exposed through `Expander` and the *_device functions, which take raw device
pointers (ints) such as torch's tensor.data_ptr().

There is no CPU fallback: if the shared library or a CUDA device is missing,
the calls raise.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libpcg_b200.so")

P = 4611686018326724609
PRG_AES, PRG_CHACHA8 = 0, 1
POLYMUL_V1, POLYMUL_MERGE, POLYMUL_4STEP, POLYMUL_SQUARE = 0, 1, 2, 3
OUT_HASH_DOMAIN = 0x6F75745F68617368

_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_vp = C.c_void_p

EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p)


class Request(C.Structure):
    _fields_ = [("N", C.c_int), ("c", C.c_int), ("t", C.c_int), ("party", C.c_int),
                ("seed", C.c_uint64), ("arrival_s", C.c_double)]


class Result(C.Structure):
    _fields_ = [("digest_x", C.c_uint64), ("digest_z", C.c_uint64), ("submit_s", C.c_double),
                ("start_s", C.c_double), ("done_s", C.c_double), ("status", C.c_int),
                ("reserved", C.c_int)]


class PcgError(RuntimeError):
    """A library call failed; .code is the PCGB_E* value."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libpcg_b200.so not built ({LIB_PATH}); run __graft_entry__.build()")
    L = C.CDLL(LIB_PATH)
    L.pcgb_last_error.restype = C.c_char_p
    sig = {
        "pcgb_version": ([], C.c_int),
        "pcgb_is_cuda_available": ([], C.c_int),
        "pcgb_device_name": ([C.c_char_p, C.c_size_t], C.c_int),
        "pcgb_runtime_version": ([C.c_char_p, C.c_size_t], C.c_int),
        "pcgb_set_device": ([C.c_int], C.c_int),
        "pcgb_get_device": ([C.POINTER(C.c_int)], C.c_int),
        "pcgb_sm_count": ([C.POINTER(C.c_int)], C.c_int),
        "pcgb_malloc": ([C.POINTER(_vp), C.c_size_t], C.c_int),
        "pcgb_free": ([_vp], C.c_int),
        "pcgb_memcpy_h2d": ([_vp, _vp, C.c_size_t, _vp], C.c_int),
        "pcgb_memcpy_d2h": ([_vp, _vp, C.c_size_t, _vp], C.c_int),
        "pcgb_memset": ([_vp, C.c_int, C.c_size_t, _vp], C.c_int),
        "pcgb_stream_synchronize": ([_vp], C.c_int),
        "pcgb_device_synchronize": ([], C.c_int),
        "pcgb_trim_pool": ([], C.c_int),
        "pcgb_triples_device": ([C.c_int, C.c_int] + [_vp] * 7 + [_vp], C.c_int),
        "pcgb_verify_ole_device": ([C.c_int] + [_vp] * 5 + [_vp], C.c_int),
        "pcgb_verify_triples_device": ([C.c_int] + [_vp] * 7 + [_vp], C.c_int),
        "pcgb_default_stream": ([], _vp),
        "pcgb_dpf_batch_full_eval": ([C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, C.c_int, _vp, _vp,
                                      _vp, C.c_int], C.c_int),
        "pcgb_dpf_batch_full_eval_device": ([C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, C.c_int,
                                             _vp, _vp, C.c_int, C.POINTER(_vp)], C.c_int),
        "pcgb_gmw_position_add_gates": ([C.c_int], C.c_size_t),
        "pcgb_gmw_position_add": ([C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
                                  C.c_int),
        "pcgb_gmw_dltsft_gates": ([C.c_int, C.c_int], C.c_size_t),
        "pcgb_gmw_dltsft": ([C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                             _vp], C.c_int),
        "pcgb_dpf_batch_full_eval_convert_device": ([C.c_int, C.c_int, C.c_int, _vp, _vp, _vp,
                                                     C.c_int, _vp, _vp, C.c_int, _vp, _vp, _vp],
                                                    C.c_int),
        "pcgb_dpf_batch_full_eval_convert_device_dx": ([C.c_int, C.c_int, C.c_int, _vp, _vp,
                                                        _vp, C.c_int, _vp, _vp, C.c_int, _vp,
                                                        _vp, _vp], C.c_int),
        "pcgb_dpf_out_convert_device": ([_vp, C.c_int, C.c_size_t, _vp, _vp, _vp, _vp], C.c_int),
        "pcgb_dpf_out_scatter_g_conv_device": ([_vp, C.c_int, C.c_size_t, C.c_int, C.c_int, _vp,
                                                _vp, C.c_int, _vp], C.c_int),
        "pcgb_out_beaver_open_device": ([C.c_int, C.c_int] + [_vp] * 6 + [_vp], C.c_int),
        "pcgb_out_beaver_close_device": ([C.c_int, C.c_int] + [_vp] * 6 + [_vp], C.c_int),
        "pcgb_add_mod_p_device": ([_vp, _vp, _vp, C.c_size_t, _vp], C.c_int),
        "pcgb_dpf_out_sums": ([_vp, C.c_int, C.c_size_t, C.c_uint64, _u64p, _u64p], C.c_int),
        "pcgb_dpf_out_scatter_g": ([_vp, C.c_int, C.c_size_t, C.c_int, C.c_int, C.c_uint64, _u64p,
                                    _u64p, C.c_int], C.c_int),
        "pcgb_dpf_out_sums_noalloc": ([_vp, C.c_int, C.c_size_t, C.c_uint64, _vp, _vp, _vp],
                                      C.c_int),
        "pcgb_poly_mul_supported": ([C.c_int, C.c_uint64, C.c_int, C.c_char_p, C.c_size_t],
                                    C.c_int),
        "pcgb_poly_mul_u64": ([C.c_int, _u64p, _u64p, _u64p, C.c_int, C.c_int, C.c_uint64,
                               C.POINTER(C.c_double)], C.c_int),
        "pcgb_aes128_expand_key": ([_u8p, _u8p], C.c_int),
        "pcgb_aes128_ecb_encrypt": ([_u8p, _u8p, _u8p, C.c_int], C.c_int),
        "pcgb_aes_tree_round_keys": ([_u8p, C.c_int, _u8p], C.c_int),
        "pcgb_dpf_keyed_full_eval": ([C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp],
                                     C.c_int),
        "pcgb_dpf_keyed_full_eval_multi": ([C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                            C.c_int, C.c_int, C.POINTER(_vp), C.POINTER(_vp),
                                            _vp, C.POINTER(_vp), _vp], C.c_int),
        "pcgb_poly_mul_device": ([_vp, _vp, _vp, C.c_int, C.c_int, _vp], C.c_int),
        "pcgb_poly_mul_device_multi": ([C.c_int, _vp, _vp, _vp, _vp, _vp], C.c_int),
        "pcgb_expander_create": ([C.POINTER(_vp), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _vp,
                                  _vp], C.c_int),
        "pcgb_expander_destroy": ([_vp], C.c_int),
        "pcgb_expander_info": ([_vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                C.POINTER(C.c_size_t)], C.c_int),
        "pcgb_expand_device": ([_vp, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp], C.c_int),
        "pcgb_expand_batch_device": ([C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
                                     C.c_int),
        "pcgb_expand_host": ([_vp, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp], C.c_int),
        "pcgb_expand_g_device": ([_vp, C.c_int, _vp, _vp, _vp, _vp, _vp], C.c_int),
        "pcgb_expander_set_profiling": ([_vp, C.c_int], C.c_int),
        "pcgb_expander_set_graph": ([_vp, C.c_int], C.c_int),
        "pcgb_expander_create_shard": ([_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _vp,
                                        _vp, C.c_int, C.c_int], C.c_int),
        "pcgb_expander_shard": ([_vp] * 5, C.c_int),
        "pcgb_expander_create_public_a0": ([C.POINTER(_vp), C.c_int, C.c_int, C.c_int, C.c_int,
                                            C.c_int, _vp, _vp], C.c_int),
        "pcgb_reduce_mod_p": ([_vp, _vp, C.c_size_t, _vp], C.c_int),
        "pcgb_expand_from_g_device": ([_vp] * 6 + [_vp], C.c_int),
        "pcgb_dpf_out_scatter_g_device": ([_vp, C.c_int, C.c_size_t, C.c_int, C.c_int, _vp, _vp,
                                           C.c_int, _vp], C.c_int),
        "pcgb_expander_autotune": ([_vp, C.POINTER(C.c_int)], C.c_int),
        "pcgb_expander_leaf_shape": ([_vp, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
        "pcgb_expander_set_leaf_shape": ([_vp, C.c_int, C.c_int], C.c_int),
        "pcgb_expand_host_async": ([_vp, C.c_int] + [_vp] * 7, C.c_int),
        "pcgb_expander_wait": ([_vp], C.c_int),
        "pcgb_expander_stage_times": ([_vp, C.POINTER(C.c_float), C.c_int], C.c_int),
        "pcgb_launch_count": ([], C.c_ulonglong),
        "pcgb_arx_peak": ([C.POINTER(C.c_double), C.POINTER(C.c_float)], C.c_int),
        "pcgb_arx_peak_samples": ([C.c_int, C.c_int, C.POINTER(C.c_double)], C.c_int),
        "pcgb_arx_peak_variant": ([C.c_uint32, C.c_int, C.c_int, C.POINTER(C.c_double)], C.c_int),
        "pcgb_event_create": ([C.POINTER(_vp)], C.c_int),
        "pcgb_event_destroy": ([_vp], C.c_int),
        "pcgb_event_record": ([_vp, _vp], C.c_int),
        "pcgb_event_elapsed": ([_vp, _vp, C.POINTER(C.c_float)], C.c_int),
        "pcgb_noise": ([C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int, _u64p, _u64p], C.c_int),
        "pcgb_public_a": ([C.c_int, C.c_int, C.c_uint64, _vp], C.c_int),
        "pcgb_deal_keys_device": ([_vp, C.c_uint64, _vp, _vp, _vp, _vp, _vp], C.c_int),
        "pcgb_server_create": ([C.POINTER(_vp), C.c_int, C.c_size_t, C.c_int, C.c_uint64], C.c_int),
        "pcgb_server_prepare": ([_vp, C.c_int, C.c_int, C.c_int], C.c_int),
        "pcgb_server_submit": ([_vp, C.POINTER(Request), C.POINTER(C.c_uint64)], C.c_int),
        "pcgb_server_wait": ([_vp, C.c_uint64, C.POINTER(Result), C.c_int], C.c_int),
        "pcgb_server_run_trace": ([_vp, C.POINTER(Request), C.c_int, C.POINTER(Result),
                                   C.c_double], C.c_int),
        "pcgb_server_stats": ([_vp, C.POINTER(C.c_int), C.POINTER(C.c_int),
                               C.POINTER(C.c_size_t), C.POINTER(C.c_int)], C.c_int),
        "pcgb_server_destroy": ([_vp, C.c_int], C.c_int),
        "pcgb_digest_device": ([_vp, C.c_size_t, _vp, _vp], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    return L


lib = _load()


def _check(rc):
    if rc != 0:
        raise PcgError(rc, lib.pcgb_last_error().decode(errors="replace"))


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _u8(x):
    if isinstance(x, (bytes, bytearray, memoryview)):
        return np.frombuffer(bytes(x), dtype=np.uint8).copy()
    return np.ascontiguousarray(x, dtype=np.uint8).reshape(-1)


def _blocks(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.uint64).reshape(-1, 2)
    if n is not None and a.shape[0] < n:
        raise ValueError(f"expected at least {n} blocks, got {a.shape[0]}")
    return a


# ---- device / runtime (poly_mul_cuda.h:13-16) ------------------------------
def is_cuda_available():
    return lib.pcgb_is_cuda_available() == 1


def device_name():
    buf = C.create_string_buffer(256)
    return buf.value.decode() if lib.pcgb_device_name(buf, 256) == 0 else "unavailable"


def runtime_version():
    buf = C.create_string_buffer(64)
    return buf.value.decode() if lib.pcgb_runtime_version(buf, 64) == 0 else "unavailable"


def set_device(dev):
    _check(lib.pcgb_set_device(dev))


def sm_count():
    n = C.c_int(0)
    _check(lib.pcgb_sm_count(C.byref(n)))
    return n.value


class DeviceBuffer:
    """Owning device allocation made by the library (no torch needed)."""

    def __init__(self, nbytes):
        self.nbytes = int(nbytes)
        p = C.c_void_p()
        _check(lib.pcgb_malloc(C.byref(p), max(self.nbytes, 1)))
        self.ptr = p.value

    def upload(self, arr):
        arr = np.ascontiguousarray(arr)
        assert arr.nbytes <= self.nbytes
        _check(lib.pcgb_memcpy_h2d(self.ptr, _p(arr), arr.nbytes, None))
        return self

    def upload_at(self, arr, offset):
        """Copy a host array into the buffer at byte `offset`."""
        arr = np.ascontiguousarray(arr)
        assert offset + arr.nbytes <= self.nbytes
        _check(lib.pcgb_memcpy_h2d(self.ptr + offset, _p(arr), arr.nbytes, None))
        return self

    def download(self, dtype, count):
        out = np.empty(count, dtype=dtype)
        _check(lib.pcgb_memcpy_d2h(_p(out), self.ptr, out.nbytes, None))
        return out

    def free(self):
        if self.ptr:
            lib.pcgb_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def to_device(arr):
    arr = np.ascontiguousarray(arr)
    return DeviceBuffer(arr.nbytes).upload(arr)


def synchronize():
    _check(lib.pcgb_device_synchronize())


def triples_device(N, party, d_x1, d_z1, d_x2, d_z2, d_a, d_b, d_c, stream=None):
    """One party's Beaver-triple slot shares from two ring OLEs (device)."""
    _check(lib.pcgb_triples_device(N, party, d_x1, d_z1, d_x2, d_z2, d_a, d_b, d_c, stream))


def verify_ole_device(N, d_x0, d_z0, d_x1, d_z1, d_bad, stream=None):
    """d_bad (one u64 on the device) := slots where x0*x1 != z0+z1."""
    _check(lib.pcgb_verify_ole_device(N, d_x0, d_z0, d_x1, d_z1, d_bad, stream))


def verify_triples_device(N, d_a0, d_b0, d_c0, d_a1, d_b1, d_c1, d_bad, stream=None):
    """d_bad (one u64 on the device) := slots where (a0+a1)(b0+b1) != c0+c1."""
    _check(lib.pcgb_verify_triples_device(N, d_a0, d_b0, d_c0, d_a1, d_b1, d_c1, d_bad, stream))


def reduce_mod_p(d_dst, d_src, count, stream=None):
    """d_dst[i] = d_src[i] mod p for any 64-bit words (device)."""
    _check(lib.pcgb_reduce_mod_p(d_dst, d_src, count, stream))


def trim_pool():
    """Return the library pool's cached scratch on the current device."""
    _check(lib.pcgb_trim_pool())


def launch_count():
    """Kernel launches issued by the library so far."""
    return lib.pcgb_launch_count()


def arx_peak():
    """(G int-ops/s, ms) of the ChaCha8 ARX throughput probe."""
    g, ms = C.c_double(), C.c_float()
    _check(lib.pcgb_arx_peak(C.byref(g), C.byref(ms)))
    return g.value, ms.value


def arx_peak_samples(reps=15, iters=16384):
    """G int-ops/s of each of `reps` launches of the ARX probe."""
    out = (C.c_double * reps)()
    _check(lib.pcgb_arx_peak_samples(reps, iters, out))
    return list(out)


def arx_peak_variant(add_mask, reps=7, iters=16384):
    """G int-ops/s of `reps` launches of the probe with the quarter-round
    adds of add_mask issued on the FMA pipe (pcgb_arx_peak_variant)."""
    out = (C.c_double * reps)()
    _check(lib.pcgb_arx_peak_variant(add_mask, reps, iters, out))
    return list(out)


def default_stream():
    return lib.pcgb_default_stream()


class Event:
    """CUDA event recorded on a library stream (default: the library's own)."""

    def __init__(self):
        p = C.c_void_p()
        _check(lib.pcgb_event_create(C.byref(p)))
        self.h = p.value

    def record(self, stream=None):
        _check(lib.pcgb_event_record(self.h, stream))

    def elapsed_ms(self, stop):
        ms = C.c_float()
        _check(lib.pcgb_event_elapsed(self.h, stop.h, C.byref(ms)))
        return ms.value

    def __del__(self):
        try:
            lib.pcgb_event_destroy(self.h)
        except Exception:
            pass


# ---- DPF (dpf_gpu.h:55-75) -------------------------------------------------
def _exchange_cb(exchange):
    """Wrap `exchange(my: ndarray[count,2]) -> peer ndarray` as a C callback."""
    if exchange is None:
        return None

    def cb(my, peer, count, user):
        try:
            m = np.ctypeslib.as_array(C.cast(my, C.POINTER(C.c_uint64)), shape=(count, 2))
            p = np.ctypeslib.as_array(C.cast(peer, C.POINTER(C.c_uint64)), shape=(count, 2))
            p[:] = np.asarray(exchange(m.copy()), dtype=np.uint64).reshape(count, 2)
            return 0
        except Exception:
            return 1

    return EXCHANGE_FN(cb)


def dpf_gpu_batch_full_eval(B, n, w, roots, dltsft, round_keys=None, party=0, exchange=None,
                            prg=PRG_AES):
    """Interactive batched full-domain evaluation; returns leaves [B*2^n, 2].

    exchange(my) -> peer shares (None = peer shares are zero, the reference
    benches' stub exchange).
    """
    roots = _blocks(roots, B)
    dltsft = _blocks(dltsft)
    out = np.zeros((B << n, 2), dtype=np.uint64)
    cb = _exchange_cb(exchange)
    rk = None if round_keys is None else _u8(round_keys)
    _check(lib.pcgb_dpf_batch_full_eval(B, n, w, _p(roots), _p(dltsft), _p(rk), party,
                                        C.cast(cb, C.c_void_p) if cb else None, None, _p(out), prg))
    return out


def dpf_gpu_batch_full_eval_device(B, n, w, roots, dltsft, round_keys=None, party=0,
                                   exchange=None, prg=PRG_AES):
    """Same, leaves stay on the device: returns the device pointer (int),
    valid until the next dpf_gpu_* call."""
    roots = _blocks(roots, B)
    dltsft = _blocks(dltsft)
    cb = _exchange_cb(exchange)
    rk = None if round_keys is None else _u8(round_keys)
    d = C.c_void_p()
    _check(lib.pcgb_dpf_batch_full_eval_device(B, n, w, _p(roots), _p(dltsft), _p(rk), party,
                                               C.cast(cb, C.c_void_p) if cb else None, None, prg,
                                               C.byref(d)))
    return d.value


# ---- boolean preprocessing, two-party GMW (dpf.cpp:171-283, adder.h:22-63) --
def gmw_position_add_gates(off_bits):
    """AND gates (triple rows) of the Kogge-Stone position adder."""
    return int(lib.pcgb_gmw_position_add_gates(off_bits))


def gmw_dltsft_gates(n, w):
    """AND gates (triple rows) of the DltSft circuit."""
    return int(lib.pcgb_gmw_dltsft_gates(n, w))


def _bool_triples(triples, rows, B):
    words = rows * ((B + 31) // 32)
    out = [np.ascontiguousarray(v, dtype=np.uint32).reshape(-1) for v in triples]
    if len(out) != 3 or any(v.size < words for v in out):
        raise ValueError(f"triples need 3 arrays of {words} uint32 words")
    return out


def gmw_position_add(party, my_off, off_bits, triples, exchange):
    """XOR shares of alpha = off0 + off1 (off_bits + 1 bits) for B instances.

    my_off: this party's B offsets; triples: (a, b, c) bit-sliced AND-triple
    shares, gmw_position_add_gates(off_bits) rows of ceil(B/32) words;
    exchange(my) -> peer message, as for the interactive DPF."""
    my_off = np.ascontiguousarray(my_off, dtype=np.uint64).reshape(-1)
    B = my_off.size
    ta, tb, tc = _bool_triples(triples, gmw_position_add_gates(off_bits), B)
    out = np.zeros(B, np.uint64)
    cb = _exchange_cb(exchange)
    _check(lib.pcgb_gmw_position_add(party, B, off_bits, _p(my_off), _p(ta), _p(tb), _p(tc),
                                     C.cast(cb, C.c_void_p) if cb else None, None, _p(out)))
    return out


def gmw_dltsft(party, alpha_share, delta_share, n, w, triples, exchange):
    """DltSft shares [B * n/w * (2^w-1), 2] of [digit_i(alpha) == k] * Delta.

    Returns (delta_share with lsb(Delta) forced, dltsft)."""
    alpha_share = np.ascontiguousarray(alpha_share, dtype=np.uint64).reshape(-1)
    B = alpha_share.size
    delta = _blocks(delta_share, B)[:B].copy()
    ta, tb, tc = _bool_triples(triples, gmw_dltsft_gates(n, w), B)
    out = np.zeros((B * (n // w) * ((1 << w) - 1), 2), np.uint64)
    cb = _exchange_cb(exchange)
    _check(lib.pcgb_gmw_dltsft(party, B, n, w, _p(alpha_share), _p(delta), _p(ta), _p(tb), _p(tc),
                               C.cast(cb, C.c_void_p) if cb else None, None, _p(out)))
    return delta, out


# ---- output layer (leaf_convert_cuda.h:43-52) ------------------------------
def dpf_out_sums(d_leaves, B, D, prime=P):
    """Per-instance sumC (mod p) and sumT of the device leaves."""
    sc, st = np.zeros(B, np.uint64), np.zeros(B, np.uint64)
    _check(lib.pcgb_dpf_out_sums(d_leaves, B, D, prime, sc, st))
    return sc, st


def dpf_out_scatter_g_device(d_leaves, B, D, t, party, d_cw, d_g, N, stream=None):
    """Folded g of the B instances into device d_g; CWs on the device."""
    _check(lib.pcgb_dpf_out_scatter_g_device(d_leaves, B, D, t, party, d_cw, d_g, N, stream))


def dpf_gpu_batch_full_eval_convert_device(B, n, w, roots, dltsft, d_conv, d_sumC, d_sumT,
                                           round_keys=None, party=0, exchange=None,
                                           prg=PRG_AES):
    """Interactive evaluation fused with the convert pass: converted words
    (B * 2^n) and sums into the device buffers; no leaves are stored."""
    roots = _blocks(roots, B)
    dltsft = _blocks(dltsft)
    cb = _exchange_cb(exchange)
    rk = None if round_keys is None else _u8(round_keys)
    _check(lib.pcgb_dpf_batch_full_eval_convert_device(
        B, n, w, _p(roots), _p(dltsft), _p(rk), party, C.cast(cb, C.c_void_p) if cb else None,
        None, prg, d_conv, d_sumC, d_sumT))


def dpf_gpu_batch_full_eval_convert_device_dx(B, n, w, roots, dltsft, d_conv, d_sumC, d_sumT,
                                              exchange_device, round_keys=None, party=0,
                                              prg=PRG_AES):
    """As dpf_gpu_batch_full_eval_convert_device, with the per-level CW
    shares exchanged between device arrays: exchange_device(d_my, d_peer,
    count) gets device pointers to `count` 16-byte shares and must fill
    d_peer (and have it landed) before returning."""
    roots = _blocks(roots, B)
    dltsft = _blocks(dltsft)

    def cb(my, peer, count, user):
        try:
            exchange_device(my, peer, count)
            return 0
        except Exception:
            return 1

    fn = EXCHANGE_FN(cb)
    rk = None if round_keys is None else _u8(round_keys)
    _check(lib.pcgb_dpf_batch_full_eval_convert_device_dx(
        B, n, w, _p(roots), _p(dltsft), _p(rk), party, C.cast(fn, C.c_void_p), None, prg, d_conv,
        d_sumC, d_sumT))


def dpf_out_convert_device(d_leaves, B, D, d_conv, d_sumC, d_sumT, stream=None):
    """Sums of the B instances into device d_sumC/d_sumT and each leaf's
    converted word C | tau << 63 into d_conv (B*D words)."""
    _check(lib.pcgb_dpf_out_convert_device(d_leaves, B, D, d_conv, d_sumC, d_sumT, stream))


def dpf_out_scatter_g_conv_device(d_conv, B, D, t, party, d_cw, d_g, N, stream=None):
    """Folded g from the converted words of dpf_out_convert_device."""
    _check(lib.pcgb_dpf_out_scatter_g_conv_device(d_conv, B, D, t, party, d_cw, d_g, N, stream))


def out_beaver_open_device(B, party, d_sumC, d_sumT, d_beta, d_r, d_s, d_de, stream=None):
    """This party's Beaver opening [<A> - r | <B> - s] (2B words) into d_de."""
    _check(lib.pcgb_out_beaver_open_device(B, party, d_sumC, d_sumT, d_beta, d_r, d_s, d_de,
                                           stream))


def out_beaver_close_device(B, party, d_de_my, d_de_peer, d_r, d_s, d_rs, d_cw, stream=None):
    """This party's share of CW = A*B from both openings."""
    _check(lib.pcgb_out_beaver_close_device(B, party, d_de_my, d_de_peer, d_r, d_s, d_rs, d_cw,
                                            stream))


def add_mod_p_device(d, u, v, count, stream=None):
    """d = (u + v) mod p over `count` device words."""
    _check(lib.pcgb_add_mod_p_device(d, u, v, count, stream))


def dpf_out_scatter_g(d_leaves, B, D, t, party, CW, N, prime=P):
    """Folded g (N residues) of the B instances' output layer."""
    CW = np.ascontiguousarray(CW, np.uint64)
    if B > 0 and CW.size < B:
        raise ValueError("CW needs B entries")
    g = np.zeros(N, np.uint64)
    _check(lib.pcgb_dpf_out_scatter_g(d_leaves, B, D, t, party, prime,
                                      CW, g, N))
    return g


# ---- poly-mul (poly_mul_cuda.h:14-31) --------------------------------------
def _supported(variant, prime, N):
    buf = C.create_string_buffer(256)
    ok = lib.pcgb_poly_mul_supported(variant, prime, N, buf, 256)
    return ok == 1, buf.value.decode()


def _mul(variant, a, b, batch, N, prime):
    a = np.ascontiguousarray(a, np.uint64).reshape(-1)
    b = np.ascontiguousarray(b, np.uint64).reshape(-1)
    if batch > 0 and (a.size < batch * N or b.size < batch * N):
        raise ValueError(f"poly-mul operands need batch*N = {batch * N} words")
    out = np.zeros(batch * N, np.uint64)
    ms = C.c_double(0)
    _check(lib.pcgb_poly_mul_u64(variant, out, a, b, batch, N, prime, C.byref(ms)))
    return out, ms.value


def poly_mul_supported(prime, N):
    return _supported(POLYMUL_V1, prime, N)


def poly_mul_u64(a, b, batch, N, prime=P):
    return _mul(POLYMUL_V1, a, b, batch, N, prime)


def poly_mul_gpuntt_supported(prime, N):
    return _supported(POLYMUL_MERGE, prime, N)


def poly_mul_u64_gpuntt(a, b, batch, N, prime=P):
    return _mul(POLYMUL_MERGE, a, b, batch, N, prime)


def poly_mul_gpuntt_4step_supported(prime, N):
    return _supported(POLYMUL_4STEP, prime, N)


def poly_mul_u64_gpuntt_4step(a, b, batch, N, prime=P):
    return _mul(POLYMUL_4STEP, a, b, batch, N, prime)


def poly_mul_gpuntt_square_supported(prime, N):
    return _supported(POLYMUL_SQUARE, prime, N)


def poly_mul_u64_gpuntt_square(a, b, batch, N, prime=P):
    return _mul(POLYMUL_SQUARE, a, b, batch, N, prime)


def poly_mul_device(d_c, d_a, d_b, batch, N, stream=None):
    _check(lib.pcgb_poly_mul_device(d_c, d_a, d_b, batch, N, stream))


# ---- AES (aes_gpu.h:13-19) --------------------------------------------------
def aes128_expand_key_host(key):
    rk = np.zeros(176, np.uint8)
    _check(lib.pcgb_aes128_expand_key(_u8(key), rk))
    return rk


def aes128_ecb_encrypt_gpu(keys, data):
    keys = _u8(keys)
    data = _u8(data)
    count = data.size // 16
    out = np.zeros(count * 16, np.uint8)
    _check(lib.pcgb_aes128_ecb_encrypt(keys, data, out, count))
    return out


def aes_tree_round_keys(master, nk):
    rk = np.zeros(176 * nk, np.uint8)
    _check(lib.pcgb_aes_tree_round_keys(_u8(master), nk, rk))
    return rk


# ---- keyed DPF / synthetic material ------------------------------------------
def dpf_keyed_full_eval_device(K, n, w, prg, d_roots, d_cws, d_leaves, round_keys=None,
                               stream=None):
    rk = None if round_keys is None else _u8(round_keys)
    _check(lib.pcgb_dpf_keyed_full_eval(K, n, w, prg, d_roots, d_cws, _p(rk), d_leaves, stream))


def dpf_keyed_full_eval_multi_device(groups, w, prg, round_keys=None, stream=None):
    """groups: [(K, n, d_roots, d_cws, d_leaves), ...] with device pointers;
    all groups share w and the PRG.  One launch per top-walk stage."""
    G = len(groups)
    Ks = (C.c_int * G)(*[int(g[0]) for g in groups])
    ns = (C.c_int * G)(*[int(g[1]) for g in groups])
    ptrs = [(C.c_void_p * G)(*[g[i] for g in groups]) for i in (2, 3, 4)]
    rk = None if round_keys is None else _u8(round_keys)
    _check(lib.pcgb_dpf_keyed_full_eval_multi(G, Ks, ns, w, prg, ptrs[0], ptrs[1], _p(rk),
                                              ptrs[2], stream))


def noise(N, c, t, seed, party):
    pos, val = np.zeros(c * t, np.uint64), np.zeros(c * t, np.uint64)
    _check(lib.pcgb_noise(N, c, t, seed, party, pos, val))
    return pos, val


def public_a(N, c, a_seed):
    a = np.zeros(max(c - 1, 1) * N, np.uint64)
    _check(lib.pcgb_public_a(N, c, a_seed, _p(a)))
    return a


class Expander:
    """Resident per-shape state of the fused PCG-OLE expansion (one device)."""

    def __init__(self, N, c, t, w=1, prg=PRG_CHACHA8, public_a=None, master_key=None,
                 rank=0, world=1, a0_public=False):
        """public_a: a_1 .. a_{c-1} (a_0 = 1, the reference's convention), or
        with a0_public=True all of a_0 .. a_{c-1}.  rank/world: this
        expander's shard of the pair blocks (see pcgb_expander_create_shard);
        Q is then the shard's own pair count."""
        self.N, self.c, self.t, self.w, self.prg = N, c, t, w, prg
        pa = None if public_a is None else np.ascontiguousarray(public_a, np.uint64)
        mk = None if master_key is None else _u8(master_key)
        h = C.c_void_p()
        if a0_public:
            if (rank, world) != (0, 1):
                raise ValueError("a0_public expanders are not sharded")
            _check(lib.pcgb_expander_create_public_a0(C.byref(h), N, c, t, w, prg, _p(pa),
                                                      _p(mk)))
        else:
            _check(lib.pcgb_expander_create_shard(C.byref(h), N, c, t, w, prg, _p(pa), _p(mk),
                                                  rank, world))
        self.h = h.value
        K, L, nk, sb = C.c_int(), C.c_int(), C.c_int(), C.c_size_t()
        _check(lib.pcgb_expander_info(self.h, C.byref(K), C.byref(L), C.byref(nk), C.byref(sb)))
        self.K, self.levels, self.nk, self.scratch_bytes = K.value, L.value, nk.value, sb.value
        r, wd, ql, qt = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _check(lib.pcgb_expander_shard(self.h, C.byref(r), C.byref(wd), C.byref(ql), C.byref(qt)))
        self.rank, self.world, self.Q, self.Q_total = r.value, wd.value, ql.value, qt.value

    def close(self):
        if getattr(self, "h", None):
            lib.pcgb_expander_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def expand_device(self, party, d_roots, d_cws, d_cw_out, d_pos, d_val, d_x, d_z, stream=None):
        _check(lib.pcgb_expand_device(self.h, party, d_roots, d_cws, d_cw_out, d_pos, d_val, d_x,
                                      d_z, stream))

    def expand_host(self, party, roots, cws, cw_out, pos, val):
        roots = _blocks(roots, self.K)
        cws = _blocks(cws, self.K * self.levels * self.nk)
        cw_out = np.ascontiguousarray(cw_out, np.uint64)
        pos = np.ascontiguousarray(pos, np.uint64)
        val = np.ascontiguousarray(val, np.uint64)
        x, z = np.zeros(self.N, np.uint64), np.zeros(self.N, np.uint64)
        _check(lib.pcgb_expand_host(self.h, party, _p(roots), _p(cws), _p(cw_out), _p(pos),
                                    _p(val), _p(x), _p(z)))
        return x, z

    def expand_g_device(self, party, d_roots, d_cws, d_cw_out, d_g, stream=None):
        _check(lib.pcgb_expand_g_device(self.h, party, d_roots, d_cws, d_cw_out, d_g, stream))

    def deal_keys_device(self, seed, d_roots0, d_roots1, d_cws, d_cw_out, stream=None):
        _check(lib.pcgb_deal_keys_device(self.h, seed, d_roots0, d_roots1, d_cws, d_cw_out,
                                         stream))

    def expand_from_g_device(self, d_g, d_pos, d_val, d_x, d_z, stream=None):
        """Step 4 (x, z) from c*c caller-computed folded blocks g_ij."""
        _check(lib.pcgb_expand_from_g_device(self.h, d_g, d_pos, d_val, d_x, d_z, stream))

    def set_graph(self, enable=True):
        """Replay expand_device as a CUDA graph (see pcgb_expander_set_graph)."""
        _check(lib.pcgb_expander_set_graph(self.h, 1 if enable else 0))

    def autotune(self):
        """Pick the fused leaf kernel's shape (leaves per thread, CTA size)
        for this expansion shape; returns the CTA size."""
        v = C.c_int()
        _check(lib.pcgb_expander_autotune(self.h, C.byref(v)))
        K, L, nk, sb = C.c_int(), C.c_int(), C.c_int(), C.c_size_t()
        _check(lib.pcgb_expander_info(self.h, C.byref(K), C.byref(L), C.byref(nk), C.byref(sb)))
        self.scratch_bytes = sb.value
        return v.value

    def set_leaf_shape(self, tpb, leaves_per_thread):
        """Pin the fused leaf kernel's shape (one of the autotuner's candidates)."""
        _check(lib.pcgb_expander_set_leaf_shape(self.h, int(tpb), int(leaves_per_thread)))
        K, L, nk, sb = C.c_int(), C.c_int(), C.c_int(), C.c_size_t()
        _check(lib.pcgb_expander_info(self.h, C.byref(K), C.byref(L), C.byref(nk), C.byref(sb)))
        self.scratch_bytes = sb.value

    def leaf_shape(self):
        """(CTA threads, leaves per thread) of the fused leaf kernel."""
        tpb, lpt = C.c_int(), C.c_int()
        _check(lib.pcgb_expander_leaf_shape(self.h, C.byref(tpb), C.byref(lpt)))
        return tpb.value, lpt.value

    def set_profiling(self, slots):
        """Record per-stage events for the next `slots` expansions (0 = off)."""
        _check(lib.pcgb_expander_set_profiling(self.h, int(slots)))
        self._slots = int(slots)

    def stage_times(self):
        """[(tops, leaf_gather, x, ntt) ms] of the recorded expansions."""
        n = max(getattr(self, "_slots", 0), 1)
        ms = (C.c_float * (4 * n))()
        r = lib.pcgb_expander_stage_times(self.h, ms, n)
        if r < 0:
            _check(r)
        return [tuple(ms[4 * i: 4 * i + 4]) for i in range(r)]


def expand_batch_device(requests, stream=None):
    """Several expansions as one batch (pcgb_expand_batch_device).
    requests: list of (Expander, party, d_roots, d_cws, d_cw_out, d_pos, d_val,
    d_x, d_z), the pointers device addresses (ints)."""
    n = len(requests)
    if n == 0:
        return
    col = lambda k: (C.c_void_p * n)(*[r[k] for r in requests])
    _check(lib.pcgb_expand_batch_device(n, (C.c_void_p * n)(*[r[0].h for r in requests]),
                                        (C.c_int * n)(*[r[1] for r in requests]), col(2), col(3),
                                        col(4), col(5), col(6), col(7), col(8), stream))


def digest_device(d_v, n, stream=None):
    """Order-independent 64-bit digest of n device words (bit-exactness checks)."""
    out = DeviceBuffer(8)
    _check(lib.pcgb_digest_device(d_v, n, out.ptr, stream))
    _check(lib.pcgb_stream_synchronize(stream))
    return int(out.download(np.uint64, 1)[0])


class Server:
    """Continuous-batching expansion server on the current device.
    max_in_flight (default 8 x n_streams) above n_streams lets small
    requests of mixed shapes run as batches (pcgb_server_create)."""

    def __init__(self, n_streams=4, mem_budget=0, max_in_flight=None, a_seed=7):
        h = C.c_void_p()
        _check(lib.pcgb_server_create(C.byref(h), n_streams, mem_budget,
                                      max_in_flight or 8 * n_streams, a_seed))
        self.h = h.value

    def prepare(self, N, c, t):
        _check(lib.pcgb_server_prepare(self.h, N, c, t))

    def submit(self, N, c, t, seed, party=0):
        r = Request(N, c, t, party, seed, 0.0)
        tk = C.c_uint64()
        _check(lib.pcgb_server_submit(self.h, C.byref(r), C.byref(tk)))
        return tk.value

    def wait(self, ticket, timeout_ms=-1):
        res = Result()
        _check(lib.pcgb_server_wait(self.h, ticket, C.byref(res), timeout_ms))
        return res

    def run_trace(self, reqs, timeout_s=600.0):
        """reqs: list of (N, c, t, party, seed, arrival_s); returns list of Result."""
        arr = (Request * len(reqs))(*[Request(*r) for r in reqs])
        out = (Result * len(reqs))()
        _check(lib.pcgb_server_run_trace(self.h, arr, len(reqs), out, timeout_s))
        return list(out)

    def stats(self):
        p, f, b, n = C.c_int(), C.c_int(), C.c_size_t(), C.c_int()
        _check(lib.pcgb_server_stats(self.h, C.byref(p), C.byref(f), C.byref(b), C.byref(n)))
        return {"pending": p.value, "in_flight": f.value, "bytes_in_flight": b.value,
                "plans": n.value}

    def close(self, timeout_ms=60000):
        if getattr(self, "h", None):
            h, self.h = self.h, None
            _check(lib.pcgb_server_destroy(h, timeout_ms))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

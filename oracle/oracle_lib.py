"""ctypes bindings for the CPU oracle (oracle/liboracle.so) and for the
reference code compiled from its own sources (oracle/_ref/*.so).

Test infrastructure only: used by tests/, the smoke check and bench.py's CPU
baseline leg; the library under test never imports this module.
"""
import ctypes as C
import os

import numpy as np

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
P = 4611686018326724609
PRG_AES, PRG_CHACHA8 = 0, 1

u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")

# A node array is a uint64 array of shape (..., 2): [..., 0] = lo, [..., 1] = hi.


class Blk(C.Structure):
    _fields_ = [("lo", C.c_uint64), ("hi", C.c_uint64)]


class Shape(C.Structure):
    _fields_ = [(k, C.c_int) for k in ("N", "c", "t", "w", "prg", "n", "levels", "nk", "K")]


EXCHANGE_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p)

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(ORACLE_DIR, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle not built: run `make -C oracle`")
        L = C.CDLL(path)
        L.orc_prime.restype = C.c_uint64
        L.orc_chacha8_block.argtypes = [u32p, C.c_uint64, C.c_uint64, u32p]
        L.orc_tree_hash_chacha8.argtypes = [u64p, u64p, C.c_size_t, C.c_int]
        L.orc_out_hash_lo64.argtypes = [Blk]
        L.orc_out_hash_lo64.restype = C.c_uint64
        L.orc_aes128_expand_key.argtypes = [u8p, u8p]
        L.orc_aes128_encrypt.argtypes = [u8p, u8p, u8p]
        L.orc_aes_tree_round_keys.argtypes = [u8p, C.c_int, u8p]
        L.orc_tree_hash_aes.argtypes = [u64p, u64p, C.c_size_t, C.c_int, u8p]
        L.orc_dpf_batch_full_eval.argtypes = [C.c_int, C.c_int, C.c_int, u64p, u64p,
                                              C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, u64p]
        L.orc_dpf_batch_full_eval_2p.argtypes = [C.c_int, C.c_int, C.c_int, u64p, u64p, u64p,
                                                 u64p, C.c_void_p, C.c_int, u64p, u64p, C.c_void_p]
        L.orc_dpf_keyed_full_eval.argtypes = [C.c_int, C.c_int, C.c_int, u64p, u64p,
                                              C.c_void_p, C.c_int, u64p]
        L.orc_dpf_eval.argtypes = [Blk, u64p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_uint64]
        L.orc_dpf_eval.restype = Blk
        L.orc_dpf_deal.argtypes = [C.c_int, C.c_int, Blk, Blk, C.c_uint64, C.c_uint64,
                                   C.c_void_p, C.c_int, u64p, C.POINTER(C.c_uint64),
                                   C.c_void_p, C.c_void_p]
        L.orc_out_sums.argtypes = [u64p, C.c_int, C.c_size_t, u64p, u64p]
        L.orc_out_scatter_g.argtypes = [u64p, C.c_int, C.c_size_t, C.c_int, C.c_int, u64p,
                                        u64p, C.c_int]
        L.orc_poly_mul.argtypes = [u64p, u64p, u64p, C.c_int, C.c_int]
        L.orc_poly_mul_schoolbook.argtypes = [u64p, u64p, u64p, C.c_int]
        L.orc_ntt_forward.argtypes = [u64p, C.c_int, C.c_int]
        L.orc_triples.argtypes = [C.c_int, C.c_int, u64p, u64p, u64p, u64p, u64p, u64p, u64p]
        L.orc_mulmod.argtypes = [C.c_uint64, C.c_uint64]
        L.orc_mulmod.restype = C.c_uint64
        L.orc_rnd.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
        L.orc_rnd.restype = C.c_uint64
        L.orc_shape_init.argtypes = [C.POINTER(Shape), C.c_int, C.c_int, C.c_int, C.c_int,
                                     C.c_int]
        L.orc_noise.argtypes = [C.POINTER(Shape), C.c_uint64, C.c_int, u64p, u64p]
        L.orc_public_a.argtypes = [C.POINTER(Shape), C.c_uint64, u64p]
        L.orc_deal_keys.argtypes = [C.POINTER(Shape), C.c_uint64, C.c_void_p, u64p, u64p,
                                    u64p, u64p]
        L.orc_expand.argtypes = [C.POINTER(Shape), C.c_int, u64p, u64p, u64p, u64p, u64p,
                                 u64p, C.c_void_p, C.c_uint64, C.c_int, u64p, u64p,
                                 C.c_void_p]
        L.orc_step4.argtypes = [C.c_int, C.c_int, C.c_int, u64p, u64p, u64p, u64p, u64p, u64p]
        L.orc_mt64_fill.argtypes = [C.c_uint64, u64p, C.c_size_t]
        L.orc_bench_sample.argtypes = [C.POINTER(Shape), C.c_int, u64p, u64p, u64p, u64p,
                                       C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_bench_block.argtypes = [C.POINTER(Shape), C.c_int, u64p, u64p, u64p, u64p,
                                      C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def blocks(n):
    return np.zeros((n, 2), dtype=np.uint64)


def chacha8_block(key_words, counter, nonce):
    out = np.zeros(16, np.uint32)
    lib().orc_chacha8_block(np.ascontiguousarray(key_words, np.uint32), counter, nonce, out)
    return out


def out_hash_lo64(lo, hi):
    return lib().orc_out_hash_lo64(Blk(int(lo), int(hi)))


def aes_expand_key(key16):
    rk = np.zeros(176, np.uint8)
    lib().orc_aes128_expand_key(np.ascontiguousarray(key16, np.uint8), rk)
    return rk


def aes_encrypt(rk, pt16):
    out = np.zeros(16, np.uint8)
    lib().orc_aes128_encrypt(rk, np.ascontiguousarray(pt16, np.uint8), out)
    return out


def aes_tree_round_keys(master16, nk):
    rks = np.zeros(176 * nk, np.uint8)
    lib().orc_aes_tree_round_keys(np.ascontiguousarray(master16, np.uint8), nk, rks)
    return rks


def tree_hash(parents, nk, prg=PRG_CHACHA8, rks=None):
    parents = np.ascontiguousarray(parents, np.uint64).reshape(-1, 2)
    out = blocks(parents.shape[0] * nk)
    if prg == PRG_CHACHA8:
        lib().orc_tree_hash_chacha8(out, parents, parents.shape[0], nk)
    else:
        lib().orc_tree_hash_aes(out, parents, parents.shape[0], nk, rks)
    return out


def dpf_batch_full_eval(B, n, w, roots, dltsft, prg=PRG_CHACHA8, rks=None, exchange=None):
    """exchange: None (peer share = 0) or python callable(my ndarray) -> peer ndarray."""
    out = blocks(B << n)
    cb = None
    if exchange is not None:
        def _cb(my, peer, count, user):
            m = np.ctypeslib.as_array(C.cast(my, C.POINTER(C.c_uint64)), shape=(count, 2))
            p = np.ctypeslib.as_array(C.cast(peer, C.POINTER(C.c_uint64)), shape=(count, 2))
            p[:] = exchange(m.copy())
        cb = EXCHANGE_FN(_cb)
    rc = lib().orc_dpf_batch_full_eval(B, n, w, np.ascontiguousarray(roots, np.uint64),
                                       np.ascontiguousarray(dltsft, np.uint64),
                                       _ptr(rks), prg, C.cast(cb, C.c_void_p) if cb else None,
                                       None, out)
    assert rc == 0, rc
    return out


def dpf_full_eval_2p(B, n, w, roots0, roots1, dlt0, dlt1, prg=PRG_CHACHA8, rks=None):
    l0, l1 = blocks(B << n), blocks(B << n)
    nk = (1 << w) - 1
    cws = blocks(B * (n // w) * nk)
    rc = lib().orc_dpf_batch_full_eval_2p(B, n, w, roots0, roots1, dlt0, dlt1, _ptr(rks), prg,
                                          l0, l1, _ptr(cws))
    assert rc == 0, rc
    return l0, l1, cws


def dpf_keyed_full_eval(K, n, w, roots, cws, prg=PRG_CHACHA8, rks=None):
    out = blocks(K << n)
    rc = lib().orc_dpf_keyed_full_eval(K, n, w, np.ascontiguousarray(roots, np.uint64),
                                       np.ascontiguousarray(cws, np.uint64), _ptr(rks), prg, out)
    assert rc == 0, rc
    return out


def dpf_deal(n, w, root0, delta, alpha, beta, prg=PRG_CHACHA8, rks=None, dlt0=None):
    nk = (1 << w) - 1
    levels = n // w
    cws = blocks(levels * nk)
    cw_out = C.c_uint64(0)
    dlt1 = blocks(levels * nk) if dlt0 is not None else None
    rc = lib().orc_dpf_deal(n, w, Blk(*map(int, root0)), Blk(*map(int, delta)), alpha, beta,
                            _ptr(rks), prg, cws, C.byref(cw_out), _ptr(dlt0), _ptr(dlt1))
    assert rc == 0, rc
    return cws, cw_out.value, dlt1


def out_sums(leaves, B, D):
    sc, st = np.zeros(B, np.uint64), np.zeros(B, np.uint64)
    lib().orc_out_sums(np.ascontiguousarray(leaves, np.uint64), B, D, sc, st)
    return sc, st


def out_scatter_g(leaves, B, D, t, party, CW, N):
    g = np.zeros(N, np.uint64)
    lib().orc_out_scatter_g(np.ascontiguousarray(leaves, np.uint64), B, D, t, party,
                            np.ascontiguousarray(CW, np.uint64), g, N)
    return g


def poly_mul(a, b, N):
    a = np.ascontiguousarray(a, np.uint64).reshape(-1)
    b = np.ascontiguousarray(b, np.uint64).reshape(-1)
    c = np.zeros_like(a)
    lib().orc_poly_mul(c, a, b, a.size // N, N)
    return c


def ntt_forward(a, N):
    """Negacyclic forward NTT (slot k = A(psi^(2k+1))) of each length-N row."""
    x = np.array(a, dtype=np.uint64).reshape(-1).copy()
    lib().orc_ntt_forward(x, x.size // N, N)
    return x


def triples(N, party, x1, z1, x2, z2):
    """One party's (a, b, c) Beaver-triple slot shares from two ring OLEs."""
    arrs = [np.ascontiguousarray(v, np.uint64) for v in (x1, z1, x2, z2)]
    a, b, c = (np.zeros(N, np.uint64) for _ in range(3))
    lib().orc_triples(N, party, *arrs, a, b, c)
    return a, b, c


def poly_mul_schoolbook(a, b, N):
    c = np.zeros(N, np.uint64)
    lib().orc_poly_mul_schoolbook(c, np.ascontiguousarray(a, np.uint64),
                                  np.ascontiguousarray(b, np.uint64), N)
    return c


def mt64(seed, n):
    out = np.zeros(n, np.uint64)
    lib().orc_mt64_fill(seed, out, n)
    return out


def shape(N, c, t, w=1, prg=PRG_CHACHA8):
    s = Shape()
    assert lib().orc_shape_init(C.byref(s), N, c, t, w, prg) == 0
    return s


def noise(s, seed, party):
    n = s.c * s.t
    pos, val = np.zeros(n, np.uint64), np.zeros(n, np.uint64)
    lib().orc_noise(C.byref(s), seed, party, pos, val)
    return pos, val


def public_a(s, a_seed):
    a = np.zeros(max(s.c - 1, 1) * s.N, np.uint64)
    lib().orc_public_a(C.byref(s), a_seed, a)
    return a


def deal_keys(s, seed, rks=None):
    r0, r1 = blocks(s.K), blocks(s.K)
    cws = blocks(s.K * s.levels * s.nk)
    cw_out = np.zeros(s.K, np.uint64)
    rc = lib().orc_deal_keys(C.byref(s), seed, _ptr(rks), r0, r1, cws, cw_out)
    assert rc == 0, rc
    return r0, r1, cws, cw_out


def expand(s, party, roots, cws, cw_out, pos, val, a, rks=None, blocks_mask=(1 << 64) - 1,
           threads=1, want_g=False):
    x, z = np.zeros(s.N, np.uint64), np.zeros(s.N, np.uint64)
    g = np.zeros(s.c * s.c * s.N, np.uint64) if want_g else None
    rc = lib().orc_expand(C.byref(s), party, roots, cws, cw_out, pos, val, a, _ptr(rks),
                          blocks_mask, threads, x, z, _ptr(g))
    assert rc == 0, rc
    return (x, z, g) if want_g else (x, z)


def step4(N, c, t, pos, val, a_all, g):
    """x, z from the c*c block outputs g and all c public polynomials a_all
    (a_0 included)."""
    x, z = np.zeros(N, np.uint64), np.zeros(N, np.uint64)
    rc = lib().orc_step4(N, c, t, np.ascontiguousarray(pos, np.uint64),
                         np.ascontiguousarray(val, np.uint64),
                         np.ascontiguousarray(a_all, np.uint64), np.ascontiguousarray(g, np.uint64),
                         x, z)
    assert rc == 0, rc
    return x, z


# ---- reference code compiled from its own sources (oracle/_ref) -----------
_ref_cpu = None
_ref_gpu = None


def ref_cpu():
    """CPU_baseline/chacha8.h + ntt.h, compiled in place; None if not built."""
    global _ref_cpu
    if _ref_cpu is None:
        path = os.path.join(ORACLE_DIR, "_ref", "libref_cpu.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.ref_chacha8_keystream.argtypes = [u8p, C.c_uint64, C.c_uint64, u8p, C.c_size_t]
        L.ref_ntt_poly_mul.argtypes = [u64p, u64p, u64p, C.c_int, C.c_int]
        L.ref_ntt_forward.argtypes = [u64p, C.c_int, C.c_int]
        L.ref_negacyclic_psi.argtypes = [C.c_int]
        L.ref_negacyclic_psi.restype = C.c_uint64
        _ref_cpu = L
    return _ref_cpu


def ref_gpu():
    """GPU_baseline/common/*.cu compiled for sm_100a; None if not built."""
    global _ref_gpu
    if _ref_gpu is None:
        path = os.path.join(ORACLE_DIR, "_ref", "libref_gpu.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.ref_last_error.restype = C.c_char_p
        L.ref_dpf_batch_full_eval.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p,
                                              C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                              C.c_void_p, C.c_void_p, C.c_int]
        L.ref_dpf_batch_full_eval_device.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p,
                                                     C.c_void_p, C.c_void_p, C.c_int,
                                                     C.c_void_p, C.c_void_p, C.c_int,
                                                     C.POINTER(C.c_void_p)]
        L.ref_dpf_out_sums.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.c_uint64, u64p, u64p]
        L.ref_dpf_out_scatter_g.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.c_int, C.c_int,
                                            C.c_uint64, u64p, u64p, C.c_int]
        L.ref_poly_mul_u64.argtypes = [u64p, u64p, u64p, C.c_int, C.c_int, C.c_uint64,
                                       C.POINTER(C.c_double)]
        L.ref_aes128_ecb_encrypt_gpu.argtypes = [u8p, u8p, u8p, C.c_int]
        L.ref_h2d.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        L.ref_malloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
        L.ref_free.argtypes = [C.c_void_p]
        _ref_gpu = L
    return _ref_gpu


def bench_block(s, party, roots, cws, cw_out, a, blk, n_polymuls, threads):
    """Wall seconds of one whole (i,j) block of one party's expansion (all its
    keys through DPF + convert + scatter) plus n_polymuls step-4 products, on
    `threads` host threads."""
    sec = C.c_double()
    rc = lib().orc_bench_block(C.byref(s), party, np.ascontiguousarray(roots, np.uint64),
                               np.ascontiguousarray(cws, np.uint64),
                               np.ascontiguousarray(cw_out, np.uint64),
                               np.ascontiguousarray(a, np.uint64), blk, n_polymuls, threads,
                               C.byref(sec))
    assert rc == 0, rc
    return sec.value


def bench_sample(s, party, roots, cws, cw_out, a, n_blocks, keys_per_block, n_polymuls, threads):
    """Times a bounded sample of one party's expansion on the host:
    DPF + convert of n_blocks x keys_per_block keys and n_polymuls negacyclic
    products of length N, on `threads` threads.  Returns (t_dpf_s, t_ntt_s)."""
    t1, t2 = C.c_double(), C.c_double()
    rc = lib().orc_bench_sample(C.byref(s), party, np.ascontiguousarray(roots, np.uint64),
                                np.ascontiguousarray(cws, np.uint64),
                                np.ascontiguousarray(cw_out, np.uint64),
                                np.ascontiguousarray(a, np.uint64), n_blocks, keys_per_block,
                                n_polymuls, threads, C.byref(t1), C.byref(t2))
    assert rc == 0, rc
    return t1.value, t2.value

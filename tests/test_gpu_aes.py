"""AES-128 drop-ins against the FIPS-197 vector and the oracle
(GPU_baseline/test/aes_gpu.cpp restated)."""
import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu


def test_fips197_kat(pcg):
    key = np.arange(16, dtype=np.uint8)
    pt = bytes.fromhex("00112233445566778899aabbccddeeff")
    out = pcg.aes128_ecb_encrypt_gpu(key, pt)
    assert out.tobytes().hex() == "69c4e0d86a7b0430d8cdb78070b4c55a"


def test_random_blocks_match_oracle(pcg):
    count = 8192
    r = O.mt64(0xC0FFEE, 2 * count * 16).astype(np.uint8)
    keys, data = r[: count * 16], r[count * 16:]
    out = pcg.aes128_ecb_encrypt_gpu(keys, data)
    for i in range(0, count, 37):
        rk = O.aes_expand_key(keys[16 * i: 16 * i + 16])
        assert (out[16 * i: 16 * i + 16] == O.aes_encrypt(rk, data[16 * i: 16 * i + 16])).all()


def test_key_schedule_and_tree_keys_match_oracle(pcg):
    rng = np.random.default_rng(2)
    for _ in range(16):
        k = rng.integers(0, 256, 16, dtype=np.uint8)
        assert (pcg.aes128_expand_key_host(k) == O.aes_expand_key(k)).all()
    for nk in (1, 3, 7, 15):
        m = rng.integers(0, 256, 16, dtype=np.uint8)
        assert (pcg.aes_tree_round_keys(m, nk) == O.aes_tree_round_keys(m, nk)).all()

"""Seeded synthetic Goldilocks inputs: ChaCha20 (RFC 8439 block function) keyed by a 32-byte
seed, read as little-endian u64 words.

Element i of a stream is word i of the keystream (block i // 8, nonce 0).  A word >= p is
redrawn: it is replaced by the first word < p of block i of the keystream with nonce 1 (a
second independent stream), so every element depends on its index only and the device
generator (glc_fill_random) produces the same values in parallel.
"""
from __future__ import annotations

import hashlib

import numpy as np

P = 0xFFFFFFFF00000001
_CONST = np.array([0x61707865, 0x3320646E, 0x79622D32, 0x6B206574], dtype=np.uint32)


def seed_bytes(seed) -> bytes:
    """32-byte key from an int / str / bytes seed (ints and strings are hashed with SHA-256)."""
    if isinstance(seed, (bytes, bytearray)) and len(seed) == 32:
        return bytes(seed)
    if isinstance(seed, int):
        seed = seed.to_bytes(8, "little", signed=False)
    if isinstance(seed, str):
        seed = seed.encode()
    return hashlib.sha256(bytes(seed)).digest()


def _rotl(x, n):
    return (x << np.uint32(n)) | (x >> np.uint32(32 - n))


def chacha20_blocks(key: bytes, counters: np.ndarray, nonce: int = 0) -> np.ndarray:
    """Keystream blocks for the given 32-bit counters: array (len(counters), 16) of uint32."""
    k = np.frombuffer(key, dtype="<u4").astype(np.uint32)
    n = len(counters)
    st = np.empty((16, n), dtype=np.uint32)
    st[0:4] = _CONST[:, None]
    st[4:12] = k[:, None]
    st[12] = counters.astype(np.uint32)
    st[13] = np.uint32(nonce & 0xFFFFFFFF)
    st[14] = np.uint32((nonce >> 32) & 0xFFFFFFFF)
    st[15] = np.uint32(0)
    x = st.copy()

    def qr(a, b, c, d):
        x[a] += x[b]; x[d] ^= x[a]; x[d] = _rotl(x[d], 16)
        x[c] += x[d]; x[b] ^= x[c]; x[b] = _rotl(x[b], 12)
        x[a] += x[b]; x[d] ^= x[a]; x[d] = _rotl(x[d], 8)
        x[c] += x[d]; x[b] ^= x[c]; x[b] = _rotl(x[b], 7)

    with np.errstate(over="ignore"):
        for _ in range(10):
            qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15)
            qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14)
        x += st
    return x.T.copy()


def _words(blocks: np.ndarray) -> np.ndarray:
    # 16 LE u32 -> 8 LE u64 per block
    return blocks.astype("<u4").view("<u8").reshape(-1)


def random_field_elements(seed, count: int, offset: int = 0) -> np.ndarray:
    """Elements offset .. offset+count of the stream, uniform in [0, p)."""
    key = seed_bytes(seed)
    if count == 0:
        return np.zeros(0, dtype=np.uint64)
    first, last = offset // 8, (offset + count - 1) // 8
    words = _words(chacha20_blocks(key, np.arange(first, last + 1, dtype=np.uint64)))
    out = words[offset - first * 8: offset - first * 8 + count].astype(np.uint64).copy()
    bad = np.nonzero(out >= np.uint64(P))[0]
    for j in bad:
        idx = offset + int(j)
        alt = _words(chacha20_blocks(key, np.array([idx], dtype=np.uint64), nonce=1))
        ok = alt[alt < np.uint64(P)]
        out[j] = ok[0] if len(ok) else alt[0] % np.uint64(P)
    return out


def fill_device(buf, seed, offset: int = 0, stream=None) -> None:
    """Fills a device buffer with elements offset.. of the stream (glc_fill_random), same values
    as random_field_elements."""
    from ._buffers import as_slice, stream_handle
    from ._lib import call
    ptr, n = as_slice(buf)
    call("glc_fill_random", ptr, n, offset, seed_bytes(seed), stream_handle(stream))

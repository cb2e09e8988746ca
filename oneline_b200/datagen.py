"""Seeded synthetic documents and pattern sets (ctypes over gen/libolgen.so).

* ``generate(profile, nbytes, seed)`` — the reference's test-document generator
  (crates/oneline-core/src/datagen.rs:159-253), restated in ``gen/datagen.c``.
* ``corpus(nbytes, seed)`` — the benchmark documents (depth walk 0..16 rendered as
  ``|`` runs, 5% empty lines, 70% marker lines, printable payloads of mean 40 B).
* ``patterns_*`` — the benchmark pattern sets.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GEN_SRC = os.path.join(HERE, "gen", "datagen.c")
GEN_LIB = os.path.join(HERE, "gen", "libolgen.so")

REPEAT, SHORT_LINES, MIXED, LONG_LINES, PROSE, NESTED = range(6)
PROFILES = {"repeat": REPEAT, "short-lines": SHORT_LINES, "mixed": MIXED, "long-lines": LONG_LINES,
            "prose": PROSE, "nested": NESTED}
ALL_PROFILES = (REPEAT, SHORT_LINES, MIXED, LONG_LINES, PROSE, NESTED)


def build(force: bool = False) -> str:
    if not force and os.path.exists(GEN_LIB) and os.path.getmtime(GEN_LIB) >= os.path.getmtime(GEN_SRC):
        return GEN_LIB
    subprocess.run(["gcc", "-O3", "-fPIC", "-shared", GEN_SRC, "-o", GEN_LIB, "-lm"], check=True)
    return GEN_LIB


_lib = None


def _l():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(GEN_LIB)
        u64 = ctypes.c_uint64
        L.olg_generate_profile.argtypes = [ctypes.c_int, u64, u64, ctypes.c_void_p, u64]
        L.olg_generate_profile.restype = u64
        L.olg_generate_corpus.argtypes = [u64, u64, ctypes.c_void_p, u64]
        L.olg_generate_corpus.restype = u64
        L.olg_generate_patterns.argtypes = [ctypes.c_int, ctypes.c_void_p, u64, u64, ctypes.c_uint32,
                                            ctypes.c_void_p, u64, ctypes.c_void_p]
        L.olg_generate_patterns.restype = u64
        L.olg_lognormal_sizes.argtypes = [u64, ctypes.c_uint32, ctypes.c_double, ctypes.c_double, u64, u64,
                                          ctypes.c_void_p]
        L.olg_poisson_arrivals.argtypes = [u64, ctypes.c_uint32, ctypes.c_double, ctypes.c_void_p]
        L.olg_prose_word.argtypes = [ctypes.c_uint32, ctypes.c_char_p]
        L.olg_prose_word.restype = ctypes.c_uint32
        L.olg_rng_seed_state.argtypes = [u64]
        L.olg_rng_seed_state.restype = u64
        L.olg_rng_next.argtypes = [ctypes.POINTER(u64)]
        L.olg_rng_next.restype = u64
        _lib = L
    return _lib


class Rng:
    """xorshift64* of crates/oneline-core/src/datagen.rs:53-82."""

    def __init__(self, seed: int):
        self._s = ctypes.c_uint64(_l().olg_rng_seed_state(seed & (2**64 - 1)))

    def next_u64(self) -> int:
        return _l().olg_rng_next(ctypes.byref(self._s))

    def below(self, n: int) -> int:
        return (self.next_u64() >> 11) % n

    def range(self, lo: int, hi: int) -> int:
        return lo + self.below(hi - lo)

    def chance(self, percent: int) -> bool:
        return self.below(100) < percent


def generate(profile: int, nbytes: int, seed: int) -> bytes:
    cap = nbytes + 65536
    buf = np.empty(cap, np.uint8)
    n = _l().olg_generate_profile(profile, nbytes, seed, buf.ctypes.data, cap)
    assert n != 2**64 - 1
    return buf[:n].tobytes()


def prose_vocabulary() -> list[bytes]:
    out = []
    b = ctypes.create_string_buffer(16)
    for i in range(4096):
        n = _l().olg_prose_word(i, b)
        out.append(b.raw[:n])
    return out


def corpus_into(buf: np.ndarray, seed: int) -> None:
    """Fill the whole uint8 array `buf` with the benchmark document for `seed`."""
    n = _l().olg_generate_corpus(buf.size, seed, buf.ctypes.data, buf.size)
    assert n == buf.size


def corpus(nbytes: int, seed: int) -> np.ndarray:
    buf = np.empty(nbytes, np.uint8)
    corpus_into(buf, seed)
    return buf


def _patterns(kind: int, text: np.ndarray, seed: int, n: int) -> list[bytes]:
    cap = n * 1024 + 16
    blob = np.empty(cap, np.uint8)
    lens = np.zeros(n, np.uint32)
    w = _l().olg_generate_patterns(kind, text.ctypes.data, text.size, seed, n, blob.ctypes.data, cap,
                                   lens.ctypes.data)
    assert w != 2**64 - 1
    out, at = [], 0
    for ln in lens:
        out.append(blob[at: at + ln].tobytes())
        at += int(ln)
    return out


def patterns_single(text: np.ndarray, seed: int) -> list[bytes]:
    """One 12-byte pattern sampled from the text."""
    return _patterns(0, text, seed, 1)


def patterns_eight(text: np.ndarray, seed: int) -> list[bytes]:
    """8 patterns of 4,8,...,1024 B; even indices from the text, odd random bytes."""
    return _patterns(1, text, seed, 8)


def patterns_dictionary(text: np.ndarray, seed: int, n: int = 10_000) -> list[bytes]:
    """`n` patterns of U[4,64] B: 60% text substrings, 40% random printable ASCII."""
    return _patterns(2, text, seed, n)


def lognormal_sizes(seed: int, n: int, median: float, sigma: float, lo: int, hi: int) -> np.ndarray:
    out = np.zeros(n, np.uint64)
    _l().olg_lognormal_sizes(seed, n, median, sigma, lo, hi, out.ctypes.data)
    return out


def poisson_arrivals(seed: int, n: int, rate: float) -> np.ndarray:
    out = np.zeros(n, np.float64)
    _l().olg_poisson_arrivals(seed, n, rate, out.ctypes.data)
    return out

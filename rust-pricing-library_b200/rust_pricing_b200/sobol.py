"""Joe--Kuo 6.21201 Sobol direction words.

The reference embeds the decoded 21,201 x 32 direction matrix as
``crates/pricing/data/joe-kuo-6.21201-u32be.bin`` (format in
``crates/pricing/data/README.md``: an 8-byte magic ``JK621201``, big-endian
version 1, dimension count 21201, bit count 32, then dimension-major big-endian
words).  That asset was generated from SciPy's ``_sobol_direction_numbers.npz``
(primitive polynomials and initial direction integers of the published Joe--Kuo
set).  This module regenerates the same matrix from the SciPy data with the
standard Bratley--Fox recurrence, so the table never has to be copied, and
checks the result against the asset's published SHA-256 digest.
"""
from __future__ import annotations

import hashlib
import os
import struct

import numpy as np

DIMENSIONS = 21201
BITS = 32
MAGIC = b"JK621201"
# SHA-256 of the reference's complete asset (header + words), from its README.
ASSET_SHA256 = "189f65c4e4fcf7455efb7618f3dafbbbaf70303fc35ecd380fa28a67ab896900"

_CACHE: dict[int, np.ndarray] = {}


def _scipy_tables():
    import scipy.stats  # noqa: F401  (locates the package)

    path = os.path.join(os.path.dirname(scipy.stats.__file__), "_sobol_direction_numbers.npz")
    data = np.load(path)
    return data["poly"].astype(np.int64), data["vinit"].astype(np.int64)


def direction_words(dimensions: int = DIMENSIONS) -> np.ndarray:
    """Direction words, shape (dimensions, 32), uint32, bit 0 first.

    Dimension 0 is the van der Corput sequence.  For dimension d >= 1 with
    primitive polynomial of degree s (bit_length - 1 of the encoded polynomial,
    whose inner bits are the coefficients a_1..a_{s-1}) the integers m_k follow
    m_k = 2 a_1 m_{k-1} ^ 4 a_2 m_{k-2} ^ ... ^ 2^s m_{k-s} ^ m_{k-s}, and the
    word for bit k is m_k << (31 - k).
    """
    if not 1 <= dimensions <= DIMENSIONS:
        raise ValueError(f"dimension count {dimensions} outside 1..{DIMENSIONS}")
    cached = _CACHE.get(dimensions)
    if cached is not None:
        return cached
    full = _CACHE.get(DIMENSIONS)
    if full is not None:
        return full[:dimensions]
    poly, vinit = _scipy_tables()
    m = np.zeros((dimensions, BITS), dtype=np.int64)
    m[0, :] = 1
    if dimensions > 1:
        degree = np.array([int(p).bit_length() - 1 for p in poly[1:dimensions]], dtype=np.int64)
        rows = np.arange(1, dimensions)
        for s in np.unique(degree):
            sel = rows[degree == s]
            m[sel, :s] = vinit[sel, :s]
            coeff = [((poly[sel] >> (s - 1 - k)) & 1) for k in range(s)]
            for j in range(s, BITS):
                value = m[sel, j - s].copy()
                for k in range(s):
                    value ^= coeff[k] * (m[sel, j - k - 1] << (k + 1))
                m[sel, j] = value
    shifts = (BITS - 1 - np.arange(BITS)).astype(np.int64)
    words = (m << shifts[None, :]).astype(np.uint64).astype(np.uint32)
    _CACHE[dimensions] = words
    return words


def asset_bytes(words: np.ndarray) -> bytes:
    """The reference's asset layout of a full direction matrix."""
    header = MAGIC + struct.pack(">III", 1, words.shape[0], BITS)
    return header + words.astype(">u4").tobytes()


def verify_full_table() -> bool:
    """True when the regenerated matrix hashes to the reference's digest."""
    return hashlib.sha256(asset_bytes(direction_words(DIMENSIONS))).hexdigest() == ASSET_SHA256

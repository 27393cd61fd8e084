"""BLAKE3-256 (O'Connor, Aumasson, Neves, Wilcox-O'Hearn, 2020), pure Python.

The published algorithm: 1024-byte chunks compressed in 64-byte blocks, chunk
chaining values merged in a left-balanced binary tree, 7-round compression of
16 message words on a 16-word state.  Only the hash mode (no key, no derive,
32-byte output) is needed: the reference's request fingerprints are
`blake3-256:` + hex of the hash of a canonical byte encoding.
"""
from __future__ import annotations

import struct

_IV = (0x6A09E667, 0xBB67AE85, 0x3C6EF372, 0xA54FF53A, 0x510E527F, 0x9B05688C, 0x1F83D9AB, 0x5BE0CD19)
_PERM = (2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8)
_CHUNK_START, _CHUNK_END, _PARENT, _ROOT = 1, 2, 4, 8
_M = 0xFFFFFFFF


def _rotr(x: int, n: int) -> int:
    return ((x >> n) | (x << (32 - n))) & _M


def _g(s, a, b, c, d, mx, my):
    s[a] = (s[a] + s[b] + mx) & _M
    s[d] = _rotr(s[d] ^ s[a], 16)
    s[c] = (s[c] + s[d]) & _M
    s[b] = _rotr(s[b] ^ s[c], 12)
    s[a] = (s[a] + s[b] + my) & _M
    s[d] = _rotr(s[d] ^ s[a], 8)
    s[c] = (s[c] + s[d]) & _M
    s[b] = _rotr(s[b] ^ s[c], 7)


def _compress(cv, block_words, counter: int, block_len: int, flags: int):
    s = list(cv) + list(_IV[:4]) + [counter & _M, (counter >> 32) & _M, block_len, flags]
    m = list(block_words)
    for r in range(7):
        _g(s, 0, 4, 8, 12, m[0], m[1])
        _g(s, 1, 5, 9, 13, m[2], m[3])
        _g(s, 2, 6, 10, 14, m[4], m[5])
        _g(s, 3, 7, 11, 15, m[6], m[7])
        _g(s, 0, 5, 10, 15, m[8], m[9])
        _g(s, 1, 6, 11, 12, m[10], m[11])
        _g(s, 2, 7, 8, 13, m[12], m[13])
        _g(s, 3, 4, 9, 14, m[14], m[15])
        if r < 6:
            m = [m[i] for i in _PERM]
    return [s[i] ^ s[i + 8] for i in range(8)]


def _words(block: bytes):
    return struct.unpack("<16I", block.ljust(64, b"\0"))


class _Output:
    """A node's inputs, compressed as a chaining value or as the root."""

    def __init__(self, cv, words, counter, block_len, flags):
        self.cv, self.words, self.counter, self.block_len, self.flags = cv, words, counter, block_len, flags

    def chaining_value(self):
        return _compress(self.cv, self.words, self.counter, self.block_len, self.flags)

    def root(self) -> bytes:
        return struct.pack("<8I", *_compress(self.cv, self.words, 0, self.block_len, self.flags | _ROOT))


def _chunk_output(chunk: bytes, index: int) -> _Output:
    cv = list(_IV)
    blocks = [chunk[i:i + 64] for i in range(0, len(chunk), 64)] or [b""]
    for k, block in enumerate(blocks):
        flags = (_CHUNK_START if k == 0 else 0) | (_CHUNK_END if k == len(blocks) - 1 else 0)
        if k == len(blocks) - 1:
            return _Output(cv, _words(block), index, len(block), flags)
        cv = _compress(cv, _words(block), index, 64, flags)
    raise AssertionError("unreachable")


def _parent(left, right) -> _Output:
    return _Output(list(_IV), tuple(left) + tuple(right), 0, 64, _PARENT)


def blake3(data: bytes) -> bytes:
    """The 32-byte BLAKE3 hash of `data`."""
    chunks = [data[i:i + 1024] for i in range(0, len(data), 1024)] or [b""]
    stack = []
    for index, chunk in enumerate(chunks[:-1]):
        cv = _chunk_output(chunk, index).chaining_value()
        total = index + 1
        while total & 1 == 0:
            cv = _parent(stack.pop(), cv).chaining_value()
            total >>= 1
        stack.append(cv)
    out = _chunk_output(chunks[-1], len(chunks) - 1)
    while stack:
        out = _parent(stack.pop(), out.chaining_value())
    return out.root()

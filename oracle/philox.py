"""Philox4x32-10 restated on the CPU (test infrastructure: a checker for the
CUDA path's counter-based generator, never product code).

The reference draws its numbers from a 48-bit linear congruential generator
(src/core/misc/sampler.hpp:22-36); the CUDA path replaces it with the
counter-based Philox4x32-10 of Salmon, Moraes, Dror and Shaw, "Parallel
random numbers: as easy as 1, 2, 3" (SC'11).  This module restates the
published algorithm independently of the device code, vectorised over numpy
arrays, and carries the generator's published known-answer vectors
(Random123's kat_vectors for philox4x32 with 10 rounds), so that tests can pin
the restatement first and then the device generator against it.
"""
import numpy as np

M0, M1 = 0xD2511F53, 0xCD9E8D57   # round multipliers
W0, W1 = 0x9E3779B9, 0xBB67AE85   # Weyl key increments

# (counter c0..c3, key k0 k1) -> output, from the Random123 distribution.
KNOWN_ANSWERS = [
    ((0x00000000, 0x00000000, 0x00000000, 0x00000000, 0x00000000, 0x00000000),
     (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF),
     (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344, 0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


def philox4x32_10(ctr_key):
    """ctr_key: (n, 6) unsigned 32-bit words (c0, c1, c2, c3, k0, k1) -> (n, 4)."""
    a = np.asarray(ctr_key, dtype=np.uint64).reshape(-1, 6)
    c0, c1, c2, c3, k0, k1 = (a[:, i].copy() for i in range(6))
    mask = np.uint64(0xFFFFFFFF)
    for _ in range(10):
        p0 = np.uint64(M0) * c0
        p1 = np.uint64(M1) * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & mask
        hi1, lo1 = p1 >> np.uint64(32), p1 & mask
        c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
        k0 = (k0 + np.uint64(W0)) & mask
        k1 = (k1 + np.uint64(W1)) & mask
    return np.stack([c0, c1, c2, c3], 1).astype(np.uint32)

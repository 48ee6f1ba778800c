"""Known-answer test of the noise source's Philox4x32-10 block function
(Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
SC'11), which the device uses for the reference's common-random-numbers noise
(one stream shared by all particles and FIC trials, run_CMAES.cpp:640-657).

The vectors are the published known answers of Philox4x32 with 10 rounds
(counter, key -> output).  A plain-Python restatement of the round function
(multipliers 0xD2511F53 / 0xCD9E8D57, Weyl key increments 0x9E3779B9 /
0xBB67AE85) reproduces them on the CPU; the device function must give the
same words for them and for random inputs."""
import numpy as np
import pytest

import bnm_cuda_b200 as B

KAT = [  # counter[4], key[2] -> output[4]
    ((0x00000000, 0x00000000, 0x00000000, 0x00000000), (0x00000000, 0x00000000),
     (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff, 0xffffffff, 0xffffffff, 0xffffffff), (0xffffffff, 0xffffffff),
     (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
]


def philox4x32_10(c, k):
    c, (k0, k1) = list(c), k
    for _ in range(10):
        p0, p1 = 0xD2511F53 * c[0], 0xCD9E8D57 * c[2]
        c = [(p1 >> 32) ^ c[1] ^ k0, p1 & 0xFFFFFFFF, (p0 >> 32) ^ c[3] ^ k1, p0 & 0xFFFFFFFF]
        k0, k1 = (k0 + 0x9E3779B9) & 0xFFFFFFFF, (k1 + 0xBB67AE85) & 0xFFFFFFFF
    return tuple(c)


def test_restatement_reproduces_published_vectors():
    for c, k, want in KAT:
        assert philox4x32_10(c, k) == want


@pytest.mark.gpu
def test_device_philox_matches_published_vectors_and_restatement():
    rng = np.random.default_rng(7)
    rnd = rng.integers(0, 2**32, size=(200, 6), dtype=np.uint64).astype(np.uint32)
    inp = np.concatenate([np.array([list(c) + list(k) for c, k, _ in KAT], np.uint32), rnd])
    got = B.philox_probe(inp)
    for i, (c, k, want) in enumerate(KAT):
        assert tuple(int(x) for x in got[i]) == want, (i, [hex(int(x)) for x in got[i]])
    for i in range(len(KAT), len(inp)):
        assert tuple(int(x) for x in got[i]) == philox4x32_10(inp[i, :4].tolist(), inp[i, 4:].tolist())

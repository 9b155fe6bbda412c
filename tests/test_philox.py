"""The Brownian-dynamics noise: FP32 normals from a Philox4x32-10 stream keyed by
(seed, particle, step).  A NumPy Philox4x32-10 is pinned to the published
known-answer vectors of the Random123 library (J. K. Salmon et al., SC11), and
the device's noise, read back through msg_bd_step, must equal its Box-Muller
transform of the same counters."""
import numpy as np
import pytest

import helpers as Hp

M0, M1 = 0xD2511F53, 0xCD9E8D57
W0, W1 = 0x9E3779B9, 0xBB67AE85
CTR2 = 0x4D4F4C53      # third counter word of the library's noise stream


def philox4x32_10(ctr, key):
    """Vectorised over the rows of ctr [n][4] (uint32); key [2]."""
    c = [np.asarray(ctr[:, k], np.uint64) for k in range(4)]
    k0, k1 = np.uint64(key[0]), np.uint64(key[1])
    mask = np.uint64(0xFFFFFFFF)
    for r in range(10):
        if r:
            k0 = (k0 + np.uint64(W0)) & mask
            k1 = (k1 + np.uint64(W1)) & mask
        p0 = np.uint64(M0) * c[0]
        p1 = np.uint64(M1) * c[2]
        c = [(p1 >> np.uint64(32)) ^ c[1] ^ k0, p1 & mask, (p0 >> np.uint64(32)) ^ c[3] ^ k1, p0 & mask]
    return np.stack(c, axis=1).astype(np.uint32)


@pytest.mark.parametrize("ctr,key,want", [
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
])
def test_philox_known_answers(ctr, key, want):
    got = philox4x32_10(np.array([ctr], np.uint64), key)[0]
    assert [int(x) for x in got] == want


def box_muller3(r):
    """The library's transform of one Philox output block into three normals (FP32)."""
    inv = np.float32(2.0 ** -32)
    u1 = (r[:, 0].astype(np.float32) + np.float32(1)) * inv
    u2 = r[:, 1].astype(np.float32) * inv
    u3 = (r[:, 2].astype(np.float32) + np.float32(1)) * inv
    u4 = r[:, 3].astype(np.float32) * inv
    m1 = np.sqrt(np.float32(-2) * np.log(u1))
    m2 = np.sqrt(np.float32(-2) * np.log(u3))
    a1 = 2.0 * np.pi * u2.astype(np.float64)
    a2 = 2.0 * np.pi * u4.astype(np.float64)
    return np.stack([m1 * np.cos(a1), m1 * np.sin(a1), m2 * np.cos(a2)], axis=1)


@pytest.mark.gpu
def test_device_noise_is_the_philox_stream():
    from molsim_b200 import Engine

    s = dict(Hp.colloid_small())
    t = Hp.oracle_table(s)
    g = Engine(s, t)
    seed, nsteps, n = 0x1234ABCD5678, 3, int(s["np"])
    _, xi = g.BDStep(nsteps, seed=seed, return_noise=True, energies=False)
    for step in range(nsteps):
        ctr = np.zeros((n, 4), np.uint64)
        ctr[:, 0] = np.arange(n)
        ctr[:, 1] = step
        ctr[:, 2] = CTR2
        want = box_muller3(philox4x32_10(ctr, [seed & 0xFFFFFFFF, seed >> 32]))
        assert np.abs(xi[step] - want).max() < 5e-5, step
    flat = xi.reshape(-1)
    assert abs(flat.mean()) < 0.05 and abs(flat.var() - 1.0) < 0.1
    # a second handle with the same seed draws the same numbers; another seed does not
    g2 = Engine(s, t)
    _, xi2 = g2.BDStep(nsteps, seed=seed, return_noise=True, energies=False)
    assert np.array_equal(xi, xi2)
    g3 = Engine(s, t)
    _, xi3 = g3.BDStep(1, seed=seed + 1, return_noise=True, energies=False)
    assert not np.allclose(xi3[0], xi[0])

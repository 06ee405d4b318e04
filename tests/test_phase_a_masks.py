"""CPU property tests of the row-mask identities the tier-1 context-modelling kernel relies on
(t1enc.cu, phase A), on random 64-bit and 32-bit row masks of one 4-row stripe:

- the significance-propagation membership computed by sweeps that stop as soon as no lower row
  seeds a sample outside the runs already filled equals the one computed by sweeping until
  nothing changes (the least fixpoint);
- at that fixpoint the newly significant samples are the coded ones whose bit is 1 (N = K & B);
- dilating an OR of rows equals the OR of their dilations;
- the lane's own two columns taken by one shift equal bits 1-2 of its 4-bit window.

The GPU tests check the same kernel end to end (codewords byte-equal to the oracle's); these pin
the algebra on many more stripes than any image holds."""
import numpy as np
import pytest


def _dil(m, full):
    return (m | (m << 1) | (m >> 1)) & full


def _fill(M, seeds, full):
    # carry-propagate run fill: every run of M bits upward from a seed bit
    seeds &= M
    return M & ((~((M + seeds) & full)) | seeds) & full


def _stripe(rng, bits):
    full = (1 << bits) - 1
    r = lambda p: int(sum(1 << i for i in range(bits) if rng.random() < p))  # noqa: E731
    O = [r(0.2) for _ in range(6)]                       # significance before the pass, rows -1..4
    Bm = [r(0.5) for _ in range(4)]                      # this bit-plane's bits, rows 0..3
    C = [(~O[j + 1]) & full for j in range(4)]           # candidates: not yet significant
    E = [C[j] & _dil(O[j] | O[j + 1] | O[j + 2], full) for j in range(4)]
    M = [C[j] & Bm[j] for j in range(4)]
    return full, O, Bm, C, E, M


def _sweep(N, M, E, full):
    for j in range(4):
        seeds = M[j] & (E[j] | (((N[j] | N[j + 2]) << 1) & full) | N[j])
        N[j + 1] = _fill(M[j], seeds, full)


def _fixpoint_until_unchanged(M, E, full):
    N = [0] * 6
    while True:
        old = list(N)
        _sweep(N, M, E, full)
        if N == old:
            return N


def _fixpoint_early_exit(M, E, full):
    N = [0] * 6
    if not any(M):
        return N
    while True:
        _sweep(N, M, E, full)
        more = 0
        for j in range(3):
            more |= M[j] & ((N[j + 2] << 1) & full) & ~N[j + 1]
        if not more:
            return N


@pytest.mark.parametrize("bits", [32, 64])
def test_fixpoint_early_exit_and_new_significance(bits):
    rng = np.random.default_rng(bits)
    for _ in range(3000):
        full, O, Bm, C, E, M = _stripe(rng, bits)
        ref = _fixpoint_until_unchanged(M, E, full)
        got = _fixpoint_early_exit(M, E, full)
        assert got == ref
        for j in range(4):
            K = C[j] & (E[j] | (((got[j] | got[j + 1] | got[j + 2]) << 1) & full) | got[j])
            assert got[j + 1] == K & Bm[j]


@pytest.mark.parametrize("bits", [32, 64])
def test_dilation_of_or_and_own_columns(bits):
    rng = np.random.default_rng(100 + bits)
    full = (1 << bits) - 1
    for _ in range(2000):
        a, b, c = (int(rng.integers(0, 1 << 62)) & full for _ in range(3))
        assert _dil(a | b | c, full) == _dil(a, full) | _dil(b, full) | _dil(c, full)
        for c0 in range(0, bits, 2 if bits == 64 else 1):
            win4 = ((a >> (c0 - 1)) if c0 else (a << 1)) & 0xF
            assert (a >> c0) & 3 == (win4 >> 1) & 3

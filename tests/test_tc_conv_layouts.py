"""Layout model of the tensor-core convolutions (csrc/conv_bf16.cu, csrc/tc05.cuh),
recomputed from the constants in the sources. CPU only.

The MMAs read their operands through shared-memory descriptors in the no-swizzle canonical
layouts: K-major — element (row r, k) at start + (r/8)·SBO + (r mod 8)·16 + (k/8)·LBO +
(k mod 8)·2 bytes — and MN-major — element (mn, k) at start + (mn/8)·SBO + (mn mod 8)·2 +
(k/8)·LBO + (k mod 8)·16 — for BF16 and one K step of 16. For every descriptor a kernel
builds, the tests check that each element it addresses is the staged value the convolution
needs at that (row, k), and that every byte an MMA can read lies inside the CTA's dynamic
shared memory."""
import os
import re

import numpy as np
import pytest

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "femtools.jl_b200", "csrc")


def src(name):
    with open(os.path.join(CSRC, name)) as f:
        return f.read()


def const(text, name):
    return int(re.search(rf"constexpr int {name} = (\d+);", text).group(1))


S = src("conv_bf16.cu")
SEG, FROWS, NSTAGE = const(S, "SEG"), const(S, "FROWS"), const(S, "NSTAGE")
HALO = SEG + 2
FSLAB = (FROWS + 2) * HALO * 16
SMEM_CAP = 227 * 1024
CASES = [(16, 16), (16, 32), (32, 16), (32, 32)]


def kmajor(start, lbo, sbo, rows, ks=16):
    r = np.arange(rows)[:, None]
    k = np.arange(ks)[None, :]
    return start + (r // 8) * sbo + (r % 8) * 16 + (k // 8) * lbo + (k % 8) * 2


def mnmajor(start, lbo, sbo, mn, ks=16):
    m = np.arange(mn)[:, None]
    k = np.arange(ks)[None, :]
    return start + (m // 8) * sbo + (m % 8) * 2 + (k // 8) * lbo + (k % 8) * 16


def conv_smem(ci, co):
    a = ci // 8 * FSLAB
    b = 9 * ci // 8 * co * 16
    bias = b + NSTAGE * a
    bar = bias + co * 4
    return dict(A=a, B=b, BIAS=bias, BAR=bar, BYTES=bar + 32)


def wgrad_smem(ci, co):
    ns, nso, nr = ci // 8, co // 8, FROWS + 2
    a = nr * ns * HALO * 16
    by = FROWS * nso * SEG * 16
    stage = a + by
    reach = ((FROWS - 1) * ns * HALO + 2 + SEG - 16) * 16 + 15 * HALO * 16 + 256
    tail = max(reach - stage, 0)
    return dict(NS=ns, NSO=nso, A=a, BY=by, STAGE=stage, REACH=reach, BYTES=2 * stage + tail + 32)


def test_constants_match_the_kernel_structs():
    # the Python restatement of the shared-memory structs against the expressions in the source
    assert "static constexpr int A = CI / 8 * FSLAB;" in S
    assert "static constexpr int B = 9 * CI / 8 * CO * 16;" in S
    assert "static constexpr int BIAS = B + NSTAGE * A;" in S
    assert "static constexpr int STAGE = A + BY;" in S
    assert "static constexpr int BYTES = 2 * STAGE + TAIL + 32;" in S
    assert re.search(r"REACH = \(\(FROWS - 1\) \* NS \* HALO \+ 2 \+ SEG - 16\) \* 16 \+ 15 \* HALO \* 16 \+ 256", S)
    assert re.search(r"constexpr int FSLAB = \(FROWS \+ 2\) \* HALO \* 16;", S)


def test_descriptor_fields_and_offsets():
    # start address, LBO and SBO are 14-bit fields in 16-byte units; the kernels add offsets
    # to a base descriptor, which stays exact while shared addresses are below 2^18 bytes
    t = src("tc05.cuh")
    assert "(saddr >> 4) & 0x3FFFu" in t and "(1ull << 46)" in t
    for ci, co in CASES:
        assert conv_smem(ci, co)["BYTES"] < 1 << 18 and wgrad_smem(ci, co)["BYTES"] < 1 << 18
        assert FSLAB % 16 == 0 and (HALO * 16) < (1 << 18)
    # instruction descriptor: F32 accumulate, BF16 A and B, N/8 at bit 17, M/16 at bit 24
    m = re.search(r"return \(1u << 4\) \| \(1u << 7\) \| \(1u << 10\) \| \(\(uint32_t\)\(N >> 3\) << 17\) \| "
                  r"\(\(uint32_t\)\(M >> 4\) << 24\);", t)
    assert m


@pytest.mark.parametrize("ci,co", CASES)
def test_forward_operands_address_the_staged_values(ci, co):
    sm = conv_smem(ci, co)
    assert sm["BYTES"] <= SMEM_CAP
    nr = FROWS + 2
    for st in range(NSTAGE):
        base = sm["B"] + st * sm["A"]
        for u in range(FROWS):
            for tap in range(9):
                ky, kx = divmod(tap, 3)
                for c0 in range(0, ci, 16):
                    got = kmajor(base + (c0 // 8) * FSLAB + ((u + ky) * HALO + kx) * 16, FSLAB, 128, SEG)
                    m = np.arange(SEG)[:, None]
                    c = c0 + np.arange(16)[None, :]
                    want = base + (((c // 8) * nr + u + ky) * HALO + m + kx) * 16 + (c % 8) * 2
                    assert np.array_equal(got, want)
                    # inside this stage's halo block
                    assert got.min() >= base and got.max() + 2 <= base + sm["A"]
    # weights: chunk j of row co at (j·co + co)·16, the k-th value of the chunk at + 2·(k mod 8)
    for tap in range(9):
        for c0 in range(0, ci, 16):
            k0 = tap * ci + c0
            got = kmajor(k0 // 8 * co * 16, co * 16, 128, co)
            n = np.arange(co)[:, None]
            k = k0 + np.arange(16)[None, :]
            want = ((k // 8) * co + n) * 16 + (k % 8) * 2
            assert np.array_equal(got, want) and got.max() + 2 <= sm["B"]
    # two accumulator columns per output row set within the allocation
    assert FROWS * co <= (64 if FROWS * co <= 64 else 128)


@pytest.mark.parametrize("ci,co", CASES)
def test_weight_gradient_operands_address_the_staged_values(ci, co):
    sm = wgrad_smem(ci, co)
    assert sm["BYTES"] <= SMEM_CAP
    ns, nso = sm["NS"], sm["NSO"]
    for st in range(2):
        base = st * sm["STAGE"]
        reach = 0
        for u in range(FROWS):
            for kx in range(3):
                for ks in range(SEG // 16):
                    got = mnmajor(base + (u * ns * HALO + kx + 16 * ks) * 16, 128, HALO * 16, 128)
                    reach = max(reach, got.max() + 2 - base)
                    # rows ky·ci + c (ky < 3) are the staged input of kernel row ky, channel c
                    m = np.arange(3 * ci)[:, None]
                    ky, c = m // ci, m % ci
                    p = 16 * ks + np.arange(16)[None, :]
                    want = base + (((u + ky) * ns + c // 8) * HALO + p + kx) * 16 + (c % 8) * 2
                    assert np.array_equal(got[:3 * ci], want)
                    # B: the output gradient of row u, co group n/8, pixel p
                    gb = mnmajor(base + sm["A"] + (u * nso * SEG + 16 * ks) * 16, 128, SEG * 16, co)
                    n = np.arange(co)[:, None]
                    wb = base + sm["A"] + ((u * nso + n // 8) * SEG + p) * 16 + (n % 8) * 2
                    assert np.array_equal(gb, wb)
                    assert gb.max() + 2 <= base + sm["STAGE"]
        # the rows past 3·ci read further, but never past the allocation
        assert reach <= sm["REACH"]
        assert base + reach <= sm["BYTES"] - 32
    # three kernel rows of a column fit in the M = 128 block; three accumulator column sets
    assert 3 * ci <= 128 and 3 * co <= 128

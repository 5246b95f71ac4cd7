"""CPU model of the compile-time Stockham schedule of the FFT passes.

The sm_100a line passes (``k_line_tma`` in ``csrc/tr_nufft.cu``) run the
stages of ``csrc/tr_fft.cuh`` (``CtStage`` with two buffers, ``CtStageIP`` in
place) with the radix order, butterfly indexing and twiddle steps fixed at
compile time.  This file restates that index arithmetic in NumPy for every
compiled length and tile width and checks, without a GPU:

* the radix order factors each length;
* the two-buffer schedule and the in-place schedule (every butterfly of a stage
  read before any is written back) both give the DFT;
* in place, each stage writes every element of the [L][W] tile exactly once,
  so one barrier between a stage's reads and its writes is enough;
* the thread counts and the one-tile shared-memory size let six 320-thread
  CTAs (32 registers each) share an SM.
"""

from __future__ import annotations

import numpy as np
import pytest

CT_LENGTHS = [60, 80, 100, 120, 140, 160, 200, 240, 320]


def ct_width(L):                      # tr_nufft.cu: ct_width
    return 8 if L >= 240 else 16


def ct_radices(L):                    # tr_fft.cuh: ct_radix (7s, 5s, 3s, then 8s, 4s, 2s)
    out, n = [], L
    for r in (7, 5, 3, 8, 4, 2):
        while n % r == 0:
            out.append(r)
            n //= r
    assert n == 1, L
    return out


def ct_radices_p(P, L):               # tr_fft.cuh: ct_radix_p (P = 1: two passes at 320 and 160)
    if P == 1 and L == 320:
        return [20, 16]
    if P == 1 and L == 160:
        return [10, 16]
    return ct_radices(L)


def ct_rounds(L, W, NT):              # tr_nufft.cu: ct_rounds
    return sum(-(-(L // r) * W // NT) for r in ct_radices(L))


def line_threads(L, W):               # tr_nufft.cu: line_threads
    return 320 if ct_rounds(L, W, 320) < ct_rounds(L, W, 256) else 256


def _stage(src, L, W, R, Ns, tw, inv):
    """One Stockham stage over the [L][W] tile `src` (flat); returns (dst, write indices)."""
    NB = L // R
    step = L // (Ns * R)
    idx = np.arange(NB * W)
    j, w = idx // W, idx % W
    k = j % Ns
    v = np.stack([src[(j + r * NB) * W + w] for r in range(R)])            # (R, NB*W)
    if Ns > 1:
        t = np.stack([tw[(k * r * step) % L] for r in range(R)])
        v = v * (np.conj(t) if inv else t)
    sgn = 1.0 if inv else -1.0
    m = np.arange(R)
    dft = np.exp(sgn * 2j * np.pi * np.outer(m, m) / R)
    out = dft @ v
    d0 = (j // Ns) * Ns * R + k
    widx = np.stack([(d0 + r * Ns) * W + w for r in range(R)])
    dst = np.empty_like(src)
    dst[widx.ravel()] = out.ravel()
    return dst, widx.ravel()


def _run(x, L, W, inv, in_place, plan=0):
    tw = np.exp(-2j * np.pi * np.arange(L) / L)
    buf = x.reshape(-1).astype(np.complex128)
    Ns = 1
    for R in ct_radices_p(plan, L):
        new, widx = _stage(buf, L, W, R, Ns, tw, inv)
        if in_place:
            # every element written exactly once: reads-then-barrier-then-writes is race-free
            assert np.array_equal(np.sort(widx), np.arange(L * W))
        buf = new
        Ns *= R
    return buf.reshape(L, W)


@pytest.mark.parametrize("L", CT_LENGTHS)
@pytest.mark.parametrize("inv", [False, True])
@pytest.mark.parametrize("in_place", [False, True])
def test_schedule_is_the_dft(L, inv, in_place):
    W = ct_width(L)
    assert int(np.prod(ct_radices(L))) == L
    rng = np.random.default_rng(L + 7 * inv)
    x = rng.standard_normal((L, W)) + 1j * rng.standard_normal((L, W))
    y = _run(x, L, W, inv, in_place)
    ref = np.fft.ifft(x, axis=0) * L if inv else np.fft.fft(x, axis=0)
    assert np.max(np.abs(y - ref)) < 1e-9 * np.max(np.abs(ref))


@pytest.mark.parametrize("L", [160, 320])
@pytest.mark.parametrize("inv", [False, True])
@pytest.mark.parametrize("in_place", [False, True])
def test_two_pass_plan_is_the_dft(L, inv, in_place):
    """Radix plan 1 (20 x 16 at 320, 10 x 16 at 160): the same Stockham indexing
    and twiddle steps with composite radices give the DFT in two passes."""
    assert len(ct_radices_p(1, L)) == 2 and int(np.prod(ct_radices_p(1, L))) == L
    W = 8
    rng = np.random.default_rng(L + 3 * inv)
    x = rng.standard_normal((L, W)) + 1j * rng.standard_normal((L, W))
    y = _run(x, L, W, inv, in_place, plan=1)
    ref = np.fft.ifft(x, axis=0) * L if inv else np.fft.fft(x, axis=0)
    assert np.max(np.abs(y - ref)) < 1e-9 * np.max(np.abs(ref))


def ct_swz_row(m, sw):                # tr_fft.cuh: ct_swz_row (rows 2i, 2i+1 exchanged in odd blocks)
    return m ^ ((m // sw) & 1) if sw else m


@pytest.mark.parametrize("L", [160, 320])
def test_two_pass_row_swizzle(L):
    """With 64-byte rows (W = 8) the first pass's rows R0 j + r of the two
    butterflies j, j + 1 of a half-warp would share a bank half; the swizzle
    is a permutation of the tile's rows that gives them opposite halves, and
    the second pass's rows j + R0 r (consecutive j) stay in opposite halves."""
    r0, r1 = ct_radices_p(1, L)
    sw = r0                                        # ct_swz_p: even first radix, 8-column rows
    assert r0 % 2 == 0
    rows = [ct_swz_row(m, sw) for m in range(L)]
    assert sorted(rows) == list(range(L))
    for j in range(0, L // r0, 2):                 # stage 0: half-warp = butterflies j, j + 1 (8 columns each)
        for r in range(r0):
            assert ct_swz_row(r0 * j + r, sw) % 2 != ct_swz_row(r0 * (j + 1) + r, sw) % 2
    nb = L // r1                                   # stage 1 reads rows j + nb r, nb = r0
    assert nb == r0
    for j in range(0, nb, 2):
        for r in range(r1):
            assert ct_swz_row(j + nb * r, sw) % 2 != ct_swz_row(j + 1 + nb * r, sw) % 2


@pytest.mark.parametrize("L", CT_LENGTHS)
def test_in_place_tiles_fit_six_ctas(L):
    W = ct_width(L)
    NT = line_threads(L, W)
    smem = (L * W + L) * 8 + 128                   # line_tma_smem_bytes
    assert 6 * (smem + 1024) <= 228 * 1024         # per-CTA reserve included
    if NT == 320:                                  # __launch_bounds__(320, 5): 32 registers measured
        assert 6 * NT * 32 <= 65536 and 6 * NT <= 2048
    # the workload's lengths: the 8-column y tiles and 16-column z tiles both take 320 threads
    if L in (160, 320):
        assert NT == 320 and ct_rounds(L, W, 320) < ct_rounds(L, W, 256)

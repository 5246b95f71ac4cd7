"""CPU model of the gridding launch's block decoding and of the z passes'
empty-column test (``csrc/tr_nufft.cu``).

* ``k_spread`` spreads its zero-fill CTAs among the work items: CTA b of
  T = n_work + nz is zero-fill group floor(b nz / T) when floor((b + 1) nz / T)
  steps past it, else work item b - floor(b nz / T).  Every work item and every
  zero-fill group is taken by exactly one CTA, work items keep their order
  (heaviest first), and the zero-fill CTAs are evenly spaced.
* ``lines_unoccupied``: a z-pass CTA of W lines starting at inner index q0
  (q = (y OSX + x) ncol + column) is skipped only when every line's tile column
  (y / 4, x / 4) is unoccupied; with ncol a multiple of W (the only case the
  host passes a mask) a CTA never mixes columns.
"""

from __future__ import annotations

import numpy as np
import pytest


def decode(b, n_work, nz):
    T = n_work + nz
    zlo, zhi = b * nz // T, (b + 1) * nz // T
    return ("zero", zlo) if zhi > zlo else ("work", b - zlo)


@pytest.mark.parametrize("n_work,nz", [(0, 5), (7, 0), (1, 1), (133_000, 4_480), (61, 3), (5, 17), (96, 96)])
def test_zero_fill_ctas_interleave_exactly(n_work, nz):
    T = n_work + nz
    got = [decode(b, n_work, nz) for b in range(T)]
    works = [i for kind, i in got if kind == "work"]
    zeros = [i for kind, i in got if kind == "zero"]
    assert works == list(range(n_work))           # each once, in order (heaviest first)
    assert zeros == list(range(nz))
    if nz > 1 and n_work > 0:
        pos = np.array([b for b, (kind, _) in enumerate(got) if kind == "zero"])
        gaps = np.diff(pos)
        assert gaps.max() - gaps.min() <= 1        # evenly spaced


def lines_unoccupied(mask, q0, W, inner, ncol, osx, nt2):
    q1 = min(q0 + W, inner) - 1
    for yx in range(q0 // ncol, q1 // ncol + 1):
        y, x = divmod(yx, osx)
        if mask[(y >> 2) * nt2 + (x >> 2)]:
            return False
    return True


@pytest.mark.parametrize("osy,osx,ncol,W", [(25, 30, 16, 16), (80, 80, 96, 16), (320, 320, 96, 16), (20, 24, 32, 16)])
def test_column_skip_never_mixes_columns(osy, osx, ncol, W):
    rng = np.random.default_rng(osy * osx + ncol)
    nt1, nt2 = -(-osy // 4), -(-osx // 4)
    mask = rng.integers(0, 2, nt1 * nt2).astype(bool)
    inner = osy * osx * ncol
    assert ncol % W == 0
    for q0 in range(0, inner, W):
        cols = {((q // ncol) // osx >> 2, ((q // ncol) % osx) >> 2) for q in range(q0, min(q0 + W, inner))}
        assert len(cols) == 1                      # one (y, x) tile column per CTA
        (ty, tx), = cols
        assert lines_unoccupied(mask, q0, W, inner, ncol, osx, nt2) == (not mask[ty * nt2 + tx])

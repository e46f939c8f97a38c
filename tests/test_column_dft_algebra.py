"""The algebra the tensor-core column DFT (csrc/hybrid_p1g.cuh) rests on,
restated in numpy on the CPU: for two real columns a, b packed as z = a + ib,

* the spectrum rows ky and M - ky follow from two real products with the
  cos / -sin tables over ky < M/2 (Hermitian symmetry of A = DFT(a) and
  B = DFT(b)), the Nyquist row from the table's zero row ky = 0 of S
  replaced by (-1)^y;
* by ky parity, the tables over y < M/2 suffice: the rows at y + M/2 are
  (-1)^ky times those at y (one image atom pair per table atom, the odd
  rows negated);
* the plane-row bookkeeping of the stores: rows ky = p + 2 r (staging row
  2 r + part) from ky = p, and rows M - ky (staging row 2 (127 - r) + part)
  from ky = M/2 + 2 - p, cover every row of both parities exactly once with
  ky = 0 / M/2 handled by the Nyquist lane."""
import numpy as np

M = 512
KR = 128


def tables():
    """C, S over ky = p + 2 r (rows [p][r]) and y < M/2, as the table kernel builds them."""
    y = np.arange(M // 2)
    C = np.zeros((2, KR, M // 2))
    S = np.zeros((2, KR, M // 2))
    for p in range(2):
        ky = p + 2 * np.arange(KR)
        ang = 2 * np.pi * ((ky[:, None] * y[None, :]) % M) / M
        C[p] = np.cos(ang)
        S[p] = -np.sin(ang)
    S[0, 0] = np.where(y % 2, -1.0, 1.0)  # the Nyquist row in the zero row ky = 0
    return C, S


def test_parity_symmetry_of_the_tables():
    y = np.arange(M)
    for ky in (0, 1, 2, 7, 128, 255):
        c = np.cos(2 * np.pi * ky * y / M)
        s = -np.sin(2 * np.pi * ky * y / M)
        sign = -1.0 if ky % 2 else 1.0
        np.testing.assert_allclose(c[M // 2:], sign * c[:M // 2], atol=1e-12)
        np.testing.assert_allclose(s[M // 2:], sign * s[:M // 2], atol=1e-12)
    nyq = np.where(y % 2, -1.0, 1.0)
    np.testing.assert_allclose(nyq[M // 2:], nyq[:M // 2])  # even: the Nyquist row takes + too


def test_packed_column_spectrum_from_the_half_tables():
    rng = np.random.default_rng(5)
    a, b = rng.standard_normal(M), rng.standard_normal(M)
    ref = np.fft.fft(a + 1j * b)  # unnormalised, exp(-2 pi i ky y / M)
    C, S = tables()
    lo, hi = slice(0, M // 2), slice(M // 2, M)
    Z = np.zeros(M, complex)
    for p in range(2):
        sign = -1.0 if p else 1.0  # negate-A on the atom at y + M/2 for odd rows
        ReA = C[p] @ a[lo] + sign * (C[p] @ a[hi])
        ReB = C[p] @ b[lo] + sign * (C[p] @ b[hi])
        ImA = S[p] @ a[lo] + sign * (S[p] @ a[hi])
        ImB = S[p] @ b[lo] + sign * (S[p] @ b[hi])
        for r in range(KR):
            ky = p + 2 * r
            if ky == 0:
                Z[0] = ReA[r] + 1j * ReB[r]
                Z[M // 2] = ImA[r] + 1j * ImB[r]  # the Nyquist row from S's row 0
                continue
            Z[ky] = (ReA[r] - ImB[r]) + 1j * (ImA[r] + ReB[r])
            Z[M - ky] = (ReA[r] + ImB[r]) + 1j * (ReB[r] - ImA[r])
    np.testing.assert_allclose(Z, ref, rtol=0, atol=1e-9 * np.abs(ref).max())


def test_store_rows_cover_every_plane_row_once():
    hits = np.zeros(2 * M, int)  # plane rows 2 ky + part
    for p in range(2):
        for start, row_of in ((p, lambda r: 2 * r), (M // 2 + 2 - p, lambda r: 2 * (KR - 1 - r))):
            # a 4-D store of 128 ky rows (stride 2) x 2 parts from staging rows 0 .. 255
            for j in range(KR):
                ky = start + 2 * j
                for part in range(2):
                    if ky < M:  # rows past the planes are dropped
                        hits[2 * ky + part] += 1
        # staging row of each lane r in both passes agrees with the store's row j
        for r in range(KR):
            ky = p + 2 * r
            assert (ky - p) // 2 == r
            if ky:
                assert (M - ky - (M // 2 + 2 - p)) // 2 == KR - 1 - r
    hits[2 * (M // 2)] += 1  # the Nyquist row, stored by the threads
    hits[2 * (M // 2) + 1] += 1
    # ky = 0's mirror (row M) is dropped, so every row is written exactly once
    assert (hits == 1).all(), np.nonzero(hits != 1)

"""The oracle's E4M3 restatement (CPU): every code round-trips, rounding is
to nearest with ties to even (normal and subnormal), values saturate at
+-448, and the per-row / per-column quantizers use max|x| / 448 scales."""
import numpy as np

from oracle import oracle


def test_every_code_round_trips():
    tab = oracle.e4m3_table()
    codes = [q for q in range(256) if (q & 0x7F) != 0x7F]
    back = oracle.f32_to_e4m3(tab[codes])
    for q, b in zip(codes, back):
        assert b == q or (q & 0x7F) == 0 and (b & 0x7F) == 0
    assert np.isnan(tab[0x7F]) and np.isnan(tab[0xFF])
    assert tab[0x7E] == 448.0 and tab[0x08] == 2.0 ** -6 and tab[0x01] == 2.0 ** -9


def test_rounding_ties_to_even_and_saturation():
    cases = {
        1.0625: 1.0,          # tie between 1.0 (mantissa 0) and 1.125 (1): even -> 1.0
        1.1875: 1.25,         # tie between 1.125 (1) and 1.25 (2): even -> 1.25
        1.07: 1.125,
        2.0 ** -10: 0.0,      # subnormal tie between 0 and 2^-9: even -> 0
        3 * 2.0 ** -10: 2.0 ** -8,  # tie between 2^-9 (1) and 2^-8 (2): even -> 2^-8
        2.0 ** -6 * 15.5 / 16: 2.0 ** -6,  # subnormal rounding up into the smallest normal
        440.0: 448.0,         # 448 = 1.75 * 2^8 is the largest finite value
        464.0: 448.0,
        1e6: 448.0,
        -1e6: -448.0,
        -0.3: -0.3125,
    }
    tab = oracle.e4m3_table()
    for x, want in cases.items():
        q = oracle.f32_to_e4m3(np.float32(x))
        assert tab[q] == np.float32(want), (x, tab[q], want)


def test_row_and_column_quantizers():
    rng = np.random.default_rng(0)
    rp = np.array([0, 3, 3, 7, 8], np.int32)
    vals = (rng.standard_normal(8) * 0.1).astype(np.float16)
    vals[7] = 0
    scale, q = oracle.quant_rows(rp, vals)
    tab = oracle.e4m3_table()
    for r in range(4):
        seg = vals[rp[r]:rp[r + 1]].astype(np.float32)
        m = np.abs(seg).max() if seg.size else 0.0
        s = np.float32(m) / np.float32(448.0) if m > 0 else np.float32(1.0)
        assert scale[r] == s
        if seg.size:
            np.testing.assert_array_equal(q[rp[r]:rp[r + 1]], oracle.f32_to_e4m3(seg / s))
            if m > 0:
                assert np.abs(tab[q[rp[r]:rp[r + 1]]]).max() == 448.0
    B = rng.uniform(-3, 3, (20, 12)).astype(np.float16)
    B[:, 5] = 0
    qb, sb = oracle.quant_cols(B, ldq=16)
    assert qb.shape == (20, 16) and (qb[:, 12:] == 0).all()
    assert sb[5] == 1.0 and (qb[:, 5] == 0).all()
    for n in (0, 7, 11):
        s = np.float32(np.abs(B[:, n].astype(np.float32)).max()) / np.float32(448.0)
        assert sb[n] == s
        np.testing.assert_array_equal(qb[:, n], oracle.f32_to_e4m3(B[:, n].astype(np.float32) / s))

"""The CPU oracle against known answers (hand-derived from the reference's
formulas), the reference's own narrowing headers, and its committed golden
fixtures. CPU only."""
import json
import os

import numpy as np
import pytest

import ref_pins

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def csr(rows, ncols=None):
    """rows: list of [(col, val), ...] -> CSR arrays (entries kept in order)."""
    row = [0]
    col, val = [], []
    for r in rows:
        for c, v in r:
            col.append(c)
            val.append(v)
        row.append(len(col))
    return (np.array(row, np.uint32), np.array(col, np.uint32), np.array(val, np.float64))


A4 = csr([[(0, 4.0), (1, -1.0)], [(1, 4.0), (0, -1.0), (2, -1.0)],
          [(2, 4.0), (1, -1.0), (3, -1.0)], [(3, 3.0), (2, -1.0)]])


# ------------------------------------------------------------- narrowing
@pytest.mark.parametrize("rng,code", [(0, 0), (255, 0), (256, 1), (65535, 1), (65536, 2),
                                      (2**32 - 1, 2), (2**32, 3)])
def test_define_int_type_boundaries(oracle, rng, code):
    # bit_operations.h:119-129: <=255 u8, <=65535 u16, <=2^32-1 u32, else u64
    assert oracle.define_int_type(rng) == code


def test_encode_hash_config1(oracle):
    # 32^3 cube: nnz 223232 (u32), 32768 columns / rows (u16), F64 = 6
    h = oracle.encode_hash(223232, 32768, 32768, 32768)
    assert h == 6 | (2 << 3) | (1 << 5) | (1 << 7) | (1 << 9) == 694
    # matrix.h:80-84: reduced precision forces the F32 code (5)
    assert oracle.encode_hash(223232, 32768, 32768, 32768, reduced=True) == 693


def test_narrowing_pinned_to_reference():
    R = ref_pins.load()
    if R is None:
        pytest.skip("reference narrowing headers not available")
    import oracle_py as O
    for r in [0, 1, 200, 255, 256, 4000, 65535, 65536, 10**6, 2**32 - 1, 2**32, 2**40]:
        assert O.define_int_type(r) == R.ref_define_int_type(r)
    rng = np.random.default_rng(3)
    for _ in range(200):
        a = [int(v) for v in rng.choice([10, 300, 70000, 5 * 10**9], 4)]
        for f32 in (0, 1):
            assert O.encode_hash(*a, f32=bool(f32)) == R.ref_encode_hash(*a, f32)


def test_core_split_pinned_to_reference(oracle):
    R = ref_pins.load()
    if R is None:
        pytest.skip("reference headers not available")
    for n in [1, 7, 8, 9, 100, 1000, 32768, 123457]:
        for nc in [1, 2, 3, 8, 16, 100]:
            cs = R.ref_split_range_f64(n, nc)
            for c in range(nc):
                off, sz = oracle.core_range(n, nc, c)
                assert off == min(n, cs * c)
                assert sz == min(cs, n - off)


# ------------------------------------------------------------- SpMV
def test_spmv_kat_nv1(oracle):
    row, col, val = A4
    y = oracle.csr_ax_y(row, col, val, np.array([1.0, 2, 3, 4]), 1)
    assert y.tolist() == [2.0, 4.0, 6.0, 9.0]


def test_spmv_kat_nv3(oracle):
    row, col, val = A4
    x = np.array([[i + 1 + 10 * k for k in range(3)] for i in range(4)], np.float64)
    y = oracle.csr_ax_y(row, col, val, x.ravel(), 3)
    assert y.reshape(4, 3).tolist() == [[2, 32, 62], [4, 24, 44], [6, 26, 46], [9, 29, 49]]


def test_spmv_accumulation_order(oracle):
    # csr_matvec.inl:222-230 adds entry by entry from 0: ((0+1e16)+1)-1e16 = 0
    row, col, val = csr([[(0, 1e16), (1, 1.0), (2, -1e16)]], 3)
    assert oracle.csr_ax_y(row, col, val, np.ones(3), 1, ncols=3)[0] == 0.0


def test_spmv_no_fma(oracle):
    # each product is rounded before the add: -1 + rn((1-2^-30)(1+2^-30)) = 0,
    # a fused multiply-add would give -2^-60
    e = 2.0**-30
    row, col, val = csr([[(0, -1.0), (1, 1 + e)]], 2)
    y = oracle.csr_ax_y(row, col, val, np.array([1.0, 1 - e]), 1, ncols=2)
    assert y[0] == 0.0


def test_axpy_accumulates_into_y(oracle):
    # csr_matvec.inl:106-120: y += x*val directly into y, entry by entry
    row, col, val = csr([[(0, 1.0), (1, -1e16)]], 2)
    y = oracle.csr_ax_y(row, col, val, np.array([1.0, 1.0]), 1, ncols=2, axpy_y=np.array([1e16]))
    assert y[0] == 0.0  # (1e16 + 1) rounds to 1e16, minus 1e16


def test_spmv_f32(oracle):
    row, col, val = A4
    y = oracle.csr_ax_y(row, col, val.astype(np.float32), np.array([1, 2, 3, 4], np.float32), 1)
    assert y.dtype == np.float32 and y.tolist() == [2.0, 4.0, 6.0, 9.0]


# ------------------------------------------------------------- compress / transpose / inverse
def test_compress_kat(oracle):
    # csr_matrix.inl:86-170 on an off-diagonal block of 4 rows x 6 columns
    row = np.array([0, 2, 2, 3, 4], np.uint32)
    col = np.array([4, 1, 1, 5], np.uint32)
    r, c, ri, ci = oracle.compress(row, col, 6)
    assert r.tolist() == [0, 2, 3, 4]
    assert ri.tolist() == [0, 2, 3]
    assert ci.tolist() == [1, 4, 5]
    assert c.tolist() == [1, 0, 0, 2]


def test_transpose_kat(oracle):
    row, col, val = csr([[(0, 1.0)], [(0, 0.5), (1, 0.5)], [(1, 1.0)]], 2)
    tr, tc, tv = oracle.transpose(row, col, val, 2)
    assert tr.tolist() == [0, 2, 4]
    assert tc.tolist() == [0, 1, 1, 2]
    assert tv.tolist() == [1.0, 0.5, 0.5, 1.0]


def test_inverse_kat(oracle):
    inv = oracle.inverse(np.array([[2.0, 0.0], [0.0, 4.0]]))
    assert inv.tolist() == [[0.5, 0.0], [0.0, 0.25]]
    a = np.array([[4.0, -1, 0], [-1, 4, -1], [0, -1, 4]])
    np.testing.assert_allclose(oracle.inverse(a), np.linalg.inv(a), rtol=1e-14, atol=1e-15)
    a32 = a.astype(np.float32)
    inv32 = oracle.inverse(a32)
    assert inv32.dtype == np.float32
    np.testing.assert_allclose(inv32, np.linalg.inv(a), rtol=1e-6)


def test_inv_diag_precision(oracle):
    # csr_matrix.h:326-327: 1/a computed in double from the stored value
    row, col, val = csr([[(0, 3.0)], [(1, 7.0)]], 2)
    d = oracle.inv_diag(row, col, val)
    assert d.tolist() == [1.0 / 3.0, 1.0 / 7.0]
    d32 = oracle.inv_diag(row, col, val, f32=True)
    assert d32.tolist() == [np.float32(1.0 / 3.0), np.float32(1.0 / 7.0)]
    s = oracle.inv_diag(row, col, val, sqrt=True)
    assert s.tolist() == [np.sqrt(1.0 / 3.0), np.sqrt(1.0 / 7.0)]


@pytest.mark.parametrize("order", [1, 2, 3, 4])
def test_chebyshev_coefficients(oracle, order):
    # chebyshev.inl:50-127: 1 - t q(t) is the Chebyshev polynomial of the
    # interval [lower, upper], normalised to 1 at t = 0
    mn, mx, frac = 0.05, 1.9, 0.3
    c = oracle.cheby_coeffs(mn, mx, order, frac)
    up = mx * 1.1
    lo = (up - mn) * np.float64(np.float32(frac)) + mn
    th, de = (up + lo) / 2, (up - lo) / 2
    for t in np.linspace(lo, up, 7):
        q = sum(c[i] * t**i for i in range(order))
        cheb = np.polynomial.chebyshev.chebval((th - t) / de, [0] * order + [1])
        cheb0 = np.polynomial.chebyshev.chebval(th / de, [0] * order + [1])
        assert abs((1 - t * q) - cheb / cheb0) < 1e-10


# ------------------------------------------------------------- generator
def test_cube_generator_kat(oracle):
    row, col, val = oracle.generate_cube(3, 3, 3)
    q = 9.0  # 1/h^2 with h = 1/3
    # centre (13): diag 6q, six neighbours in the order -z, -y, -x, +x, +y, +z
    c = slice(row[13], row[14])
    assert col[c].tolist() == [13, 4, 10, 12, 14, 16, 22]
    assert val[c].tolist() == [6 * q] + [-q] * 6
    # corner (0): boundary sides add 2q (cube.inl:105-145)
    c = slice(row[0], row[1])
    assert col[c].tolist() == [0, 1, 3, 9]
    assert val[c].tolist() == [9 * q, -q, -q, -q]
    row, col, val = oracle.generate_cube(32, 32, 32)
    assert len(col) == 223232


# ------------------------------------------------------------- reduction orders
def canon_reference(terms, nv):
    """Independent numpy statement of the kernels' fixed reduction order."""
    n = terms.shape[0]
    R = 256 // nv
    ntiles = -(-n // R)
    B = min(ntiles, 1184)
    part = np.zeros((B, nv))
    for b in range(B):
        acc = np.zeros(256)
        for tile in range(b, ntiles, B):
            for t in range(256):
                i = tile * R + t // nv
                if i < n:
                    acc[t] = acc[t] + terms[i, t % nv]
        ws = np.zeros((8, nv))
        for w in range(8):
            lane = acc[32 * w:32 * w + 32].copy()
            off = 16
            while off >= nv:
                lane = lane + lane[np.arange(32) ^ off]
                off //= 2
            ws[w] = lane[:nv]
        s = ws[0].copy()
        for w in range(1, 8):
            s = s + ws[w]
        part[b] = s
    out = np.zeros(nv)
    for k in range(nv):
        lane = np.zeros(32)
        for l in range(32):
            a = 0.0
            for bb in range(l, B, 32):
                a = a + part[bb, k]
            lane[l] = a
        for off in (16, 8, 4, 2, 1):
            lane = lane + lane[np.arange(32) ^ off]
        out[k] = lane[0]
    return out


@pytest.mark.parametrize("n,nv", [(1, 1), (300, 1), (5000, 2), (777, 8), (1000, 32)])
def test_canonical_order_matches_numpy_statement(oracle, n, nv):
    rng = np.random.default_rng(n * 31 + nv)
    x = rng.standard_normal((n, nv)) * 10.0 ** rng.integers(-8, 8, (n, nv))
    y = rng.standard_normal((n, nv))
    oracle.set_reduction(1)
    try:
        got = oracle.dot(x.ravel(), y.ravel(), nv)
    finally:
        oracle.set_reduction(0)
    want = canon_reference(x * y, nv)
    assert got.tobytes() == want.tobytes()


def test_xamg_order_is_sequential(oracle):
    rng = np.random.default_rng(5)
    x = rng.standard_normal(1000) * 1e8
    y = rng.standard_normal(1000)
    s = 0.0
    for a, b in zip(x, y):
        s = s + a * b
    assert oracle.dot(x, y, 1)[0] == s


# ------------------------------------------------------------- whole solves
def test_oracle_config1_golden(oracle):
    """The oracle's 32^3 MergedPBiCGStab + Jacobi solve against its committed
    fixture (tests/golden/make_golden.py)."""
    g = json.load(open(os.path.join(GOLDEN, "oracle_solves.json")))["config1_nv1"]
    row, col, val = oracle.generate_cube(32, 32, 32)
    S = oracle.System(1)
    S.set_params(g["params"])
    S.add_level(row, col, val)
    S.setup()
    b = np.random.default_rng(g["seed"]).uniform(-1, 1, len(row) - 1)
    x, st = S.solve(b)
    assert st["iters"] == g["iters"]
    assert st["conv"].tolist() == g["conv"]
    assert st["rel_res"].tolist() == g["rel_res"]
    import scipy.sparse as sp
    A = sp.csr_matrix((val, col, row))
    assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) <= 1e-8


def test_oracle_residual_drop_multi_rhs(oracle):
    row, col, val = oracle.generate_cube(12, 12, 12)
    nv = 4
    S = oracle.System(nv)
    S.set_params({"solver": {"method": "PBiCGStab", "max_iters": 200, "rel_tolerance": 1e-10,
                             "abs_tolerance": 0},
                  "preconditioner": {"method": "Jacobi"}})
    S.add_level(row, col, val)
    S.setup()
    b = np.random.default_rng(1).uniform(-1, 1, (len(row) - 1) * nv)
    x, st = S.solve(b)
    assert all(st["conv"])
    import scipy.sparse as sp
    A = sp.csr_matrix((val, col, row))
    r = b.reshape(-1, nv) - A @ x.reshape(-1, nv)
    assert (np.linalg.norm(r, axis=0) / np.linalg.norm(b.reshape(-1, nv), axis=0)).max() <= 1e-10


def test_bf16_rounding_matches_torch(oracle):
    """The oracle's BF16 rounding (round to nearest, ties to even) equals
    torch's float32 -> bfloat16 conversion, ties and extremes included."""
    import torch
    rng = np.random.default_rng(17)
    a = np.concatenate([
        rng.standard_normal(100000).astype(np.float32) * np.float32(1e3),
        (rng.standard_normal(1000) * 1e-39).astype(np.float32),        # subnormals
        np.array([0.0, -0.0, np.inf, -np.inf, 3.4e38, -3.4e38, 1.0, 1.00390625,
                  1.01171875, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8], np.float32)])
    # exact ties: low 16 bits = 0x8000 with either parity of the kept bit
    u = rng.integers(0, 2 ** 31, 2000, dtype=np.uint32) & np.uint32(0x7F7F0000)
    ties = ((u | np.uint32(0x8000))).view(np.float32)
    a = np.concatenate([a, ties])
    want = torch.from_numpy(a).to(torch.bfloat16).to(torch.float32).numpy()
    got = oracle.round_bf16(a)
    assert got.tobytes() == want.tobytes()

"""Pins the C oracle (oracle/oracle.c) before any GPU result is compared to it.

Known answers come from the reference's own tests:
  tests/field_vectors.rs:16-182, src/field/babybear.rs:378-568,
  src/field/m31.rs:144-203, src/field/circle.rs:153-235,
  tests/ntt_cross_validation.rs:113-376, src/ntt/*/cpu_reference.rs tests,
  src/lde/mod.rs:194-271.
Fixtures come from tests/golden/gen_golden.py, an independent pure-Python
restatement that checks itself against naive DFT / coset-evaluation closed forms.
"""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from oracle import oracle as O

P = O.BB_P
MP = O.M31_P


def modpow(b, e, m):
    return pow(b, e, m)


def sha(a) -> str:
    return hashlib.sha256(np.asarray(a, dtype="<u4").tobytes()).hexdigest()


# ---- BabyBear KATs (tests/field_vectors.rs:15-116) ---------------------------
def test_bb_modulus_and_constants():
    assert P == (1 << 31) - (1 << 27) + 1
    assert O.bb_to_monty(1) == (1 << 32) % P == 0x0FFFFFFE
    assert O.bb_from_monty(O.bb_to_monty(1)) == 1
    assert O.bb_to_monty(0) == 0
    assert (P * 0x77FFFFFF + 1) % (1 << 32) == 0  # babybear.rs:561-568
    assert O.bb_from_monty(1476048622) == 440564289  # babybear.rs:35-37


def test_bb_arithmetic_kats():
    a, b = O.bb_to_monty(123), O.bb_to_monty(456)
    assert O.bb_from_monty(O.bb_mul(a, b)) == 56088
    pm1 = O.bb_to_monty(P - 1)
    assert O.bb_from_monty(O.bb_mul(pm1, pm1)) == 1
    assert O.bb_from_monty(O.bb_add(pm1, O.bb_to_monty(1))) == 0
    assert O.bb_from_monty(O.bb_sub(0, O.bb_to_monty(1))) == P - 1
    for v in (0, 1, 2, 42, 1000, P - 1, P - 2):
        assert O.bb_from_monty(O.bb_to_monty(v)) == v
    assert O.bb_from_monty(O.bb_reduce(21)) == 21
    assert O.bb_from_monty(O.bb_reduce(P + 5)) == 5
    one = O.bb_to_monty(1)
    assert O.bb_monty_reduce(one * one) == one


def test_bb_inverse_kats():
    seven = O.bb_to_monty(7)
    inv7 = O.bb_inv(seven)
    assert O.bb_from_monty(O.bb_mul(seven, inv7)) == 1
    assert O.bb_from_monty(inv7) == modpow(7, P - 2, P)
    assert O.bb_from_monty(O.bb_inv(O.bb_to_monty(1))) == 1
    assert O.bb_from_monty(O.bb_inv(O.bb_to_monty(P - 1))) == P - 1
    for v in (1, 2, 7, 100, 999999, P - 1, 42):
        a = O.bb_to_monty(v)
        assert O.bb_from_monty(O.bb_mul(a, O.bb_inv(a))) == 1


def test_bb_root_orders():
    one = O.bb_to_monty(1)
    for k in range(1, 28):
        g = O.bb_two_adic_generator(k)
        v = g
        for _ in range(k):
            v = O.bb_mul(v, v)
        assert v == one
        v = g
        for _ in range(k - 1):
            v = O.bb_mul(v, v)
        assert v != one
    pm1, c = P - 1, 0
    while pm1 % 2 == 0:
        pm1 //= 2
        c += 1
    assert (c, pm1) == (27, 15)


# ---- M31 / circle KATs (tests/field_vectors.rs:118-182, circle.rs tests) ----
def test_m31_kats():
    assert MP == 2147483647
    assert O.m31_mul(123, 456) == 56088
    assert O.m31_mul(MP - 1, MP - 1) == 1
    assert O.m31_add(MP - 1, 1) == 0
    assert O.m31_add(MP - 1, MP - 1) == MP - 2
    assert O.m31_sub(0, 1) == MP - 1
    assert O.m31_sub(8, 3) == 5
    inv7 = O.m31_inv(7)
    assert O.m31_mul(7, inv7) == 1 and inv7 == modpow(7, MP - 2, MP)
    assert O.m31_inv(1) == 1 and O.m31_inv(MP - 1) == MP - 1
    assert O.m31_reduce(0) == 0 and O.m31_reduce(MP) == 0
    assert O.m31_mul(42, O.m31_inv(42)) == 1


def test_circle_generator():
    L = O.lib()
    g = L.orc_circle_subgroup_gen(31)
    assert (g.x, g.y) == (2, 1268011823)
    assert O.m31_add(O.m31_mul(g.x, g.x), O.m31_mul(g.y, g.y)) == 1
    p = g
    for _ in range(30):
        p = L.orc_circle_double(p)
    assert (p.x, p.y) != (1, 0)
    p = L.orc_circle_double(p)
    assert (p.x, p.y) == (1, 0)
    d, a = L.orc_circle_double(g), L.orc_circle_add(g, g)
    assert (d.x, d.y) == (a.x, a.y)


# ---- NTT KATs and structural tests -------------------------------------------
def test_bb_polynomial_multiplication():  # ntt_cross_validation.rs:113-148
    a = O.bb_forward([O.bb_to_monty(1), O.bb_to_monty(2), 0, 0])
    b = O.bb_forward([O.bb_to_monty(3), O.bb_to_monty(4), 0, 0])
    c = O.bb_inverse([O.bb_mul(int(x), int(y)) for x, y in zip(a, b)])
    assert [O.bb_from_monty(int(v)) for v in c] == [3, 10, 8, 0]


def _naive_dft_bitrev(x):
    n = len(x)
    log_n = n.bit_length() - 1
    w = O.bb_from_monty(O.bb_two_adic_generator(log_n))
    nat = [sum(int(x[i]) * pow(w, i * k, P) for i in range(n)) % P for k in range(n)]
    rev = [int(format(k, f"0{log_n}b")[::-1], 2) for k in range(n)]
    return [nat[r] for r in rev]


@pytest.mark.parametrize("log_n", [2, 3, 4, 8, 10])
def test_bb_forward_matches_plonky3_property(log_n):  # ntt_cross_validation.rs:43-110
    n = 1 << log_n
    x = [(i * 7 + 3) % P for i in range(n)]
    got = O.bb_from_monty_array(O.bb_forward(O.bb_to_monty_array(x)))
    assert list(got) == _naive_dft_bitrev(x)


def test_bb_inverse_of_plonky3_forward():  # ntt_cross_validation.rs:151-182
    vals = list(range(1, 17))
    ev = _naive_dft_bitrev(vals)
    got = O.bb_from_monty_array(O.bb_inverse(O.bb_to_monty_array(ev)))
    assert list(got) == vals


def test_m31_constant_and_zero_polys():  # ntt_cross_validation.rs:347-376
    assert list(O.m31_forward([1, 0, 0, 0])) == [1, 1, 1, 1]
    x = np.zeros(16, np.uint32)
    x[0] = 1
    assert np.all(O.m31_forward(x) == 1)
    for log_n in range(1, 9):
        assert not O.m31_forward(np.zeros(1 << log_n, np.uint32)).any()


def test_m31_linearity_and_roundtrip():  # ntt_cross_validation.rs:300-344
    n = 16
    a = np.array([i + 1 for i in range(n)], np.uint32)
    b = np.array([i * 3 + 2 for i in range(n)], np.uint32)
    fa, fb = O.m31_forward(a), O.m31_forward(b)
    fab = O.m31_forward([O.m31_add(int(x), int(y)) for x, y in zip(a, b)])
    assert list(fab) == [O.m31_add(int(x), int(y)) for x, y in zip(fa, fb)]
    for log_n in range(1, 13):
        n = 1 << log_n
        x = O.lcg(n, n * 11111 + 98765, MP)
        f = O.m31_forward(x)
        assert not np.array_equal(f, x)
        assert np.array_equal(O.m31_inverse(f), x)


def test_bb_linearity_roundtrip_edges():  # babybear/cpu_reference.rs:196-297
    n = 16
    a = O.bb_to_monty_array([i + 1 for i in range(n)])
    b = O.bb_to_monty_array([i * 3 + 2 for i in range(n)])
    fab = O.bb_forward([O.bb_add(int(x), int(y)) for x, y in zip(a, b)])
    fa, fb = O.bb_forward(a), O.bb_forward(b)
    assert list(fab) == [O.bb_add(int(x), int(y)) for x, y in zip(fa, fb)]
    for n in (4, 256, 1024, 4096):
        x = O.lcg(n, 12345 + n, P, monty=True)
        assert np.array_equal(O.bb_inverse(O.bb_forward(x)), x)
    assert not O.bb_forward(np.zeros(16, np.uint32)).any()
    assert list(O.bb_forward([O.bb_to_monty(42)])) == [O.bb_to_monty(42)]
    for bad in ([], [1, 2, 3]):
        with pytest.raises(O.InvalidSize):
            O.bb_forward(bad)
        with pytest.raises(O.InvalidSize):
            O.m31_inverse(bad)


def test_bb_twiddle_inverses():  # babybear/twiddles.rs:32-75
    fwd, inv = O.bb_twiddles(4), O.bb_twiddles(4, inverse=True)
    one = O.bb_to_monty(1)
    assert all(O.bb_mul(int(f), int(i)) == one for f, i in zip(fwd, inv))
    assert fwd[0] == one and fwd[1] == one and fwd[3] == one


# ---- oracle vs the independent restatement's fixtures -----------------------
def test_oracle_matches_golden_ntts(golden):
    meta, arr = golden
    fns = {"bb_forward": O.bb_forward, "bb_inverse": O.bb_inverse,
           "m31_forward": O.m31_forward, "m31_inverse": O.m31_inverse}
    for key, fn in fns.items():
        assert meta[key]
        for case in meta[key]:
            got = fn(arr[case["input"]])
            assert np.array_equal(got, arr[case["output"]]), (key, case["log_n"])


def test_oracle_matches_golden_twiddles(golden):
    meta, _ = golden
    for case in meta["bb_twiddles"]:
        t = O.bb_twiddles(case["log_n"], case["inverse"])
        assert sha(t) == case["sha256"] and list(t[:16]) == case["head"]
    for case in meta["m31_twiddles"]:
        t = O.m31_twiddles(case["log_n"], case["inverse"])
        assert sha(t) == case["sha256"] and list(t[:16]) == case["head"]


def test_oracle_matches_golden_lde(golden):
    meta, arr = golden
    for case in meta["bb_lde"]:
        ln, b, ab = case["log_n"], case["batch"], case["added_bits"]
        inp = O.lcg(b << ln, case["seed"], P, monty=True)
        if "input" in case:
            assert np.array_equal(inp, arr[case["input"]])
        out = O.bb_coset_lde(inp, ln, b, ab, case.get("shift_monty", 0))
        assert sha(out) == case["sha256"], case
        par = O.bb_coset_lde(inp, ln, b, ab, case.get("shift_monty", 0), threads=4)
        assert np.array_equal(out, par)
    for case in meta["m31_lde"]:
        ln, b, ab = case["log_n"], case["batch"], case["added_bits"]
        out = O.m31_lde(arr[case["input"]], ln, b, ab)
        assert np.array_equal(out, arr[case["output"]])


def test_reference_lde_shift_default():
    # lde/mod.rs:59, :158 -- shift = two_adic_generator(log_n_ext + 1)
    assert O.bb_from_monty(O.bb_two_adic_generator(22)) == 570250684
    assert O.bb_from_monty(O.bb_two_adic_generator(23)) == 1267047229


# ---- KoalaBear (planned in the reference, README.md:20; no reference code) ---
# The oracle runs the BabyBear code path over KoalaBear's constants, so the
# BabyBear pins above cover the algorithm; these pin the constants and the
# transforms against closed forms computed here in plain Python.
KP = O.KB_P


def _kb_from(a):
    return [O.kb_from_monty(int(v)) for v in np.asarray(a).ravel()]


def _kb_to(a):
    return np.array([O.kb_to_monty(int(v)) for v in a], dtype=np.uint32)


def _bitrev(k, bits):
    return int(format(k, f"0{bits}b")[::-1], 2) if bits else 0


def test_kb_constants():
    assert KP == (1 << 31) - (1 << 24) + 1
    assert (KP - 1) == (1 << 24) * 127
    assert O.kb_to_monty(1) == (1 << 32) % KP
    assert O.kb_to_monty(5) == (5 << 32) % KP
    for v in (0, 1, 2, 12345, KP - 1):
        assert O.kb_from_monty(O.kb_to_monty(v)) == v
    rinv = pow(1 << 32, -1, KP)
    for a, b in ((3, 5), (KP - 1, KP - 2), (1 << 30, 987654321)):
        assert O.kb_mul(a, b) == a * b * rinv % KP
    # 3 generates the multiplicative group: 3^((p-1)/q) != 1 for q in {2, 127}
    assert pow(3, (KP - 1) // 2, KP) != 1 and pow(3, (KP - 1) // 127, KP) != 1


@pytest.mark.parametrize("k", [0, 1, 2, 5, 13, 23, 24])
def test_kb_two_adic_generator_order(k):
    g = O.kb_from_monty(O.kb_two_adic_generator(k))
    assert g == pow(3, (KP - 1) >> k, KP)
    assert pow(g, 1 << k, KP) == 1
    if k:
        assert pow(g, 1 << (k - 1), KP) == KP - 1


def _kb_naive_dft_bitrev(x):
    n = len(x)
    log_n = n.bit_length() - 1
    w = pow(3, (KP - 1) >> log_n, KP)
    nat = [sum(int(x[i]) * pow(w, i * k, KP) for i in range(n)) % KP for k in range(n)]
    return [nat[_bitrev(k, log_n)] for k in range(n)]


@pytest.mark.parametrize("log_n", [1, 2, 3, 5, 8, 10])
def test_kb_forward_is_bitreversed_dft(log_n):
    n = 1 << log_n
    x = [(i * 7919 + 11) % KP for i in range(n)]
    assert _kb_from(O.kb_forward(_kb_to(x))) == _kb_naive_dft_bitrev(x)
    # inverse: bit-reversed evaluations back to coefficients, times n^-1 n
    assert _kb_from(O.kb_inverse(_kb_to(_kb_naive_dft_bitrev(x)))) == x


def test_kb_twiddles_and_batches():
    tw, itw = O.kb_twiddles(6), O.kb_twiddles(6, inverse=True)
    for s in range(6):
        g = pow(3, (KP - 1) >> (s + 1), KP)
        for j in range(1 << s):
            assert O.kb_from_monty(int(tw[(1 << s) - 1 + j])) == pow(g, j, KP)
            assert O.kb_from_monty(int(itw[(1 << s) - 1 + j])) == pow(g, KP - 1 - j, KP)
    x = O.lcg(5 << 7, 77, KP, monty=True)
    fw = O.kb_forward_batch(x, 7, 5, threads=3)
    for c in range(5):
        assert np.array_equal(fw[c << 7:(c + 1) << 7], O.kb_forward(x[c << 7:(c + 1) << 7]))
    assert np.array_equal(O.kb_inverse_batch(fw, 7, 5), x)
    with pytest.raises(O.InvalidSize):
        O.kb_forward(np.zeros(1 << 25, dtype=np.uint32))


@pytest.mark.parametrize("log_n,batch,added,shift", [(3, 2, 1, 0), (4, 1, 2, 0), (0, 3, 2, 0), (5, 2, 1, 3)])
def test_kb_coset_lde_is_coset_evaluation(log_n, batch, added, shift):
    n, ext = 1 << log_n, log_n + added
    x = O.lcg(batch * n, 900 + log_n, KP, monty=True)
    out = O.kb_coset_lde(x, log_n, batch, added, O.kb_to_monty(shift) if shift else 0)
    g = shift or pow(3, (KP - 1) >> (ext + 1), KP)        # default: two_adic_generator(ext + 1)
    w = pow(3, (KP - 1) >> ext, KP)
    for c in range(batch):
        coeffs = _kb_from(O.kb_inverse(x[c * n:(c + 1) * n]))   # bit-reversed evaluations -> coefficients
        want = [sum(a * pow(g * pow(w, k, KP) % KP, i, KP) for i, a in enumerate(coeffs)) % KP
                for k in range(1 << ext)]
        got = _kb_from(out[c << ext:(c + 1) << ext])
        assert got == [want[_bitrev(r, ext)] for r in range(1 << ext)], c
    assert np.array_equal(out, O.kb_coset_lde(x, log_n, batch, added, O.kb_to_monty(shift) if shift else 0, threads=2))


# ---- CM31 = M31[i] / (i^2 + 1) (planned in the reference, TODOS.md:27-31) ----
def test_cm31_mul_is_complex_product():
    rng = np.random.default_rng(3)
    a = rng.integers(0, MP, 2 * 64, dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, MP, 2 * 64, dtype=np.uint64).astype(np.uint32)
    got = O.cm31_mul(a, b)
    for k in range(64):
        ar, ai, br, bi = (int(a[2 * k]), int(a[2 * k + 1]), int(b[2 * k]), int(b[2 * k + 1]))
        assert int(got[2 * k]) == (ar * br - ai * bi) % MP
        assert int(got[2 * k + 1]) == (ar * bi + ai * br) % MP
    i = np.array([0, 1], np.uint32)
    assert list(O.cm31_mul(i, i)) == [MP - 1, 0]  # i^2 = -1


def test_cm31_ntt_is_componentwise():
    log_n, batch = 6, 3
    re = O.lcg(batch << log_n, 5, MP)
    im = O.lcg(batch << log_n, 6, MP)
    pairs = np.empty(2 * re.size, np.uint32)
    pairs[0::2], pairs[1::2] = re, im
    fw = O.cm31_ntt(pairs, log_n, batch)
    n = 1 << log_n
    for c in range(batch):
        col = fw[2 * c * n:2 * (c + 1) * n]
        assert np.array_equal(col[0::2], O.m31_forward(re[c * n:(c + 1) * n]))
        assert np.array_equal(col[1::2], O.m31_forward(im[c * n:(c + 1) * n]))
    assert np.array_equal(O.cm31_ntt(fw, log_n, batch, inverse=True), pairs)
    # C-linearity: transform(i * x) = i * transform(x)
    i_pairs = O.cm31_mul(np.tile(np.array([0, 1], np.uint32), re.size), pairs)
    assert np.array_equal(O.cm31_ntt(i_pairs, log_n, batch),
                          O.cm31_mul(np.tile(np.array([0, 1], np.uint32), re.size), fw))


# ---- canonic-coset circle FFT / circle LDE (Stwo-style; not in the reference) ---
# Pinned here against its definition, evaluated directly in Python integers:
# domain odds(k) ordered h_0..h_{n/2-1}, conj(h_0).., h_i = (1 + 4i) G_{2^(k+1)};
# storage r holds f(D[bitrev_k(r)]); coefficient r multiplies
# y^{r_0} x^{r_1} pi(x)^{r_2} ..., pi(x) = 2x^2 - 1.
def _cadd(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % MP, (a[0] * b[1] + a[1] * b[0]) % MP)


def _cmul(p, m):
    r, b = (1, 0), p
    while m:
        if m & 1:
            r = _cadd(r, b)
        b = _cadd(b, b)
        m >>= 1
    return r


def _gen(k):
    g = (2, 1268011823)  # circle.rs:17-20, order 2^31
    for _ in range(31 - k):
        g = _cadd(g, g)
    return g


def _domain(k):
    n = 1 << k
    g = _gen(k + 1)
    half = [_cmul(g, 1 + 4 * i) for i in range(n // 2)]
    return half + [(x, (-y) % MP) for (x, y) in half]


def _basis(r, k, pt):
    x, y = pt
    v = y if r & 1 else 1
    for j in range(1, k):
        if (r >> j) & 1:
            v = v * x % MP
        x = (2 * x * x - 1) % MP
    return v


def _circle_eval(coeffs, k_dom):
    """Values of sum_r c_r b_r on D_{k_dom}, bit-reversed storage order."""
    dom = _domain(k_dom)
    n = 1 << k_dom
    nat = [sum(int(c) * _basis(r, k_dom, p) for r, c in enumerate(coeffs)) % MP for p in dom]
    return [nat[_bitrev(r, k_dom)] for r in range(n)]


@pytest.mark.parametrize("log_n", [1, 2, 3, 4, 6])
def test_circle_fft_is_basis_evaluation(log_n):
    c = O.lcg(1 << log_n, 70 + log_n, MP)
    assert list(O.circle_ntt(c, log_n)) == _circle_eval(c, log_n)
    assert np.array_equal(O.circle_ntt(O.circle_ntt(c, log_n), log_n, inverse=True), c)


@pytest.mark.parametrize("log_n,added", [(1, 1), (2, 1), (3, 2), (4, 1), (5, 3)])
def test_circle_lde_is_low_degree_extension(log_n, added):
    """The extension evaluates, on the bigger canonic coset, the same circle
    polynomial that interpolates the input: a genuine low-degree extension."""
    x = O.lcg(2 << log_n, 90 + log_n, MP)
    out = O.circle_lde(x, log_n, 2, added)
    n, n_ext = 1 << log_n, 1 << (log_n + added)
    for c in range(2):
        coeffs = O.circle_ntt(x[c * n:(c + 1) * n], log_n, inverse=True)
        assert list(out[c * n_ext:(c + 1) * n_ext]) == _circle_eval(coeffs, log_n + added)
    assert np.array_equal(O.circle_lde(x, log_n, 2, added, threads=2), out)
    tw = O.circle_twiddles(log_n + added)
    assert np.array_equal(O.circle_twiddles(log_n + added, inverse=True),
                          np.array([pow(int(t), MP - 2, MP) for t in tw], np.uint32))

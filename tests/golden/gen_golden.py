#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/ from an independent restatement.

This is a second, pure-Python restatement of the reference's CPU path, written
with Python integers and `pow(.., -1, p)` (no Montgomery REDC code, no shared
code with oracle/oracle.c).  Before writing anything it checks itself against
closed forms that the reference's own tests pin:

* BabyBear forward == bit-reversal of the natural-order DFT with
  omega = two_adic_generator(log n)  (tests/ntt_cross_validation.rs:43-110,
  the Plonky3 Radix2Dit cross-check; Plonky3's TWO_ADIC_GENERATOR 0x1a427a41 =
  440564289 is the reference's root, src/field/babybear.rs:35-37).
* BabyBear inverse of the bit-reversed DFT recovers the input
  (tests/ntt_cross_validation.rs:151-182) and (1+2x)(3+4x) = [3,10,8,0]
  (:113-148).
* M31 forward == the butterfly network written as a direct sum
  out[k] = sum_i c_i prod_{L in bits(i)} (-1)^{k_L} T_L[k >> (L+1)]
  (src/ntt/m31/cpu_reference.rs:61-74), constant poly -> all ones (:347-361).
* Coset LDE == evaluations of the interpolant on shift * <omega_ext> in
  bit-reversed order (src/lde/mod.rs:127-176).

Run:  python tests/golden/gen_golden.py      (writes fixtures next to itself)
"""
from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

BB_P = 2013265921
M31_P = (1 << 31) - 1
R = 1 << 32
R_INV = pow(R, -1, BB_P)
BB_ROOT = 440564289  # canonical primitive 2^27-th root (babybear.rs:35)


# ---------------------------------------------------------------- BabyBear ---
def to_m(v: int) -> int: return (v * R) % BB_P
def from_m(m: int) -> int: return (m * R_INV) % BB_P
def mm(a: int, b: int) -> int: return (a * b * R_INV) % BB_P  # Montgomery product


def bb_gen(k: int) -> int:
    """two_adic_generator(k) in canonical form."""
    return pow(BB_ROOT, 1 << (27 - k), BB_P)


def bb_tw(log_n: int, inverse: bool) -> list[list[int]]:
    """Per-layer twiddles in Montgomery form (babybear.rs:83-97)."""
    out = []
    for s in range(log_n):
        g = bb_gen(s + 1)
        if inverse:
            g = pow(g, -1, BB_P)
        out.append([to_m(pow(g, j, BB_P)) for j in range(1 << s)])
    return out


def bb_forward(d: list[int]) -> list[int]:
    d = list(d)
    n = len(d)
    log_n = n.bit_length() - 1
    tw = bb_tw(log_n, False)
    for layer in reversed(range(log_n)):
        half = 1 << layer
        for blk in range(0, n, 2 * half):
            for j in range(half):
                a, b = d[blk + j], d[blk + j + half]
                d[blk + j] = (a + b) % BB_P
                d[blk + j + half] = mm((a - b) % BB_P, tw[layer][j])
    return d


def bb_inverse(d: list[int], normalize: bool = True) -> list[int]:
    d = list(d)
    n = len(d)
    log_n = n.bit_length() - 1
    tw = bb_tw(log_n, True)
    for layer in range(log_n):
        half = 1 << layer
        for blk in range(0, n, 2 * half):
            for j in range(half):
                t = mm(d[blk + j + half], tw[layer][j])
                a = d[blk + j]
                d[blk + j] = (a + t) % BB_P
                d[blk + j + half] = (a - t) % BB_P
    if normalize and n > 1:
        inv_n = to_m(pow(n, -1, BB_P))
        d = [mm(x, inv_n) for x in d]
    return d


def bitrev(i: int, bits: int) -> int:
    return int(format(i, f"0{bits}b")[::-1], 2) if bits else 0


def bb_naive_dft_bitrev(x_canon: list[int]) -> list[int]:
    n = len(x_canon)
    log_n = n.bit_length() - 1
    w = bb_gen(log_n)
    nat = [sum(x_canon[i] * pow(w, i * k, BB_P) for i in range(n)) % BB_P for k in range(n)]
    return [nat[bitrev(k, log_n)] for k in range(n)]


def bb_lde(inp: list[int], log_n: int, batch: int, added: int, shift_m: int | None) -> list[int]:
    n, ln_ext = 1 << log_n, log_n + added
    n_ext = 1 << ln_ext
    shift = from_m(shift_m) if shift_m else bb_gen(ln_ext + 1)
    out = []
    for c in range(batch):
        col = bb_inverse(inp[c * n:(c + 1) * n]) if n > 1 else list(inp[c * n:(c + 1) * n])
        col = col + [0] * (n_ext - n)
        col = [mm(v, to_m(pow(shift, i, BB_P))) for i, v in enumerate(col)]
        out += bb_forward(col) if n_ext > 1 else col
    return out


def bb_lde_naive(inp: list[int], log_n: int, batch: int, added: int) -> list[int]:
    n, ln_ext = 1 << log_n, log_n + added
    n_ext = 1 << ln_ext
    shift = bb_gen(ln_ext + 1)
    w_n, w_e = bb_gen(log_n), bb_gen(ln_ext)
    inv_n = pow(n, -1, BB_P)
    out = []
    for c in range(batch):
        ev_nat = [from_m(inp[c * n + bitrev(k, log_n)]) for k in range(n)]
        coef = [inv_n * sum(ev_nat[k] * pow(w_n, (n - 1) * i * k, BB_P) for k in range(n)) % BB_P
                for i in range(n)]
        nat = [sum(coef[i] * pow(shift * pow(w_e, k, BB_P), i, BB_P) for i in range(n)) % BB_P
               for k in range(n_ext)]
        out += [to_m(nat[bitrev(k, ln_ext)]) for k in range(n_ext)]
    return out


# --------------------------------------------------------------------- M31 ---
def cadd(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % M31_P, (a[0] * b[1] + a[1] * b[0]) % M31_P)


def cdbl(a):
    return ((2 * a[0] * a[0] - 1) % M31_P, (2 * a[0] * a[1]) % M31_P)


CIRCLE_GEN = (2, 1268011823)


def subgroup_gen(k: int):
    p = CIRCLE_GEN
    for _ in range(31 - k):
        p = cdbl(p)
    return p


def m31_tw(log_n: int, inverse: bool) -> list[list[int]]:
    """Layer l: x (y on the last layer) of the l-times-doubled odds(log_n) coset
    at bit-reversed positions (m31/twiddles.rs:19-68).  Points are enumerated by
    repeated addition, not scalar multiplication: same group elements."""
    init, step, ls = subgroup_gen(log_n + 1), subgroup_gen(log_n), log_n
    out = []
    for layer in range(log_n):
        size = 1 << ls
        pts, cur = [], init
        for _ in range(size):
            pts.append(cur)
            cur = cadd(cur, step)
        half = size // 2
        coord = 1 if layer == log_n - 1 else 0
        row = [pts[bitrev(i, ls - 1)][coord] for i in range(half)]
        if inverse:
            row = [pow(t, -1, M31_P) if t else 0 for t in row]
        out.append(row)
        init, step, ls = cdbl(init), cdbl(step), ls - 1
    return out


def m31_forward(d: list[int]) -> list[int]:
    d = list(d)
    n = len(d)
    log_n = n.bit_length() - 1
    tw = m31_tw(log_n, False)
    for layer in reversed(range(log_n)):
        half = 1 << layer
        for bi, blk in enumerate(range(0, n, 2 * half)):
            t = tw[layer][bi]
            for j in range(half):
                a, b = d[blk + j], d[blk + j + half]
                tb = b * t % M31_P
                d[blk + j] = (a + tb) % M31_P
                d[blk + j + half] = (a - tb) % M31_P
    return d


def m31_inverse(d: list[int]) -> list[int]:
    d = list(d)
    n = len(d)
    log_n = n.bit_length() - 1
    tw = m31_tw(log_n, True)
    for layer in range(log_n):
        half = 1 << layer
        for bi, blk in enumerate(range(0, n, 2 * half)):
            t = tw[layer][bi]
            for j in range(half):
                a, b = d[blk + j], d[blk + j + half]
                d[blk + j] = (a + b) % M31_P
                d[blk + j + half] = (a - b) * t % M31_P
    inv_n = pow(n, -1, M31_P)
    return [x * inv_n % M31_P for x in d]


def m31_forward_direct(c: list[int]) -> list[int]:
    n = len(c)
    log_n = n.bit_length() - 1
    tw = m31_tw(log_n, False)
    out = []
    for k in range(n):
        s = [(-1 if (k >> L) & 1 else 1) * tw[L][k >> (L + 1)] for L in range(log_n)]
        acc = 0
        for i in range(n):
            term = c[i]
            for L in range(log_n):
                if (i >> L) & 1:
                    term = term * s[L] % M31_P
            acc += term
        out.append(acc % M31_P)
    return out


def m31_lde(inp: list[int], log_n: int, batch: int, added: int) -> list[int]:
    n, n_ext = 1 << log_n, 1 << (log_n + added)
    out = []
    for c in range(batch):
        col = inp[c * n:(c + 1) * n]
        col = m31_inverse(col) if n > 1 else list(col)
        col = col + [0] * (n_ext - n)
        out += m31_forward(col) if n_ext > 1 else col
    return out


# ------------------------------------------------------------------- data ----
def lcg(n: int, seed: int, p: int) -> list[int]:
    s, out = seed, []
    for _ in range(n):
        s = (s * 6364136223846793005 + 1) & ((1 << 64) - 1)
        out.append((s >> 33) % p)
    return out


def sha(vals) -> str:
    return hashlib.sha256(np.asarray(vals, dtype="<u4").tobytes()).hexdigest()


# ------------------------------------------------------------- self-checks ---
def self_check() -> None:
    # Plonky3 property and the reference's fixed patterns
    for log_n in (2, 3, 4, 8):
        n = 1 << log_n
        x = [(i * 7 + 3) % BB_P for i in range(n)]
        got = [from_m(v) for v in bb_forward([to_m(v) for v in x])]
        assert got == bb_naive_dft_bitrev(x), log_n
    x = [1, 2, 3, 4]
    assert [from_m(v) for v in bb_forward([to_m(v) for v in x])] == bb_naive_dft_bitrev(x)
    # Plonky3 forward -> our inverse recovers 1..16
    vals = list(range(1, 17))
    ev = bb_naive_dft_bitrev(vals)
    assert [from_m(v) for v in bb_inverse([to_m(v) for v in ev])] == vals
    # (1+2x)(3+4x)
    a = bb_forward([to_m(1), to_m(2), 0, 0])
    b = bb_forward([to_m(3), to_m(4), 0, 0])
    c = bb_inverse([mm(u, v) for u, v in zip(a, b)])
    assert [from_m(v) for v in c] == [3, 10, 8, 0]
    # M31: direct sum, constant poly, round trip
    for log_n in range(1, 7):
        n = 1 << log_n
        c = lcg(n, n * 11111 + 98765, M31_P)
        assert m31_forward(c) == m31_forward_direct(c), log_n
        assert m31_inverse(m31_forward(c)) == c
    assert m31_forward([1, 0, 0, 0]) == [1, 1, 1, 1]
    # LDE against naive coset evaluation
    for (ln, b, ab) in ((2, 2, 1), (3, 2, 1), (3, 1, 2), (4, 2, 1)):
        inp = [to_m(v) for v in lcg(b << ln, 42, BB_P)]
        assert bb_lde(inp, ln, b, ab, None) == bb_lde_naive(inp, ln, b, ab), (ln, b, ab)


# -------------------------------------------------------------- fixtures ----
def main() -> None:
    self_check()
    fx: dict = {"bb_forward": [], "bb_inverse": [], "m31_forward": [], "m31_inverse": [],
                "bb_lde": [], "m31_lde": [], "bb_twiddles": [], "m31_twiddles": []}
    arrays: dict[str, np.ndarray] = {}

    def put(key: str, vals) -> str:
        arrays[key] = np.asarray(vals, dtype=np.uint32)
        return key

    for log_n in range(0, 11):
        n = 1 << log_n
        # BabyBear: reference pattern (i*7+3) and the LCG (test_utils.rs seeds)
        x = [to_m((i * 7 + 3) % BB_P) for i in range(n)]
        y = [to_m(v) for v in lcg(n, n * 11111 + 98765, BB_P)]
        for tag, inp in (("pattern", x), ("lcg", y)):
            fwd = bb_forward(inp) if n > 1 else list(inp)
            inv = bb_inverse(inp) if n > 1 else list(inp)
            fx["bb_forward"].append({"log_n": log_n, "tag": tag, "input": put(f"bbf_in_{tag}_{log_n}", inp),
                                     "output": put(f"bbf_out_{tag}_{log_n}", fwd)})
            fx["bb_inverse"].append({"log_n": log_n, "tag": tag, "input": put(f"bbi_in_{tag}_{log_n}", inp),
                                     "output": put(f"bbi_out_{tag}_{log_n}", inv)})
        c = lcg(n, n * 11111 + 98765, M31_P)
        fwd = m31_forward(c) if n > 1 else list(c)
        inv = m31_inverse(c) if n > 1 else list(c)
        fx["m31_forward"].append({"log_n": log_n, "input": put(f"m31f_in_{log_n}", c),
                                  "output": put(f"m31f_out_{log_n}", fwd)})
        fx["m31_inverse"].append({"log_n": log_n, "input": put(f"m31i_in_{log_n}", c),
                                  "output": put(f"m31i_out_{log_n}", inv)})
    for log_n in (1, 2, 5, 8, 12):
        for inverse in (False, True):
            flat = [v for layer in bb_tw(log_n, inverse) for v in layer]
            fx["bb_twiddles"].append({"log_n": log_n, "inverse": inverse, "sha256": sha(flat),
                                      "head": flat[:16]})
            flat = [v for layer in m31_tw(log_n, inverse) for v in layer]
            fx["m31_twiddles"].append({"log_n": log_n, "inverse": inverse, "sha256": sha(flat),
                                       "head": flat[:16]})
    # LDE cases: the reference's own (src/lde/mod.rs:194-271, seed 42) plus edges.
    lde_cases = [(8, 4, 1, True), (8, 4, 2, True), (12, 8, 1, False), (0, 3, 1, True),
                 (1, 2, 2, True), (5, 3, 3, True), (10, 2, 1, False)]
    for (ln, b, ab, full) in lde_cases:
        inp = [to_m(v) for v in lcg(b << ln, 42, BB_P)]
        out = bb_lde(inp, ln, b, ab, None)
        rec = {"log_n": ln, "batch": b, "added_bits": ab, "seed": 42, "sha256": sha(out)}
        if full:
            rec["input"] = put(f"lde_in_{ln}_{b}_{ab}", inp)
            rec["output"] = put(f"lde_out_{ln}_{b}_{ab}", out)
        fx["bb_lde"].append(rec)
    # g = 31 (Plonky3 convention) shift mode, separately oracled
    inp = [to_m(v) for v in lcg(4 << 6, 7, BB_P)]
    out = bb_lde(inp, 6, 4, 1, to_m(31))
    fx["bb_lde"].append({"log_n": 6, "batch": 4, "added_bits": 1, "seed": 7, "shift_monty": to_m(31),
                         "sha256": sha(out), "input": put("lde31_in", inp), "output": put("lde31_out", out)})
    for (ln, b, ab) in ((6, 3, 1), (4, 2, 2), (9, 2, 1)):
        inp = lcg(b << ln, 1234 + ln, M31_P)
        out = m31_lde(inp, ln, b, ab)
        fx["m31_lde"].append({"log_n": ln, "batch": b, "added_bits": ab, "sha256": sha(out),
                              "input": put(f"m31lde_in_{ln}_{b}_{ab}", inp),
                              "output": put(f"m31lde_out_{ln}_{b}_{ab}", out)})

    np.savez_compressed(HERE / "golden.npz", **arrays)
    (HERE / "golden.json").write_text(json.dumps(fx, indent=1) + "\n")
    print(f"wrote {len(arrays)} arrays, {sum(a.size for a in arrays.values())} values")


if __name__ == "__main__":
    main()

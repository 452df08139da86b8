"""
oracle.pyoracle — the reference's CPU algorithms restated on Python integers.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py): the checker for the GPU
path, never the product. Each function cites the reference file:line it
follows; the arithmetic is the reference's, so results are bit-identical to
running the reference itself (tests/test_oracle_golden.py pins that).
"""

from __future__ import annotations

# zkgpu/field.py:17 (r) and zkgpu/curve.py:29 (P)
R = 21888242871839275222246405745257275088548364400416034343698204186575808495617
P = 21888242871839275222246405745257275088696311157297823662689037894645226208583
B = 3
G = (1, 2)
JACOBIAN_IDENTITY = (1, 1, 0)
SCALAR_BITS = R.bit_length()  # 254

Jacobian = tuple[int, int, int]
Affine = tuple[int, int] | None  # None is the point at infinity

# ------------------------------------------------------------------
# Montgomery constants (zkgpu/field256_gpu.py:282-287)
# ------------------------------------------------------------------


def montgomery_constants(p: int) -> dict[str, int]:
    return {
        "r2": pow(2, 512, p),
        "r_inv": pow(2**256, -1, p),
        "n_inv": -pow(p, -1, 2**64) % 2**64,
        "one": 2**256 % p,
    }


def to_mont(v: int, p: int) -> int:
    return v * 2**256 % p


def from_mont(v: int, p: int) -> int:
    return v * pow(2**256, -1, p) % p


def mont_mul(a: int, b: int, p: int) -> int:
    """Montgomery product a * b * 2^-256 mod p of two Montgomery-form values."""
    return a * b * pow(2**256, -1, p) % p


# ------------------------------------------------------------------
# Roots of unity and the NTT (zkgpu/ntt.py:53-203, zkgpu/domain.py)
# ------------------------------------------------------------------

_MR_BASES = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41)


def is_probable_prime(n: int) -> bool:
    """zkgpu/ntt.py:53-71"""
    if n < 2:
        return False
    for q in _MR_BASES:
        if n % q == 0:
            return n == q
    s = ((n - 1) & -(n - 1)).bit_length() - 1
    d = (n - 1) >> s
    for a in _MR_BASES:
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def quadratic_non_residue(mod: int) -> int:
    """zkgpu/ntt.py:74-95"""
    if mod < 3 or not is_probable_prime(mod):
        raise ValueError(f"NTT modulus must be an odd prime, got {mod}")
    g = 2
    while pow(g, (mod - 1) // 2, mod) != mod - 1:
        g += 1
    return g


def get_ntt_root(n: int, mod: int) -> int:
    """zkgpu/ntt.py:98-124"""
    if n < 1 or n & (n - 1):
        raise ValueError(f"NTT size must be a power of 2, got {n}")
    g = quadratic_non_residue(mod)
    if (mod - 1) % n:
        raise ValueError(f"NTT of size {n} not supported for mod={mod}: not divisible by n.")
    return pow(g, (mod - 1) // n, mod)


def _bit_reverse_copy(a: list[int]) -> list[int]:
    """zkgpu/ntt.py:132-141"""
    n = len(a)
    bits = n.bit_length() - 1
    out = a[:]
    for i in range(n):
        rev = int(f"{i:0{bits}b}"[::-1], 2) if bits else 0
        if rev > i:
            out[i], out[rev] = out[rev], out[i]
    return out


def ntt(a: list[int], mod: int = R, invert: bool = False) -> list[int]:
    """Iterative Cooley-Tukey DIT with bit-reversed input (zkgpu/ntt.py:149-203)."""
    n = len(a)
    if n == 0:
        return []
    if n & (n - 1):
        raise ValueError(f"NTT length must be a power of 2, got {n}")
    omega = get_ntt_root(n, mod)
    if invert:
        omega = pow(omega, mod - 2, mod)
    if n == 1:
        return [a[0] % mod]
    a = _bit_reverse_copy([v % mod for v in a])
    length = 2
    while length <= n:
        w_len = pow(omega, n // length, mod)
        half = length >> 1
        for i in range(0, n, length):
            w = 1
            for j in range(half):
                u = a[i + j]
                v = a[i + j + half] * w % mod
                a[i + j] = (u + v) % mod
                a[i + j + half] = (u - v) % mod
                w = w * w_len % mod
        length <<= 1
    if invert:
        n_inv = pow(n, mod - 2, mod)
        a = [x * n_inv % mod for x in a]
    return a


def ntt_np(a, mod: int, invert: bool = False):
    """
    The same transform on a NumPy int64 array, one vectorised stage at a time,
    as the reference's ntt_gpu (zkgpu/ntt_gpu.py:128-153) runs it; for moduli
    below 2^32, where every product fits uint64. Returns an int64 array.
    """
    import numpy as np

    if mod >= 2**32:
        raise ValueError("ntt_np needs mod < 2^32")
    n = len(a)
    omega = get_ntt_root(n, mod)
    if invert:
        omega = pow(omega, mod - 2, mod)
    x = np.mod(np.asarray(a, dtype=np.int64), mod).astype(np.uint64)
    if n == 1:
        return x.astype(np.int64)
    bits = n.bit_length() - 1
    idx = np.arange(n, dtype=np.int64)
    rev = np.zeros(n, dtype=np.int64)
    for b in range(bits):
        rev |= ((idx >> b) & 1) << (bits - 1 - b)
    x = x[rev]
    table = np.ones(n // 2, dtype=np.uint64)  # omega^j, j < n/2
    for j in range(1, n // 2):
        table[j] = table[j - 1] * np.uint64(omega) % np.uint64(mod)
    m = np.uint64(mod)
    length = 2
    while length <= n:
        half = length >> 1
        groups = x.reshape(-1, length)
        upper, lower = groups[:, :half].copy(), groups[:, half:]
        v = lower * table[:: n // length] % m
        groups[:, :half] = (upper + v) % m
        groups[:, half:] = (upper + m - v) % m
        length <<= 1
    if invert:
        x = x * np.uint64(pow(n, mod - 2, mod)) % m
    return x.astype(np.int64)


def scale_by_powers(values: list[int], g: int, mod: int) -> list[int]:
    """zkgpu/domain.py:33-39"""
    out, power = [], 1
    for v in values:
        out.append(v * power % mod)
        power = power * g % mod
    return out


def coset_offset(size: int, mod: int = R) -> int:
    """Radix2Domain's default coset shift (zkgpu/domain.py:71-83); 5 for BN254 Fr."""
    g = quadratic_non_residue(mod)
    while pow(g, size, mod) == 1:
        g += 1
    return g


def coset_fft(coeffs: list[int], g: int, mod: int = R) -> list[int]:
    """zkgpu/domain.py:122-128"""
    return ntt(scale_by_powers(coeffs, g, mod), mod)


def coset_ifft(evals: list[int], g: int, mod: int = R) -> list[int]:
    """zkgpu/domain.py:130-135"""
    return scale_by_powers(ntt(evals, mod, invert=True), pow(g, -1, mod), mod)


def domain_elements(n: int, mod: int = R) -> list[int]:
    """Radix2Domain.elements (zkgpu/domain.py:100-102)"""
    return scale_by_powers([1] * n, get_ntt_root(n, mod), mod)


# ------------------------------------------------------------------
# G1 in Jacobian coordinates (zkgpu/curve.py:213-324)
# ------------------------------------------------------------------


def on_curve(x: int, y: int) -> bool:
    """zkgpu/curve.py:105-110"""
    return (y * y - pow(x, 3, P) - B) % P == 0


def to_jacobian(q: Affine) -> Jacobian:
    """zkgpu/curve.py:213-218"""
    return JACOBIAN_IDENTITY if q is None else (q[0], q[1], 1)


def from_jacobian(j: Jacobian) -> Affine:
    """zkgpu/curve.py:221-233 (None for the identity)."""
    x, y, z = j
    if z == 0:
        return None
    zi = pow(z, -1, P)
    zi2 = zi * zi % P
    out = (x * zi2 % P, y * zi2 % P * zi % P)
    assert on_curve(*out)
    return out


def jacobian_double(j: Jacobian) -> Jacobian:
    """EFD dbl-2009-l (zkgpu/curve.py:236-252)."""
    x1, y1, z1 = j
    if z1 == 0 or y1 == 0:
        return JACOBIAN_IDENTITY
    a = x1 * x1 % P
    b = y1 * y1 % P
    c = b * b % P
    d = 2 * ((x1 + b) * (x1 + b) - a - c) % P
    e = 3 * a % P
    f = e * e % P
    x3 = (f - 2 * d) % P
    y3 = (e * (d - x3) - 8 * c) % P
    z3 = 2 * y1 * z1 % P
    return (x3, y3, z3)


def jacobian_add(j1: Jacobian, j2: Jacobian) -> Jacobian:
    """EFD add-2007-bl (zkgpu/curve.py:255-281)."""
    x1, y1, z1 = j1
    x2, y2, z2 = j2
    if z1 == 0:
        return j2
    if z2 == 0:
        return j1
    z1z1 = z1 * z1 % P
    z2z2 = z2 * z2 % P
    u1 = x1 * z2z2 % P
    u2 = x2 * z1z1 % P
    s1 = y1 * z2 % P * z2z2 % P
    s2 = y2 * z1 % P * z1z1 % P
    h = (u2 - u1) % P
    r = 2 * (s2 - s1) % P
    if h == 0:
        return jacobian_double(j1) if r == 0 else JACOBIAN_IDENTITY
    i = 4 * h * h % P
    j = h * i % P
    v = u1 * i % P
    x3 = (r * r - j - 2 * v) % P
    y3 = (r * (v - x3) - 2 * s1 * j) % P
    z3 = ((z1 + z2) * (z1 + z2) - z1z1 - z2z2) * h % P
    return (x3, y3, z3)


def jacobian_add_affine(j1: Jacobian, x2: int, y2: int) -> Jacobian:
    """EFD madd-2007-bl (zkgpu/curve.py:284-303)."""
    x1, y1, z1 = j1
    if z1 == 0:
        return (x2, y2, 1)
    z1z1 = z1 * z1 % P
    u2 = x2 * z1z1 % P
    s2 = y2 * z1 % P * z1z1 % P
    h = (u2 - x1) % P
    r = 2 * (s2 - y1) % P
    if h == 0:
        return jacobian_double(j1) if r == 0 else JACOBIAN_IDENTITY
    hh = h * h % P
    i = 4 * hh % P
    j = h * i % P
    v = x1 * i % P
    x3 = (r * r - j - 2 * v) % P
    y3 = (r * (v - x3) - 2 * y1 * j) % P
    z3 = ((z1 + h) * (z1 + h) - z1z1 - hh) % P
    return (x3, y3, z3)


def neg(q: Affine) -> Affine:
    return None if q is None else (q[0], -q[1] % P)


def jacobian_mul(q: Affine, k: int) -> Jacobian:
    """Left-to-right double-and-add, scalar used as given (zkgpu/curve.py:306-324)."""
    if k < 0:
        q, k = neg(q), -k
    if k == 0 or q is None:
        return JACOBIAN_IDENTITY
    acc = JACOBIAN_IDENTITY
    for bit in bin(k)[2:]:
        acc = jacobian_double(acc)
        if bit == "1":
            acc = jacobian_add_affine(acc, q[0], q[1])
    return acc


def scalar_mul(q: Affine, k: int) -> Affine:
    """Point.__mul__ (zkgpu/curve.py:153-159)."""
    return from_jacobian(jacobian_mul(q, k))


def affine_add(a: Affine, b: Affine) -> Affine:
    """Point.__add__ (zkgpu/curve.py:116-137), via Jacobian for brevity (same result)."""
    if a is None:
        return b
    if b is None:
        return a
    return from_jacobian(jacobian_add_affine(to_jacobian(a), b[0], b[1]))


# ------------------------------------------------------------------
# MSM (zkgpu/msm.py)
# ------------------------------------------------------------------

MAX_WINDOW_SIZE = 16


def pippenger_window_size(n: int) -> int:
    """zkgpu/msm.py:112-121"""
    return min(range(1, MAX_WINDOW_SIZE + 1), key=lambda w: -(-SCALAR_BITS // w) * (n + 2 ** (w + 1)))


def _window_sum(coords: list[tuple[int, int]], digits: list[int], bucket_count: int) -> Jacobian:
    """zkgpu/msm.py:156-177 (buckets, then the running-sum trick)."""
    buckets = [JACOBIAN_IDENTITY] * bucket_count
    for (x, y), d in zip(coords, digits, strict=True):
        if d:
            buckets[d] = jacobian_add_affine(buckets[d], x, y)
    running = JACOBIAN_IDENTITY
    total = JACOBIAN_IDENTITY
    for k in range(bucket_count - 1, 0, -1):
        running = jacobian_add(running, buckets[k])
        total = jacobian_add(total, running)
    return total


def combine_windows(window_sums: list[Jacobian], w: int) -> Jacobian:
    """Horner from the top window (zkgpu/msm.py:180-193)."""
    acc = window_sums[-1]
    for win in range(len(window_sums) - 2, -1, -1):
        for _ in range(w):
            acc = jacobian_double(acc)
        acc = jacobian_add(acc, window_sums[win])
    return acc


def msm_pippenger(coords: list[tuple[int, int]], scalars: list[int], w: int | None = None) -> Affine:
    """Pippenger on affine coordinates, scalars reduced mod r (zkgpu/msm.py:196-207)."""
    if len(coords) != len(scalars):
        raise ValueError("Length mismatch")
    if not coords:
        return None
    if w is None:
        w = pippenger_window_size(len(coords))
    reduced = [s % R for s in scalars]
    num_windows = -(-SCALAR_BITS // w)
    mask = (1 << w) - 1
    sums = [
        _window_sum(coords, [(s >> (win * w)) & mask for s in reduced], 1 << w)
        for win in range(num_windows)
    ]
    return from_jacobian(combine_windows(sums, w))


def msm_double_and_add(coords: list[tuple[int, int]], scalars: list[int]) -> Affine:
    """Straus/Shamir simultaneous double-and-add (zkgpu/msm.py:61-104)."""
    terms = [((x, y) if s >= 0 else (x, -y % P), abs(s)) for (x, y), s in zip(coords, scalars, strict=True)]
    max_bits = max((s.bit_length() for _, s in terms), default=0)
    acc = JACOBIAN_IDENTITY
    for bit in range(max_bits - 1, -1, -1):
        acc = jacobian_double(acc)
        for (x, y), s in terms:
            if (s >> bit) & 1:
                acc = jacobian_add_affine(acc, x, y)
    return from_jacobian(acc)

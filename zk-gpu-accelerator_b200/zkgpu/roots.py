"""
zkgpu.roots — roots of unity for the NTT, derived on the host.

The same derivation as the reference (zkgpu/ntt.py:46-124): every size's root
comes from the smallest quadratic non-residue g of the field (5 for BN254's
r), as w_n = g^((p - 1) / n), so get_ntt_root(n / 2) == get_ntt_root(n)^2 and
the roots match snarkjs's. The checks, and their ValueError messages, are
the reference's: the size must be a power of two, the modulus an odd prime,
and n must divide p - 1.
"""

from __future__ import annotations

import functools

# Deterministic for n < 3.3e24 (Sorenson & Webster 2015); a strong
# probable-prime test above that.
_MILLER_RABIN_BASES = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41)


def is_probable_prime(n: int) -> bool:
    if n < 2:
        return False
    for p in _MILLER_RABIN_BASES:
        if n % p == 0:
            return n == p
    s = ((n - 1) & -(n - 1)).bit_length() - 1
    d = (n - 1) >> s
    for a in _MILLER_RABIN_BASES:
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


@functools.cache
def quadratic_non_residue(mod: int) -> int:
    """Smallest quadratic non-residue of F_mod; ValueError unless mod is an odd prime."""
    if mod < 3 or not is_probable_prime(mod):
        raise ValueError(f"NTT modulus must be an odd prime, got {mod}")
    g = 2
    while pow(g, (mod - 1) // 2, mod) != mod - 1:
        g += 1
    return g


def get_ntt_root(n: int, mod: int, non_residue: int | None = None) -> int:
    """A primitive n-th root of unity of F_mod for n a power of two (see module docstring)."""
    if n < 1 or n & (n - 1):
        raise ValueError(f"NTT size must be a power of 2, got {n}")
    default_g = quadratic_non_residue(mod)
    g = default_g if non_residue is None else non_residue
    if (mod - 1) % n != 0:
        raise ValueError(
            f"NTT of size {n} not supported for mod={mod}: (mod-1) = {mod - 1} is not divisible by n."
        )
    omega = pow(g, (mod - 1) // n, mod)
    if n > 1 and pow(omega, n // 2, mod) != mod - 1:
        raise ValueError(
            f"{g} gives no primitive {n}-th root of unity mod {mod}; it must be a quadratic non-residue"
        )
    return omega


def default_coset_offset(size: int, mod: int) -> int | None:
    """The coset shift Radix2Domain uses: the smallest g >= the non-residue with g^size != 1
    (zkgpu/domain.py:71-83 of the reference); None if the domain is all of F_mod*."""
    g = quadratic_non_residue(mod)
    while g < mod:
        if pow(g, size, mod) != 1:
            return g
        g += 1
    return None

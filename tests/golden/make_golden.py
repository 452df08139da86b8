"""
Regenerate the golden fixtures in tests/golden/ by running the reference itself.

    python tests/golden/make_golden.py --reference /path/to/zk-gpu-accelerator [--quick]
    (or ZKGPU_REFERENCE=/path/to/zk-gpu-accelerator python tests/golden/make_golden.py)

The reference (erihhh6/zk-gpu-accelerator) is pure Python, so its CPU path is
imported directly from the `src` folder of the checkout given and
run on inputs regenerated from seeds by zkgpu/workloads.py (loaded by file
path, since the reference's package is also named zkgpu). Only results are
stored: big integers as hex strings, and for large transforms the SHA-256 of
the output rows (Montgomery form, little-endian uint64 limbs) plus a few
sample values. Nothing at test time reads the reference; the fixtures carry
its answers.

Contents
  known.json  known answers from the reference's own tests and constants
  field.json  Montgomery rows and mul/add/sub results for five moduli
  ntt.json    NTT / inverse / coset transforms, sizes 1..4096 in full, 2^16 and 2^20 by hash
  curve.json  exact Jacobian results of add / add_affine / double
  msm.json    Pippenger MSM results (small explicit cases; 2^12, 2^14, 2^16 by seed)
  field64.json  int64-field mul/add/pow (zkgpu/field_gpu.py's CPU path) and NTTs over
                moduli below 2^63, the moduli of the reference's own tests

`--only field64.json` (or any other name) rewrites that file alone.
"""

from __future__ import annotations

import argparse
import hashlib
import importlib.util
import json
import os
import random
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent


def _load_workloads():
    path = REPO / "zk-gpu-accelerator_b200" / "zkgpu" / "workloads.py"
    spec = importlib.util.spec_from_file_location("zkb_workloads", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def hx(v: int) -> str:
    return f"{v:x}"


def rows_digest(values: list[int], mod: int, montgomery: bool = True) -> str:
    """SHA-256 of the rows the GPU produces for these values (Montgomery form by default)."""
    h = hashlib.sha256()
    for v in values:
        h.update((v * 2**256 % mod if montgomery else v).to_bytes(32, "little"))
    return h.hexdigest()


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[1])
    ap.add_argument("--reference", default=os.environ.get("ZKGPU_REFERENCE"),
                    help="checkout of the reference repository (or set ZKGPU_REFERENCE)")
    ap.add_argument("--quick", action="store_true", help="skip the 2^16 MSM and 2^20 NTT")
    ap.add_argument("--only", help="write this fixture file alone (field64.json)")
    args = ap.parse_args()
    if not args.reference:
        ap.error("give the reference checkout with --reference or ZKGPU_REFERENCE")
    sys.path.insert(0, str(Path(args.reference) / "src"))
    if args.only == "field64.json":
        field64_fixtures()
        return

    from zkgpu import field256_gpu as ref_f256  # the reference's package
    from zkgpu.curve import (
        JACOBIAN_IDENTITY,
        G,
        P,
        Point,
        from_jacobian,
        jacobian_add,
        jacobian_add_affine,
        jacobian_double,
        jacobian_mul,
    )
    from zkgpu.domain import Radix2Domain
    from zkgpu.field import FIELD_MODULUS as R
    from zkgpu.msm import msm_double_and_add, msm_naive, msm_pippenger, pippenger_window_size
    from zkgpu.ntt import get_ntt_root, ntt, quadratic_non_residue

    wl = _load_workloads()
    ref_f256._gpu_available = False  # its CPU path: identical rows (reference tests :88-94)
    import warnings

    warnings.simplefilter("ignore")

    def dump(name: str, obj: object) -> None:
        (HERE / name).write_text(json.dumps(obj, indent=1, sort_keys=True) + "\n")
        print(f"wrote {name}", file=sys.stderr)

    # ---- known answers (reference tests/test_field256_gpu.py:60-85, test_domain.py:15-16,
    # test_curve.py:26-29, test_ntt.py:135-138, test_msm.py:170-171)
    fr, fq = ref_f256.BN254_FR, ref_f256.BN254_FQ
    dump(
        "known.json",
        {
            "r": hx(R),
            "p": hx(P),
            "fr_ninv": hx(fr._n_inv),
            "fq_ninv": hx(fq._n_inv),
            "fr_r2": hx(fr._r2),
            "fq_r2": hx(fq._r2),
            "fr_one_row": [hx(v) for v in fr.from_ints([1]).tolist()[0]],
            "root_2_28": hx(Radix2Domain(2**28).omega),
            "root_2_28_generator_7": hx(get_ntt_root(2**28, R, non_residue=7)),
            "qnr": {"998244353": quadratic_non_residue(998244353), "r": quadratic_non_residue(R)},
            "two_g": [hx((G * 2).x), hx((G * 2).y)],
            "pippenger_window_size": {str(n): pippenger_window_size(n) for n in (0, 100, 1000, 10000, 100000, 2**16, 2**20, 2**22)},
            "coset_offset_fr": Radix2Domain(8).coset_offset,
        },
    )

    # ---- field ops: the reference test's operand construction (test_field256_gpu.py:46-52)
    def operands(p: int, seed: int):
        edge = sorted({e % p for e in (0, 1, 2, p - 1, p - 2, p // 2, 2**64 - 1, 2**128 - 1, 2**192 - 1)})
        rng = random.Random(seed)
        a = [x for x in edge for _ in edge] + [rng.randrange(p) for _ in range(200)]
        b = edge * len(edge) + [rng.randrange(p) for _ in range(200)]
        return a, b

    field = {}
    for modulus in (R, P, 2**255 - 19, 3, 2**64 + 13):
        F = ref_f256.Field256(modulus)
        a, b = operands(modulus, 1)
        A, B = F.from_ints(a), F.from_ints(b)

        def rows(x):
            return [hx(sum(int(l) << (64 * j) for j, l in enumerate(r))) for r in x.tolist()]

        field[hx(modulus)] = {
            "n_inv": hx(F._n_inv),
            "r2": hx(F._r2),
            "a": [hx(v) for v in a],
            "b": [hx(v) for v in b],
            "a_rows": rows(A),
            "mul_rows": rows(F.mul(A, B)),
            "add_rows": rows(F.add(A, B)),
            "sub_rows": rows(F.sub(A, B)),
        }
    dump("field.json", field)

    # ---- NTT (zkgpu/ntt.py, zkgpu/domain.py), inputs as the reference test draws them
    small = {}
    for n in (1, 2, 4, 8, 64, 1024, 4096):
        rng = random.Random(n)
        a = [rng.randrange(R) for _ in range(n)]
        d = Radix2Domain(n)
        outs = {"fwd": ntt(a, R), "inv": ntt(a, R, invert=True)}
        if d.coset_offset is not None:
            outs["coset_fwd"] = d.coset_fft(a)
            outs["coset_inv"] = d.coset_ifft(a)
        entry = {"coset_offset": d.coset_offset, "input_seed": n}
        for key, vals in outs.items():
            if n <= 1024:  # in full; larger ones by digest (inputs regenerate from random.Random(n))
                entry[key] = [hx(v) for v in vals]
            else:
                entry[key + "_sha256"] = rows_digest(vals, R)
        small[str(n)] = entry
    large = {}
    sizes = [] if args.quick else [2**16, 2**20]
    for n in sizes:
        t0 = time.time()
        seed = 1000 + n.bit_length()
        a = wl.rows_to_ints(wl.uniform_fr(seed, n))
        d = Radix2Domain(n)
        fwd, inv = ntt(a, R), ntt(a, R, invert=True)
        entry = {
            "seed": seed,
            "generator": "uniform_fr",
            "input_sha256": rows_digest(a, R),
            "fwd_sha256": rows_digest(fwd, R),
            "inv_sha256": rows_digest(inv, R),
            "fwd_samples": {str(i): hx(fwd[i]) for i in (0, 1, n // 2, n - 1)},
        }
        if n <= 2**16:
            entry["coset_fwd_sha256"] = rows_digest(d.coset_fft(a), R)
            entry["coset_inv_sha256"] = rows_digest(d.coset_ifft(a), R)
        large[str(n)] = entry
        print(f"ntt 2^{n.bit_length() - 1}: {time.time() - t0:.1f}s", file=sys.stderr)
    dump("ntt.json", {
        "small": small,
        "large": large,
        "elements": {str(n): [hx(v) for v in Radix2Domain(n).elements()] for n in (8, 256)},
    })

    # ---- curve: exact Jacobian results (reference tests/test_curve_gpu.py:45-100)
    def jacobians(n: int, seed: int):
        rng = random.Random(seed)
        return [jacobian_mul(G * rng.randrange(1, R), rng.randrange(2, 2**64)) for _ in range(n)]

    def negate(j):
        return (j[0], -j[1] % P, j[2])

    def jh(j):
        return [hx(c) for c in j]

    js = jacobians(12, 1)
    a = js + js[:4] + js[4:8] + [JACOBIAN_IDENTITY] * 2 + js[8:10]
    b = js[::-1] + js[:4] + [negate(j) for j in js[4:8]] + js[10:12] + [JACOBIAN_IDENTITY] * 2
    add_case = {"a": [jh(j) for j in a], "b": [jh(j) for j in b], "out": [jh(jacobian_add(x, y)) for x, y in zip(a, b)]}
    js = jacobians(10, 2)
    pts = [from_jacobian(j) for j in jacobians(10, 3)]
    same = [from_jacobian(j) for j in js[:4]]
    acc = js + js[:4] + [negate(j) for j in js[4:8]] + [JACOBIAN_IDENTITY] * 2
    q = pts + same + [from_jacobian(j) for j in js[4:8]] + pts[:2]
    mixed_case = {
        "a": [jh(j) for j in acc],
        "b": [[hx(p.x), hx(p.y)] for p in q],
        "out": [jh(jacobian_add_affine(j, p.x, p.y)) for j, p in zip(acc, q)],
    }
    js = [*jacobians(10, 4), JACOBIAN_IDENTITY, (1, 2, 1), (5, 0, 1)]
    dbl_case = {"a": [jh(j) for j in js], "out": [jh(jacobian_double(j)) for j in js]}
    to_affine = {"a": [jh(j) for j in jacobians(6, 5)], "out": [[hx(p.x), hx(p.y)] for p in map(from_jacobian, jacobians(6, 5))]}
    dump("curve.json", {"add": add_case, "add_affine": mixed_case, "double": dbl_case, "to_affine": to_affine})

    # ---- MSM
    def pt(p):
        return None if p.is_identity() else [hx(p.x), hx(p.y)]

    cases = []
    rng = random.Random(29)  # reference tests/test_msm.py:58-63
    points = [G * rng.randint(1, 2**32) for _ in range(30)]
    scalars = [rng.randint(0, 2**32) for _ in range(30)]
    cases.append({"name": "small-scalars-30", "points": [pt(p) for p in points], "scalars": [hx(s) for s in scalars],
                  "expected": pt(msm_naive(points, scalars))})
    rng = random.Random(31)  # :66-72
    points = [G * rng.randint(1, 2**32) for _ in range(12)]
    scalars = [rng.randrange(R) for _ in range(12)]
    cases.append({"name": "full-scalars-12", "points": [pt(p) for p in points], "scalars": [hx(s) for s in scalars],
                  "expected": pt(msm_double_and_add(points, scalars))})
    rng = random.Random(37)  # :262-271
    step = G * rng.randrange(1, R)
    points = [G * rng.randrange(1, R)]
    for _ in range(399):
        points.append(points[-1] + step)
    scalars = [rng.randrange(R) for _ in points]
    cases.append({"name": "uniform-400", "points": [pt(p) for p in points], "scalars": [hx(s) for s in scalars],
                  "expected": pt(msm_pippenger(points, scalars))})
    rng = random.Random(41)  # :307-312
    bools = [rng.randrange(2) for _ in points]
    cases.append({"name": "boolean-400", "points": [pt(p) for p in points], "scalars": [hx(s) for s in bools],
                  "expected": pt(msm_pippenger(points, bools))})
    heavy = [G * k for k in range(1, 201)]  # :286-291
    cases.append({"name": "one-heavy-bucket-200", "points": [pt(p) for p in heavy], "scalars": [hx(2**200 + 12345)] * 200,
                  "expected": pt(msm_pippenger(heavy, [2**200 + 12345] * 200))})
    for name, pts_, sc in (("cancel", [G, -G], [7, 7]), ("double", [G, G], [5, 5]), ("zeros", [G, G], [0, 0]),
                           ("r-times-g", [G], [R]), ("minus-5", [G * 3], [-5]), ("r-plus-7", [G * 3], [R + 7]),
                           ("huge", [G * 3], [2**300 + 1])):
        cases.append({"name": name, "points": [pt(p) for p in pts_], "scalars": [hx(s % R) for s in sc],
                      "raw_scalars": [str(s) for s in sc], "expected": pt(msm_pippenger(pts_, sc))})
    seeded = []
    plan = [(2**12, "uniform"), (2**12, "skewed"), (2**14, "uniform")]
    if not args.quick:
        plan.append((2**16, "uniform"))
    for n, kind in plan:
        t0 = time.time()
        bseed, sseed = 2000 + n.bit_length(), 3000 + n.bit_length() + (kind == "skewed")
        ks = wl.rows_to_ints(wl.base_scalars(bseed, n))
        bases = [G * k for k in ks]
        sc_rows = wl.uniform_fr(sseed, n) if kind == "uniform" else wl.skewed_scalars(sseed, n)
        sc = wl.rows_to_ints(sc_rows)
        res = msm_pippenger(bases, sc)
        h = hashlib.sha256()
        for p in bases:
            h.update((p.x * 2**256 % P).to_bytes(32, "little") + (p.y * 2**256 % P).to_bytes(32, "little"))
        seeded.append({"n": n, "kind": kind, "base_seed": bseed, "scalar_seed": sseed,
                       "bases_sha256": h.hexdigest(), "bases_first": [hx(bases[0].x), hx(bases[0].y)],
                       "expected": pt(res)})
        print(f"msm {kind} 2^{n.bit_length() - 1}: {time.time() - t0:.1f}s", file=sys.stderr)
    dump("msm.json", {"cases": cases, "seeded": seeded})
    field64_fixtures()


def i64_digest(values: list[int]) -> str:
    """SHA-256 of int64 values as little-endian 8-byte words (the GPU's output bytes)."""
    return hashlib.sha256(b"".join(v.to_bytes(8, "little", signed=True) for v in values)).hexdigest()


def field64_fixtures() -> None:
    """
    field64.json from the reference's int64 path: zkgpu/field_gpu.py with its
    GPU flag off (its NumPy / Python-int fallback) and zkgpu/ntt.py's NTT, on
    the moduli of the reference's tests/test_field_gpu.py:19-25 and
    tests/test_ntt.py:14-35.
    """
    import warnings

    import numpy as np
    from zkgpu import field_gpu as ref_f64  # the reference's package
    from zkgpu.ntt import ntt

    warnings.simplefilter("ignore")
    ref_f64._gpu_available = False
    field_moduli = [7, 998_244_353, 3_037_000_500, 3_037_000_501, 2**61 - 1, 2**63 - 25]
    primes = {7, 998_244_353, 2**61 - 1, 2**63 - 25}
    ops = {}
    for mod in field_moduli:
        rng = random.Random(mod)
        # operands over all of int64: negative and unreduced values included
        a = [rng.randrange(-(2**63), 2**63) for _ in range(64)] + [mod - 1, 0, 2**63 - 1, -(2**63)]
        b = [rng.randrange(-(2**63), 2**63) for _ in range(64)] + [mod - 1, mod - 1, -(2**63), 2**63 - 1]
        A, B = np.array(a, dtype=np.int64), np.array(b, dtype=np.int64)
        entry = {
            "a": a,
            "b": b,
            "mul": ref_f64.gpu_batch_mul(A, B, mod).tolist(),
            "add": ref_f64.gpu_batch_add(A, B, mod).tolist(),
            "pow": {str(e): ref_f64.gpu_batch_pow(B, e, mod).tolist() for e in (0, 1, 2, 65537, 2**70 + 3)},
        }
        if mod in primes:
            inv = [v if v % mod else 1 for v in a]  # zero has no inverse
            entry["inv_bases"] = inv
            entry["pow"]["-3"] = ref_f64.gpu_batch_pow(np.array(inv, dtype=np.int64), -3, mod).tolist()
        ops[str(mod)] = entry
    ntt_moduli = [998_244_353, 12_289, 2_147_483_641 * 2**32 + 1]
    transforms = {}
    for mod in ntt_moduli:
        per = {}
        for n in (1, 2, 8, 256, 4096):
            rng = random.Random(n)  # the reference test's draw (tests/test_ntt.py:226-229)
            a = [rng.randrange(mod) for _ in range(n)]
            fwd, inv = ntt(a, mod), ntt(a, mod, invert=True)
            if n <= 256:
                per[str(n)] = {"fwd": fwd, "inv": inv}
            else:
                per[str(n)] = {"fwd_sha256": i64_digest(fwd), "inv_sha256": i64_digest(inv),
                               "fwd_samples": {str(i): fwd[i] for i in (0, 1, n // 2, n - 1)}}
        edge = [mod + 5, 2 * mod + 1 if 2 * mod + 1 <= 2**63 - 1 else -1, 2**63 - 1, -(2**63)] + [0] * 4
        per["unreduced"] = {"input": edge, "fwd": ntt(edge, mod), "inv": ntt(edge, mod, invert=True)}
        transforms[str(mod)] = per
    (HERE / "field64.json").write_text(json.dumps({"ops": ops, "ntt": transforms}, sort_keys=True) + "\n")
    print("wrote field64.json", file=sys.stderr)


if __name__ == "__main__":
    main()

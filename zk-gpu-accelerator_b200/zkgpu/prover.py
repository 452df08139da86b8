"""
zkgpu.prover — a Groth16-shaped prover job with every step on the device.

What one proof computes (the reference's demo/prover_simulation.py:1-25,
:137-150, :201-214), for a domain H of m points and coset offset g = 5
(zkgpu/domain.py:78-83):

  quotient  a, b, c = iNTT(A), iNTT(B), iNTT(C)         3 inverse NTTs
            A', B', C' = NTT_g(a), NTT_g(b), NTT_g(c)    3 coset NTTs
            H' = (A' B' - C') / (g^m - 1)                  one fused pointwise pass
            h = iNTT_g(H')                                 1 inverse coset NTT
  MSMs      sum z_i [A_i], sum z_i [B_i]                   witness z, m points each
            sum z_i [L_i]                                  private part z[2:], m - 2 points
            sum h_i [H_i]                                  h[:m-1], m - 1 points

over one resident base set (the demo's stand-in proving key: one point set,
a prefix per query). A satisfied circuit (C = A B on H) makes h's top
coefficient zero, which check_quotient verifies as the demo does.

ProofJob holds one job's device buffers and hands out its work stage by
stage as plain launch descriptors, so that a scheduler (zkgpu.serving) can
batch the stages of many jobs into shared launches; prove_plain runs one job
alone through the one-at-a-time entry points (the baseline that batching is
measured against).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Any

import numpy as np

from zkgpu import _native, _rows
from zkgpu.curve import R, Point
from zkgpu.field256_gpu import BN254_FR, LIMBS

COSET = 5  # the smallest quadratic non-residue of BN254 Fr (zkgpu/domain.py:78-83)
MSM_NAMES = ("A", "B", "L", "H")
NUM_PUBLIC = 1  # as the demo: z[0] = 1, z[1] public, z[2:] private
_RESULT_WORDS = 16

# job stages, in order
STAGE_INTT, STAGE_COSET, STAGE_QUOTIENT, STAGE_MSM, STAGE_DONE = range(5)


def vanishing_inverse(m: int) -> int:
    """1 / Z_H(g) = 1 / (g^m - 1) for the coset offset g."""
    return pow((pow(COSET, m, R) - 1) % R, -1, R)


@dataclass
class ProofRequest:
    """One job's inputs on the host, plain canonical rows: the values of A z,
    B z and C z on H, and the witness z (the MSM scalars)."""

    m: int
    a: np.ndarray
    b: np.ndarray
    c: np.ndarray
    witness: np.ndarray
    _host: Any = None

    @property
    def nbytes(self) -> int:
        return 4 * self.m * 32

    def host_rows(self) -> Any:
        """a, b, c, z and the row 1 / Z_H(g) in one pinned host tensor (built once, shared by
        every job made from this request)."""
        if self._host is None:
            z_inv = np.array([_native.limbs(vanishing_inverse(self.m))], dtype=np.uint64)
            self._host = _pinned(np.concatenate([self.a, self.b, self.c, self.witness, z_inv]))
        return self._host


def synthetic_request(seed: int, m: int) -> ProofRequest:
    """A satisfied stand-in circuit (the demo's): A, B uniform on H, C = A B,
    and a witness-like z with z[0] = 1 (60% in {0, 1}, 20% < 2^32, 20% uniform)."""
    from zkgpu import workloads as wl

    a = wl.uniform_fr(seed, m)
    b = wl.uniform_fr(seed + 1, m)
    ab = BN254_FR.mul(BN254_FR.to_montgomery(a), BN254_FR.to_montgomery(b))
    c = BN254_FR.from_montgomery(ab).cpu().numpy()
    z = wl.skewed_scalars(seed + 2, m)
    z[0] = (1, 0, 0, 0)
    return ProofRequest(m, a, b, c, z)


def _pinned(rows: np.ndarray) -> Any:
    torch = _native.torch_module()
    return torch.from_numpy(np.ascontiguousarray(rows, dtype=np.uint64).view(np.int64)).pin_memory()


class ProofJob:
    """
    One job's device state. Buffers are allocated at construction (the
    scheduler's admission step); bytes() is what they take, which the HBM
    budget counts. The stages hand out launch descriptors:

      ntt_entries(stage)   transforms of that stage: (in, out, n, invert, coset)
      quotient_args()      the fused pointwise step (a, b, c, z, out, n)
      msm_entries()        the four MSMs: (points, scalars, n, result row)
    """

    def __init__(self, request: ProofRequest, bases: Any, job_id: int = 0) -> None:
        torch = _native.require_cuda()
        m = request.m
        if m < 4 or m & (m - 1):
            raise ValueError(f"domain size must be a power of 2 of at least 4, got {m}")
        if int(bases.shape[0]) < m:
            raise ValueError(f"the base set has {int(bases.shape[0])} points, the job needs {m}")
        self.id = job_id
        self.m = m
        self.request = request
        self.bases = bases
        self.stage = STAGE_INTT
        # host side, pinned for asynchronous upload: a, b, c, z and the row 1 / Z_H(g)
        self.host = request.host_rows()
        # every device buffer of the job is a view into ONE allocation (a serving loop admits
        # hundreds of jobs at once, and seven allocations a job measured ~0.5 ms of host time)
        rows = (4 * m + 1) + 3 * m + 3 * m + 3 * m + m + m
        self._mem = torch.empty((rows * LIMBS + 4 * _RESULT_WORDS,), dtype=torch.int64, device="cuda")
        views, at = [], 0
        for count in (4 * m + 1, 3 * m, 3 * m, 3 * m, m, m):
            views.append(self._mem[at : at + count * LIMBS].view(count, LIMBS))
            at += count * LIMBS
        self.plain, self.abc, self.coef, self.ev, self.h, self.h_plain = views
        # plain: a, b, c, z and 1 / Z_H(g); abc: Montgomery values on H; coef: a, b, c coefficients;
        # ev: values on the coset; h: Montgomery; h_plain: h's plain coefficients
        self.z_inv = self.plain[4 * m:]
        self.results = self._mem[at:].view(4, _RESULT_WORDS)
        self.done_event = None
        self.arrival = 0.0
        self.admitted = 0.0

    def bytes(self) -> int:
        """Device bytes held by this job (its buffers; workspaces are the scheduler's)."""
        return (4 + 3 + 3 + 3 + 1 + 1) * self.m * 32 + 32 * 5

    # ---- stage work ---------------------------------------------------------

    def upload(self) -> None:
        """Pinned host rows to the device, then A, B, C into Montgomery form (current stream)."""
        self.copy_rows()
        self.to_montgomery()

    def copy_rows(self) -> None:
        """The pinned host rows (a, b, c, z, 1 / Z_H(g)) to the device (current stream)."""
        self.plain.copy_(self.host, non_blocking=True)

    def to_montgomery(self) -> None:
        """A, B, C into Montgomery form (current stream, after copy_rows)."""
        f = BN254_FR._field()
        _native.check(_native.lib().zkb_field_to_mont(ctypes.byref(f), _native.ptr(self.plain),
                                                       _native.ptr(self.abc), 3 * self.m, _native.stream_ptr()),
                      "zkb_field_to_mont")

    def witness_rows(self) -> Any:
        return self.plain[3 * self.m : 4 * self.m]

    def ntt_entries(self, stage: int) -> list[tuple[int, int, int, bool, int | None]]:
        m, row = self.m, 32 * self.m
        if stage == STAGE_INTT:  # values on H -> coefficients
            return [(_native.ptr(self.abc) + k * row, _native.ptr(self.coef) + k * row, m, True, None)
                    for k in range(3)]
        if stage == STAGE_COSET:  # coefficients -> values on g H
            return [(_native.ptr(self.coef) + k * row, _native.ptr(self.ev) + k * row, m, False, COSET)
                    for k in range(3)]
        if stage == STAGE_QUOTIENT:  # quotient values on g H -> h's coefficients
            return [(_native.ptr(self.coef), _native.ptr(self.h), m, True, COSET)]
        return []

    def quotient_args(self) -> tuple[int, int, int, int, int, int]:
        """(A' B' - C') / Z_H(g) into the first coefficient buffer (free after the coset NTTs)."""
        m, row = self.m, 32 * self.m
        ev = _native.ptr(self.ev)
        return (ev, ev + row, ev + 2 * row, _native.ptr(self.z_inv), _native.ptr(self.coef), m)

    def msm_entries(self) -> list[tuple[int, int, int, int]]:
        m = self.m
        z = _native.ptr(self.witness_rows())
        b = _native.ptr(self.bases)
        res = _native.ptr(self.results)
        skip = (NUM_PUBLIC + 1) * 32
        return [
            (b, z, m, res),                              # A: sum z_i [A_i]
            (b, z, m, res + 8 * _RESULT_WORDS),          # B: sum z_i [B_i]
            (b, z + skip, m - NUM_PUBLIC - 1, res + 16 * _RESULT_WORDS),  # L: private witness
            (b, _native.ptr(self.h_plain), m - 1, res + 24 * _RESULT_WORDS),  # H: h[:m-1]
        ]

    def h_to_plain(self) -> None:
        f = BN254_FR._field()
        _native.check(_native.lib().zkb_field_from_mont(ctypes.byref(f), _native.ptr(self.h),
                                                         _native.ptr(self.h_plain), self.m, _native.stream_ptr()),
                      "zkb_field_from_mont")

    # ---- results ------------------------------------------------------------

    def msm_points(self) -> dict[str, Point]:
        from zkgpu.batch import results_to_points

        return dict(zip(MSM_NAMES, results_to_points(self.results), strict=True))

    def h_ints(self) -> list[int]:
        return _rows.limbs_to_ints(self.h_plain.cpu().numpy().view(np.uint64))

    def check_quotient(self) -> None:
        """h must have degree <= m - 2 for a satisfied circuit (the demo's check)."""
        top = self.h_plain[self.m - 1].cpu().numpy().view(np.uint64)
        if top.any():
            raise RuntimeError("the quotient is not a polynomial of degree <= m - 2")


def msm_table_jobs(table: Any, entries: list[tuple[int, int, int, int]]) -> Any:
    """zkb_msm_job rows for MSM entries (points, scalars, n, result) whose points are a prefix
    of the base set that `table` (a FixedBaseTable) was built from: the table takes their place."""
    jobs = (_native.ZkbMsmJob * max(len(entries), 1))()
    for j, (_, sc, n, res) in enumerate(entries):
        if n > table.n:
            raise ValueError(f"an MSM of {n} points over a table of {table.n}")
        jobs[j].points, jobs[j].scalars, jobs[j].n, jobs[j].result = _native.ptr(table.table), sc, n, res
        jobs[j].window_size = table.window_size
    return jobs


def prove_plain(job: ProofJob, workspaces: dict[str, Any] | None = None, table: Any = None) -> None:
    """One job alone, one call per operation (7 zkb_ntt, 1 pointwise, 4 MSMs) on the
    current stream: the one-at-a-time form the batched scheduler is compared with. With a
    FixedBaseTable of the job's base set, each MSM is one zkb_msm_fixed_batch call of one
    job over it, else one zkb_msm call."""
    lib = _native.lib()
    f = BN254_FR._field()
    s = _native.stream_ptr()
    m = job.m
    ws = workspaces if workspaces is not None else {}
    ntt_bytes = lib.zkb_ntt_workspace_bytes(m)
    if "ntt" not in ws or ws["ntt"].numel() < ntt_bytes:
        ws["ntt"] = _native.workspace(ntt_bytes)
    g = _native.u64_array(_native.limbs(COSET))
    job.upload()
    for stage in (STAGE_INTT, STAGE_COSET):
        for src, dst, n, inv, coset in job.ntt_entries(stage):
            _native.check(lib.zkb_ntt(ctypes.byref(f), src, dst, n, int(inv), None, g if coset else None,
                                      _native.ptr(ws["ntt"]), ntt_bytes, s), "zkb_ntt")
    _native.check(lib.zkb_quotient_pointwise(*job.quotient_args(), s), "zkb_quotient_pointwise")
    for src, dst, n, inv, coset in job.ntt_entries(STAGE_QUOTIENT):
        _native.check(lib.zkb_ntt(ctypes.byref(f), src, dst, n, int(inv), None, g, _native.ptr(ws["ntt"]),
                                  ntt_bytes, s), "zkb_ntt")
    job.h_to_plain()
    for k, (pts, sc, n, res) in enumerate(job.msm_entries()):
        key = f"msm{k}"
        if table is not None:
            jobs = msm_table_jobs(table, [(pts, sc, n, res)])
            need = lib.zkb_msm_fixed_batch_workspace_bytes(jobs, 1)
            if key not in ws or ws[key].numel() < need:
                ws[key] = _native.workspace(need)
            _native.check(lib.zkb_msm_fixed_batch(jobs, 1, _native.ptr(ws[key]), need, s), "zkb_msm_fixed_batch")
            continue
        need = lib.zkb_msm_workspace_bytes(n, 0)
        if key not in ws or ws[key].numel() < need:
            ws[key] = _native.workspace(need)
        _native.check(lib.zkb_msm(pts, sc, n, 0, res, _native.ptr(ws[key]), need, s), "zkb_msm")
    job.stage = STAGE_DONE

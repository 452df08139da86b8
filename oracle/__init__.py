"""
oracle — CPU restatements of the reference's BN254 hot-path algorithms.

TEST INFRASTRUCTURE ONLY. This package is the checker that the GPU results
are compared against. Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg (and its `--impl reference` arm) may import, call, link or
run anything here, and only as the checker or as the timed CPU baseline,
never as the product. The zkgpu package never imports it.

Two restatements of the same algorithms, both following the reference
erihhh6/zk-gpu-accelerator file by file (cited per function):
  - pyoracle : Python integers, line for line with the reference's CPU path
               (zkgpu/field.py, ntt.py, domain.py, curve.py, msm.py); for small
               cases.
  - c_oracle : the same algorithms in C (zk_oracle.c, 4 x 64-bit Montgomery
               limbs), built by oracle/Makefile into oracle/libzk_oracle.so;
               fast enough for 2^16-point MSMs and 2^20-point NTTs, and
               multi-threaded for the timed CPU baseline.

Parity is pinned: tests/test_oracle_golden.py checks both against golden
vectors produced by running the reference itself (tests/golden/make_golden.py)
and against the known answers in the reference's own tests (gnark's
Montgomery constants, snarkjs's 2^28 root of unity, py_ecc's 2G, r*G = O).
"""

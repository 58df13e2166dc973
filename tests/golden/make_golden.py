#!/usr/bin/env python
"""Generates the golden fixtures in tests/golden/ from the REFERENCE itself.

Run in a checkout where the reference sources are available (default
/root/reference, override with VBCSR_REFERENCE) after ``oracle/build_ref.sh``
and ``python -m vbcsr_b200._build``:

    python tests/golden/make_golden.py [--only-hermitian]

Two sources:
* the reference C++ core (oracle/_ref/libvbcsr_ref.so, built from the
  reference's own headers) for mult / mult_dense / adjoints, spmm with
  thresholds, filter_blocks, transpose, set_random, the KPM recurrence and
  the complex Chebyshev propagation loop;
* the reference's Python ``VBCSR.create_random`` (vbcsr/matrix.py), executed
  unmodified on this repository's host core (construction is host-only), for
  the random-matrix generator's stream.

Fixtures are small .npz files; the tests read them without the reference.
"""
from __future__ import annotations

import importlib
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle.oracle import Reference  # noqa: E402
from vbcsr_b200 import workloads as W  # noqa: E402

REF_SRC = Path(os.environ.get("VBCSR_REFERENCE", "/root/reference"))


def save(name, **arrays):
    np.savez_compressed(HERE / f"{name}.npz", **arrays)
    print("wrote", name)


def blockcsr_arrays(prefix, H):
    return {f"{prefix}_bsz": H.block_sizes, f"{prefix}_rp": H.row_ptr, f"{prefix}_ci": H.col_ind,
            f"{prefix}_val": H.values}


def core_fixtures(ref: Reference):
    rng = np.random.default_rng(2024)
    for name, H in {
        "apply_vbcsr": W.random_symmetric_blocks(60, seed=101),
        "apply_cplx": W.random_pattern(30, 2, 6, 4, seed=102, dtype=np.complex128),
        "apply_csr": W.random_pattern(80, 1, 1, 5, seed=103),
    }.items():
        R = ref.matrix(H)
        x = rng.normal(size=H.N)
        X = rng.normal(size=(H.N, 5))
        if np.iscomplexobj(H.values):
            x = x + 1j * rng.normal(size=H.N)
            X = X + 1j * rng.normal(size=(H.N, 5))
        save(name, **blockcsr_arrays("A", H), x=x, X=X, y=R.mult(x), ya=R.mult(x, adjoint=True),
             Y=R.mult_dense(X), Ya=R.mult_dense(X, adjoint=True), kind=np.array(R.kind()),
             norms=R.block_norms())
    P = W.random_symmetric_blocks(50, seed=104)
    P.values *= 0.1
    R = ref.matrix(P)
    out = blockcsr_arrays("A", P)
    for k, thr in enumerate([0.0, 1e-3, 0.05, 0.3]):
        C = R.spmm(R, thr).to_blockcsr()
        out.update({f"C{k}_rp": C.row_ptr, f"C{k}_ci": C.col_ind, f"C{k}_val": C.values, f"thr{k}": np.array(thr)})
    T = R.transpose().to_blockcsr()
    out.update({"T_rp": T.row_ptr, "T_ci": T.col_ind, "T_val": T.values})
    F = R.duplicate()
    F.filter_blocks(0.5)
    Fb = F.to_blockcsr()
    out.update({"F_rp": Fb.row_ptr, "F_ci": Fb.col_ind, "F_val": Fb.values, "F_thr": np.array(0.5)})
    save("spmm_threshold", **out)
    A = W.ring_blocks(4, 2)
    Rr = ref.matrix(A)
    C0 = Rr.spmm(Rr, 0.0).to_blockcsr()
    C6 = Rr.spmm(Rr, 0.6).to_blockcsr()
    save("ring", **blockcsr_arrays("A", A), C0_rp=C0.row_ptr, C0_ci=C0.col_ind, C0_val=C0.values,
         C6_rp=C6.row_ptr, C6_ci=C6.col_ind, C6_val=C6.values)
    H = W.random_pattern(25, 1, 5, 3, seed=105)
    Z = W.random_pattern(25, 1, 5, 3, seed=105, dtype=np.complex128)
    save("set_random", bsz=H.block_sizes, real=ref.matrix(H).set_random(3, 77, True),
         real_raw=ref.matrix(H).set_random(2, 5, False), cplx=ref.matrix(Z).set_random(3, 77, True))
    L, _ = W.tmd_lattice(5, seed=106)
    V = np.where(rng.random((L.N, 4)) < 0.5, -1.0, 1.0)
    save("kpm_tmd5", **blockcsr_arrays("A", L), V=V, mu=ref.matrix(L).kpm_moments(V, 40))
    Lz, _ = W.tmd_lattice(3, seed=107, bond_phase=True)
    psi = rng.normal(size=Lz.N) + 1j * rng.normal(size=Lz.N)
    coeffs = rng.normal(size=12) + 1j * rng.normal(size=12)
    save("cheb_apply_cplx", **blockcsr_arrays("A", Lz), psi=psi, coeffs=coeffs,
         out=ref.matrix(Lz).cheb_apply(coeffs, psi))


def hermitian_fixtures(ref: Reference):
    """spmm_hermitian of the reference core: a real symmetric and a complex
    Hermitian (bond-phase lattice) operand, squared at several thresholds."""
    P = W.random_symmetric_blocks(24, seed=109)
    P.values *= 0.1
    Z, _ = W.tmd_lattice(3, seed=108, bond_phase=True, dtype=np.complex128)
    out = {}
    for tag, H, thrs in (("R", P, [0.0, 1e-3, 0.05]), ("Z", Z, [0.0, 3e-3, 6e-3])):
        R = ref.matrix(H)
        out.update(blockcsr_arrays(tag, H))
        for k, thr in enumerate(thrs):
            C = R.spmm_hermitian(R, thr).to_blockcsr()
            out.update({f"{tag}C{k}_rp": C.row_ptr, f"{tag}C{k}_ci": C.col_ind, f"{tag}C{k}_val": C.values,
                        f"{tag}thr{k}": np.array(thr)})
    save("spmm_hermitian", **out)


def reference_python_package():
    """The reference's vbcsr package modules (matrix.py & co.) without its
    __init__ (which needs ase), bound to this repository's vbcsr_core."""
    from vbcsr_b200 import _core

    sys.modules["vbcsr_core"] = _core.load()
    pkg = types.ModuleType("vbcsr_ref")
    pkg.__path__ = [str(REF_SRC / "vbcsr")]
    sys.modules["vbcsr_ref"] = pkg
    return importlib.import_module("vbcsr_ref.matrix")


def create_random_fixtures():
    refmat = reference_python_package()
    out = {}
    cases = [(30, 1, 4, 0.1, np.float64, 42), (40, 2, 5, 0.2, np.float64, 7), (25, 1, 3, 0.15, np.complex128, 11)]
    for k, (nb, lo, hi, dens, dt, seed) in enumerate(cases):
        M = refmat.VBCSR.create_random(nb, lo, hi, dens, dtype=dt, seed=seed)
        out.update({f"m{k}_args": np.array([nb, lo, hi, dens, seed, int(dt == np.complex128)], dtype=np.float64),
                    f"m{k}_rp": np.asarray(M.row_ptr), f"m{k}_ci": np.asarray(M.col_ind),
                    f"m{k}_bsz": np.asarray(M.graph.block_sizes), f"m{k}_val": M.get_values()})
    save("create_random", **out)


if __name__ == "__main__":
    ref = Reference()
    if "--only-hermitian" not in sys.argv:
        core_fixtures(ref)
        create_random_fixtures()
    hermitian_fixtures(ref)

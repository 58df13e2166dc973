"""The reference's own Python package, unchanged, on top of this repository's
``vbcsr_core`` (the drop-in boundary: vbcsr/__init__.py:16-27 puts
$VBCSR_BUILD_DIR first on sys.path and imports ``vbcsr_core`` by name).

Runs where the reference checkout exists (the one oracle/build_ref.sh built
the reference core from, or $VBCSR_REFERENCE) and skips elsewhere.  Each
check runs in a child process so that the reference package and its
``vbcsr_core`` import never mix with this process's modules; the child
writes no bytecode into the reference tree.  A test-only stand-in for the
``ase`` package (the reference imports it for its atomic-structure classes,
which this engine does not provide) is written to a temporary directory.

What runs here needs no GPU: the import, every native attribute the
reference's wrapper reaches for, the host-side construction paths
(create_random, from_scipy, add_block / assemble, to_dense, get_values) and
the placeholders of the out-of-scope atomic classes.  The device paths under
the same calls are covered on the GPU by tests/test_api_gpu.py."""
import json
import os
import re
import subprocess
import sys
import textwrap
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "vbcsr_b200"
GOLDEN = Path(__file__).resolve().parent / "golden"

# Methods of the reference's ImageContainer wrapper (periodic images,
# k-sampling): not part of this engine.
_OUT_OF_SCOPE = {"add_blocks", "axpy_into", "redistribute_into", "sample_k"}


def _reference():
    from oracle.oracle import reference_root

    ref = reference_root()
    if ref is None or not (ref / "vbcsr" / "__init__.py").exists():
        pytest.skip("reference checkout not present on this machine")
    if not any(PKG.glob("vbcsr_core*.so")):
        pytest.skip("vbcsr_core not built")
    return ref


def _run(ref: Path, tmp_path: Path, body: str) -> dict:
    stub = tmp_path / "ase_stub" / "ase"
    stub.mkdir(parents=True, exist_ok=True)
    (stub / "__init__.py").write_text("class Atoms:\n    pass\n")
    (stub / "data.py").write_text("chemical_symbols = ['X', 'H', 'He', 'Li', 'Be', 'B', 'C', 'N', 'O']\n")
    (stub / "io.py").write_text("def read(*a, **k):\n    raise RuntimeError('ase stand-in')\n")
    script = tmp_path / "child.py"
    script.write_text(
        "import json, sys\n"
        f"sys.path[:0] = [{str(stub.parent)!r}, {str(ref)!r}]\n"
        "import numpy as np\n"
        "import vbcsr\n"
        "out = {'core_file': vbcsr.vbcsr_core.__file__}\n" + textwrap.dedent(body) + "\nprint(json.dumps(out))\n"
    )
    env = dict(os.environ, VBCSR_BUILD_DIR=str(PKG), VBCSR_PREFER_BUILD="1", PYTHONDONTWRITEBYTECODE="1",
               CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", ""))
    env.pop("PYTHONPATH", None)
    proc = subprocess.run([sys.executable, str(script)], cwd=str(tmp_path), env=env, capture_output=True,
                          text=True, timeout=300)
    assert proc.returncode == 0, proc.stdout + proc.stderr
    out = json.loads(proc.stdout.strip().splitlines()[-1])
    assert Path(out["core_file"]).resolve().parent == PKG.resolve(), out["core_file"]
    return out


def test_reference_package_imports_on_dropin(tmp_path):
    ref = _reference()
    out = _run(ref, tmp_path, """
        out['exports'] = sorted(n for n in ('VBCSR', 'DistVector', 'DistMultiVector', 'DistGraph', 'AtomicData',
                                            'ImageContainer', 'AssemblyMode') if hasattr(vbcsr, n))
        import scipy.sparse.linalg as sla
        A = vbcsr.VBCSR.create_random(12, 2, 3, density=0.3, seed=5)
        out['linear_operator'] = isinstance(A, sla.LinearOperator)
    """)
    assert out["exports"] == sorted(["VBCSR", "DistVector", "DistMultiVector", "DistGraph", "AtomicData",
                                     "ImageContainer", "AssemblyMode"])
    assert out["linear_operator"]


def test_every_native_attribute_the_wrapper_uses_exists(tmp_path):
    """Scans the reference wrapper for `_core.<name>` and `vbcsr_core.<name>`
    and checks each against the classes of this vbcsr_core."""
    ref = _reference()
    used_core, used_mod = set(), set()
    for f in (ref / "vbcsr").glob("*.py"):
        src = f.read_text()
        used_core |= set(re.findall(r"(?<!\w)_core\.([A-Za-z_]\w*)", src))
        used_mod |= set(re.findall(r"vbcsr_core\.([A-Za-z_]\w*)", src))
    used_core -= _OUT_OF_SCOPE
    out = _run(ref, tmp_path, f"""
        core = vbcsr.vbcsr_core
        classes = [core.BlockSpMat_Double, core.BlockSpMat_Complex, core.DistVector_Double,
                   core.DistVector_Complex, core.DistMultiVector_Double, core.DistMultiVector_Complex,
                   core.DistGraph]
        out['missing_attr'] = sorted(n for n in {sorted(used_core)!r}
                                     if not any(hasattr(c, n) for c in classes))
        out['missing_mod'] = sorted(n for n in {sorted(used_mod)!r} if not hasattr(core, n))
    """)
    assert out["missing_attr"] == [], out["missing_attr"]
    assert out["missing_mod"] == [], out["missing_mod"]


def test_reference_create_random_on_dropin_matches_golden(tmp_path):
    """The reference's create_random (vbcsr/matrix.py:331-410: one add_block
    per block, then assemble) through this core gives the matrices that the
    reference's own core gave (tests/golden/create_random.npz)."""
    import numpy as np

    ref = _reference()
    d = np.load(GOLDEN / "create_random.npz")
    args = [[float(v) for v in d[f"m{k}_args"]] for k in range(3)]
    out = _run(ref, tmp_path, f"""
        res = []
        for nb, lo, hi, dens, seed, cplx in {args!r}:
            M = vbcsr.VBCSR.create_random(int(nb), int(lo), int(hi), float(dens),
                                          dtype=np.complex128 if cplx else np.float64, seed=int(seed))
            v = M.get_values()
            res.append({{'rp': np.asarray(M.row_ptr).tolist(), 'ci': np.asarray(M.col_ind).tolist(),
                        'bsz': list(M.graph.block_sizes), 're': np.real(v).tolist(), 'im': np.imag(v).tolist(),
                        'kind': M.matrix_kind}})
        out['mats'] = res
    """)
    for k, m in enumerate(out["mats"]):
        assert np.array_equal(m["rp"], d[f"m{k}_rp"])
        assert np.array_equal(m["ci"], d[f"m{k}_ci"])
        assert np.array_equal(m["bsz"], d[f"m{k}_bsz"])
        v = np.asarray(m["re"]) + 1j * np.asarray(m["im"])
        assert np.array_equal(v, d[f"m{k}_val"])


def test_reference_from_scipy_kinds_and_values(tmp_path):
    """from_scipy (vbcsr/matrix.py:877-976): BSR with square blocks -> BSR
    kind, any other format -> CSR kind; to_dense reproduces the input."""
    ref = _reference()
    out = _run(ref, tmp_path, """
        import scipy.sparse as sp
        rng = np.random.default_rng(11)
        D = rng.random((24, 24)) * (rng.random((24, 24)) < 0.2)
        res = {}
        for name, m in (('bsr', sp.bsr_matrix(D, blocksize=(3, 3))), ('csr', sp.csr_matrix(D)),
                        ('coo', sp.coo_matrix(D)), ('bsr_c', sp.bsr_matrix(D + 1j * D.T, blocksize=(4, 4)))):
            A = vbcsr.VBCSR.from_scipy(m)
            v = A.get_values()
            res[name] = [A.matrix_kind, float(np.abs(A.to_dense() - m.toarray()).max()), str(A.dtype),
                         np.asarray(A.row_ptr).tolist(), np.asarray(A.col_ind).tolist(),
                         list(A.graph.block_sizes), np.real(v).tolist(), np.imag(v).tolist()]
        out['res'] = res
    """)
    res = out["res"]
    assert res["bsr"][0] == "bsr" and res["bsr_c"][0] == "bsr"
    assert res["csr"][0] == "csr" and res["coo"][0] == "csr"
    assert all(r[1] == 0.0 for r in res.values())
    assert res["bsr_c"][2] == "complex128"
    # this repository's bulk from_scipy builds the same matrices
    import numpy as np
    import scipy.sparse as sp

    from vbcsr_b200 import VBCSR

    rng = np.random.default_rng(11)
    D = rng.random((24, 24)) * (rng.random((24, 24)) < 0.2)
    for name, m in (("bsr", sp.bsr_matrix(D, blocksize=(3, 3))), ("csr", sp.csr_matrix(D)),
                    ("coo", sp.coo_matrix(D)), ("bsr_c", sp.bsr_matrix(D + 1j * D.T, blocksize=(4, 4)))):
        A = VBCSR.from_scipy(m)
        kind, _, dt, rp, ci, bsz, re_, im_ = res[name]
        assert A.matrix_kind == kind and str(A.dtype) == dt
        assert np.array_equal(A.row_ptr, rp) and np.array_equal(A.col_ind, ci)
        assert np.array_equal(np.asarray(A.graph.block_sizes), bsz)
        v = A.get_values()
        assert np.array_equal(np.real(v), re_) and np.array_equal(np.imag(v), im_)


def test_out_of_scope_atomic_classes_raise(tmp_path):
    """The atomic-structure placeholders import, and raise when built."""
    ref = _reference()
    out = _run(ref, tmp_path, """
        errs = {}
        for name, make in (('AtomicData', lambda: vbcsr.vbcsr_core.AtomicData()),
                           ('ImageContainer', lambda: vbcsr.vbcsr_core.ImageContainer(None)),
                           ('ImageContainer_Complex', lambda: vbcsr.vbcsr_core.ImageContainer_Complex(None))):
            try:
                make()
                errs[name] = None
            except RuntimeError as e:
                errs[name] = str(e)
        out['errs'] = errs
        out['phase'] = [str(vbcsr.vbcsr_core.PhaseConvention.R_ONLY),
                        str(vbcsr.vbcsr_core.PhaseConvention.R_AND_POSITION)]
    """)
    for name, msg in out["errs"].items():
        assert msg and "not available in the B200 engine" in msg, (name, msg)
    assert len(out["phase"]) == 2

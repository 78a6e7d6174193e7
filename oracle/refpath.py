"""Where the reference checkout and the BLAS the oracle links against are found.

TEST INFRASTRUCTURE ONLY: used by the oracle's build recipe callers
(__graft_entry__.build, tests/conftest.py) and the golden-fixture generators.

The reference checkout is named by the environment variable PYQCM_REFERENCE_ROOT.
When it is unset, the checkout location of this build container is used if it
exists (that is where the oracle is compiled; the GPU box only loads the prebuilt
oracle/_ref library). `reference_root(required=True)` raises with a clear message
when neither is there.
"""
from __future__ import annotations

import glob
import os
import sysconfig

ENV = "PYQCM_REFERENCE_ROOT"
_CONTAINER_DEFAULT = "/root/reference"


def reference_root(required: bool = False) -> str | None:
    root = os.environ.get(ENV)
    if root:
        if not os.path.isdir(root):
            raise RuntimeError(f"{ENV}={root} is not a directory")
        return root
    if os.path.isdir(_CONTAINER_DEFAULT):
        return _CONTAINER_DEFAULT
    if required:
        raise RuntimeError(f"the reference checkout is needed here: set {ENV} to its directory")
    return None


def reference_file(relpath: str) -> str:
    return os.path.join(reference_root(required=True), relpath)


def openblas_library() -> str:
    """The OpenBLAS shared library bundled with this interpreter's site-packages
    (LP64, exports the LAPACK routines the oracle's shims call). Override with
    QED_ORACLE_BLASLIB."""
    env = os.environ.get("QED_ORACLE_BLASLIB")
    if env:
        return env
    site = sysconfig.get_paths()["purelib"]
    for pat in ("*.libs/libopenblasp-r0-*.so", "*.libs/libopenblas*.so*", "numpy.libs/libscipy_openblas*.so"):
        hits = sorted(glob.glob(os.path.join(site, pat)))
        if hits:
            return hits[0]
    raise RuntimeError("no OpenBLAS library found in site-packages: set QED_ORACLE_BLASLIB")


def make_args() -> list[str]:
    """make variables for oracle/ref_build (REF and BLASLIB)."""
    lib = openblas_library()
    return [f"REF={reference_root(required=True)}", f"BLASLIB={lib}", f"BLASDIR={os.path.dirname(lib)}"]

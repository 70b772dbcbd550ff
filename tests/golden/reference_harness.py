"""Import the reference PolyBin3D (Python sources, read in place) for fixture generation.

Only usable where the reference tree exists (the development container).  The reference's
`from .cython import utils` is served by the Cython kernels compiled from its own
utils.pyx into oracle/_ref/ (oracle/build_ref.sh), and its `backend='mkl'` FFT module is a
stand-in wrapping scipy.fft in FP64 (pyfftw and mkl_fft are not installed here), as the
reference's `to_fourier`/`to_real` (base.py:189-194, 218-223) call it.
"""
import importlib
import importlib.util
import os
import sys
import types

import numpy as np
import scipy.fft

# the reference tree's root (the directory holding PolyBin3D/): required, no default
REF_ROOT = os.environ.get("PB_REFERENCE_ROOT", "")
_REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def available():
    return bool(REF_ROOT) and os.path.isfile(os.path.join(REF_ROOT, "PolyBin3D", "base.py"))


def _mkl_shim(workers):
    m = types.ModuleType("mkl_fft")
    m.rfftn = lambda a, axes=(0, 1, 2): scipy.fft.rfftn(a, axes=axes, workers=workers)
    m.irfftn = lambda a, axes=(0, 1, 2): scipy.fft.irfftn(a, axes=axes, workers=workers)
    m.fftn = lambda a, axes=(0, 1, 2): scipy.fft.fftn(a, axes=axes, workers=workers)
    m.ifftn = lambda a, axes=(0, 1, 2): scipy.fft.ifftn(a, axes=axes, workers=workers)
    return m


def load_reference(workers=None):
    """Return the reference package `PolyBin3D` (with .base/.pspec/.bspec loaded)."""
    if "PolyBin3D" in sys.modules and hasattr(sys.modules["PolyBin3D"], "BSpec"):
        return sys.modules["PolyBin3D"]
    if not available():
        raise RuntimeError("reference tree not found: set PB_REFERENCE_ROOT to the directory holding PolyBin3D/")
    sys.dont_write_bytecode = True
    workers = workers or os.cpu_count()
    sys.modules["mkl_fft"] = _mkl_shim(workers)
    # compiled reference kernels
    refdir = os.path.join(_REPO, "oracle", "_ref")
    spec_files = [f for f in os.listdir(refdir) if f.startswith("pb_ref_utils") and f.endswith(".so")]
    if not spec_files:
        raise RuntimeError("oracle/_ref not built: run oracle/build_ref.sh")
    spec = importlib.util.spec_from_file_location("pb_ref_utils", os.path.join(refdir, spec_files[0]))
    utils = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(utils)
    pkg = types.ModuleType("PolyBin3D")
    pkg.__path__ = [os.path.join(REF_ROOT, "PolyBin3D")]
    sys.modules["PolyBin3D"] = pkg
    cy = types.ModuleType("PolyBin3D.cython")
    cy.__path__ = []
    cy.utils = utils
    sys.modules["PolyBin3D.cython"] = cy
    sys.modules["PolyBin3D.cython.utils"] = utils
    for name in ("base", "pspec", "bspec"):
        mod = importlib.import_module("PolyBin3D." + name)
        for k in dir(mod):
            if k in ("PolyBin3D", "PSpec", "BSpec"):
                setattr(pkg, k, getattr(mod, k))
    return pkg

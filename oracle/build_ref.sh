#!/usr/bin/env bash
# Recipe: compile the reference's own Cython grid kernels (PolyBin3D/cython/utils.pyx)
# from the source where it lies, into oracle/_ref/ only.  The shipped cpython-39 .so of
# the reference is never used.  Needs the reference tree; on a machine without it this
# script exits 0 after saying so (the prebuilt oracle/_ref/ travels with the repository).
#
# Flags follow PolyBin3D/cython/setup.py:13-14 (-fopenmp -O3 -ffast-math), minus the
# -march=broadwell pin so the object runs on any x86-64 host; libmvec/libm as there.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
# PB_REFERENCE_ROOT: the reference tree's root (the directory holding PolyBin3D/); required
if [ -z "${PB_REFERENCE_ROOT:-}" ]; then
    echo "build_ref: PB_REFERENCE_ROOT not set; keeping prebuilt $HERE/_ref" >&2
    exit 0
fi
SRC="$PB_REFERENCE_ROOT/PolyBin3D/cython/utils.pyx"
OUT="$HERE/_ref"
if [ ! -f "$SRC" ]; then
    echo "build_ref: reference source not present; keeping prebuilt $OUT" >&2
    exit 0
fi
mkdir -p "$OUT/build"
PY=${PYTHON:-python}
EXT=$($PY -c "import sysconfig; print(sysconfig.get_config_var('EXT_SUFFIX'))")
PYINC=$($PY -c "import sysconfig; print(sysconfig.get_paths()['include'])")
NPINC=$($PY -c "import numpy; print(numpy.get_include())")
$PY -m cython -3 "$SRC" -o "$OUT/build/pb_ref_utils.c" --module-name pb_ref_utils
/usr/bin/gcc -shared -fPIC -fopenmp -O3 -ffast-math -DNPY_NO_DEPRECATED_API=NPY_1_7_API_VERSION \
    -I"$PYINC" -I"$NPINC" "$OUT/build/pb_ref_utils.c" -o "$OUT/pb_ref_utils$EXT" -lmvec -lm
echo "build_ref: built $OUT/pb_ref_utils$EXT"

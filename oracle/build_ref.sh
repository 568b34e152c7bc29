#!/bin/bash
# Build the reference's own Cython kernels (polyspec/cython/tauNL_utils.pyx with
# wignerSymbols-cpp.cpp, and ideal_fisher.pyx) from the reference checkout into
# oracle/_ref, as the checker for the pixel-product kernels.  Nothing is copied:
# cython reads the .pyx in place and writes its generated sources under
# oracle/_ref/build; the compilers read the reference's .cpp/.h in place.
# Flags follow the reference's setup.py (-fopenmp -O3 -ffast-math
# -march=broadwell); its GSL link libraries are dropped (ideal_fisher uses none).
set -euo pipefail
REF=${1:-${PS_REFERENCE_ROOT:-}}
[ -n "$REF" ] || { echo "usage: build_ref.sh <reference checkout> (or set PS_REFERENCE_ROOT)"; exit 1; }
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
SRC="$REF/polyspec/cython"
[ -f "$SRC/tauNL_utils.pyx" ] || { echo "no reference checkout at $REF"; exit 1; }
mkdir -p "$OUT/build"
PY=python
EXT=$($PY -c "import sysconfig; print(sysconfig.get_config_var('EXT_SUFFIX'))")
PYINC=$($PY -c "import sysconfig; print(sysconfig.get_paths()['include'])")
NPINC=$($PY -c "import numpy; print(numpy.get_include())")
FLAGS="-fopenmp -O3 -ffast-math -march=broadwell -fPIC -shared -DNPY_NO_DEPRECATED_API=NPY_1_7_API_VERSION"
if [ ! -f "$OUT/tauNL_utils$EXT" ] || [ "$SRC/tauNL_utils.pyx" -nt "$OUT/tauNL_utils$EXT" ]; then
  $PY -m cython -3 --cplus -I "$SRC" -o "$OUT/build/tauNL_utils.cpp" "$SRC/tauNL_utils.pyx"
  /usr/bin/g++ $FLAGS -I"$SRC" -I"$PYINC" -I"$NPINC" "$OUT/build/tauNL_utils.cpp" "$SRC/wignerSymbols-cpp.cpp" \
    -o "$OUT/tauNL_utils$EXT"
fi
if [ ! -f "$OUT/ideal_fisher$EXT" ] || [ "$SRC/ideal_fisher.pyx" -nt "$OUT/ideal_fisher$EXT" ]; then
  $PY -m cython -3 -o "$OUT/build/ideal_fisher.c" "$SRC/ideal_fisher.pyx"
  /usr/bin/gcc $FLAGS -I"$PYINC" -I"$NPINC" "$OUT/build/ideal_fisher.c" -o "$OUT/ideal_fisher$EXT" -lm
fi
rm -rf "$OUT/build"
echo "built $OUT/tauNL_utils$EXT $OUT/ideal_fisher$EXT"

#!/usr/bin/env bash
# Compile the reference's own C extension (`pyvl.cvl`) from its sources, where they
# lie, into oracle/_ref/.  Test infrastructure only: the product never loads it.
#
# Usage: oracle/build_ref.sh [--if-present] [REFERENCE_ROOT]
#
# REFERENCE_ROOT defaults to $PYVL_REFERENCE_ROOT, else to the checkout this build recipe
# was written against (/root/reference).  With --if-present a missing tree is not an error
# (the prebuilt oracle/_ref, if any, is kept).
#
# The output, oracle/_ref/cvl<EXT_SUFFIX>, is the unmodified reference induction,
# topology and line-force code (src/core/*.c + src/*.c, built the way the
# reference's CMakeLists.txt:60-95 builds it, plus -O3 -fopenmp).  It is git-ignored
# and travels to the GPU host as a prebuilt file; nothing here needs the reference
# tree at run time.
set -euo pipefail
IF_PRESENT=0
if [ "${1:-}" = "--if-present" ]; then
  IF_PRESENT=1
  shift
fi
REF="${1:-${PYVL_REFERENCE_ROOT:-/root/reference}}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
PY="${PYTHON:-python3}"
if [ ! -d "$REF/src/core" ]; then
  echo "reference sources not found under $REF" >&2
  if [ "$IF_PRESENT" = 1 ]; then
    exit 0
  fi
  exit 1
fi
EXT_SUFFIX="$($PY -c 'import sysconfig;print(sysconfig.get_config_var("EXT_SUFFIX"))')"
PY_INC="$($PY -c 'import sysconfig;print(sysconfig.get_paths()["include"])')"
NP_INC="$($PY -c 'import numpy;print(numpy.get_include())')"
mkdir -p "$OUT"
gcc -O3 -fopenmp -fPIC -shared -std=c17 -DCVL_ASSERTS \
  -I"$PY_INC" -I"$NP_INC" \
  "$REF"/src/module.c "$REF"/src/allocator.c "$REF"/src/geoidobject.c \
  "$REF"/src/lineobject.c "$REF"/src/surfaceobject.c "$REF"/src/meshobject.c \
  "$REF"/src/referenceframeobject.c "$REF"/src/core/*.c \
  -o "$OUT/cvl$EXT_SUFFIX" -lm
echo "built $OUT/cvl$EXT_SUFFIX"

#!/bin/sh
# Compiles the reference's own compiled core (mom25d_core.cpp, pybind11 + OpenMP) from its sources where they lie
# under the read-only reference checkout, into oracle/_ref/ (git-ignored). Used only as a checker and as the
# timed CPU baseline; nothing in the product links it.
set -e
REF=${MOM25D_REFERENCE:-/root/reference}
SRC="$REF/src/mom25d/core"
OUT="$(cd "$(dirname "$0")" && pwd)/_ref"
[ -f "$SRC/mom25d_core.cpp" ] || { echo "reference core sources not found under $SRC" >&2; exit 1; }
mkdir -p "$OUT"
EXT=$(python3 -c 'import sysconfig; print(sysconfig.get_config_var("EXT_SUFFIX"))')
g++ -w -O3 -fopenmp -shared -fPIC -std=c++17 $(python3 -m pybind11 --includes) -I"$SRC" \
    "$SRC/mom25d_core.cpp" -o "$OUT/_core$EXT"
echo "built $OUT/_core$EXT"

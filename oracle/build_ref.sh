#!/usr/bin/env bash
# Builds the reference CPU core (bwpm._core: Solver, transmission_matrix, reflection_matrix,
# longitudinal_wavenumber) from the reference sources, unchanged, into oracle/_ref/.
# Test infrastructure only: the built module is the checker and the timed CPU baseline, never
# part of the product path. Needs the reference tree (BWPM_REFERENCE, default: a `reference`
# directory beside this repository) and pybind11.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${BWPM_REFERENCE:-$(cd "$HERE/../.." && pwd)/reference}"
OUT="$HERE/_ref"
if [ ! -f "$REF/cpp/src/solver.cpp" ]; then
  echo "reference sources not found at $REF; skipping oracle/_ref build" >&2
  exit 0
fi
mkdir -p "$OUT"
PY="${PYTHON:-python3}"
SUFFIX="$($PY -c 'import sysconfig; print(sysconfig.get_config_var("EXT_SUFFIX"))')"
INC="$($PY -m pybind11 --includes)"
g++ -O2 -std=c++20 -fopenmp -fPIC -shared \
  -I "$REF/cpp/include" -isystem "$REF/cpp/third_party/pocketfft" $INC \
  "$REF/cpp/src/interface.cpp" "$REF/cpp/src/solver.cpp" "$REF/cpp/python/bindings.cpp" \
  -o "$OUT/_core$SUFFIX"
echo "built $OUT/_core$SUFFIX"

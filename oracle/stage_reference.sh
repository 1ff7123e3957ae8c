#!/usr/bin/env bash
# Installs the reference package, unchanged, into baseline/_ref/ (git-ignored; it travels with
# the working tree) so that the reference's own Python callers can run against this library:
# - `pip install` of the reference from a copy of its tree (its build writes into the source
#   directory), offline from the local wheelhouse, with its CUDA core built for sm_100a
#   (BWPM_ENABLE_CUDA=ON, CMAKE_CUDA_ARCHITECTURES=100a): bwpm.fast, bwpm.adapter, ... and the
#   reference's compiled bwpm._core (CPU Solver and its own cuFFT-based CudaSolver);
# - the reference's test files and golden files copied beside it (baseline/_ref/tests,
#   baseline/_ref/reference), where the reference's tests look for them.
# Test infrastructure only: nothing of the product path imports baseline/_ref.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REPO="$(cd "$HERE/.." && pwd)"
REF="${BWPM_REFERENCE:-$(cd "$REPO/.." && pwd)/reference}"
OUT="$REPO/baseline/_ref"
if [ ! -f "$REF/pyproject.toml" ]; then
  echo "reference tree not found at $REF; skipping baseline/_ref" >&2
  exit 0
fi
SRC="$(mktemp -d)/bwpm_src"
cp -r "$REF" "$SRC"
rm -rf "$OUT"
"${PYTHON:-python3}" -m pip install --no-index --no-build-isolation --no-deps \
  --find-links /opt/wheelhouse --target "$OUT" \
  -C cmake.define.BWPM_ENABLE_CUDA=ON -C cmake.define.CMAKE_CUDA_ARCHITECTURES=100a "$SRC"
cp -r "$REF/tests" "$OUT/tests"
cp -r "$REF/reference" "$OUT/reference"
rm -rf "$SRC"
echo "staged the reference package, its tests and golden files in $OUT"

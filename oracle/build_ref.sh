#!/usr/bin/env bash
# Test infrastructure: compiles the reference's compiled CPU engine
# (cpp/native.cpp of KuboMSD, one C++17/OpenMP source file with pybind11
# bindings) from where it lies under the reference checkout into
# oracle/_ref/_native<ext-suffix>.so.  Nothing is copied into the repository;
# the output directory is git-ignored.  Used only by tests/, the oracle checks
# and bench.py's CPU baseline arm.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
# the reference checkout: $KUBOMSD_REFERENCE, else `reference` beside the repository
REF="${KUBOMSD_REFERENCE:-$(dirname "$(dirname "$HERE")")/reference}"
OUT="$HERE/_ref"
SRC="$REF/cpp/native.cpp"
if [[ ! -f "$SRC" ]]; then
    echo "reference source $SRC not present; nothing to build" >&2
    exit 0
fi
mkdir -p "$OUT"
PY="${PYTHON:-python3}"
SUFFIX="$("$PY" -c 'import sysconfig; print(sysconfig.get_config_var("EXT_SUFFIX"))')"
TARGET="$OUT/_native$SUFFIX"
if [[ -f "$TARGET" && "$TARGET" -nt "$SRC" ]]; then
    echo "$TARGET"
    exit 0
fi
INCLUDES="$("$PY" -m pybind11 --includes)"
# The reference's own flags (setup.py): C++17, -O3, OpenMP, portable code.
g++ -O3 -fopenmp -shared -fPIC -std=c++17 $INCLUDES "$SRC" -o "$TARGET.tmp"
mv "$TARGET.tmp" "$TARGET"
echo "$TARGET"

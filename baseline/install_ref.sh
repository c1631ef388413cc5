#!/usr/bin/env bash
# Installs negfpy (the reference, pure Python) into baseline/_ref, offline,
# for bench.py's timing of negfpy's own transmission().  The source tree is
# read-only, so pip builds from a copy under /tmp.  Usage:
#   NEGFPY_SRC=<negfpy project root> bash baseline/install_ref.sh
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
src="${NEGFPY_SRC:?set NEGFPY_SRC to the negfpy project root}"
tmp="$(mktemp -d /tmp/negfpy_src.XXXXXX)"
cp -r "$src"/. "$tmp"/
python -m pip install --no-index --no-build-isolation --no-deps --find-links /opt/wheelhouse \
    --target "$here/_ref" --upgrade "$tmp"
rm -rf "$tmp"

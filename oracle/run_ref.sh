#!/usr/bin/env bash
# Run every reference binary built by oracle/build_ref.py and collect its outputs.
# Test infrastructure only.  Usage (on a GPU machine, from the repository root):
#   bash oracle/run_ref.sh <dest>      # copies <case>/output and the console log to <dest>/<case>/
set -euo pipefail
if [ $# -ne 1 ]; then echo "usage: bash oracle/run_ref.sh <dest>" >&2; exit 2; fi
dest=$1
root=$(cd "$(dirname "$0")" && pwd)/_ref
for d in "$root"/*/; do
  [ -x "$d/ggb_ref" ] || continue
  name=$(basename "$d")
  mkdir -p "$dest/$name"
  ( cd "$d/run" && ../ggb_ref ) > "$dest/$name/console.log" 2>&1
  cp -r "$d/output" "$dest/$name/"
  cp "$d/case.json" "$dest/$name/"
done

#!/usr/bin/env bash
# Builds the reference's own native module (kerighan/lib-magnet src/*.cpp, pybind11) from the sources
# where they lie, into oracle/_ref/. Used only as a test oracle and as the timed CPU baseline.
# Needs the reference checkout (MAGNET_REFERENCE_DIR, else the folder `reference` beside the repository); on a machine
# without it the prebuilt oracle/_ref/ module is used as it is.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${MAGNET_REFERENCE_DIR:-$(cd "$HERE/../.." && pwd)/reference}"
OUT="$HERE/_ref"
SUFFIX="$(python3-config --extension-suffix 2>/dev/null || python3 -c 'import sysconfig;print(sysconfig.get_config_var("EXT_SUFFIX"))')"
TARGET="$OUT/_magnet$SUFFIX"
if [ ! -d "$REF/src" ]; then
  if [ -f "$TARGET" ]; then echo "reference sources absent; keeping prebuilt $TARGET"; exit 0; fi
  echo "reference sources absent and no prebuilt oracle module" >&2; exit 1
fi
mkdir -p "$OUT"
newest_src=$(ls -t "$REF"/src/*.cpp "$REF"/src/*.hpp "$REF"/src/*.h | head -1)
if [ -f "$TARGET" ] && [ "$TARGET" -nt "$newest_src" ]; then echo "up to date: $TARGET"; exit 0; fi
# -DNDEBUG as setuptools adds it (pybind11 3.x asserts on the GIL otherwise); plain -O3 as the reference's setup.py
g++ -O3 -DNDEBUG -pthread -shared -fPIC -std=c++17 $(python3 -m pybind11 --includes) \
    "$REF"/src/*.cpp -o "$TARGET.tmp"
mv "$TARGET.tmp" "$TARGET"
echo "built $TARGET"

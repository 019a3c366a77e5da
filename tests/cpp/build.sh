#!/usr/bin/env bash
# Builds the C and C++ boundary tests into tests/cpp/_build/:
#  - c99_header: include/sparkit_b200.h compiled as strict C99 and linked
#    against sparkit_b200/libsparkit_b200.so (needs only gcc);
#  - dropin_test: include/sparkit_b200.hpp compiled with the sparkit
#    reference's own headers (REF_ROOT, default /root/reference) and linked
#    against libsparkit_b200.so and the compiled reference
#    (oracle/_ref/libsparkit_ref.so, made by oracle/build_ref.sh), so that
#    the reference's solvers and the device overloads run side by side.
#    Skipped when the reference sources are absent; the built binary then
#    has to come from a machine that has them.
# Both binaries find the libraries through an $ORIGIN-relative rpath.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
ROOT="$(cd "$HERE/../.." && pwd)"
OUT="$HERE/_build"
REF_ROOT="${REF_ROOT:-/root/reference}"
mkdir -p "$OUT"
RPATH='-Wl,-rpath,$ORIGIN/../../../sparkit_b200:$ORIGIN/../../../oracle/_ref'

gcc -std=c99 -pedantic -Wall -Wextra -Werror -I "$ROOT/include" "$HERE/c99_header.c" \
    -L "$ROOT/sparkit_b200" -l:libsparkit_b200.so "$RPATH" -o "$OUT/c99_header"
echo "built $OUT/c99_header"

if [ ! -f "$REF_ROOT/sparkit/config.hpp.in" ] || [ ! -f "$ROOT/oracle/_ref/libsparkit_ref.so" ]; then
  echo "tests/cpp/build.sh: reference sources or oracle/_ref not found; dropin_test not built" >&2
  exit 0
fi
JSON_INC=""
for cand in \
  "$(python3 -c 'import sysconfig;print(sysconfig.get_paths()["purelib"])' 2>/dev/null)/include/cudnn_frontend/thirdparty" \
  /usr/include /usr/local/include; do
  if [ -f "$cand/nlohmann/json.hpp" ]; then JSON_INC="$cand"; break; fi
done
g++ -std=c++20 -O2 -Wall -Wextra -ffp-contract=off \
    -I "$ROOT/include" -I "$ROOT/oracle/_ref/gen" -I "$REF_ROOT" -I "$JSON_INC" \
    "$HERE/dropin_test.cpp" \
    -L "$ROOT/sparkit_b200" -l:libsparkit_b200.so -L "$ROOT/oracle/_ref" -l:libsparkit_ref.so "$RPATH" \
    -o "$OUT/dropin_test"
echo "built $OUT/dropin_test"

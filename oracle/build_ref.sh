#!/usr/bin/env bash
# Builds oracle/_ref/libsparkit_ref.so: the UNMODIFIED sparkit reference,
# compiled from its sources where they lie (REF_ROOT, default
# /root/reference), plus oracle/ref_shim.cpp (this repository's extern "C"
# access layer).  Test infrastructure only; outputs go to oracle/_ref/ and
# nothing is copied out of the reference tree.
#
# The reference's own CMake build cannot run here (its cmake_utilities
# submodule is empty and Catch2 is absent), so this recipe does what its
# sparkit/CMakeLists.txt does for the shared library: generate config.hpp
# from config.hpp.in (value_type = double, size_type = std::ptrdiff_t, as in
# CMakeLists.txt:6-8) and compile the listed .cpp files with -O3 -DNDEBUG.
# nlohmann/json (needed by sparkit/data/import.hpp:15) comes from the copy
# that ships in the Python environment's cudnn_frontend headers.
set -euo pipefail

HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF_ROOT="${REF_ROOT:-/root/reference}"
OUT="$HERE/_ref"
# The g++ on PATH, not $CXX: a toolchain that links libstdc++ statically
# gives the library a private iostream state, which crashes the reference's
# istream-based Matrix Market reader once another libstdc++ (numpy's) is in
# the process.  REF_CXX overrides.
CXX="${REF_CXX:-g++}"

if [ ! -f "$REF_ROOT/sparkit/config.hpp.in" ]; then
  echo "build_ref.sh: reference sources not found at $REF_ROOT; skipping" >&2
  exit 0
fi

JSON_INC=""
for cand in \
  "$(python3 -c 'import sysconfig;print(sysconfig.get_paths()["purelib"])' 2>/dev/null)/include/cudnn_frontend/thirdparty" \
  /usr/include /usr/local/include; do
  if [ -f "$cand/nlohmann/json.hpp" ]; then JSON_INC="$cand"; break; fi
done
if [ -z "$JSON_INC" ]; then
  echo "build_ref.sh: nlohmann/json.hpp not found; cannot build the reference" >&2
  exit 1
fi

mkdir -p "$OUT/gen/sparkit" "$OUT/obj"
sed -e 's/\${PROJECT_NAME}/sparkit/' \
    -e 's/\${PROJECT_VERSION_MAJOR}/0/' \
    -e 's/\${PROJECT_VERSION_MINOR}/1/' \
    -e 's/\${PROJECT_VERSION_PATCH}/0/' \
    -e 's/\${sparkit_DEFAULT_VALUE_TYPE}/double/' \
    -e 's/\${sparkit_DEFAULT_SIZE_TYPE}/std::ptrdiff_t/' \
    -e 's/\${[A-Z_a-z]*}//g' \
    "$REF_ROOT/sparkit/config.hpp.in" > "$OUT/gen/sparkit/config.hpp.tmp"
# config.hpp needs <cstddef> for std::ptrdiff_t
{ echo '#include <cstddef>'; cat "$OUT/gen/sparkit/config.hpp.tmp"; } > "$OUT/gen/sparkit/config.hpp"
rm -f "$OUT/gen/sparkit/config.hpp.tmp"

FLAGS=(-std=c++20 -O3 -DNDEBUG -fPIC -ffp-contract=off
       -I "$OUT/gen" -I "$REF_ROOT" -I "$JSON_INC")

# The source list of sparkit/CMakeLists.txt's shared library.
SRCS=$(sed -n '/add_library(sparkit_shared_library/,/)/p' "$REF_ROOT/sparkit/CMakeLists.txt" \
       | grep -o 'data/[A-Za-z_]*\.cpp')

pids=()
objs=()
for s in $SRCS; do
  o="$OUT/obj/$(basename "$s" .cpp).o"
  objs+=("$o")
  if [ ! -f "$o" ] || [ "$REF_ROOT/sparkit/$s" -nt "$o" ]; then
    "$CXX" "${FLAGS[@]}" -c "$REF_ROOT/sparkit/$s" -o "$o" &
    pids+=($!)
  fi
done
shim_o="$OUT/obj/ref_shim.o"
if [ ! -f "$shim_o" ] || [ "$HERE/ref_shim.cpp" -nt "$shim_o" ]; then
  "$CXX" "${FLAGS[@]}" -c "$HERE/ref_shim.cpp" -o "$shim_o" &
  pids+=($!)
fi
for p in "${pids[@]}"; do wait "$p"; done
"$CXX" -shared -o "$OUT/libsparkit_ref.so" "${objs[@]}" "$shim_o" -lpthread
echo "built $OUT/libsparkit_ref.so"

#!/usr/bin/env bash
# Test infrastructure only: compiles the reference's own CPU implementation
# (CPU_version1, FP64, single-threaded) from its sources where they lie, plus
# the shim in this directory, into oracle/_ref/.  Nothing is copied into the
# repository; the outputs are git-ignored build products.
#
#   oracle/build_ref.sh [REFERENCE_ROOT]
#
# REFERENCE_ROOT defaults to $DTWJ_REFERENCE_ROOT, else /root/reference (where
# the reference tree is mounted on the machine that builds the fixtures).
# Exit code 2: no reference sources there (nothing built).
#
# Produces
#   oracle/_ref/libref.so   C ABI around the reference functions (ref_shim.cpp)
#   oracle/_ref/ref_join    one reference join per process (ref_join_main.cpp)
#
# Recipe: every CPU_version1/*.cpp and CPU_version1/allmatrixop/*.cpp except
# the executable's main (AAAA.cpp), g++ -std=c++17 -O2 -include cstring (the
# `-include` supplies the <cstring> several reference files forget).
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${DTWJ_REFERENCE_ROOT:-/root/reference}}/CPU_version1"
OUT="$HERE/_ref"
OBJ="$OUT/obj"
if [ ! -d "$REF" ]; then
  echo "reference sources not found at $REF" >&2
  exit 2
fi
mkdir -p "$OBJ"
CXX="${CXX:-g++}"
FLAGS="-std=c++17 -O2 -fPIC -include cstring -w"
pids=()
objs=()
while IFS= read -r -d '' src; do
  base="$(basename "$src")"
  case "$base" in
    AAAA.cpp) continue ;;
  esac
  rel="${src#$REF/}"
  o="$OBJ/$(echo "$rel" | tr '/ ' '__').o"
  objs+=("$o")
  if [ ! -f "$o" ] || [ "$src" -nt "$o" ]; then
    "$CXX" $FLAGS -I"$REF" -c "$src" -o "$o" &
    pids+=($!)
    if [ "${#pids[@]}" -ge 8 ]; then wait "${pids[0]}"; pids=("${pids[@]:1}"); fi
  fi
done < <(find "$REF" -maxdepth 2 \( -path "$REF/*.cpp" -o -path "$REF/allmatrixop/*.cpp" \) -print0 | sort -z)
for p in "${pids[@]}"; do wait "$p"; done
"$CXX" $FLAGS -I"$REF" -c "$HERE/ref_shim.cpp" -o "$OBJ/ref_shim.o"
"$CXX" -shared -o "$OUT/libref.so" "${objs[@]}" "$OBJ/ref_shim.o"
"$CXX" $FLAGS -I"$REF" "$HERE/ref_join_main.cpp" "${objs[@]}" "$OBJ/ref_shim.o" -o "$OUT/ref_join"
echo "built $OUT/libref.so $OUT/ref_join"

#!/bin/bash
# TEST INFRASTRUCTURE: builds the reference's own CUDA programs, unmodified,
# from their sources under the reference checkout, linked with ref_shim.c
# (trace + seed wrappers).  Output: oracle/_ref/{mdp,maxbs}_<alg> (git-ignored).
# The sources are compiled where they lie; nothing is copied.
#   usage: oracle/build_ref.sh [reference_dir]
# The reference directory comes from the argument, else TS_REFERENCE_DIR, else
# the checkout location of the machine this repository is built on (this
# script is the one place that names it).
set -u
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-${TS_REFERENCE_DIR:-/root/reference}}"
OUT="$HERE/_ref"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
if [ ! -d "$REF/src" ]; then
  echo "reference sources not found at $REF; nothing built"
  exit 0
fi
mkdir -p "$OUT"
gcc -O2 -c "$HERE/ref_shim.c" -o "$OUT/ref_shim.o" || exit 1
build_one() {  # problem_dir file_prefix bin_prefix alg_suffix bin_suffix
  local src="$REF/src/$1/$2-$4.cu" exe="$OUT/$3_$5"
  if [ "$exe" -nt "$src" ] && [ "$exe" -nt "$HERE/ref_shim.c" ]; then return 0; fi
  if "$NVCC" -O3 -gencode arch=compute_100a,code=sm_100a -ccbin g++ "$src" "$OUT/ref_shim.o" \
       -Xlinker --wrap=cudaMemcpy -Xlinker --wrap=srand -o "$exe" > "$exe.build.log" 2>&1; then
    echo "built $exe"
  else
    echo "NOT BUILDABLE: $src (see $exe.build.log)"
    rm -f "$exe"
  fi
}
export -f build_one
export REF OUT NVCC HERE
{
for p in "mdp GPU-MDP mdp" "maxbisection GPU-MAXBS maxbs"; do
  set -- $p
  for a in "CSR csr" "Hash hash" "WSwap wswap" "CSR-Bitset csr-bitset" "CSR-BuscaBinaria csr-bb" \
           "CSR-Bitset-BuscaBinaria csr-bitset-bb"; do
    set -- $p $a
    echo "$1 $2 $3 $4 $5"
  done
done
} | xargs -P 6 -L 1 bash -c 'build_one "$0" "$1" "$2" "$3" "$4"'
# the reference's instance converter (host C++, one source file)
if [ ! "$OUT/convert_mwis" -nt "$REF/src/convert_mwis.cpp" ]; then
  if g++ -O2 -std=c++17 "$REF/src/convert_mwis.cpp" -o "$OUT/convert_mwis" > "$OUT/convert_mwis.build.log" 2>&1; then
    echo "built $OUT/convert_mwis"
  else
    echo "NOT BUILDABLE: $REF/src/convert_mwis.cpp"
  fi
fi

#!/usr/bin/env bash
# Build the reference's own quasi/quasi.cpp and quasi/quasi-stb.cpp against
# oracle/shim (FFTW-MPI + MPI stand-ins, ranks as threads) into oracle/_ref/.
#
# TEST INFRASTRUCTURE ONLY.  The reference ships no build system and needs
# FFTW 3.3 with fftw3-mpi and an MPI with the MPI-2 C++ bindings, none of which
# exist in this image, so as distributed it is unbuildable.  This recipe
# compiles its translation units unchanged except for six substitutions made
# on a copy written to oracle/_ref/ (git-ignored, never committed):
#   0. `int main(argc, argv)` -> `void quasi_ref_main(argc, argv)`: the shim's
#      main runs it once per emulated rank on a thread; the reference's main
#      relies on the implicit `return 0` that only `main` gets
#   1. the compile-time grid  (Nx = Ny = Nz = 256 / 512)  -> run-time QUASI_NX/NY/NZ
#   2. the hard-coded /oasis/... output prefix             -> QUASI_OUTDIR
#   3. the loop bound (L1 > 1e-6 / loopLim)                -> also nLoop < QUASI_MAXSTEPS
#   4. stepL1 / stepSave                                   -> QUASI_STEPL1 / QUASI_STEPSAVE
#   5. text dump precision (ostream default: 6 digits)     -> 17 significant digits
# Usage: oracle/build_ref.sh [reference_root]   (default: $QUASI_REFERENCE, else the
# reference checkout of the build container, /root/reference); exit code 3 when
# the sources are absent (the GPU box uses the prebuilt oracle/_ref)
set -euo pipefail
REF="${1:-${QUASI_REFERENCE:-/root/reference}}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
CXX="${CXX:-g++}"
if [ ! -f "$REF/quasi/quasi.cpp" ]; then
  echo "build_ref: reference sources not found under $REF (set QUASI_REFERENCE)" >&2
  exit 3
fi
mkdir -p "$OUT"

patch_src() {   # $1 = source, $2 = patched copy
  sed -E \
    -e 's/^int main\(int argc, char\* argv\[\]\) \{/void quasi_ref_main(int argc, char* argv[]) {/' \
    -e 's/const ptrdiff_t Nx = [0-9]+, Ny = [0-9]+, Nz = [0-9]+;/const ptrdiff_t Nx = quasi_shim_grid(0), Ny = quasi_shim_grid(1), Nz = quasi_shim_grid(2);/' \
    -e 's#"/oasis/scratch/[^"]*"#quasi_shim_outdir()#g' \
    -e 's/while \(L1 > limL1\)/while (L1 > limL1 \&\& nLoop < quasi_shim_int("QUASI_MAXSTEPS", 500))/' \
    -e 's/const int loopLim = [0-9]+;/const int loopLim = quasi_shim_int("QUASI_MAXSTEPS", 10);/' \
    -e 's/const int stepL1 = ([0-9]+);/const int stepL1 = quasi_shim_int("QUASI_STEPL1", \1);/' \
    -e 's/const int stepSave = ([0-9]+);/const int stepSave = quasi_shim_int("QUASI_STEPSAVE", \1);/' \
    -e 's/_output << /_output << std::setprecision(17) << /g' \
    -e 's/std::setprecision\((8|16)\)/std::setprecision(17)/g' \
    "$1" > "$2"
  # every substitution must have happened exactly where expected
  grep -q '^void quasi_ref_main' "$2"
  grep -q 'quasi_shim_grid(0)' "$2"
  grep -q 'quasi_shim_outdir()' "$2"
  grep -q 'QUASI_MAXSTEPS' "$2"
  grep -q 'QUASI_STEPL1' "$2"
}

FLAGS="-O2 -std=gnu++17 -pthread -I$HERE/shim -w"
$CXX -O2 -std=gnu++20 -pthread -I"$HERE/shim" -c "$HERE/shim/shim.cpp" -o "$OUT/shim.o"
for v in quasi quasi-stb; do
  patch_src "$REF/quasi/$v.cpp" "$OUT/${v}_patched.cpp"
  $CXX $FLAGS -c "$OUT/${v}_patched.cpp" -o "$OUT/${v}.o"
  $CXX -O2 -pthread "$OUT/${v}.o" "$OUT/shim.o" -o "$OUT/${v}_ref"
done
echo "build_ref: built $OUT/quasi_ref $OUT/quasi-stb_ref"

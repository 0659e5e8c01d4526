#!/usr/bin/env bash
# Builds the reference vlasolve binary (OpenMP, no MPI, FP64) from the
# read-only reference tree into oracle/_ref/. Test infrastructure only: the
# binary is used to produce golden vectors and as the timed CPU baseline.
#
# The reference does not compile unmodified with g++ 13, so a scratch copy of
# its src/ is taken under oracle/_ref/src, patched for syntax only, compiled,
# and then deleted. The patches never touch arithmetic:
#   1. drop the stray `template <>` before partial specialisations
#      (slice21Iterator.hxx, subgridIterator.hxx, sliceNNIterator.hxx);
#   2. `static const double` -> `static constexpr double` for an in-class
#      initialiser (subgridIterator.hxx);
#   3. the aliasing sprintf(fname,"%s.ND",fname) in the snapshot writer
#      (vlasovSolver21.hxx) becomes strcat, so snapshot files get their names;
#   4. built with _FORTIFY_SOURCE off, because myIO::writeTag writes one byte
#      past its tag buffer (strcpy of the terminating NUL).
#
# The reference tree is taken from VLS_REFERENCE_DIR; unset, the recipe looks
# in the read-only checkout of this build machine.  Without the tree it
# builds nothing and exits 0 (a machine that only runs prebuilt files).
set -euo pipefail
REF=${VLS_REFERENCE_DIR:-/root/reference}
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
if [ ! -f "$REF/src/vlasolve.cpp" ]; then
  echo "reference tree not found at $REF; skipping reference build" >&2
  exit 0
fi
mkdir -p "$OUT"
rm -rf "$OUT/src"
cp -r "$REF/src" "$OUT/src"
chmod -R u+w "$OUT/src"
S="$OUT/src"
for f in slice21Iterator.hxx subgridIterator.hxx sliceNNIterator.hxx; do
  sed -i '/^template <>$/{N;s/^template <>\ntemplate </template </}' "$S/$f"
done
sed -i 's/static const double N_INT_P_INV/static constexpr double N_INT_P_INV/' "$S/subgridIterator.hxx"
sed -i 's/sprintf(fname,"%s.ND",fname);/strcat(fname,".ND");/' "$S/vlasovSolver21.hxx"
g++ -O3 -fopenmp -DUSE_OPENMP -DNDEBUG -w -fpermissive \
    -U_FORTIFY_SOURCE -D_FORTIFY_SOURCE=0 \
    -o "$OUT/vlasolve" "$S/vlasolve.cpp"
rm -rf "$OUT/src"
echo "built $OUT/vlasolve"

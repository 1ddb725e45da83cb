#!/usr/bin/env bash
# Test infrastructure: builds the unmodified DollarStoreSCF C++ sources into
# oracle/_ref/libdssref.so together with oracle/ref_harness.cpp (a driver the
# reference itself lacks: it has no main()).  Only the tests, the smoke check
# and bench.py's reference arm load the result; the product never links it.
#
# The reference is written for MSVC.  g++ needs four mechanical edits, all of
# them in declarations (no arithmetic changes):
#   lalib/LalibDeclarations.hpp:15  opaque `enum MatrixSymmetryFlags;` -> `: int`
#   lalib/Matrix.hpp:8              matching enum base `: int`
#   lalib/Vector.ipp:20             `Vector<T>::Vector<T>(` -> `Vector<T>::Vector(`
#   lalib/MatrixAlgebra.ipp:534     same for WeightedMatrixSum
# plus a forced include that brings std::isnan/std::isinf into scope.
# The edits are applied to a transient shadow tree under oracle/_ref/.src that
# is deleted after the build, so no reference source is kept in the repository
# or shipped anywhere; only the built .so stays in oracle/_ref/.
#
# LAPACK: the reference calls dspev_/dspsv_/dgesv_/dgesvd_ (lalib/Lapack.cpp:6-9)
# and vendors no LAPACK.  The OpenBLAS 0.3.15 bundled with the opencv wheel in
# this image exports those names unprefixed; it is linked by path.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${DSS_REFERENCE_SRC:-/root/reference/src}"
OUT="$HERE/_ref"
if [ ! -d "$REF" ]; then
  echo "build_ref.sh: reference sources not found at $REF; skipping" >&2
  exit 0
fi
SITE="$(python -c 'import sysconfig; print(sysconfig.get_paths()["purelib"])')"
BLASDIR="$SITE/opencv_python_headless.libs"
BLAS="$(ls "$BLASDIR"/libopenblasp-*.so 2>/dev/null | head -1 || true)"
if [ -z "$BLAS" ]; then
  echo "build_ref.sh: no OpenBLAS with LAPACK symbols found under $BLASDIR" >&2
  exit 1
fi
mkdir -p "$OUT"
SHADOW="$OUT/.src"
rm -rf "$SHADOW"
mkdir -p "$SHADOW"
cp -r "$REF/." "$SHADOW/"
sed -i 's/enum MatrixSymmetryFlags;/enum MatrixSymmetryFlags : int;/' "$SHADOW/lalib/LalibDeclarations.hpp"
sed -i 's/enum MatrixSymmetryFlags {/enum MatrixSymmetryFlags : int {/' "$SHADOW/lalib/Matrix.hpp"
sed -i 's/Vector<T>::Vector<T>(/Vector<T>::Vector(/' "$SHADOW/lalib/Vector.ipp"
sed -i 's/WeightedMatrixSum<T>::WeightedMatrixSum<T>(/WeightedMatrixSum<T>::WeightedMatrixSum(/' "$SHADOW/lalib/MatrixAlgebra.ipp"
printf '#include <cmath>\nusing std::isnan;\nusing std::isinf;\n' > "$SHADOW/compat.h"

# The files on the single-point RHF path and what they pull in.
SRCS="chem/GaussianIntegral.cpp chem/GTO.cpp chem/BasisReader.cpp chem/XYZReader.cpp
chem/Molecule.cpp chem/Element.cpp chem/scf/SCFSolver.cpp chem/scf/SCFBasis.cpp
chem/scf/SCFCommon.cpp chem/scf/SCFDIIS.cpp chem/scf/ExactCoulomb.cpp chem/scf/Energy.cpp
chem/scf/Damping.cpp chem/scf/Population.cpp chem/scf/Output.cpp chem/scf/WriteOrbitals.cpp
chem/scf/Gradient.cpp
lalib/Lapack.cpp lalib/Complex.cpp lalib/PrintMatrix.cpp lalib/LBFGS.cpp
util/FormattedStream.cpp util/TextReader.cpp util/TextUtil.cpp util/Time.cpp util/Parallel.cpp"
OBJDIR="$SHADOW/obj"
mkdir -p "$OBJDIR"
CXXFLAGS="-std=c++17 -O2 -fPIC -fpermissive -w -include $SHADOW/compat.h"
pids=()
for s in $SRCS; do
  o="$OBJDIR/$(echo "$s" | tr '/' '_').o"
  g++ $CXXFLAGS -c "$SHADOW/$s" -o "$o" &
  pids+=($!)
done
for p in "${pids[@]}"; do wait "$p"; done
g++ $CXXFLAGS -I"$SHADOW" -c "$HERE/ref_harness.cpp" -o "$OBJDIR/ref_harness.o"
g++ -shared -o "$OUT/libdssref.so" "$OBJDIR"/*.o "$BLAS" \
    -Wl,--disable-new-dtags -Wl,-rpath,"$BLASDIR" -Wl,-rpath-link,"$BLASDIR" -lpthread

# The drop-in variant: the same reference objects with chem/scf/ExactCoulomb.cpp
# replaced by the engine's shim (dollarstorescf_b200/shim/ExactCoulomb_gpu.cpp),
# linked against the engine library.  Used by the GPU drop-in test only.
DSS_PKG="$(cd "$HERE/.." && pwd)/dollarstorescf_b200"
if [ -f "$DSS_PKG/libdss.so" ]; then
  g++ $CXXFLAGS -I"$SHADOW" -I"$(cd "$HERE/.." && pwd)/include" -c "$DSS_PKG/shim/ExactCoulomb_gpu.cpp" \
      -o "$SHADOW/ExactCoulomb_gpu.o"
  g++ -shared -o "$OUT/libdssref_gpu.so" $(ls "$OBJDIR"/*.o | grep -v chem_scf_ExactCoulomb.cpp.o) \
      "$SHADOW/ExactCoulomb_gpu.o" "$BLAS" "$DSS_PKG/libdss.so" \
      -Wl,--disable-new-dtags -Wl,-rpath,"$BLASDIR" -Wl,-rpath-link,"$BLASDIR" \
      -Wl,-rpath,'$ORIGIN/../../dollarstorescf_b200' -lpthread
  echo "built $OUT/libdssref_gpu.so"
fi
rm -rf "$SHADOW"
echo "built $OUT/libdssref.so"

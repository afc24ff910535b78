#!/bin/sh
# Builds the checkers that run the reference's OWN code, compiled from its
# sources read in place (never copied), into oracle/_ref/ (git-ignored).
# TEST INFRASTRUCTURE ONLY.
#
#   oracle/_ref/libfemlib_ref.so  femlib's element path (ElementRegGrid ->
#       ElementHex -> MaterialQuad(StrainLin) -> Gauss2) in FP64, entry
#       oracle/femlib_k0.cpp: the element stiffness K0.
#   oracle/_ref/libnc_ref.so      SamplesGenerator's NumericalCoarsening (the
#       force-driven coarsened tensor and parameters) with all of femlib,
#       Utilities and StepperCPU's Newton stepper, as the reference ships it
#       (cfgScalar float), entry oracle/ref_nc.cpp; PARDISO, absent from the
#       tree, is replaced by oracle/ref_shim/pardiso_eigen.cpp (the
#       reference's vendored Eigen sparse LU).
#   oracle/_ref/libfastfem_ref.so fast_fem's FEM3DFun (setParam's energy loop,
#       f, df and the field chain rule) and the PiecewiseConstant{,Sym,Cubic}3D
#       fields, entry
#       oracle/ref_fastfem.cpp; topoOptLib, absent from the tree, is replaced
#       by the stand-in headers of oracle/ref_shim/ whose Homogenize() runs the
#       oracle's FP64 solve.
#
# usage: sh oracle/build_ref.sh [reference-tree]   (or FEMH_REFERENCE_TREE);
# without the tree the build is skipped and the tests that use it skip too.
set -e
REF=${1:-${FEMH_REFERENCE_TREE:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
F="$REF/femlib/src"
[ -d "$F" ] || { echo "reference tree not found at $REF; skipping"; exit 0; }
mkdir -p "$OUT/obj"
COMMON="-std=c++11 -fPIC -include iterator -include cfloat -include cstring -w"

# 1. femlib element path, FP64
if [ ! -f "$OUT/libfemlib_ref.so" ] || [ "$HERE/femlib_k0.cpp" -nt "$OUT/libfemlib_ref.so" ]; then
g++ $COMMON -O1 -shared -DUSE_DOUBLE_FOR_SCALAR \
    -I"$REF/femlib/include" -I"$REF/Utilities/include" -Wl,--no-undefined -o "$OUT/libfemlib_ref.so" \
    "$HERE/femlib_k0.cpp" "$F/ElementRegGrid.cpp" "$F/ElementMesh.cpp" "$F/Element.cpp" \
    "$F/ElementHex.cpp" "$F/MaterialQuad.cpp" "$F/Material.cpp" "$F/Quadrature.cpp" \
    "$F/StrainLin.cpp" "$F/StrainEne.cpp" "$F/femError.cpp"
fi

# 2. NumericalCoarsening (float, as shipped) + femlib + Utilities + Newton stepper
INC="-I$REF/femlib/include -I$REF/Utilities/include -I$REF/StepperCPU/include -I$REF/SamplesGenerator"
NC="$OUT/libnc_ref.so"
if [ ! -f "$NC" ] || [ "$HERE/ref_nc.cpp" -nt "$NC" ] || [ "$HERE/ref_shim/pardiso_eigen.cpp" -nt "$NC" ]; then
  SRCS=""
  for s in "$F"/*.cpp "$REF/Utilities/src/"*.cpp "$REF/StepperCPU/src/StepperNewton.cpp" \
           "$REF/StepperCPU/src/StepperNewton2D.cpp" "$REF/SamplesGenerator/NumericalCoarsening.cpp"; do
    case "$(basename "$s")" in
      EigenUtil.cpp|MatTable.cpp) continue ;;   # EigenUtil.cpp does not compile (EigenUtil.hpp:69); MatTable is unused
    esac
    SRCS="$SRCS $s"
  done
  # the 2-D files define file-scope names that the 3-D files define too
  # (makeGauss2, makeUniform4, oneEleV); they are renamed in those two
  # translation units only, so the one library holds both
  for s in $SRCS "$HERE/ref_nc.cpp" "$HERE/ref_shim/pardiso_eigen.cpp"; do echo "$s"; done |
    xargs -P "$(nproc)" -I{} sh -c 'case "{}" in
        */Quadrature2D.cpp) X="-DmakeGauss2=makeGauss2_2d -DmakeUniform4=makeUniform4_2d" ;;
        */ElementRegGrid2D.cpp) X="-DoneEleV=oneEleV_2d" ;;
        *) X="" ;; esac
      g++ '"$COMMON"' -O2 '"$INC"' $X -c "{}" -o "'"$OUT"'/obj/nc_$(basename "{}" .cpp).o"'
  g++ -shared -fPIC -fopenmp -Wl,--no-undefined -o "$NC" "$OUT"/obj/nc_*.o
fi

# 3. fast_fem FEM3DFun against the stand-in topoOptLib headers
FF="$OUT/libfastfem_ref.so"
if [ -f "$HERE/ref_fastfem.cpp" ] && { [ ! -f "$FF" ] || [ "$HERE/ref_fastfem.cpp" -nt "$FF" ] ||
     [ -n "$(find "$HERE/ref_shim" -newer "$FF" -name '*.h')" ] || [ "$HERE/libfemh_oracle.so" -nt "$FF" ]; }; then
  g++ $COMMON -O2 -shared -I"$HERE/ref_shim" -I"$HERE" -I"$REF/fast_fem" -I"$REF/femlib/include" \
      -Wl,--no-undefined -o "$FF" "$HERE/ref_fastfem.cpp" "$REF/fast_fem/FEM3DFun.cpp" \
      "$REF/fast_fem/ArrayUtil.cpp" "$REF/fast_fem/PiecewiseConstant3D.cpp" \
      "$REF/fast_fem/PiecewiseConstantCubic3D.cpp" "$REF/fast_fem/PiecewiseConstantSym3D.cpp" \
      "$REF/fast_fem/RealFun.cpp" \
      -L"$HERE" -lfemh_oracle -Wl,-rpath,'$ORIGIN/..' -fopenmp
fi
echo "built $OUT"

#!/bin/sh
# Builds oracle/_ref/libfemlib_ref.so from the reference's own femlib sources,
# read in place (never copied), plus oracle/femlib_k0.cpp (this project's C
# entry point).  Test infrastructure only: it cross-checks the oracle's element
# stiffness against the reference's code.  Needs the reference tree (default
# /root/reference); without it the build is skipped and the tests that use the
# library skip too.
set -e
REF=${1:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref/libfemlib_ref.so"
F="$REF/femlib/src"
[ -d "$F" ] || { echo "reference tree not found at $REF; skipping"; exit 0; }
mkdir -p "$HERE/_ref"
# femlib element path: ElementRegGrid -> ElementHex -> MaterialQuad(StrainLin) -> Gauss2
g++ -std=c++11 -O1 -fPIC -shared -include iterator -include cfloat -DUSE_DOUBLE_FOR_SCALAR \
    -I"$REF/femlib/include" -I"$REF/Utilities/include" -w -Wl,--no-undefined -o "$OUT" \
    "$HERE/femlib_k0.cpp" "$F/ElementRegGrid.cpp" "$F/ElementMesh.cpp" "$F/Element.cpp" \
    "$F/ElementHex.cpp" "$F/MaterialQuad.cpp" "$F/Material.cpp" "$F/Quadrature.cpp" \
    "$F/StrainLin.cpp" "$F/StrainEne.cpp" "$F/femError.cpp"
echo "built $OUT"

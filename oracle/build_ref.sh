#!/usr/bin/env bash
# Build the reference's own CUDA step kernels (engrab6/lbmPonD) for sm_100a,
# driven by oracle/ref_main.cu.  TEST INFRASTRUCTURE ONLY: the binaries pin
# the FP64 oracle against the reference and time the reference kernels on
# the GPU; nothing in the product links them.
#
#   oracle/build_ref.sh <D1Q5|D3Q27|D3Q125> <double|float> <nx> <ny> <nz> [scheme] [bc]
#
# scheme selects the interpolation call of LBMpull among the reference's own
# alternatives at steps.cu:444-463 (the live one is propagate<4>, :451):
#   lagr4 (default)     as shipped
#   lagr2, lagr3, lagr5 the template order of the live call changed
#   weno5               :451 commented, :458 propagateWENO<3,5> uncommented
#   gap2                :451 commented, :449 propagate_nonequal_1D<2> uncommented
#   nu3                 :451 commented, :453 propagateNR_1D uncommented, and
#                       consts.h:12 NRMESH defined (node positions in Cell::p)
# Only comment markers and the template argument change; the binary name
# carries the scheme unless it is lagr4.
#
# On D3Q125 the shipped calcStep launches PonDstepD3Q125 (update.cu:97) and
# LBMpull takes its fixed-stencil D3Q125 block (steps.cu:366); both switches
# are `#if defined D3Q125 && 1`.  For a D3Q125 scheme other than lagr4 the
# two `&& 1` become `&& 0`, so the step runs PonDstep -> LBMpull's generic
# branch with the selected interpolation call (the reference's own
# alternative, as for the other lattices).
#
# bc = mirror sets the `outflow` flags of steps.cu.  On the D1Q5 / D3Q27
# path only propagate<N>'s counts (steps.cu:1004-1013): the stencil is
# reflected at every face with the populations reversed and u negated
# (Cell::mirrX/Y/Z, structs.cuh:552-578).  On D3Q125 only the launched
# PonDstepD3Q125's counts (steps.cu:167-191): the same reflection through
# the reverse tables.  periodic (default) leaves them off.  With the
# Lagrange schemes only (the other propagators never read the flag).
#
# The reference sources stay where they are (read-only); patched copies live
# in a temporary directory and only the binary is written, into oracle/_ref/.
# Patches (the lattice, precision and grid size are compile-time constants in
# the reference):
#   consts.h:7       the live lattice #define
#   params.h:13      USE_DOUBLE -> USE_FLOAT for the float build
#   params.h:160-161 cudaPointerAttributes::memoryType -> type (CUDA >= 11)
#   structs.cuh:10-12 LSizeX/Y/Z (grid = LSize * brick(4,1,1))
#   im2D.h           replaced by a stub: the GL/GLUT window code is not on
#                    the step's path and no graphics stack exists here
set -euo pipefail
# the reference's source tree: POND_REFERENCE_DIR, else a directory named
# "reference" beside this repository
REF=${POND_REFERENCE_DIR:-$(cd "$(dirname "$0")/../.." && pwd)/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
LAT=${1:?lattice}; PREC=${2:?precision}; NX=${3:?nx}; NY=${4:?ny}; NZ=${5:?nz}; SCHEME=${6:-lagr4}; BC=${7:-periodic}
case "$BC" in
  periodic) ;;
  mirror) case "$SCHEME" in lagr*) ;; *) echo "mirror: Lagrange schemes only" >&2; exit 2;; esac ;;
  *) echo "bad bc $BC" >&2; exit 2;;
esac
case "$SCHEME" in lagr2|lagr3|lagr4|lagr5|weno5|gap2|nu3) ;; *) echo "bad scheme $SCHEME" >&2; exit 2;; esac
case "$LAT" in D1Q5|D3Q27|D3Q125) ;; *) echo "bad lattice $LAT" >&2; exit 2;; esac
case "$PREC" in double|float) ;; *) echo "bad precision $PREC" >&2; exit 2;; esac
if (( NX % 4 != 0 )); then echo "nx must be a multiple of 4 (brick.x)" >&2; exit 2; fi
if [ ! -f "$REF/steps.cu" ]; then echo "reference sources not found at $REF" >&2; exit 3; fi
NVCC=${NVCC:-nvcc}
EXTRA=()
mkdir -p "$OUT"
BIN="$OUT/ref_pond_${LAT}_${PREC}_${NX}x${NY}x${NZ}"
if [ "$SCHEME" != lagr4 ]; then BIN="${BIN}_${SCHEME}"; fi
if [ "$BC" = mirror ]; then BIN="${BIN}_mirror"; fi
TMP=$(mktemp -d /tmp/pond_ref.XXXXXX)
trap 'rm -rf "$TMP"' EXIT
cp "$REF"/*.cu "$REF"/*.cuh "$REF"/*.h "$REF"/*.hpp "$TMP"/
sed -i "s/^ #define D1Q5\$/ #define ${LAT}/" "$TMP/consts.h"
grep -q "^ #define ${LAT}\$" "$TMP/consts.h"
sed -i "s/^const long int LSizeX=.*/const long int LSizeX=$((NX / 4));/; s/^const long int LSizeY=.*/const long int LSizeY=${NY};/; s/^const long int LSizeZ=.*/const long int LSizeZ=${NZ};/" "$TMP/structs.cuh"
sed -i 's/ptrAt\.memoryType/ptrAt.type/g' "$TMP/params.h"
if [ "$PREC" = float ]; then sed -i 's/^#define USE_DOUBLE$/#define USE_FLOAT/' "$TMP/params.h"; fi
if [ "$BC" = mirror ]; then
  [ "$(grep -c '^    const bool outflow=0;$' "$TMP/steps.cu")" -ge 1 ]
  sed -i 's/^    const bool outflow=0;$/    const bool outflow=1;/' "$TMP/steps.cu"
fi
LIVE='^\( *newfh = propagate *\)<4>\((make_ftype3(coord)-vi\[i\], i, uT,M4);\)$'
grep -q "$LIVE" "$TMP/steps.cu"
case "$SCHEME" in
  lagr2|lagr3|lagr5) sed -i "s/$LIVE/\1<${SCHEME#lagr}>\2/" "$TMP/steps.cu" ;;
  weno5|gap2|nu3)
    sed -i "s/$LIVE/\/\/&/" "$TMP/steps.cu"
    case "$SCHEME" in
      weno5) PAT='newfh = propagateWENO<3,5>(make_ftype3(coord)-vi\[i\], i, uT, vi\[i\].x, Niter);' ;;
      gap2)  PAT='newfh = propagate_nonequal_1D<2>(make_ftype3(coord)-vi\[i\], i, uT);' ;;
      nu3)   PAT='newfh = propagateNR_1D(c0_st.p-vi\[i\],coord, i, uT);' ;;
    esac
    grep -q "^// *${PAT}\$" "$TMP/steps.cu"
    sed -i "s/^\/\/\( *${PAT}\)\$/\1/" "$TMP/steps.cu"
    grep -q "^ *${PAT}\$" "$TMP/steps.cu"
    if [ "$SCHEME" = nu3 ]; then
      sed -i 's/^\/\/ *#define NRMESH$/#define NRMESH/' "$TMP/consts.h"
      grep -q '^#define NRMESH$' "$TMP/consts.h"
    fi ;;
esac
if [ "$LAT" = D3Q125 ] && [ "$SCHEME" != lagr4 ]; then
  [ "$(grep -c '^  #if defined D3Q125 && 1$' "$TMP/steps.cu" "$TMP/update.cu" | awk -F: '{s+=$2} END {print s}')" -eq 2 ]
  sed -i 's/^  #if defined D3Q125 \&\& 1$/  #if defined D3Q125 \&\& 0/' "$TMP/steps.cu" "$TMP/update.cu"
  EXTRA=(-DPOND_REF_D3Q125_PULL)  # oracle/ref_main.cu mirrors calcStep's launch switch
fi
cat > "$TMP/im2D.h" <<'EOF'
#ifndef IM2D_H
#define IM2D_H
struct image2D { void get_device(int, int) {} };
#endif
EOF
FLAGS=(-gencode arch=compute_100a,code=sm_100a -O3 -rdc=true -I"$TMP" -Xcudafe --diag_suppress=declared_but_not_referenced -w)
for f in update init lbpack diagn drop; do
  "$NVCC" "${FLAGS[@]}" -c "$TMP/$f.cu" -o "$TMP/$f.o"
done
"$NVCC" "${FLAGS[@]}" "${EXTRA[@]}" -c "$HERE/ref_main.cu" -o "$TMP/ref_main.o"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -rdc=true "$TMP"/*.o -o "$BIN"
echo "$BIN"

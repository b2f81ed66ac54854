#!/bin/sh
# Builds the MATLAB interface of libzfmm_b200 (needs MATLAB's `mex`; the
# library itself is built first with `python -m zfmm_b200.build`).
#
#   sh build_mex.sh                      hand-written gateway zfmm_b200_mex.c,
#                                        one MEX file per routine (zlfmm2dmex ...),
#                                        used by the .m wrappers in this folder
#   sh build_mex.sh --mwrap <dir> <mwrap>
#                                        mwrap-generated gateways from the .mw
#                                        specs in <dir> (the reference's
#                                        zfmm2d/matlab_linux or zfmm3d/matlab_linux),
#                                        linked against libzfmm_b200 instead of the
#                                        Fortran archive: their FORTRAN lines call
#                                        zlfmm2d_ ... which the library exports
#
# MEX, CUDA and the library path can be overridden: MEX=/path/to/mex.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
PKG=$(dirname "$HERE")
INC=$(dirname "$PKG")/include
MEX=${MEX:-mex}
LIBS="-L$PKG -lzfmm_b200 -Wl,-rpath,$PKG"
ROUTINES="zlfmm2d zhfmm2d zl2devaldirect zh2devaldirect zlfmm3d zhfmm3d zl3devaldirect zh3devaldirect"

if [ "$1" = "--mwrap" ]; then
  DIR=$2
  MWRAP=${3:-mwrap}
  cd "$DIR"
  for r in $ROUTINES; do
    [ -f "$r.mw" ] || continue
    "$MWRAP" -c99complex -list -mex "${r}mex" -mb "$r.mw"
    "$MWRAP" -c99complex -mex "${r}mex" -c "${r}mex.c" "$r.mw"
    "$MEX" -largeArrayDims -DMWF77_UNDERSCORE1 "${r}mex.c" $LIBS -output "${r}mex"
  done
  exit 0
fi

cd "$HERE"
for r in $ROUTINES; do
  "$MEX" -R2018a -I"$INC" zfmm_b200_mex.c $LIBS -output "${r}mex"
done

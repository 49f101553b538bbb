#!/bin/sh
# Builds oracle/_ref/libxts_ref.so: the reference's own hot-path translation
# units, compiled in place from the reference tree, plus oracle/ref_driver.cxx.
# TEST INFRASTRUCTURE ONLY (CPU checker and timed CPU reference arm).
#
#   oracle/build_ref.sh [REFERENCE_ROOT]      (default $XTS_REFERENCE, else /root/reference)
#
# Include order: oracle/ref_overlay (SkyGeom stand-in, cblas.h), then
# oracle/_ref/patched (a build-time copy of
# model_map/mm_cubature/convolve_pixel_psf_logsep.hpp with the one missing
# statement `keys[index] = psfidx;` added after the weight accumulation), then
# the reference tree.  Outputs go to oracle/_ref only.
set -e
REF=${1:-${XTS_REFERENCE:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$HERE/_ref
LOGSEP=xtsrcmaps/model_map/mm_cubature/convolve_pixel_psf_logsep.hpp
[ -f "$REF/$LOGSEP" ] || { echo "reference tree not found at $REF"; exit 1; }
mkdir -p "$OUT/patched/$(dirname $LOGSEP)" "$OUT/obj"
sed '/sum_wts\[index\]\.second += t \* w;/a\        keys[index] = psfidx;' "$REF/$LOGSEP" > "$OUT/patched/$LOGSEP"
[ "$(grep -c 'keys\[index\] = psfidx;' "$OUT/patched/$LOGSEP")" = 1 ] || { echo "keys fix did not apply"; exit 1; }

# the system GCC 13 (it ships libgomp); the environment's CXX may name a wrapper without it
CXX=${XTS_REF_CXX:-/usr/bin/g++}
CC=${XTS_REF_CC:-/usr/bin/gcc}
# x86-64-v3 (AVX2/FMA), not -march=native: the library is built here and runs on another host
FLAGS="-std=c++23 -O3 -march=x86-64-v3 -fopenmp -DNDEBUG -fPIC -include memory -include cstring \
  -I$HERE/ref_overlay -I$OUT/patched -I$REF -I$HERE"
TUS="exposure/exposure.cxx exposure/exposure.contract.cpp healpix/healpix.cxx math/bilerp.cxx
  psf/psf.king.cxx psf/psf.bilerp.cxx psf/psf.corrected_exposure_psf.cxx psf/psf.mean_psf.cxx
  psf/psf.partial_total_integral.cxx psf/psf.normalize.cxx psf/psf.fast_separation_lower_index.cxx
  psf/psf.psf_lookup_table_and_partial_integrals.cxx
  model_map/model_map.point_src_model_map_wcs.cxx model_map/model_map.map_integral.cxx
  model_map/model_map.map_correction_factor.cxx model_map/model_map.psf_boundary_radius.cxx
  model_map/model_map.scale_map_by_solid_angle.cxx model_map/model_map.scale_map_by_exposure.cxx
  model_map/model_map.scale_map_by_correction_factor.cxx model_map/mm_cubature/cubature.implementation.cxx"
pids=""
for tu in $TUS; do
  o="$OUT/obj/$(echo "$tu" | tr / _).o"
  $CXX $FLAGS -c "$REF/xtsrcmaps/$tu" -o "$o" &
  pids="$pids $!"
done
$CXX $FLAGS -c "$HERE/ref_driver.cxx" -o "$OUT/obj/ref_driver.o" &
pids="$pids $!"
$CC -O2 -fPIC -std=c99 -ffp-contract=off -c "$HERE/xts_oracle.c" -o "$OUT/obj/xts_oracle.o" &
pids="$pids $!"
for p in $pids; do wait $p; done
$CXX -shared -fopenmp -o "$OUT/libxts_ref.so" "$OUT"/obj/*.o -lm
echo "built $OUT/libxts_ref.so"

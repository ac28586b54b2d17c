#!/usr/bin/env bash
# Compiles HemePure's own sources, unmodified and where they lie in the reference
# tree, into single-rank CPU solvers used as the parity oracle (test
# infrastructure only; nothing in the product links or runs them).
#
#   oracle/ref/build_ref.sh [combo ...]      (default: every combo below)
#
# The reference's CMake build is not used.  Its external dependencies are
# replaced by the stand-ins in oracle/ref/shim (single-process MPI, std-backed
# boost adaptors, an idx_t-only parmetis.h, a no-op ctemplate, XDR); TinyXML is
# compiled from the reference's own dep/src tarball into the build folder.  The
# four headers CMake would configure from *.h.in templates are produced here by
# substituting the same cache values.  Outputs go to oracle/_ref/ only.
#
# Build choices follow src/CMakeLists.txt:17-111: -O3 with SSE3 intrinsics
# (HEMELB_USE_SSE3, the default; no FMA contraction is possible without -mfma),
# HEMELB_READING_GROUP_SIZE=1 so a one-rank run reads the geometry
# (src/geometry/GeometryReader.cc:643-644), neutral architecture weights, and
# one executable per kernel / boundary-condition combination, because the
# reference fixes them at compile time (src/lb/lb.h:37-48).
set -euo pipefail

REF="${HEMEPURE_REFERENCE:-/root/reference}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$(cd "$HERE/.." && pwd)/_ref"
JOBS="${JOBS:-$(nproc)}"
SRC="$REF/src"

if [ ! -d "$SRC" ]; then
  echo "build_ref: reference sources not found at $SRC" >&2
  exit 2
fi

# combo: kernel wall inlet outlet wall-inlet wall-outlet
declare -A COMBOS=(
  [lbgk_sbb_nash]="LBGK SIMPLEBOUNCEBACK NASHZEROTHORDERPRESSUREIOLET NASHZEROTHORDERPRESSUREIOLET NASHZEROTHORDERPRESSURESBB NASHZEROTHORDERPRESSURESBB"
  [lbgk_bfl_ladd_nash]="LBGK BFL LADDIOLET NASHZEROTHORDERPRESSUREIOLET LADDIOLETBFL NASHZEROTHORDERPRESSUREBFL"
  [trt_gzs_nash]="TRT GZS NASHZEROTHORDERPRESSUREIOLET NASHZEROTHORDERPRESSUREIOLET NASHZEROTHORDERPRESSUREGZS NASHZEROTHORDERPRESSUREGZS"
  [les_bfl_ladd_nash]="LBGKLESSL BFL LADDIOLET NASHZEROTHORDERPRESSUREIOLET LADDIOLETBFL NASHZEROTHORDERPRESSUREBFL"
  [lbgk_sbb_ladd_nash]="LBGK SIMPLEBOUNCEBACK LADDIOLET NASHZEROTHORDERPRESSUREIOLET LADDIOLETSBB NASHZEROTHORDERPRESSURESBB"
  [trt_gzs_ladd_nash]="TRT GZS LADDIOLET NASHZEROTHORDERPRESSUREIOLET LADDIOLETGZS NASHZEROTHORDERPRESSUREGZS"
)

if [ $# -gt 0 ]; then WANT=("$@"); else WANT=("${!COMBOS[@]}"); fi

mkdir -p "$OUT"
CXX="${CXX:-g++}"
CC="${CC:-gcc}"

# TinyXML from the reference's dependency tarball (third-party source, compiled only).
TX="$OUT/tinyxml"
if [ ! -f "$TX/libtinyxml.a" ]; then
  rm -rf "$TX.tmp"
  mkdir -p "$TX.tmp"
  tar -xzf "$REF/dep/src/tinyxml_2_6_2.tar.gz" -C "$TX.tmp"
  TXS="$(dirname "$(find "$TX.tmp" -name tinyxml.cpp | head -1)")"
  for f in tinyxml tinystr tinyxmlerror tinyxmlparser; do
    $CXX -O3 -msse3 -DTIXML_USE_STL -c "$TXS/$f.cpp" -o "$TX.tmp/$f.o"
  done
  ar rcs "$TX.tmp/libtinyxml.a" "$TX.tmp"/*.o
  mkdir -p "$TX"
  cp "$TXS/tinyxml.h" "$TXS/tinystr.h" "$TX.tmp/libtinyxml.a" "$TX/"
  rm -rf "$TX.tmp"
fi

# Stand-ins shared by every combo.
SH="$OUT/shim"
mkdir -p "$SH"
stale=0
for f in "$HERE"/shim/*.c "$HERE"/shim/*.cc "$HERE"/shim/*.h; do
  if [ ! -f "$SH/libshim.a" ] || [ "$f" -nt "$SH/libshim.a" ]; then stale=1; fi
done
if [ $stale = 1 ]; then
  $CXX -O2 -std=gnu++17 -I"$HERE/shim" -c "$HERE/shim/mpi_stub.cc" -o "$SH/mpi_stub.o"
  $CC -O2 -I"$HERE/shim" -c "$HERE/shim/xdr_stub.c" -o "$SH/xdr_stub.o"
  $CC -O2 -I"$HERE/shim" -c "$HERE/shim/parmetis_stub.c" -o "$SH/parmetis_stub.o"
  rm -f "$SH/libshim.a"
  ar rcs "$SH/libshim.a" "$SH/mpi_stub.o" "$SH/xdr_stub.o" "$SH/parmetis_stub.o"
fi

# The translation units the reference's own CMake lists name for its libraries
# (src/*/CMakeLists.txt add_library), except colloids (never configured by these
# cases); SimulationMaster.cc and main.cc are replaced by harness.cc.
mapfile -t SOURCES < <(python3 - "$SRC" <<'PY'
import os, re, sys
src = sys.argv[1]
for d in "configuration extraction reporting geometry lb net util io log".split():
    txt = re.sub(r"#.*", "", open(os.path.join(src, d, "CMakeLists.txt")).read())
    for m in re.finditer(r"add_library\(\s*\S+(.*?)\)", txt, re.S):
        for tok in m.group(1).split():
            if tok.endswith(".cc"):
                print(os.path.join(d, tok))
PY
)

configure() {  # configure <template> <output> <kernel> <wall> <inlet> <outlet> <wall-inlet> <wall-outlet>
  local in="$1" out="$2"
  mkdir -p "$(dirname "$out")"
  sed -e "s/@CMAKE_BUILD_TYPE@/Release/" -e "s/@HEMELB_OPTIMISATION@/-O3/" \
      -e "s/@HEMELB_USE_SSE3@/ON/" -e "s/@HEMELB_BUILD_TIME@/oracle/" \
      -e "s/@HEMELB_READING_GROUP_SIZE@/1/" -e "s/@HEMELB_LATTICE@/D3Q19/" \
      -e "s/@HEMELB_KERNEL@/$3/" -e "s/@HEMELB_WALL_BOUNDARY@/$4/g" \
      -e "s/@HEMELB_INLET_BOUNDARY@/$5/g" -e "s/@HEMELB_OUTLET_BOUNDARY@/$6/g" \
      -e "s/@HEMELB_WALL_INLET_BOUNDARY@/$7/" -e "s/@HEMELB_WALL_OUTLET_BOUNDARY@/$8/" \
      -e "s/@HEMELB_COMPUTE_ARCHITECTURE@/NEUTRAL/g" \
      -e "s/@HEMELB_POINTPOINT_IMPLEMENTATION@/Coalesce/" -e "s/@HEMELB_GATHERS_IMPLEMENTATION@/Separated/" \
      -e "s/@HEMELB_ALLTOALL_IMPLEMENTATION@/Separated/" -e "s/@HEMELB_SEPARATE_CONCERNS@/OFF/" \
      -e "s|@BUILD_RESOURCE_PATH@|$OUT/resources|" -e "s|@INSTALL_RESOURCE_PATH@|$OUT/resources|" \
      -e "s/#cmakedefine HEMELB_SEPARATE_CONCERNS/\/* HEMELB_SEPARATE_CONCERNS off *\//" \
      -e "s/#cmakedefine HAVE_CONSTCORRECTMPI/#define HAVE_CONSTCORRECTMPI/" \
      "$in" > "$out.tmp"
  if [ ! -f "$out" ] || ! cmp -s "$out.tmp" "$out"; then mv "$out.tmp" "$out"; else rm -f "$out.tmp"; fi
}

for combo in "${WANT[@]}"; do
  spec="${COMBOS[$combo]:-}"
  if [ -z "$spec" ]; then
    echo "build_ref: unknown combo $combo (have: ${!COMBOS[*]})" >&2
    exit 2
  fi
  read -r K W I O WI WO <<< "$spec"
  B="$OUT/$combo"
  # The reference tree is read-only: a binary newer than this recipe, the
  # harness and the stand-ins is current.
  if [ -x "$B/hemepure_ref" ] && [ -z "${FORCE:-}" ]; then
    fresh=1
    for f in "${BASH_SOURCE[0]}" "$HERE/harness.cc" $(find "$HERE/shim" -type f); do
      [ "$f" -nt "$B/hemepure_ref" ] && fresh=0
    done
    if [ $fresh = 1 ]; then echo "build_ref: $B/hemepure_ref (current)"; continue; fi
  fi
  G="$B/gen"
  mkdir -p "$B/obj"
  configure "$SRC/reporting/BuildInfo.h.in" "$G/reporting/BuildInfo.h" $K $W $I $O $WI $WO
  configure "$SRC/geometry/decomposition/DecompositionWeights.h.in" "$G/geometry/decomposition/DecompositionWeights.h" $K $W $I $O $WI $WO
  configure "$SRC/net/BuildInfo.h.in" "$G/net/BuildInfo.h" $K $W $I $O $WI $WO
  configure "$SRC/net/MpiConstness.h.in" "$G/net/MpiConstness.h" $K $W $I $O $WI $WO
  configure "$SRC/resources/path_parameters.h.in" "$G/resources/path_parameters.h" $K $W $I $O $WI $WO

  FLAGS=(-O3 -msse3 -std=gnu++17 -w -Wno-deprecated-declarations
    -DHEMELB_CODE -DHEMELB_READING_GROUP_SIZE=1 -DHEMELB_READING_GROUP_SPACING=1
    -DHEMELB_LATTICE=D3Q19 -DHEMELB_KERNEL=$K -DHEMELB_WALL_BOUNDARY=$W
    -DHEMELB_INLET_BOUNDARY=$I -DHEMELB_OUTLET_BOUNDARY=$O
    -DHEMELB_WALL_INLET_BOUNDARY=$WI -DHEMELB_WALL_OUTLET_BOUNDARY=$WO
    -DHEMELB_COMPUTE_ARCHITECTURE=NEUTRAL -DHEMELB_LOG_LEVEL=Warning
    -DHEMELB_IMAGES_TO_NULL -DHEMELB_TRACER_PARTICLES -DHEMELB_USE_SSE3
    -DTIXML_USE_STL -DHAVE_STD_ISNAN -DLINUX_SCANDIR -DHAVE_RUSAGE -DHEMELB_HAVE_CSTDINT
    -DHAVE_FOPENCOOKIE
    -I"$G" -I"$SRC" -I"$HERE/shim" -I"$TX")
  # Objects are cached by a hash of the preprocessed source and the flags, so
  # translation units that do not depend on the combo are compiled once.
  mkdir -p "$OUT/objcache"
  export CXX B SRC HERE OUT
  export FLAGS_STR="${FLAGS[*]}"
  rm -f "$B"/obj/*.o
  printf '%s\n' "${SOURCES[@]}" harness | xargs -P "$JOBS" -I{} bash -c '
    set -o pipefail
    s="{}"
    if [ "$s" = harness ]; then src="$HERE/harness.cc"; else src="$SRC/$s"; fi
    key=$({ echo "$CXX -O3 -msse3 -std=gnu++17"; $CXX $FLAGS_STR -E -P "$src"; } | sha1sum | cut -c1-40) || { echo "FAILED: $s (preprocess)"; exit 255; }
    c="$OUT/objcache/$key.o"
    if [ ! -f "$c" ]; then
      $CXX $FLAGS_STR -c "$src" -o "$c.tmp.$$" 2> "$c.log" || { echo "FAILED: $s"; head -40 "$c.log"; exit 255; }
      mv "$c.tmp.$$" "$c"
    fi
    ln -sf "$c" "$B/obj/$(echo "$s" | tr / _).o"'
  $CXX -O3 -o "$B/hemepure_ref.tmp" "$B"/obj/*.o "$SH/libshim.a" "$TX/libtinyxml.a" -lz
  mv "$B/hemepure_ref.tmp" "$B/hemepure_ref"
  echo "build_ref: $B/hemepure_ref"
done

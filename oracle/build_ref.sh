#!/bin/sh
# Test infrastructure: builds the REFERENCE QLA 1.9.0 level-1 libraries as a checker.
#
# QLA's level-1 C exists only as output of its Perl generator
# (lib/perl/build_qla.pl:36-49, invoked per library by lib/make_qla_dirs:66).
# This recipe does NOT run QLA's autotools build.  It invokes the generator
# script in place (read-only source tree), writes every generated file under
# oracle/_ref/ (git-ignored), and compiles the generated C plus the
# hand-written code templates, lib/cmath and lib/random with gcc, using the
# per-library flags of lib/make_qla_dirs:27-40.  Nothing here is copied into the
# repository's history; the product never links or calls the result.
#
# Output: oracle/_ref/libqla_ref.so  (OpenMP build of the generated code:
#         lib/perl/formatting.pl:90-127 with $have_openmp="yes").
#         Run with OMP_NUM_THREADS=1 it reproduces the serial summation order.
#
# Usage: sh oracle/build_ref.sh <reference-root>
#        (or QLA_REF_SRC=<reference-root> sh oracle/build_ref.sh)
set -e
REF=${1:-${QLA_REF_SRC:-}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$HERE/_ref
JOBS=${JOBS:-$(nproc)}

if [ -z "$REF" ]; then
  echo "build_ref.sh: name the QLA source tree as the first argument or in QLA_REF_SRC" >&2
  exit 2
fi
if [ ! -f "$REF/lib/perl/build_qla.pl" ]; then
  echo "build_ref.sh: reference tree not found at $REF" >&2
  exit 2
fi
# The reference's hand-written API headers (qla.h, qla_types.h, qla_complex.h
# ...) beside the generated ones, so that a C caller can be compiled against
# the reference's own headers from oracle/_ref alone (tests/test_c_dropin.py).
copy_api_headers() {
  mkdir -p "$OUT/gen/include"
  for h in "$REF"/include/*.h; do cp "$h" "$OUT/gen/include/"; done
}
if [ -f "$OUT/libqla_ref.so" ] && [ "$OUT/libqla_ref.so" -nt "$HERE/build_ref.sh" ]; then
  copy_api_headers
  echo "build_ref.sh: $OUT/libqla_ref.so is up to date"
  exit 0
fi

GEN=$OUT/gen
rm -rf "$GEN"
mkdir -p "$GEN/perl" "$GEN/include" "$GEN/obj"

# generator configuration normally substituted by configure (lib/perl/defines.pl.in)
cat > "$GEN/perl/defines.pl" <<'EOF'
$have_openmp = "yes";
$have_xlc = "no";
$temp_precision = "";
1;
EOF
cat > "$GEN/include/qla_config.h" <<'EOF'
#define VERSION "1.9.0"
#define PACKAGE_VERSION "1.9.0"
#define QLA_SSE_LEVEL 0
EOF

# libraries whose headers qla.h pulls in (qla.h:113-129) and whose code we compile
HDR_ONLY="qla_q qla_dq qla_q3 qla_dq3 qla_qn qla_dqn"
COMPILE="qla_int qla_f qla_d qla_df qla_f2 qla_d2 qla_df2 qla_f3 qla_d3 qla_df3 qla_fn qla_dn qla_dfn"

for dir in $COMPILE $HDR_ONLY; do
  tag=$(echo $dir | sed s/_int// | tr a-z A-Z)
  mkdir -p "$GEN/$dir"
  ( cd "$GEN/$dir" && perl "$REF/lib/perl/build_qla.pl" "$tag" "$dir.h" . > gen.log 2>&1 )
  cp "$GEN/$dir"/*.h "$GEN/include/"
done

# per-library preprocessor flags (lib/make_qla_dirs:27-40) are applied in the
# compile step below from the library name carried in the third field.
CFLAGS="-std=gnu99 -O2 -fPIC -fopenmp -DQLA_RESTRICT=restrict -I$GEN/include -I$REF/include"
: > "$GEN/compile.list"
for dir in $COMPILE; do
  for src in "$GEN/$dir"/QLA_*.c; do
    b=$(basename "$src" .c)
    echo "$src|$GEN/obj/${dir}__$b.o|$dir" >> "$GEN/compile.list"
  done
done
for sub in cmath random; do
  for src in "$REF/lib/$sub"/*.c; do
    b=$(basename "$src" .c)
    echo "$src|$GEN/obj/${sub}__$b.o|$sub" >> "$GEN/compile.list"
  done
done

export CFLAGS
xargs -P "$JOBS" -n 1 -d '\n' sh -c '
  IFS="|"; set -- $1
  case $3 in
    qla_f|qla_f2|qla_f3|qla_fn) P="-DQLA_PrecisionInt=1" ;;
    qla_d|qla_d2|qla_d3|qla_dn) P="-DQLA_PrecisionInt=2" ;;
    *) P="" ;;
  esac
  case $3 in
    *2) C="-DQLA_Colors=2" ;;
    *3) C="-DQLA_Colors=3" ;;
    qla_fn|qla_dn|qla_dfn) C="-DQLA_Colors='"'"'N'"'"'" ;;
    *) C="" ;;
  esac
  IFS=" "
  gcc $CFLAGS $P ${C:+"$C"} -c "$1" -o "$2" || { echo "compile failed: $1" >&2; exit 255; }
' _ < "$GEN/compile.list"

# -Bsymbolic: calls between reference functions resolve inside this library even
# when a same-named product library is loaded into the same process.
rm -f "$GEN/libqla_ref_all.a"
( cd "$GEN/obj" && find . -name '*.o' | sort | xargs ar rcs "$GEN/libqla_ref_all.a" )
gcc -shared -fopenmp -Wl,-Bsymbolic -o "$OUT/libqla_ref.so.tmp" \
    -Wl,--whole-archive "$GEN/libqla_ref_all.a" -Wl,--no-whole-archive -lm
mv "$OUT/libqla_ref.so.tmp" "$OUT/libqla_ref.so"
# keep the generated headers (the checker's tests include none of them, but they
# document the exact prototypes) and drop the bulky generated sources and objects
rm -rf "$GEN/obj" "$GEN/libqla_ref_all.a"
for dir in $COMPILE $HDR_ONLY; do rm -f "$GEN/$dir"/QLA_*.c; done
copy_api_headers
echo "build_ref.sh: built $OUT/libqla_ref.so"

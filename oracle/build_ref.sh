#!/usr/bin/env bash
# Builds the reference's own projector (DiuYao/CT_Forward_Projection) from its
# sources under /root/reference into oracle/_ref/ctfp_ref, for use as a parity
# oracle and as the reference benchmark arm.  TEST INFRASTRUCTURE ONLY.
#
# The sources are GBK-encoded Windows/MSVC code: they are converted to UTF-8 and
# their backslash #include paths rewritten in a temporary directory outside the
# repository (deleted afterwards); nothing but the binary lands in oracle/_ref/.
# The closed InitFile.dll is not used: the project's own CInitFile
# (ct_forward_projection_b200/compat/ini) is compiled in its place.  MSVC CRT
# calls are mapped by oracle/ref_shim/ref_compat.h.  The reference's projector
# objects are automatic variables (ForwardProjection.cpp:94) whose destructors
# delete[] members the constructors never set (e.g. aDetResponse,
# CBCTForwardProj.h:99, in the multi-material and TestI0 paths), which aborts at
# exit after the outputs are written; the host objects are built with
# -ftrivial-auto-var-init=zero so those members start as null.  The
# computation is untouched.
set -euo pipefail
REF=${REF:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT=$(cd "$HERE/.." && pwd)
OUT="$HERE/_ref"
# without the sources (e.g. on a GPU box, which uses the binary built here)
# there is nothing to build
[ -d "$REF/Source" ] || { echo "reference sources not found at $REF; oracle/_ref not built" >&2; exit 0; }
BIN="$OUT/ctfp_ref"
# rebuild only when the recipe or the shims are newer than the binary
if [ -x "$BIN" ] && [ "$BIN" -nt "$HERE/build_ref.sh" ] && [ "$BIN" -nt "$HERE/ref_shim/ref_compat.h" ] \
   && [ "$BIN" -nt "$ROOT/ct_forward_projection_b200/compat/ini/InitFile.cpp" ]; then
  exit 0
fi
mkdir -p "$OUT"
TMP=$(mktemp -d /tmp/ctfp_ref_build.XXXXXX)
trap 'rm -rf "$TMP"' EXIT
mkdir -p "$TMP/Source/CUDAFun"
for f in "$REF"/Source/*.cpp "$REF"/Source/*.h "$REF"/Source/CUDAFun/*; do
  rel=${f#"$REF"/}
  # most files are GBK; the few already in UTF-8 (with a byte-order mark) are copied
  if ! iconv -f GBK -t UTF-8 "$f" > "$TMP/$rel" 2>/dev/null; then
    sed '1s/^\xEF\xBB\xBF//' "$f" > "$TMP/$rel"
  fi
  # backslash include paths (e.g. "..\DataType.h") -> forward slashes
  sed -i -E '/^[[:space:]]*#[[:space:]]*include/ s#\\#/#g' "$TMP/$rel"
done
NVCC=${NVCC:-nvcc}
ARCH="-gencode arch=compute_100a,code=sm_100a"
INC="-I $TMP/Source -I $ROOT/ct_forward_projection_b200/compat/ini -I $HERE/ref_shim"
objs=()
for f in "$TMP"/Source/*.cpp; do
  o="$TMP/$(basename "$f").o"
  g++ -std=c++17 -O2 -w -ftrivial-auto-var-init=zero -include "$HERE/ref_shim/ref_compat.h" $INC \
    -I /usr/local/cuda/include -c "$f" -o "$o"
  objs+=("$o")
done
g++ -std=c++17 -O2 -w -I "$ROOT/ct_forward_projection_b200/compat/ini" \
  -c "$ROOT/ct_forward_projection_b200/compat/ini/InitFile.cpp" -o "$TMP/InitFile.o"
"$NVCC" $ARCH -O3 -std=c++17 -w $INC -c "$TMP/Source/CUDAFun/CBCTPolyProjGPU.cu" -o "$TMP/gpu.o"
"$NVCC" $ARCH -o "$BIN" "${objs[@]}" "$TMP/InitFile.o" "$TMP/gpu.o" -lcudart
echo "built $BIN"

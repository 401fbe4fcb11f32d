#!/usr/bin/env bash
# Builds the reference's own code from its sources where they lie under the
# reference tree (read-only; nothing is copied), outputs into oracle/_ref/:
#
#   _ref/libref_ttpc.so    the reference's TTPC channel functions
#                          (GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/AllModels.cu)
#                          compiled for the host with __device__ defined away,
#                          plus oracle/ref_channels_wrap.cpp (C entry points)
#   _ref/libref_mainen.so  the same for Figures/FigureS4_mainen/CParsed/AllModels.cu
#   _ref/neuroGPU_ttpc512  the reference's fused GPU simulator, unmodified,
#                          for sm_100a (its own Makefile uses -dc -O3 per file,
#                          GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/Makefile:154)
#   _ref/ref_atof          the reference's AllParams value parser (Util.cu,
#                          myatof) behind oracle/ref_atof_main.cpp (stdin
#                          tokens -> float bits)
#
# Test infrastructure only.  _ref/ is git-ignored but travels with the repo
# snapshot, so the GPU box uses these prebuilt files.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${NGPU_REFERENCE_DIR:-/root/reference}"
OUT="$HERE/_ref"
U="$REF/GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src"
MN="$REF/Figures/FigureS4_mainen/CParsed"
if [ ! -d "$U" ]; then
    echo "build_ref.sh: reference tree not found at $REF; keeping prebuilt $OUT" >&2
    exit 0
fi
CXX=/usr/bin/g++
[ -x "$CXX" ] || CXX=g++
mkdir -p "$OUT/shim"
# empty stand-ins for the CUDA headers the generated channel files include
: > "$OUT/shim/cuda_runtime.h"
: > "$OUT/shim/device_launch_parameters.h"
HOSTFLAGS=(-O2 -fPIC -fpermissive -w -D__device__= -I"$OUT/shim")

"$CXX" "${HOSTFLAGS[@]}" -I"$U" -x c++ -c "$U/AllModels.cu" -o "$OUT/ttpc_models.o"
"$CXX" -O2 -fPIC -DREF_TTPC -c "$HERE/ref_channels_wrap.cpp" -o "$OUT/ttpc_wrap.o"
"$CXX" -shared -o "$OUT/libref_ttpc.so" "$OUT/ttpc_models.o" "$OUT/ttpc_wrap.o"

# the Mainen header includes Util.h, which only the canonical src/ directory holds
"$CXX" "${HOSTFLAGS[@]}" -I"$MN" -I"$U" -x c++ -c "$MN/AllModels.cu" -o "$OUT/mainen_models.o"
"$CXX" -O2 -fPIC -DREF_MAINEN -c "$HERE/ref_channels_wrap.cpp" -o "$OUT/mainen_wrap.o"
"$CXX" -shared -o "$OUT/libref_mainen.so" "$OUT/mainen_models.o" "$OUT/mainen_wrap.o"

if command -v nvcc >/dev/null 2>&1; then
    GEN=(-gencode arch=compute_100a,code=sm_100a)
    objs=()
    for f in AllModels CudaStuff MainC Util kernel; do
        nvcc -m64 -dc -O3 -w "${GEN[@]}" -I"$U" -o "$OUT/ref_$f.o" -c "$U/$f.cu"
        objs+=("$OUT/ref_$f.o")
    done
    nvcc "${GEN[@]}" -o "$OUT/neuroGPU_ttpc512" "${objs[@]}"
    nvcc "${GEN[@]}" -O2 -c "$HERE/ref_atof_main.cpp" -o "$OUT/atof_main.o"
    nvcc "${GEN[@]}" -o "$OUT/ref_atof" "$OUT/atof_main.o" "$OUT/ref_Util.o"
fi
echo "build_ref.sh: built into $OUT"

#!/bin/bash
# build_ref.sh -- builds the reference's own CPU path (RIKEN-RCCS/hpl-ai,
# the x86 build of its Makefile: main.cpp, lazy_init_omp.cpp, otf_gemv.cpp,
# kernels/avx2.cpp, kernels/generic.cpp, higham_mat_impl.cpp,
# back_buffer.cpp) from the sources where they lie, without running its
# build system, into oracle/_ref/:
#
#   ref_driver.out         linked with the OpenBLAS that ships in this image
#                          (called, not inspected): the CPU baseline
#   ref_driver_netlib.out  linked with tmpi/netlib_blas.cpp (netlib loop
#                          order, fused multiply-adds): a deterministic LU for
#                          pinning the oracle bit for bit
#   libref_higham.so       the reference's higham_mat_impl.cpp alone, so that
#                          the fixture script can record the alpha and beta
#                          of Higham's matrix (--highammat) it computes
#
# MPI is replaced by the thread-rank runtime in tmpi/ (TMPI_NP ranks as
# threads of one process); main.cpp is compiled through tmpi/ref_xdump.cpp so
# that TMPI_XDUMP=<file> receives the solution vector.  Compiler flags are
# the reference Makefile's, with -march=x86-64-v3 (AVX2, FMA, F16C: the
# reference's x86 FP16 path) instead of -march=native so that the binaries
# also run on other x86 hosts, and -DTIMER_SILENT (the timers' statics are
# shared by the rank threads).
#
# TEST INFRASTRUCTURE ONLY: used by tests/, bench.py's cpu_baseline leg and
# its --impl reference arm.  Outputs are git-ignored.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${HPLAI_REFERENCE:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -f "$REF/main.cpp" ]; then
	echo "build_ref.sh: no reference tree at $REF; nothing built" >&2
	exit 0
fi
BLASDIR="${HPLAI_OPENBLAS_DIR:-$(python3 -c 'import os, cv2; print(os.path.join(os.path.dirname(os.path.dirname(cv2.__file__)), "opencv_python_headless.libs"))' 2>/dev/null || true)}"
OPENBLAS="$(ls "$BLASDIR"/libopenblas*.so 2>/dev/null | head -1 || true)"

CXX="${HPLAI_REF_CXX:-g++}"   # not $CXX: an image-level wrapper there lacks libgomp
FLAGS=(-W -Wall -Wextra -fopenmp -std=c++17 -O2 -march=x86-64-v3 -DEXTERNAL_CONV -DOTF_GEMV_OPTIMIZED -DTIMER_SILENT
	-w -I"$HERE/tmpi" -I"$REF")
OBJ="$OUT/obj"
mkdir -p "$OBJ"

stamp="$OUT/.stamp"
newest_src=$(find "$REF" "$HERE/tmpi" "$HERE/build_ref.sh" -newer "$stamp" -type f 2>/dev/null | head -1 || true)
if [ -f "$stamp" ] && [ -z "$newest_src" ] && [ -x "$OUT/ref_driver_netlib.out" ] && [ -f "$OUT/libref_higham.so" ]; then
	exit 0
fi

"$CXX" "${FLAGS[@]}" -Dmain=hplai_rank_main -c "$HERE/tmpi/ref_xdump.cpp" -o "$OBJ/main.o"
for src in lazy_init_omp.cpp otf_gemv.cpp kernels/avx2.cpp kernels/generic.cpp higham_mat_impl.cpp back_buffer.cpp; do
	"$CXX" "${FLAGS[@]}" -c "$REF/$src" -o "$OBJ/$(basename "${src%.cpp}").o" &
done
"$CXX" -std=c++17 -O2 -W -Wall -c "$HERE/tmpi/tmpi.cpp" -o "$OBJ/tmpi.o" &
"$CXX" -std=c++17 -O2 -march=x86-64-v3 -ffp-contract=off -W -Wall -c "$HERE/tmpi/netlib_blas.cpp" \
	-o "$OBJ/netlib_blas.o" &
wait
OBJS=("$OBJ/main.o" "$OBJ/lazy_init_omp.o" "$OBJ/otf_gemv.o" "$OBJ/avx2.o" "$OBJ/generic.o" "$OBJ/higham_mat_impl.o"
	"$OBJ/back_buffer.o" "$OBJ/tmpi.o")
"$CXX" -fopenmp -o "$OUT/ref_driver_netlib.out" "${OBJS[@]}" "$OBJ/netlib_blas.o" -lm -lpthread
if [ -n "$OPENBLAS" ]; then
	"$CXX" -fopenmp -o "$OUT/ref_driver.out" "${OBJS[@]}" "$OPENBLAS" -Wl,--disable-new-dtags,-rpath,"$BLASDIR" -lm -lpthread
else
	echo "build_ref.sh: no OpenBLAS found; the CPU baseline uses the netlib-order build" >&2
	cp "$OUT/ref_driver_netlib.out" "$OUT/ref_driver.out"
fi
"$CXX" -shared -o "$OUT/libref_higham.so" "$OBJ/higham_mat_impl.o" -lm
touch "$stamp"
echo "build_ref.sh: built $OUT/ref_driver.out and $OUT/ref_driver_netlib.out"

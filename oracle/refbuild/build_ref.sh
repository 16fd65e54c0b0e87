#!/usr/bin/env bash
# Builds the reference solver's own C++ sources (read in place under REF_DIR)
# against the Eigen API stand-in in shim/, together with harness.cpp, into
# oracle/_ref/.  Test infrastructure: the CPU oracle and CPU baseline only.
#
#   ref_f32       as shipped (float), the reference's flags (-O3 -mavx2 -mfma
#                 -fopenmp, build.bat:36): the timed CPU baseline
#   ref_f32_pin   float, -ffp-contract=off: bit-exact pin of the C restatement
#   ref_f64_pin   the same sources re-typed to double by a textual substitution
#                 (float->double, MatrixXf->MatrixXd, VectorXf->VectorXd, 'f'
#                 literal suffixes dropped), -ffp-contract=off: the FP64 oracle
#   ref_dropin    the shipped sources with Utilities/iterations.cpp replaced by
#                 the GPU drop-in (coldplate-solver_b200/dropin/), linked
#                 against libcoldplate.so: the reference's own outer loop
#                 running on the library
#
# The re-typed copy lives only in a temporary directory; nothing from REF_DIR
# is written into the repository.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
if [ -z "${REF_DIR:-}" ]; then
    echo "build_ref.sh: set REF_DIR to the reference checkout (the directory holding SIMPLE.cpp)" >&2
    exit 2
fi
OUT="${OUT:-$HERE/../_ref}"
CXX="${CXX:-g++}"
# the image's g++ driver does not search the system gcc directory for
# libgomp.spec; point it there explicitly when that directory exists
GOMP_B=()
[ -f /usr/lib/gcc/x86_64-linux-gnu/13/libgomp.spec ] && GOMP_B=(-B/usr/lib/gcc/x86_64-linux-gnu/13/)
if [ ! -f "$REF_DIR/SIMPLE.cpp" ]; then
    echo "build_ref.sh: no reference sources at $REF_DIR" >&2
    exit 3
fi
mkdir -p "$OUT"
TMP="$(mktemp -d /tmp/cp_refbuild.XXXXXX)"
trap 'rm -rf "$TMP"' EXIT

SRCS_REL="SIMPLE.cpp $(cd "$REF_DIR" && ls Utilities/*.cpp Utilities/solvers/cpu/*.cpp | tr '\n' ' ')"

build() {  # build <name> <srcroot> <real> <flags...>
    local name="$1" root="$2" real="$3"; shift 3
    local obj="$TMP/obj_$name"
    mkdir -p "$obj"
    local objs=()
    for s in $SRCS_REL; do
        local o="$obj/$(echo "$s" | tr '/' '_').o"
        local extra=()
        [ "$s" = "SIMPLE.cpp" ] && extra=(-Dmain=ref_main_unused)
        "$CXX" "${GOMP_B[@]}" -std=c++17 "$@" -fopenmp -w "${extra[@]}" -I"$HERE/shim" -I"$root" -I"$root/Utilities" \
            -c "$root/$s" -o "$o" &
        objs+=("$o")
    done
    "$CXX" "${GOMP_B[@]}" -std=c++17 "$@" -fopenmp -w -DREF_REAL="$real" -I"$HERE/shim" -I"$root" -I"$root/Utilities" \
        -c "$HERE/harness.cpp" -o "$obj/harness.o" &
    wait
    "$CXX" "${GOMP_B[@]}" "$@" -fopenmp "${objs[@]}" "$obj/harness.o" -o "$OUT/$name"
    echo "built $OUT/$name"
}

# float, as shipped
build ref_f32 "$REF_DIR" float -O3 -mavx2 -mfma -ftree-vectorize
build ref_f32_pin "$REF_DIR" float -O2 -ffp-contract=off

# double re-typed copy
SRC64="$TMP/src64"
mkdir -p "$SRC64"
(cd "$REF_DIR" && find . -maxdepth 1 -name 'SIMPLE.*' -print0; \
 cd "$REF_DIR" && find Utilities -maxdepth 1 \( -name '*.cpp' -o -name '*.h' \) -print0; \
 cd "$REF_DIR" && find Utilities/solvers -name '*.cpp' -print0 -o -name '*.h' -print0) \
 | (cd "$REF_DIR" && xargs -0 cp --parents -t "$SRC64")
find "$SRC64" \( -name '*.cpp' -o -name '*.h' \) -print0 | xargs -0 sed -i -E \
    -e 's/\bfloat\b/double/g' \
    -e 's/MatrixXf/MatrixXd/g' -e 's/VectorXf/VectorXd/g' \
    -e 's/\b([0-9][0-9]*\.?[0-9]*([eE][-+]?[0-9]+)?)[fF]\b/\1/g'
build ref_f64_pin "$SRC64" double -O2 -ffp-contract=off

# the reference's own outer loop (SIMPLE::runIterations) over the GPU library:
# its sources as shipped except Utilities/iterations.cpp, which is replaced by
# the drop-in coldplate-solver_b200/dropin/iterations_gpu.cpp, linked against
# coldplate-solver_b200/libcoldplate.so (found through a relative rpath)
ROOT="$(cd "$HERE/../.." && pwd)"
LIB="$ROOT/coldplate-solver_b200/libcoldplate.so"
if [ -f "$LIB" ]; then
    obj="$TMP/obj_dropin"
    mkdir -p "$obj"
    objs=()
    for s in $SRCS_REL; do
        [ "$s" = "Utilities/iterations.cpp" ] && continue
        o="$obj/$(echo "$s" | tr '/' '_').o"
        extra=()
        [ "$s" = "SIMPLE.cpp" ] && extra=(-Dmain=ref_main_unused)
        "$CXX" "${GOMP_B[@]}" -std=c++17 -O2 -fopenmp -w "${extra[@]}" -I"$HERE/shim" -I"$REF_DIR" \
            -I"$REF_DIR/Utilities" -c "$REF_DIR/$s" -o "$o" &
        objs+=("$o")
    done
    "$CXX" "${GOMP_B[@]}" -std=c++17 -O2 -fopenmp -Wall -I"$HERE/shim" -I"$REF_DIR" -I"$REF_DIR/Utilities" \
        -I"$ROOT/include" -c "$ROOT/coldplate-solver_b200/dropin/iterations_gpu.cpp" -o "$obj/iterations_gpu.o" &
    "$CXX" "${GOMP_B[@]}" -std=c++17 -O2 -fopenmp -w -DREF_REAL=float -I"$HERE/shim" -I"$REF_DIR" \
        -I"$REF_DIR/Utilities" -c "$HERE/harness.cpp" -o "$obj/harness.o" &
    wait
    "$CXX" "${GOMP_B[@]}" -fopenmp "${objs[@]}" "$obj/iterations_gpu.o" "$obj/harness.o" "$LIB" \
        -Wl,-rpath,'$ORIGIN/../../coldplate-solver_b200' -o "$OUT/ref_dropin"
    echo "built $OUT/ref_dropin"
fi

# the thermal solver (ThermalSolver/thermal_solver.cpp, one translation unit)
# against the AMGCL API stand-in in shim/amgcl: the reference's own assembly,
# solved by the stand-in to a tight tolerance; -ffp-contract=off pins it
if [ -f "$REF_DIR/ThermalSolver/thermal_solver.cpp" ]; then
    $CXX -std=c++17 -O2 -ffp-contract=off -fopenmp "${GOMP_B[@]}" -I"$HERE/shim" -I"$REF_DIR/ThermalSolver" \
        "$REF_DIR/ThermalSolver/thermal_solver.cpp" -o "$OUT/thermal_ref_pin"
    echo "built $OUT/thermal_ref_pin"
fi

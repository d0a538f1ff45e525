#!/usr/bin/env bash
# Build recipe for oracle/_ref/ (libv2rdm_ref.so, libdoci_ref.so, libfocas_ref.so):
# hilbert's OWN constraint-map,
# index-table, sizing, b/c and guess code compiled where it lies in the
# reference tree, against the test-only Psi4 stand-ins in oracle/ref_shim/.
#
# The library is test infrastructure (the bit-exact checker for the B200 maps
# and the timed CPU baseline of the reference path); the product never links it.
#
# Inputs : $V2B_REFERENCE (default /root/reference), read-only.
# Outputs: oracle/_ref/ only (git-ignored; travels with the working tree).
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
ref="${V2B_REFERENCE:-/root/reference}"
src="$ref/src/v2rdm_casscf"
out="$here/_ref"
if [ ! -f "$src/v2rdm_solver.cc" ]; then
  echo "build_ref.sh: reference sources not found under $ref" >&2
  exit 2
fi
mkdir -p "$out"

# v2rdm_solver.cc as a whole needs most of Psi4; the functions the map path
# needs only touch plain members.  Pull those definitions out by name (start:
# the definition line at column 0, end: the first closing brace at column 0)
# into a generated translation unit under _ref/.
extract() {  # $1 = file, $2... = member function names
  extract_class v2RDMSolver "$@"
}
extract_class() {  # $1 = class, $2 = file, $3... = member function names
  local cls="$1" f="$2"; shift 2
  for name in "$@"; do
    awk -v pat="${cls}::${name}\\\\(" '
      !on && $0 ~ /^[A-Za-z]/ && $0 ~ pat { on = 1 }
      on { print }
      on && $0 ~ /^}/ { on = 0; print "" }
    ' "$f"
  done
}
gen="$out/v2rdm_solver_extract.cc"
{
  echo '// generated by oracle/build_ref.sh from the reference tree; do not edit'
  echo '#include <psi4/psi4-dec.h>'
  echo '#include <psi4/libqt/qt.h>'
  echo '#include "v2rdm_solver.h"'
  echo 'using namespace psi;'
  echo 'namespace hilbert {'
  extract "$src/v2rdm_solver.cc" SymmetryPair TotalSym set_constraints \
      determine_n_primal determine_n_dual set_primal_offsets BuildConstraints \
      Guess bpsdp_Au bpsdp_ATu PackSpatialDensity
  extract "$src/oei.cc" GetOEI_external GetOEI_hubbard
  extract "$src/write_tpdm.cc" WriteTPDM WriteTPDMSpinFree
  extract "$src/write_tpdm_iwl.cc" WriteTPDM_IWL
  echo '}'
} > "$gen"

for name in SymmetryPair TotalSym set_constraints determine_n_primal determine_n_dual \
            set_primal_offsets BuildConstraints Guess bpsdp_Au bpsdp_ATu PackSpatialDensity \
            GetOEI_external GetOEI_hubbard WriteTPDM WriteTPDMSpinFree WriteTPDM_IWL; do
  grep -q "v2RDMSolver::${name}(" "$gen" || { echo "build_ref.sh: could not extract ${name}" >&2; exit 3; }
done

# -ffp-contract=off keeps a*b+c as two roundings, as in a plain x86-64 build.
# -fopenmp: the reference parallelises its maps with OpenMP (q2.cc, g2.cc,
# t2.cc, ...); every output element is still written by one thread in the
# reference's order, so results stay bit-identical.  x86-64-v3 (AVX2, FMA)
# rather than -march=native: the library is built here and also runs on the
# GPU host, whose CPU model may differ.
CXX="${CXX:-g++}"
# some images wrap g++ without the path to libgomp.spec: point -B at it
OMPB=()
if ! echo 'int main(){return 0;}' | "$CXX" -x c++ -fopenmp - -o /dev/null 2>/dev/null; then
  spec="$(ls /usr/lib/gcc/x86_64-linux-gnu/*/libgomp.spec 2>/dev/null | tail -1)"
  [ -n "$spec" ] || { echo "build_ref.sh: $CXX cannot build OpenMP code" >&2; exit 4; }
  OMPB=(-B"$(dirname "$spec")/")
fi
FLAGS=(-std=c++17 -O3 -march=x86-64-v3 -fopenmp "${OMPB[@]}" -fPIC -ffp-contract=off -w
       -I"$here/ref_shim" -I"$src" -I"$ref/src")
units=(basis d2 spin q2 g2 t1 t2 d3 d4 e3 f3 q3 tei write_opdm write_3pdm)
objs=()
for u in "${units[@]}"; do
  "$CXX" "${FLAGS[@]}" -c "$src/$u.cc" -o "$out/$u.o"
  objs+=("$out/$u.o")
done
"$CXX" "${FLAGS[@]}" -c "$gen" -o "$out/v2rdm_solver_extract.o"
"$CXX" "${FLAGS[@]}" -c "$here/ref_harness.cc" -o "$out/ref_harness.o"
"$CXX" -shared -fopenmp "${OMPB[@]}" -Wl,--no-undefined -o "$out/libv2rdm_ref.so" "${objs[@]}" \
    "$out/v2rdm_solver_extract.o" "$out/ref_harness.o"
echo "built $out/libv2rdm_ref.so"

# v2RDM-DOCI: the map files of src/v2rdm_doci, plus BuildConstraints, Guess,
# bpsdp_Au / bpsdp_ATu and SymmetryPair from v2rdm_doci_solver.cc, plus the
# part of common_init that turns POSITIVITY / CONSTRAIN_D3 into sizes,
# offsets and the block list (from "pick conditions" up to the convergence
# thresholds), which reads nothing from the wavefunction.
dsrc="$ref/src/v2rdm_doci"
dgen="$out/doci_solver_extract.cc"
{
  echo '// generated by oracle/build_ref.sh from the reference tree; do not edit'
  echo '#include <psi4/psi4-dec.h>'
  echo '#include <psi4/libqt/qt.h>'
  echo '#include "v2rdm_doci_solver.h"'
  echo 'using namespace psi;'
  echo 'namespace hilbert {'
  extract_class v2RDM_DOCISolver "$dsrc/v2rdm_doci_solver.cc" SymmetryPair TotalSym \
      BuildConstraints Guess bpsdp_Au bpsdp_ATu PackSpatialDensity
  echo 'void v2RDM_DOCISolver::common_init() {'
  awk '/pick conditions\.  default is dqg/ { on = 1 }
       /v2rdm sdp convergence thresholds/ { on = 0 }
       on { print }' "$dsrc/v2rdm_doci_solver.cc"
  echo '}'
  echo '}'
} > "$dgen"
for name in SymmetryPair TotalSym BuildConstraints Guess bpsdp_Au bpsdp_ATu PackSpatialDensity; do
  grep -q "v2RDM_DOCISolver::${name}(" "$dgen" || { echo "build_ref.sh: could not extract DOCI ${name}" >&2; exit 3; }
done
grep -q "dimensions_.push_back" "$dgen" || { echo "build_ref.sh: could not extract the DOCI sizing" >&2; exit 3; }
DFLAGS=(-std=c++17 -O3 -march=x86-64-v3 -fopenmp "${OMPB[@]}" -fPIC -ffp-contract=off -w
        -I"$here/ref_shim" -I"$dsrc" -I"$ref/src")
dobjs=()
for u in basis d2 q2 g2 d3 t1 t2 tei write_tpdm; do
  "$CXX" "${DFLAGS[@]}" -c "$dsrc/$u.cc" -o "$out/doci_$u.o"
  dobjs+=("$out/doci_$u.o")
done
"$CXX" "${DFLAGS[@]}" -c "$dgen" -o "$out/doci_solver_extract.o"
"$CXX" "${DFLAGS[@]}" -c "$here/doci_ref_harness.cc" -o "$out/doci_ref_harness.o"
"$CXX" -shared -fopenmp "${OMPB[@]}" -Wl,--no-undefined -o "$out/libdoci_ref.so" "${dobjs[@]}" \
    "$out/doci_solver_extract.o" "$out/doci_ref_harness.o"
echo "built $out/libdoci_ref.so"

# focas's C++ orbital optimizer (the DF path v2RDM-CASSCF calls,
# src/focas/C_files/*.cc), compiled from the reference sources.  Its class
# header is copied into _ref/focas/ with two lines added -- a constructor
# that takes the orbital spaces directly (the real one reads them from a
# Psi4 wavefunction) and a friend harness -- and the C_files are copied
# beside it so that their "../orbital_optimizer.h" finds that copy.
# BLAS / LAPACK: numpy's ILP64 OpenBLAS (hilbert's misc/blas.h passes 64-bit
# integers), reached through the forwarding wrappers in focas_harness.cc.
fsrc="$ref/src/focas"
fout="$out/focas"
mkdir -p "$fout/C_files"
awk '/^class OrbitalOptimizer \{/ { print "struct FocasHarnessSetup;"; print "struct FocasHarness;"; print; print "  friend struct FocasHarness;"; next }
     /OrbitalOptimizer\(std::shared_ptr<Wavefunction> reference_wavefunction, Options & options\);/ { print; print "    explicit OrbitalOptimizer(const FocasHarnessSetup &setup);"; next }
     { print }' "$fsrc/orbital_optimizer.h" > "$fout/orbital_optimizer.h"
grep -q "FocasHarnessSetup &setup" "$fout/orbital_optimizer.h" || { echo "build_ref.sh: could not patch orbital_optimizer.h" >&2; exit 3; }
cp "$fsrc"/C_files/*.cc "$fout/C_files/"
openblas="$(ls "$(python3 -c 'import numpy, os; print(os.path.dirname(numpy.__file__))')".libs/libscipy_openblas64_*.so 2>/dev/null | head -1)"
[ -n "$openblas" ] || { echo "build_ref.sh: numpy's OpenBLAS not found" >&2; exit 4; }
FFLAGS=(-std=c++17 -O2 -fPIC -ffp-contract=off -w -I"$here/ref_shim" -I"$fout" -I"$ref/src")
fobjs=()
for f in "$fout"/C_files/*.cc; do
  o="$fout/$(basename "$f" .cc).o"
  "$CXX" "${FFLAGS[@]}" -c "$f" -o "$o"
  fobjs+=("$o")
done
"$CXX" "${FFLAGS[@]}" -c "$here/focas_harness.cc" -o "$fout/focas_harness.o"
"$CXX" -shared -Wl,--no-undefined -o "$out/libfocas_ref.so" "${fobjs[@]}" "$fout/focas_harness.o" \
    "$openblas" -Wl,-rpath,"$(dirname "$openblas")"
echo "built $out/libfocas_ref.so"

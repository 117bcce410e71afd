#!/usr/bin/env bash
# Compile the reference's own C sources for this path, where they lie in the reference
# tree, into oracle/_ref/ (git-ignored; travels with the snapshot).  Test infrastructure:
#   schur_uq.so / schur_u.so / arraymul.so / schur_uq_adjoint.so / schur_u_adjoint.so :
#       kernel/schur_uq.c, kernel/schur_u.c, kernel/arraymul.c, kernel/schur_uq_adjoint.c,
#       kernel/schur_u_adjoint.c + the MEX emulation in oracle/refshim, against numpy's ILP64
#       OpenBLAS (MATLAB's BLAS ABI uses ptrdiff_t integers);
#   libref_ns.so : application/FM/ns/{flux,fhat}_ns{2,3}d.c and
#       application/FM/euler/{flux,fhat}_euler{2,3}d.c (generated point kernels);
#   libref_fbou_ns.so / libref_fbou_euler.so : application/FM/{ns,euler}/fluxes.c with the
#       generated boundary kernels fbou_{ns,euler}{2,3}d.c and the Roe matrices of
#       application/FM/getan.c (C++: they use new/delete and iostream), behind two extern "C"
#       wrappers ref_fbou and ref_getan.  ref_fbou calls fbou_{ns,euler}{2,3}d directly with
#       their own argument order (..., ng, nc, nch, ...): the dispatchers fbou_ns / fbou_euler
#       of fluxes.c name the two counts the other way round.
# Usage: oracle/build_ref.sh REFERENCE_ROOT   (or HDG_REFERENCE=REFERENCE_ROOT oracle/build_ref.sh)
set -euo pipefail
REF=${1:-${HDG_REFERENCE:-}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
[ -n "$REF" ] && [ -d "$REF/kernel" ] || { echo "reference tree not given or not found (${REF:-unset}); skipping"; exit 0; }
mkdir -p "$OUT"
OB=$(python -c 'import numpy, glob, os; print(glob.glob(os.path.join(os.path.dirname(numpy.__file__), os.pardir, "numpy.libs", "libscipy_openblas64_*.so"))[0])')
OBDIR=$(dirname "$OB"); OBNAME=$(basename "$OB")
for f in schur_uq schur_u arraymul schur_uq_adjoint schur_u_adjoint; do
  gcc -O2 -fPIC -shared -w -I"$HERE/refshim" -o "$OUT/$f.so" "$REF/kernel/$f.c" "$HERE/refshim/mexharness.c" \
      "$OB" -Wl,-rpath,"$OBDIR" -lm
done
TMP=$(mktemp -d)
cat > "$TMP/ns.c" <<CEOF
#include <math.h>
#include "$REF/application/FM/ns/flux_ns2d.c"
#include "$REF/application/FM/ns/flux_ns3d.c"
#include "$REF/application/FM/ns/fhat_ns2d.c"
#include "$REF/application/FM/ns/fhat_ns3d.c"
#include "$REF/application/FM/euler/flux_euler2d.c"
#include "$REF/application/FM/euler/flux_euler3d.c"
#include "$REF/application/FM/euler/fhat_euler2d.c"
#include "$REF/application/FM/euler/fhat_euler3d.c"
CEOF
gcc -O2 -fPIC -shared -w -std=gnu99 -o "$OUT/libref_ns.so" "$TMP/ns.c" -lm
for fam in ns euler; do
  {
    echo '#include <cmath>'
    echo '#include <cstdio>'
    echo '#include <cstdlib>'
    echo '#include <iostream>'
    echo 'using namespace std;'
    [ "$fam" = euler ] && echo "#include \"$REF/application/FM/getan.c\""
    echo "#include \"$REF/application/FM/$fam/fluxes.c\""
    echo 'extern "C" void ref_fbou(double *fh, double *fh_u, double *fh_uh, double *pg, double *udg, double *uhg,'
    echo '                         double *nl, double *ui, double *param, double time, int ib, int ng, int nch,'
    echo '                         int nc, int nd, int ncd) {'
    echo "    if (nd == 2) fbou_${fam}2d(fh, fh_u, fh_uh, pg, udg, uhg, nl, ui, param, time, ib, ng, nc, nch, nd, ncd);"
    echo "    else fbou_${fam}3d(fh, fh_u, fh_uh, pg, udg, uhg, nl, ui, param, time, ib, ng, nc, nch, nd, ncd);"
    echo '}'
    echo 'extern "C" void ref_getan(double *An, double *Anm, double *uh, double *nl, double *param, int absflag,'
    echo '                          int ng, int nch, int nd) {'
    echo '    getan(An, Anm, uh, nl, param, absflag, ng, nch, nd);'
    echo '}'
  } > "$TMP/fbou_$fam.cpp"
  g++ -O2 -fPIC -shared -w -o "$OUT/libref_fbou_$fam.so" "$TMP/fbou_$fam.cpp" -lm
done
rm -rf "$TMP"
echo "built: $(ls "$OUT")"

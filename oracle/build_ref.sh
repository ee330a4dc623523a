#!/bin/sh
# Compiles the reference's own PETSc-free functions, from the lines where
# they lie in the reference tree, into oracle/_ref/liblgh_ref_pure.so:
#   include/lgpsf_hessian/impl/glr_common_impl.h:32-73  lgh_randn, lgh_randn_at
#   include/lgpsf_hessian/impl/zsolve_impl.h:93-102     lgh_zs_cheb_count
# Only two typedefs and three math macros are supplied around them; the
# generated translation unit stays under _ref/ (git-ignored).  When the
# reference tree is absent (the GPU host) nothing is built and the committed
# golden fixtures made from this library are used instead.
#
# The reference tree is read from $LGH_REFERENCE_ROOT.  Unset, it defaults
# to /root/reference, the read-only mount of the reference project in the
# container where the fixtures were generated; set it to build elsewhere.
set -e
REF=${LGH_REFERENCE_ROOT:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
G="$REF/include/lgpsf_hessian/impl/glr_common_impl.h"
Z="$REF/include/lgpsf_hessian/impl/zsolve_impl.h"
if [ ! -f "$G" ] || [ ! -f "$Z" ]; then
  echo "build_ref.sh: reference tree not found at $REF; skipped"
  exit 0
fi
mkdir -p "$OUT"
{
  echo '#include <math.h>'
  echo 'typedef long PetscInt; typedef double PetscReal;'
  echo '#define PetscSqrtReal(x) sqrt(x)'
  echo '#define PetscCeilReal(x) ceil(x)'
  echo '#define PetscLogReal(x) log(x)'
  sed -n '32,73p' "$G"
  sed -n '93,102p' "$Z"
  echo 'double ref_randn_at (unsigned long s, long i, long j) { return lgh_randn_at (s, i, j); }'
  echo 'long ref_cheb_count (double a, double b, double t) { return (long) lgh_zs_cheb_count (a, b, t); }'
} > "$OUT/ref_pure.c"
gcc -O2 -shared -fPIC -o "$OUT/liblgh_ref_pure.so" "$OUT/ref_pure.c" -lm
echo "build_ref.sh: built $OUT/liblgh_ref_pure.so"

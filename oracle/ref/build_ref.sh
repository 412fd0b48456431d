#!/usr/bin/env bash
# Builds the reference KORAL path into a shared library for the parity
# oracle.  Test infrastructure.
#
# The reference sources are compiled where they lie (a read-only tree given
# by KORAL_REF_DIR, or else by the one-line file reference_tree beside this
# script); nothing is copied.  Problem
# selection is done with the reference's own plug-in mechanism: the
# directory oracle/ref/problems/<PROBLEM> holds a problem.h selector plus the
# plug-in files, and is put in front of the quote-include search path with
# -I- so that ko.h picks it up instead of the reference's hard-wired
# problem.h.  GSL is replaced by the declaration-only stand-in in
# oracle/ref/gsl_shim (no GSL arithmetic is on the path).
#
# Translation units left out: ko.c (main() and the time loop, whose RK2 and
# RK2IMEX bodies harness.c reproduces by calling the same operators; ko.c
# also calls count_entropy/copy_entropycount, which no reference file
# defines), silo.c (Silo writer, removed by -DNOSILO anyway) and the
# stand-alone post-processing mains (ana.c, anarel.c, avg.c, phiavg.c,
# thsli.c).
#
# usage: build_ref.sh PROBLEM OUTLIB [extra cpp flags, e.g. -DTNX=32 -DTNY=32]
#        set KORAL_REF_OPENMP=1 for an OpenMP build (CPU timing baseline).
set -euo pipefail
PROBLEM="$1"; OUTLIB="$2"; shift 2
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${KORAL_REF_DIR:-$(head -n 1 "$HERE/reference_tree")}"
PROBDIR="$HERE/problems/$PROBLEM"
[ -d "$REF" ] || { echo "reference tree $REF not present" >&2; exit 3; }
[ -f "$PROBDIR/problem.h" ] || { echo "no plug-in $PROBDIR" >&2; exit 2; }

OUTDIR="$(dirname "$OUTLIB")"
OBJDIR="$OUTLIB.objs"
mkdir -p "$OUTDIR" "$OBJDIR"

CFLAGS=(-O3 -fPIC -fcommon -ffp-contract=off -fno-fast-math -DNOSILO -w)
if [ "${KORAL_REF_OPENMP:-0}" = "1" ]; then CFLAGS+=(-fopenmp); fi
INC=(-I "$PROBDIR" -I- -I "$HERE/gsl_shim" -I "$REF")

SRCS=(finite.c frames.c magn.c metric.c misc.c mpi.c mstep.c p2u.c physics.c
      postproc.c problem.c rad.c relele.c u2p.c u2prad.c fileop.c zeroshort.c
      zsolve_quartic.c)
OBJS=()
PIDS=()
for s in "${SRCS[@]}"; do
  o="$OBJDIR/${s%.c}.o"
  gcc "${CFLAGS[@]}" "$@" "${INC[@]}" -c "$REF/$s" -o "$o" 2> "$o.log" &
  PIDS+=($!)
  OBJS+=("$o")
done
gcc "${CFLAGS[@]}" "$@" "${INC[@]}" -c "$HERE/harness.c" -o "$OBJDIR/harness.o" 2> "$OBJDIR/harness.o.log" &
PIDS+=($!)
gcc -O2 -fPIC -I "$HERE/gsl_shim" -c "$HERE/gsl_shim/gsl_shim.c" -o "$OBJDIR/gsl_shim.o" &
PIDS+=($!)
FAIL=0
for pid in "${PIDS[@]}"; do wait "$pid" || FAIL=1; done
if [ "$FAIL" = 1 ]; then grep -h -v "obsolete option '-I-'" "$OBJDIR"/*.log >&2; exit 1; fi
LINK=(-shared -Wl,-Bsymbolic -Wl,--no-undefined)
if [ "${KORAL_REF_OPENMP:-0}" = "1" ]; then LINK+=(-fopenmp); fi
gcc "${LINK[@]}" -o "$OUTLIB" "${OBJS[@]}" "$OBJDIR/harness.o" "$OBJDIR/gsl_shim.o" -lm
rm -r "$OBJDIR"   # objects are rebuilt on every call; only the library is kept
echo "built $OUTLIB"

#!/bin/bash
# build.sh -- build the reference HARM code itself, from its own sources, into
# oracle/_ref/harm_ref_<config> (one binary per grid: the reference fixes N1, N2, N3 and
# MAXBND at compile time).  TEST INFRASTRUCTURE ONLY: the binaries are the checker of the
# parity tests and the CPU baseline of the benchmark; the product never loads or runs them.
#
# The recipe does not run the reference's makefile.  In a scratch copy of the sources it
#   1. selects the torus problem (initboundcode/init.fishmon.{c,h}, bounds.fishmon.c as
#      init.c, init.h, bounds.c), and links defs.h/global.h to the GRMHD variants;
#   2. edits init.h: grid size, MAXBND, no entropy variable (NPR = 8, HOT2ENTROPY 0),
#      PRODUCTION 1, WENO line memory on (WENOMEMORY 1) with the a2c-only
#      WENO_REDUCE_A2C_LOOK_OTHER_DIRECTIONS off;
#   3. renames the problem's init_defcoord/init_grid/init_global to href_fishmon_* so that
#      oracle/ref/driver.c can wrap them with this build's run configuration, and gives
#      choose_weno_order's weight array static storage (it returns a pointer into it) and
#      points the WENO pass's primitive line at the line it reads;
#   4. writes the extern-declaration headers (decs.h and the like) from the definition
#      headers (prefixing 'extern' to the top-level definitions) and generates
#      global.defnprs.h with the reference's own generatenprs.c;
#   5. compiles every source of the reference's GRMHD object lists except main.c, plus
#      oracle/ref/driver.c, with gcc -O3 -fopenmp -fcommon, and links them with the calls of
#      advance(), fluxcalc(), post_fixup(), bound_prim_user_dir(), flux_compute_general() and
#      pass_1d_line_multipl_weno() routed through the driver's recording
#      wrappers (ld --wrap), which call the reference's own functions.
# gcc on x86-64 without -march emits no fused multiply-add, so the arithmetic is the
# IEEE operations of the source in its order.
#
# Usage: oracle/ref/build.sh [config ...]   (default: every config below)
# Environment: HARM_REF_DIR (default /root/reference), HARM_REF_JOBS (default nproc).
set -euo pipefail

REF=${HARM_REF_DIR:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
ORC=$(dirname "$HERE")
OUT="$ORC/_ref"
JOBS=${HARM_REF_JOBS:-$(nproc)}

if [ ! -f "$REF/generatenprs.c" ]; then
  echo "ref_build: reference sources not found at $REF; nothing built" >&2
  exit 0
fi

# name N1 N2 N3 MAXBND
CONFIGS=(
  "2d_32x32_b4 32 32 1 4"
  "2d_128x128_b4 128 128 1 4"
  "2d_64x64_b4 64 64 1 4"
  "2d_48x48_b6 48 48 1 6"
  "3d_32x24x8_b4 32 24 8 4"
  "3d_32x24x8_b6 32 24 8 6"
  "3d_192x96x64_b6 192 96 64 6"
  "3d_384x192x128_b6 384 192 128 6"
)

DFLAGS="-DUSINGICC=0 -DUSINGORANGE=0 -DUSINGMPI=0 -DUSINGOPENMP=1 -DUSINGMPIAVOIDFORK=0 -DUSINGMPIAVOIDMKDIR=0 -DUSINGLAPACK=0"
# -mcmodel=medium: the static arrays of the larger grids exceed 2 GB
CFLAGS="-O3 -w -fcommon -fopenmp -mcmodel=medium $DFLAGS"

mkdir -p "$OUT"
WORK=$(mktemp -d /tmp/harm_ref_build.XXXXXX)
trap 'rm -rf "$WORK"' EXIT

edit() {  # edit <file> <sed expression> <pattern that must then be present>
  sed -i -e "$2" "$1"
  grep -q -e "$3" "$1" || { echo "ref_build: edit '$2' of $1 did not apply" >&2; exit 1; }
}

build_one() {
  local name=$1 n1=$2 n2=$3 n3=$4 mb=$5
  local bin="$OUT/harm_ref_$name"
  if [ -x "$bin" ] && [ "$bin" -nt "$HERE/driver.c" ] && [ "$bin" -nt "$HERE/build.sh" ]; then
    return 0
  fi
  local src="$WORK/$name"
  cp -r "$REF" "$src"
  chmod -R u+w "$src"
  (
    cd "$src"
    cp initboundcode/init.fishmon.c init.c
    cp initboundcode/init.fishmon.h init.h
    cp initboundcode/bounds.fishmon.c bounds.c
    ln -sf defs.grmhd.h defs.h
    ln -sf global.grmhd.h global.h
    edit init.h "s/^#define N1 64\$/#define N1 $n1/" "^#define N1 $n1\$"
    edit init.h "s/^#define N2 64\$/#define N2 $n2/" "^#define N2 $n2\$"
    edit init.h "s/^#define N3 1\$/#define N3 $n3/" "^#define N3 $n3\$"
    edit init.h "s/^#define MAXBND 4 .*/#define MAXBND $mb/" "^#define MAXBND $mb\$"
    edit init.h "s/^#define DOENTROPY DOEVOLVEENTROPY/#define DOENTROPY DONOENTROPY/" "^#define DOENTROPY DONOENTROPY"
    edit init.h "s/^#define HOT2ENTROPY 1/#define HOT2ENTROPY 0/" "^#define HOT2ENTROPY 0"
    edit init.h "s/^#define PRODUCTION 0/#define PRODUCTION 1/" "^#define PRODUCTION 1"
    # WENO reconstruction needs its line memory (definit.h WENOMEMORY 0 otherwise).  With it
    # on, the memory of WENO_REDUCE_A2C_LOOK_OTHER_DIRECTIONS does not compile
    # (reconstructeno_set_arrays.c:16 loops over undeclared variables); that switch only acts
    # in the a2c path (multidir_pre_slope_lim_linetype_weno, set at higherorder_pointavg.c:2565),
    # which runs with DOENOFLUX=NOENOFLUX never, so it is turned off.
    edit init.h "s/^#define WENO_REDUCE_A2C_LOOK_OTHER_DIRECTIONS 1/#define WENO_REDUCE_A2C_LOOK_OTHER_DIRECTIONS 0/" \
         "^#define WENO_REDUCE_A2C_LOOK_OTHER_DIRECTIONS 0"
    printf '\n#undef WENOMEMORY\n#define WENOMEMORY 1\n' >> init.h
    # choose_weno_order (reconstructeno.c:2442) hands back a pointer into its own stack frame
    # (stencil_weights_array_static_other), so the WENO3 half of a reduced stencil is read
    # after that frame is gone; built here it reads as zero weights and a fully reduced edge
    # value comes out 0.  The checker runs on one thread, so the array gets static storage,
    # which gives the mix of WENO5 and WENO3 the code intends.
    edit reconstructeno.c "s/^\(\s*\)weno_weights_t stencil_weights_array_static_other\[NUM_POINTS\];/\1static weno_weights_t stencil_weights_array_static_other[NUM_POINTS];/" \
         "static weno_weights_t stencil_weights_array_static_other\[NUM_POINTS\];"
    # The line pass with precomputed indicators (slope_lim_linetype_c2e_perijk_precomputeindicators
    # interpline.c:468) computes the momentum-flux jump indicator dP of the WENO reduction
    # (compute_df_line_new interpline.c:3557) from its primitive line yprim, which that path
    # never fills: dP then comes from whatever the stack held (the cell state itself is read
    # from the stored fluxstatecent, STOREFLUXSTATE).  Its sibling pass
    # slope_lim_linetype_c2e_perijk (interpline.c:696) points yprim at the line it reads
    # (yprim=yin); the checker build does the same here, so that dP is the indicator of the
    # cells' own primitives.
    edit interpline.c "/^void slope_lim_linetype_c2e_perijk_precomputeindicators(/,/p2interp, yin, &trueijkp);/ s/\(p2interp, yin, &trueijkp);\)\$/\1 yprim=yin;/" \
         "p2interp, yin, &trueijkp); yprim=yin;"
    for fn in init_defcoord init_grid init_global; do
      edit init.c "s/^int $fn(void)/int href_fishmon_$fn(void)/" "^int href_fishmon_$fn(void)"
    done
    for h in defs.h mpidefs.h rancdefs.h kazfulleos.defsglobalprivate.h kazfulleos.superdefs.h \
             superdefs.h superdefs.pointers.h defs.user.h defs.general.h supermpidefs.h \
             mpidefs.mpi_grmhd_grray_liaison.h; do
      out=$(echo "$h" | sed 's/def/dec/')
      sed -e 's/^\(PFTYPE\|SFTYPE\|FTYPE\|void\|CTYPE\|struct\|int\|short\|MPI_Status\|MPI_Group\|MPI_Comm\|char\|double\|float\|long\) /extern \1 /' \
          -e 's/^FILE\*/extern FILE* /' -e 's/FILE \*/extern FILE* /' \
          -e 's/^mpidefs\.h/mpidecs.h/' -e 's/defs/decs/' "$h" > "$out"
    done
    gcc $CFLAGS -o generatenprs generatenprs.c
    ./generatenprs > /dev/null
    cp "$HERE/driver.c" href_driver.c
    srcs=$(sed -n '/^SRCSMANYPOINTS=/,/^#END/p;/^SRCSONEPOINT=/,/^#END/p' maketail.harm.inc \
             | grep -v '^#END' | sed 's/SRCS[A-Z]*=//; s/\\//g' | tr ' ' '\n' | grep '\.c$' | grep -v '^main\.c$')
    printf '%s\n' $srcs href_driver.c | xargs -P "$JOBS" -I{} sh -c \
      'gcc '"$CFLAGS"' -c {} -o "$(basename {} .c).o" || { echo "ref_build: compiling {} failed" >&2; exit 255; }'
    objs=$(printf '%s\n' $srcs href_driver.c | sed 's/\.c$/.o/')
    gcc -fopenmp -mcmodel=medium -no-pie -Wl,--wrap=advance,--wrap=fluxcalc,--wrap=post_fixup,--wrap=bound_prim_user_dir,--wrap=flux_compute_general,--wrap=pass_1d_line_multipl_weno \
        -o "$bin.tmp" $objs -lm
    mv "$bin.tmp" "$bin"
  )
  rm -rf "$src"
  echo "ref_build: built $bin"
}

want=("$@")
for cfg in "${CONFIGS[@]}"; do
  set -- $cfg
  if [ ${#want[@]} -gt 0 ]; then
    hit=0
    for w in "${want[@]}"; do [ "$w" = "$1" ] && hit=1; done
    [ $hit = 1 ] || continue
  fi
  build_one "$@"
done

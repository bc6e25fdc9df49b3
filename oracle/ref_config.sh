#!/bin/sh
# Generate the reference's config.h for one oracle variant from its own Config
# file, the same way the reference Makefile does (Makefile:94-96: strip
# comments/blank lines, prefix "#define"), after switching the hot-path options.
#   $1 = reference Config file, $2 = variant (iso|per|perc)_(f32|f64)[_t|_pot], $3 = out
set -e
cfg="$1"; variant="$2"; out="$3"
geom=${variant%%_*}
rest=${variant#*_}
prec=${rest%%_*}
tmp="$out.tmp"
# opening criteria of the measured configuration: theta=0.5 (parameter is
# theta^2) and errtol=0.005
sed -e 's/^TREE_OPEN_PARAM_BH .*/TREE_OPEN_PARAM_BH 0.25/' \
    -e 's/^TREE_OPEN_PARAM_REL .*/TREE_OPEN_PARAM_REL 0.005/' "$cfg" > "$tmp"
case "$geom" in
  iso)  sed -i -e '/^PERIODIC /d' -e '/^COMOVING /d' -e '/^GADGET_COMOVING_VEL_UNIT /d' "$tmp" ;;
  per)  sed -i -e '/^COMOVING /d' -e '/^GADGET_COMOVING_VEL_UNIT /d' "$tmp" ;;
  perc) sed -i -e '/^GADGET_COMOVING_VEL_UNIT /d' "$tmp" ;;
  *) echo "bad variant $variant" >&2; exit 1 ;;
esac
if [ "$prec" = "f64" ]; then echo "DOUBLE_PRECISION" >> "$tmp"; fi
# suffix _pot: the gravitational potential (GRAVITY_POTENTIAL) and its
# snapshot block (OUTPUT_GRAV_POTENTIAL, which changes nothing but the I/O)
case "$variant" in *_pot*) printf 'GRAVITY_POTENTIAL\nOUTPUT_GRAV_POTENTIAL\n' >> "$tmp" ;; esac
# suffix _v<N>: VECTOR_SIZE N (particles per tree leaf) instead of the Config's
case "$variant" in
  *_v[0-9]*) vs=${variant##*_v}; sed -i -e "s/^VECTOR_SIZE .*/VECTOR_SIZE $vs/" "$tmp" ;;
esac
sed '/^#/d; /^[[:space:]]*$/d; s/^/#define /g' "$tmp" > "$out"
rm -f "$tmp"

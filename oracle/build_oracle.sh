#!/bin/bash
# Builds the CPU oracle (bbfmm_oracle.c) in both precisions into oracle/_build/.
# -ffp-contract=off keeps every multiply and add separately rounded, like the
# reference's default gcc build for x86-64; -O3 vectorises only loops whose sums keep their
# order (no reassociation without -ffast-math), so results do not depend on it.
set -euo pipefail
HERE=$(cd "$(dirname "$0")" && pwd)
mkdir -p "$HERE/_build"
gcc -std=gnu99 -O3 -ffp-contract=off -fPIC -shared "$HERE/bbfmm_oracle.c" -o "$HERE/_build/liboracle_d.so" -lm
gcc -std=gnu99 -O3 -ffp-contract=off -fPIC -shared -DORC_SINGLE "$HERE/bbfmm_oracle.c" -o "$HERE/_build/liboracle_s.so" -lm

#!/bin/sh
# Builds the oracle's CPU restatement (aster_oracle.c) into
# oracle/_build/libaster_oracle.so. No FMA contraction: the oracle's rounding
# must follow the source expressions exactly.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
mkdir -p "$HERE/_build"
${CC:-gcc} -std=gnu11 -O2 -fPIC -shared -ffp-contract=off -fno-fast-math -Wall -Wno-unused-function \
  -o "$HERE/_build/libaster_oracle.so" "$HERE/aster_oracle.c" -lm -lpthread

#!/usr/bin/env bash
# Test infrastructure: builds the CPU restatement oracle (oracle/*.c) into
# oracle/_build/liboracle.so.  -ffp-contract=off keeps every float operation separately
# rounded, as the reference's host build does (x86-64 without FMA contraction).
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
mkdir -p "$HERE/_build"
gcc -std=c11 -O2 -fPIC -shared -ffp-contract=off -fno-fast-math -Wall -Wno-unused-function \
  -o "$HERE/_build/liboracle.so" "$HERE/oracle.c" "$HERE/oracle_common.c" "$HERE/oracle_svd.c" -lm
echo "build_oracle: wrote $HERE/_build/liboracle.so"

#!/usr/bin/env bash
# Compile a circuit plug-in (exports circuit_init / circuit_run) into a shared
# object for bin/qcs: ./compile_circuit.sh circuit.c -o circuit.so
set -euo pipefail
: "${CC:=gcc}"
PKG_DIR="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
"$CC" -fPIC -shared -I"${PKG_DIR}/../include" -std=c11 "$@"

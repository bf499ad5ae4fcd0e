#!/bin/sh
# Build the two flavours of the CPU oracle (test infrastructure) into oracle/_build/.
set -e
cd "$(dirname "$0")"
mkdir -p _build
CXX=${CXX:-g++}
FLAGS="-O2 -std=c++17 -fPIC -shared -ffp-contract=off -fno-fast-math -Wall -Wno-unused-function -pthread"
$CXX $FLAGS -DOR_PORTABLE -o _build/liboracle_p.so gf_oracle.cpp
$CXX $FLAGS -o _build/liboracle_l.so gf_oracle.cpp -lm

#!/bin/sh
# Builds the CPU oracle (test infrastructure only) into oracle/libkpz_oracle.so.
set -e
cd "$(dirname "$0")"
gcc -O2 -std=c11 -Wall -Wextra -shared -fPIC kpz_oracle.c -o libkpz_oracle.so -lm

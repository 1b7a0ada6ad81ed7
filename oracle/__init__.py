"""Test infrastructure: CPU oracles for the render loop (checkers, never the product).

  oracle.ref   ctypes view of _ref/libref_lambda.so, the reference renderer's own CPU
               code compiled in place by oracle/Makefile (`make -C oracle ref`)
  oracle.port  ctypes view of liboracle.so, the plain-C restatement in lambda_oracle.c

Only tests, the smoke check and the benchmark's CPU-baseline arm use these.
"""

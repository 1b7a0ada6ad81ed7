"""Builds the native parts in-tree: liblambda_b200.so and bin/lambda (sm_100a),
plus the oracle libraries used by the tests (oracle/liboracle.so, and
oracle/_ref/libref_lambda.so when the reference sources are present)."""

from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# The reference checkout's src/ tree, read only by the oracle recipe; override with
# LAMBDA_REF_SRC. Where it is absent the reference harness is simply not built.
REF_SRC = os.environ.get("LAMBDA_REF_SRC", "/root/reference/src")


def _make(args):
    jobs = str(min(8, os.cpu_count() or 1))
    subprocess.run(["make", "-j", jobs] + args, check=True)


def build(with_oracle: bool = True) -> None:
    _make(["-C", os.path.join(HERE, "csrc")])
    if with_oracle:
        if os.path.exists(os.path.join(ROOT, "oracle", "lambda_oracle.c")):
            _make(["-C", os.path.join(ROOT, "oracle")])
        if os.path.isdir(REF_SRC):
            _make(["-C", os.path.join(ROOT, "oracle"), "ref", "ref_gpu", f"REF_SRC={REF_SRC}"])


if __name__ == "__main__":
    build()

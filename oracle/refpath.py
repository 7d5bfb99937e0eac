"""TEST INFRASTRUCTURE ONLY — where the reference's source tree is.

The one place that names it: the environment variable LAMBDA_REFERENCE, or
the reference checkout this repository is built beside.  The oracle recipes
(oracle/Makefile, lambda_b200/host/Makefile) receive it as REF=...; on a
machine without the reference, only the prebuilt oracle/_ref libraries are
used and nothing reads this path.
"""
import os

REFERENCE = os.environ.get("LAMBDA_REFERENCE") or "/root/reference"


def present(sub=""):
    """Whether the reference tree (or a path inside it) exists here."""
    return os.path.exists(os.path.join(REFERENCE, sub))


def path(*parts):
    return os.path.join(REFERENCE, *parts)

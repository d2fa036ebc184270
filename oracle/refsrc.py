"""ORACLE — test infrastructure only: where the reference's source tree is
read from, for the recipes that compile it (oracle/ref/Makefile through
build() and tests/golden/make_ref_golden.py) and the tests that skip without
it.  The ZEBRAFLOW_REFERENCE environment variable names the tree; without it
the recipes look at the read-only mount of the reference."""
import os

DEFAULT = "/root/reference"


def reference_dir() -> str:
    return os.environ.get("ZEBRAFLOW_REFERENCE", DEFAULT)


def have_reference() -> bool:
    return os.path.isfile(os.path.join(reference_dir(), "ZebraflowWT.c"))

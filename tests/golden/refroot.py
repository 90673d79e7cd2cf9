"""Location of the mdelast checkout that the fixture generators of this directory read.

The checkout is the directory named by ``$MDELAST_REFERENCE`` or, when that is unset, a
checkout called ``reference`` beside this repository. Generators take an explicit path
first when one is given on their command line."""

import os

REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def reference_root(explicit=None) -> str:
    cands = [explicit, os.environ.get("MDELAST_REFERENCE"),
             os.path.join(os.path.dirname(REPO), "reference")]
    for c in cands:
        if c and os.path.isfile(os.path.join(c, "src", "md_driver.cpp")):
            return os.path.abspath(c)
    raise SystemExit("mdelast checkout not found: pass its path or set MDELAST_REFERENCE")

"""TEST INFRASTRUCTURE ONLY: CPU oracles for the B200 search path.

  oracle.ref   -- the reference engine itself, compiled from its sources by
                  oracle/Makefile into oracle/_ref/ (FP32 and FP64 builds)
  oracle.port  -- dmst_oracle.c, a plain-C restatement of the same algorithm

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package, and only as the checker or the timed CPU baseline -- never as part
of the product path.
"""

import os as _os

# Where the reference sources are read from when the oracle is built or
# golden fixtures are regenerated: $DMST_REFERENCE, else the first existing
# directory of the default lookup (a checkout beside this repository, then the
# build container's copy).  Nothing on the scoring path or on a GPU box reads it.
_REFERENCE_LOOKUP = (
    _os.path.join(_os.path.dirname(_os.path.dirname(_os.path.abspath(__file__))), "..", "reference"),
    "/root/reference",
)


def reference_dir() -> str | None:
    """The reference source tree, or None when none is present."""
    env = _os.environ.get("DMST_REFERENCE")
    if env:
        return env if _os.path.isdir(env) else None
    for cand in _REFERENCE_LOOKUP:
        if _os.path.isfile(_os.path.join(cand, "dummest.cc")):
            return _os.path.normpath(cand)
    return None

"""Location of the MDP source tree that the checker builds read.

Test infrastructure only.  The tree is found through the MDP_REFERENCE_ROOT
environment variable, else as a checkout named `reference` beside this
repository.  None when neither exists (e.g. on a machine that only runs the
prebuilt checker libraries).
"""
from __future__ import annotations

import os

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def reference_root() -> str | None:
    cands = [os.environ.get("MDP_REFERENCE_ROOT")]
    cands.append(os.path.join(os.path.dirname(os.path.realpath(REPO)), "reference"))
    for c in cands:
        if c and os.path.isdir(os.path.join(c, "src", "C++", "Core")):
            return c
    return None

"""The reference's own kernels, built from its sources into oracle/_ref (see
oracle/reference_build.py)."""
import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
from reference_build import REF_DIR, RefEvent, RefSim, available, lib  # noqa: E402,F401

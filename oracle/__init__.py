"""FP64 oracle for the motility-ddm analysis path.

TEST INFRASTRUCTURE ONLY: the checker that the CUDA path is compared against.
Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this package. The product (``hackathon_b200``) never does.

The C sources in this directory restate the reference's own CPU code
(motility-ddm/src/fft.js, src/ddm_ref.js, src/motility_fit.js, test/sim.mjs);
this module is a thin ctypes layer over the compiled library.
"""
from .oracle import *  # noqa: F401,F403
from .scenarios import BASE, SCENARIOS, HARNESS_SIM  # noqa: F401

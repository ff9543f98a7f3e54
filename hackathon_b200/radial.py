"""The Radial record (motility-ddm/src/ddm_ref.js:336-348): bin-averaged D,
static power P and the phase-drift least-squares sums, plus the bin geometry
the fit needs. Field names and layouts are the reference's."""
from dataclasses import dataclass

import numpy as np


@dataclass
class Radial:
    N: int
    NB: int
    L: int
    kCenter: np.ndarray  # [NB] mean |k| per bin (FFT index units)
    kNodes: np.ndarray   # [NB*knodes] effective-|k| quadrature nodes
    nModes: np.ndarray   # [NB] modes per bin
    D: np.ndarray        # [NB*L] D[b*L + tau]
    P: np.ndarray        # [NB]
    drift: np.ndarray    # [NB*L*8] drift[(b*L + tau)*8 + c]
    knodes: int = 4

    def D2(self):
        return self.D.reshape(self.NB, self.L)

    def drift3(self):
        return self.drift.reshape(self.NB, self.L, 8)

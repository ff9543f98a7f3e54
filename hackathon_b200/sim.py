"""The reference's seeded movie generator on the GPU (ddm_simulate,
hackathon_b200/csrc/sim.cu): motility-ddm/test/sim.mjs:90-186 with the same
random streams, so a parameter dict and seed give the reference's movie
(up to one grey level on pixels that sit on a rounding boundary).

Parameters follow sim.mjs's SimParams: N, T, fps, dxUm, seed,
swimmers={n, vbar, sigma, geometry}, passive={n}, Dum2s, fixed={n},
drift={speed, angleDeg}, dropFrac, dropExact, blobSigmaPx, amp, background,
noise (defaults as in sim.mjs:91-101).
"""
import ctypes as C

import numpy as np

from . import _lib


def params(sim):
    """SimParams dict -> ddm_sim_params."""
    p = _lib.SimParams()
    p.N, p.T = int(sim.get("N", 256)), int(sim.get("T", 256))
    p.fps, p.dxUm = float(sim.get("fps", 30.0)), float(sim.get("dxUm", 1.0))
    p.seed = int(sim.get("seed", 1)) & 0xFFFFFFFF
    sw = sim.get("swimmers")
    if sw and sw.get("n", 0) > 0:
        p.nSwim, p.swimVbar, p.swimSigma = int(sw["n"]), float(sw["vbar"]), float(sw["sigma"])
        p.swim2d = 1 if sw.get("geometry") == "2d" else 0
    p.nPassive = int((sim.get("passive") or {}).get("n", 0))
    p.Dum2s = float(sim.get("Dum2s", 0.0))
    p.nFixed = int((sim.get("fixed") or {}).get("n", 0))
    dr = sim.get("drift")
    if dr:
        p.hasDrift, p.driftSpeed, p.driftAngleDeg = 1, float(dr["speed"]), float(dr["angleDeg"])
    p.dropFrac = float(sim.get("dropFrac", 0.0))
    p.dropExact = int(sim.get("dropExact", 0))
    p.blobSigmaPx = float(sim.get("blobSigmaPx", 1.5))
    p.amp = float(sim.get("amp", 0.15))
    p.background = float(sim.get("background", 0.25))
    p.noise = float(sim.get("noise", 0.01))
    return p


def simulate(sim, device=True, stream=None):
    """-> (frames u8 [T, N, N]: a torch CUDA tensor if device else numpy,
    valid bool [T] numpy, truth dict meanSpeed/Vx/Vy/D)."""
    lib = _lib.load()
    p = params(sim)
    valid = np.empty(p.T, np.uint8)
    truth = np.empty(4)
    if device:
        import torch
        frames = torch.empty((p.T, p.N, p.N), dtype=torch.uint8, device="cuda")
        ptr = frames.data_ptr()
        s = torch.cuda.current_stream().cuda_stream if stream is None else stream
    else:
        frames = np.empty((p.T, p.N, p.N), np.uint8)
        ptr = frames.ctypes.data
        s = stream
    rc = lib.ddm_simulate(C.byref(p), C.c_void_p(ptr), 1 if device else 0, C.c_void_p(valid.ctypes.data),
                          C.c_void_p(truth.ctypes.data), C.c_void_p(s) if s else None)
    if rc != _lib.DDM_OK:
        from .engine import DdmArgError, DdmError
        raise (DdmArgError if rc == _lib.DDM_ERR_ARG else DdmError)(rc, lib.ddm_simulate_error().decode())
    return frames, valid.astype(bool), dict(meanSpeed=truth[0], Vx=truth[1], Vy=truth[2], D=truth[3])

"""The reference's synthetic validation matrix as data.

Restated from motility-ddm/test/sim.mjs:195-309 (BASE, SCENARIOS, HARNESS_SIM)
so that the oracle renders the same movies the reference's own integration
test (test/t_validation_matrix.mjs) runs. ``expect`` and ``checks`` are the
reference's pass criteria (sim.mjs:208-213; checkScenario
t_validation_matrix.mjs:47-67). ``published`` holds the outputs the reference
reports for each scenario (README.md section 6, "CPU validation matrix").
TEST INFRASTRUCTURE ONLY.
"""

# sim.mjs:195
BASE = dict(N=256, T=256, fps=30.0, dxUm=1.0, Dum2s=0.4, blobSigmaPx=1.5,
            amp=0.15, background=0.25, noise=0.01)


def _sc(name, sim, geometry, expect, checks, published, shuffle=False):
    s = dict(BASE)
    s.update(sim)
    return dict(name=name, sim=s, geometry=geometry, expect=expect,
                checks=checks, shuffle=shuffle, published=published)


_SW3 = dict(n=150, vbar=20.0, sigma=8.0, geometry="3d")

# sim.mjs:215-305; published values from README.md (CPU validation matrix).
SCENARIOS = [
    _sc("motile_3d", dict(seed=11, swimmers=_SW3, passive=dict(n=150)), "3d",
        "MOTILE", dict(vbar=(20, 0.2), alpha=(0.5, 0.2)),
        dict(alpha=0.50, vbar=23.4, V=0.09)),
    _sc("motile_2d", dict(seed=12, swimmers=dict(n=150, vbar=25.0, sigma=10.0, geometry="2d"),
                          passive=dict(n=100)), "2d",
        "MOTILE", dict(vbar=(25, 0.2), alpha=(0.6, 0.2)),
        dict(alpha=0.63, vbar=21.8, V=0.32)),
    _sc("sparse_swimmers", dict(seed=13, swimmers=dict(n=25, vbar=20.0, sigma=8.0, geometry="3d"),
                                passive=dict(n=300)), "3d",
        "MOTILE", dict(alpha=(25 / 325, 0.07)),
        dict(alpha=0.08, vbar=13.0, V=0.12)),
    _sc("killed_brownian", dict(seed=14, passive=dict(n=300)), "3d",
        "NOT_MOTILE", dict(), dict(alpha=0.00, V=0.08)),
    _sc("static_debris", dict(seed=15, fixed=dict(n=300)), "3d",
        "NO_DYNAMICS", dict(), dict(V=0.00)),
    _sc("shuffle_null", dict(seed=11, swimmers=_SW3, passive=dict(n=150)), "3d",
        "NO_DYNAMICS", dict(), dict(V=0.01), shuffle=True),
    _sc("flow_0deg_10ums", dict(seed=17, passive=dict(n=250), drift=dict(speed=10.0, angleDeg=0.0)),
        "3d", "DIRECTED_TRANSPORT", dict(drift=(10, 0, 0.15, 10)),
        dict(V=9.93, angle=-1.0)),
    _sc("flow_135deg_5ums", dict(seed=18, passive=dict(n=250), drift=dict(speed=5.0, angleDeg=135.0)),
        "3d", "DIRECTED_TRANSPORT", dict(drift=(5, 135, 0.15, 10)),
        dict(V=4.85, angle=135.0)),
    _sc("flow_60deg_1ums", dict(seed=19, passive=dict(n=250), drift=dict(speed=1.0, angleDeg=60.0)),
        "3d", "NOT_MOTILE", dict(), dict(alpha=0.00, V=0.86, angle=60.0)),
    _sc("motile_in_flow", dict(seed=20, swimmers=_SW3, passive=dict(n=150),
                               drift=dict(speed=8.0, angleDeg=210.0)), "3d",
        "DIRECTED_TRANSPORT", dict(drift=(8, 210, 0.2, 15)),
        dict(V=7.92, angle=-150.0)),
    _sc("dropped_frames_20pct", dict(seed=21, swimmers=_SW3, passive=dict(n=150), dropFrac=0.2),
        "3d", "MOTILE", dict(vbar=(20, 0.2), alpha=(0.5, 0.2)),
        dict(alpha=0.51, vbar=17.7, V=0.25)),
]

# sim.mjs:309: motile_3d with exactly 37 of 256 frames dropped, seed 101.
HARNESS_SIM = dict(SCENARIOS[0]["sim"])
HARNESS_SIM.update(dropExact=37, seed=101)

"""Golden cases: small coupled systems run by the reference's own CUDA kernels.

Each case is built identically on any backend that offers the
add_gel / gel_noise / set_params / reset_quiescent / set_anchor /
set_active_from / finalize / run / get interface (the reference harness, the
CPU oracle and the product's Python binding all do).  The fixtures
tests/golden/<name>.npz hold the reference's outputs after `iters`
iterations; make_golden.py writes them.
"""

CASES = {
    # one 6x6x6 gel in a 20^3 box, IBM at full strength from the first step
    "single": dict(
        dims=(20, 20, 20), nsub=2, iters=12, beta=1.0, ramp=0.0,
        gels=[dict(size=(6, 6, 6), pos=(4.75, 4.75, 4.75), type=1)],
        seed=12345, amp=1e-3, save_pop=True,
    ),
    # two small gels (types 1 and 2) 1.5 apart, even and unequal lattice dims:
    # exercises repulsion between gels, the gelType 2 pressure and the narrowed lattice
    "pair": dict(
        dims=(24, 20, 28), nsub=3, iters=15, beta=1.0, ramp=0.0,
        gels=[dict(size=(3, 3, 3), pos=(3.75, 4.75, 6.75), type=1),
              dict(size=(3, 3, 3), pos=(8.25, 4.75, 6.75), type=2)],
        seed=777, amp=1e-3, save_pop=False,
    ),
    # an anchored rod that stays quiescent until iteration 4, then fires its pulse
    "rod": dict(
        dims=(16, 16, 30), nsub=2, iters=12, beta=1.0, ramp=100.0,
        gels=[dict(size=(2, 2, 8), pos=(3.75, 3.75, 5.5), type=1, anchor=1.5, quiescent=True,
                   active_from=4)],
        seed=99, amp=1e-3, save_pop=False,
    ),
}

FLUID_FIELDS = {"rho": 1, "u": 2, "c1": 3}
MARKER_FIELDS = {"lag": 10, "Ul": 11, "Vl": 12, "Fdrag": 13, "Frep": 14, "Cl": 15, "Dl": 16, "Sl": 17}
GEL_FIELDS = {"rn": 20, "Veln": 21, "Vels": 22, "Fn": 23, "um": 24, "vm": 25, "wm": 26,
              "un_norm": 27, "vn_norm": 28, "T0": 29, "T2": 31, "rm": 32, "nmSm": 33,
              "Volm": 34, "un_robin": 36}


def build(backend_cls, case, **kw):
    """Construct and finalize a case on `backend_cls(nx, ny, nz, nsub=..)`."""
    c = CASES[case] if isinstance(case, str) else case
    sim = backend_cls(*c["dims"], nsub=c["nsub"], **kw)
    for k, g in enumerate(c["gels"]):
        sim.add_gel(g["size"], g["pos"], g["type"], k + 1)
    for k, g in enumerate(c["gels"]):
        sim.gel_noise(k, c["seed"], c["amp"])
        if g.get("quiescent"):
            sim.reset_quiescent(k)
        if "anchor" in g:
            sim.set_anchor(k, g["anchor"])
        if g.get("active_from"):
            sim.set_active_from(k, g["active_from"])
    sim.set_params(beta=c["beta"], ramp_steps=c["ramp"])
    sim.finalize()
    return sim


def collect(sim, case):
    """Read every compared field of a finished case into a dict of float64 arrays."""
    c = CASES[case] if isinstance(case, str) else case
    out = {}
    for name, fid in FLUID_FIELDS.items():
        out[name] = sim.get(fid)
    if c.get("save_pop"):
        out["pop"] = sim.get(0)
    for name, fid in MARKER_FIELDS.items():
        out[name] = sim.get(fid)
    for k in range(len(c["gels"])):
        for name, fid in GEL_FIELDS.items():
            out[f"g{k}_{name}"] = sim.get(fid, k)
    return out

"""glsm_substep_noalloc: the substep for callers that cannot allocate device
memory (a host framework owning all device memory through its own pool, a
plug-in whose host process accounts for every device byte, a real-time loop
where an allocation may synchronise the device).

Two calls in a row (parity 0, then 1) make one full two-substep velocity step.
Their output must match the handle-based entry point glsm_fluid_step_velocity
(which owns allocated buffers) started from the same state.  The test buffers
are allocated here by torch; the entry point itself allocates nothing.

Cases: a gel in the middle of the box; a gel against the x = 0 and y = 0 faces
with a uniform body force (stencils clipped at the walls, the sum of the
clipped weights below one); and no markers at all with a body force (compared
with the handle path at zero penalty strength, whose spread force is zero).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, dtype=np.float64)

CASES = {
    "centre": dict(pos=(5.75, 5.75, 5.75), force=(0.0, 0.0, 0.0), beta=1.0, markers=True),
    "wall": dict(pos=(3.25, 3.5, 5.75), force=(2e-6, -1e-6, 5e-7), beta=1.0, markers=True),
    "no_markers": dict(pos=(5.75, 5.75, 5.75), force=(1e-6, 2e-6, -3e-6), beta=0.0, markers=False),
}


def _rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _lib():
    from glsm_fluid_3d_b200 import lib

    L = lib()
    f, i, P, vp = ctypes.c_float, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p
    L.glsm_substep_noalloc.argtypes = [P, ctypes.c_int64, P, i, i, i, i, f, f, f, f, P, P, i, f, f, P, P, vp]
    L.glsm_substep_noalloc.restype = i
    L.glsm_noalloc_last_error.restype = ctypes.c_char_p
    return L


@pytest.mark.parametrize("case", list(CASES))
def test_noalloc_substeps_match_step_velocity(gpu, case):
    import torch

    from glsm_fluid_3d_b200 import System

    c = CASES[case]
    L = _lib()
    nx = ny = nz = 24
    s = System(nx, ny, nz, nsub=2)
    s.add_gel((6, 6, 6), c["pos"], 1, 1)
    s.gel_noise(0, 4242, 1e-3)
    s.set_params(beta=c["beta"], ramp_steps=0.0, force=c["force"])
    s.finalize()
    s.run(0, 3)
    s.coupler.packFromGels()  # markers of iteration 3
    N = nx * ny * nz
    pop0 = s.fluid.read("pop").astype(np.float64).reshape(19, N)
    u0 = s.fluid.read("u").reshape(N, 3)
    rho0 = s.fluid.read("rho")
    lag = s.coupler.read("lag").reshape(-1, 3)
    vel = s.coupler.read("Vl").reshape(-1, 3)
    if case == "wall":  # some stencils reach beyond the lattice
        assert (lag[:, :2] / 0.5).min() < 2.0

    # the handle-based entry point: Fluid::stepVelocity with two substeps
    s.fluid.stepVelocity(3)
    s.fluid.sync()
    want_pop = s.fluid.read("pop")
    want_u = s.fluid.read("u")
    want_ul = s.coupler.read("Ul")
    want_fd = s.coupler.read("Fdrag")
    s.close()

    M = lag.shape[0] if c["markers"] else 0
    dev = torch.device("cuda")
    pop = torch.tensor((pop0 - W[:, None]).astype(np.float32), device=dev).contiguous()
    u4 = torch.tensor(np.concatenate([u0, rho0[:, None]], axis=1).astype(np.float32), device=dev).contiguous()
    lag4 = torch.zeros((max(M, 1), 4), dtype=torch.float32, device=dev)
    vel4 = torch.zeros((max(M, 1), 4), dtype=torch.float32, device=dev)
    if M:
        lag4[:, :3] = torch.tensor(lag, device=dev)
        vel4[:, :3] = torch.tensor(vel, device=dev)
    ul4 = torch.zeros((max(M, 1), 4), dtype=torch.float32, device=dev)
    fd4 = torch.zeros((max(M, 1), 4), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    fx, fy, fz = c["force"]
    for parity in (0, 1):  # two calls in a row
        rc = L.glsm_substep_noalloc(pop.data_ptr(), N, u4.data_ptr(), nx, ny, nz, parity, 0.8, fx, fy, fz,
                                    lag4.data_ptr() if M else None, vel4.data_ptr() if M else None, M, 0.5,
                                    c["beta"], ul4.data_ptr() if M else None, fd4.data_ptr() if M else None, stream)
        assert rc == 0, L.glsm_noalloc_last_error()
    torch.cuda.synchronize()
    got_pop = pop.cpu().numpy().astype(np.float64) + W[:, None]
    got_u = u4.cpu().numpy()[:, :3]
    # same tolerances as the parity tests against the FP64 oracle
    assert _rel(got_pop, want_pop) < 1e-6
    assert _rel(got_u, want_u) < 2e-4
    if M:
        assert _rel(ul4.cpu().numpy()[:, :3], want_ul) < 2e-4
        assert _rel(fd4.cpu().numpy()[:, :3], want_fd) < 2e-5


def test_noalloc_rejects_sizes_beyond_its_limit(gpu):
    L = _lib()
    dummy = ctypes.c_void_p(16)
    rc = L.glsm_substep_noalloc(dummy, ctypes.c_int64(65 * 65 * 65), dummy, 65, 65, 65, 0, ctypes.c_float(0.8),
                                ctypes.c_float(0), ctypes.c_float(0), ctypes.c_float(0), None, None, 0,
                                ctypes.c_float(0.5), ctypes.c_float(1.0), None, None, None)
    assert rc == -1
    assert b"262144" in L.glsm_noalloc_last_error()

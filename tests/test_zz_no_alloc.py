"""glsm_substep_noalloc: the substep for callers that cannot allocate device
memory (a host framework owning all device memory through its own pool, a
plug-in whose host process accounts for every device byte, a real-time loop
where an allocation may synchronise the device).

Two calls in a row (parity 0, then 1) make one full two-substep velocity step.
Their output must match the handle-based entry point glsm_fluid_step_velocity
(which owns allocated buffers) started from the same state.  The test buffers
are allocated here by torch; the entry point itself allocates nothing.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, dtype=np.float64)


def _rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_noalloc_substeps_match_step_velocity(gpu):
    import torch

    from glsm_fluid_3d_b200 import System, lib

    L = lib()
    f, i, P, vp = ctypes.c_float, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p
    L.glsm_substep_noalloc.argtypes = [P, ctypes.c_int64, P, i, i, i, i, f, f, f, f, P, P, i, f, f, P, P, vp]
    L.glsm_substep_noalloc.restype = i
    L.glsm_noalloc_last_error.restype = ctypes.c_char_p

    nx = ny = nz = 24
    s = System(nx, ny, nz, nsub=2)
    s.add_gel((6, 6, 6), (5.75, 5.75, 5.75), 1, 1)
    s.gel_noise(0, 4242, 1e-3)
    s.set_params(beta=1.0, ramp_steps=0.0)
    s.finalize()
    s.run(0, 3)
    s.coupler.packFromGels()  # markers of iteration 3
    N = nx * ny * nz
    pop0 = s.fluid.read("pop").astype(np.float64).reshape(19, N)
    u0 = s.fluid.read("u").reshape(N, 3)
    rho0 = s.fluid.read("rho")
    lag = s.coupler.read("lag").reshape(-1, 3)
    vel = s.coupler.read("Vl").reshape(-1, 3)
    M = lag.shape[0]

    # the handle-based entry point: Fluid::stepVelocity with two substeps
    s.fluid.stepVelocity(3)
    s.fluid.sync()
    want_pop = s.fluid.read("pop")
    want_u = s.fluid.read("u")
    want_ul = s.coupler.read("Ul")
    want_fd = s.coupler.read("Fdrag")
    s.close()

    dev = torch.device("cuda")
    pop = torch.tensor((pop0 - W[:, None]).astype(np.float32), device=dev).contiguous()
    u4 = torch.tensor(np.concatenate([u0, rho0[:, None]], axis=1).astype(np.float32), device=dev).contiguous()
    lag4 = torch.zeros((M, 4), dtype=torch.float32, device=dev)
    lag4[:, :3] = torch.tensor(lag, device=dev)
    vel4 = torch.zeros((M, 4), dtype=torch.float32, device=dev)
    vel4[:, :3] = torch.tensor(vel, device=dev)
    ul4 = torch.zeros((M, 4), dtype=torch.float32, device=dev)
    fd4 = torch.zeros((M, 4), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    for parity in (0, 1):  # two calls in a row
        rc = L.glsm_substep_noalloc(pop.data_ptr(), N, u4.data_ptr(), nx, ny, nz, parity, 0.8, 0.0, 0.0, 0.0,
                                    lag4.data_ptr(), vel4.data_ptr(), M, 0.5, 1.0, ul4.data_ptr(), fd4.data_ptr(),
                                    stream)
        assert rc == 0, L.glsm_noalloc_last_error()
    torch.cuda.synchronize()
    got_pop = pop.cpu().numpy().astype(np.float64) + W[:, None]
    got_u = u4.cpu().numpy()[:, :3]
    # same tolerances as the parity tests against the FP64 oracle
    assert _rel(got_pop, want_pop) < 1e-6
    assert _rel(got_u, want_u) < 2e-4
    assert _rel(ul4.cpu().numpy()[:, :3], want_ul) < 2e-4
    assert _rel(fd4.cpu().numpy()[:, :3], want_fd) < 2e-5


def test_noalloc_rejects_sizes_beyond_its_limit(gpu):
    from glsm_fluid_3d_b200 import lib

    L = lib()
    L.glsm_noalloc_last_error.restype = ctypes.c_char_p
    dummy = ctypes.c_void_p(16)
    rc = L.glsm_substep_noalloc(dummy, ctypes.c_int64(65 * 65 * 65), dummy, 65, 65, 65, 0, ctypes.c_float(0.8),
                                ctypes.c_float(0), ctypes.c_float(0), ctypes.c_float(0), None, None, 0,
                                ctypes.c_float(0.5), ctypes.c_float(1.0), None, None, None)
    assert rc == -1
    assert b"262144" in L.glsm_noalloc_last_error()

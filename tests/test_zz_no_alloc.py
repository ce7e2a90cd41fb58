"""ggb_observables_noalloc: the entry point for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc -- code running inside another framework's memory pool (which
must own every device allocation), or a process that reserved all device memory up front.  For
them libggbtddft exports ggb_observables_noalloc, which computes the per-(l, orbital) dipole and
acceleration sums and the per-orbital norm of a set of orbitals into caller-provided buffers,
keeping its partial sums in a fixed-size array inside the library instead of allocating.

This test calls it through the C ABI on the orbitals a time step produced and checks it against
the observables the existing path (ggb_step + ggb_get_observables) recorded for that step, on two
calls in a row (the second call reuses the shared scratch left by the first).  It lives in a file
of its own that pytest collects last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_observables_noalloc_matches_time_step_observables():
    import torch

    from ggbtddft_b200 import problems as P
    from ggbtddft_b200.engine import TimePropagation, load_library

    fn = load_library().ggb_observables_noalloc

    run = P.reference_like(70, 17, 12, "Ne3", r_mask=15.0, dt_as=10.0, perturb=0.05, seed=11)
    tp = TimePropagation([run])
    tp.step(12)
    ref = tp.observables(0, per_l=True, n_steps=12)
    x = tp.orbitals(0)                      # orbitals after the last step
    st, msg = tp.status()
    tp.close()
    assert st == 0, msg

    dev = torch.device("cuda", 0)
    # the caller owns every buffer (here: torch's allocator); the entry point allocates nothing
    xd = torch.from_numpy(x.view(np.float64).copy()).to(dev)
    rd = torch.from_numpy(run.grid.r.copy()).to(dev)
    md = torch.from_numpy(run.m_active.astype(np.int32)).to(dev)
    n_l, n_orb, n_r = x.shape
    for call in range(2):
        dip = torch.full((n_l * n_orb * 2,), float("nan"), dtype=torch.float64, device=dev)
        acc = torch.full_like(dip, float("nan"))
        norm = torch.full((n_orb,), float("nan"), dtype=torch.float64, device=dev)
        rc = fn(xd.data_ptr(), rd.data_ptr(), md.data_ptr(), n_l, n_orb, n_r, dip.data_ptr(), acc.data_ptr(),
                norm.data_ptr(), torch.cuda.current_stream().cuda_stream)
        assert rc == 0, f"call {call}: status {rc}"
        torch.cuda.synchronize()
        got_dip = dip.cpu().numpy().view(np.complex128).reshape(n_l, n_orb)
        got_acc = acc.cpu().numpy().view(np.complex128).reshape(n_l, n_orb)
        tol = 1e-12 * max(np.abs(ref["dipole"][:, :, -1]).max(), 1e-300)
        assert np.abs(got_dip - ref["dipole"][:, :, -1]).max() <= tol, call
        tol = 1e-12 * max(np.abs(ref["acceleration"][:, :, -1]).max(), 1e-300)
        assert np.abs(got_acc - ref["acceleration"][:, :, -1]).max() <= tol, call
        assert np.allclose(norm.cpu().numpy(), ref["norm"][:, -1], rtol=1e-13, atol=0), call


def test_observables_noalloc_rejects_sizes_beyond_its_scratch():
    from ggbtddft_b200.engine import load_library

    fn = load_library().ggb_observables_noalloc
    one = ctypes.c_void_p(1)   # never dereferenced: the size check comes first
    # n_orb * N_l * ceil(N_r / 32) above 65536 partial sums, and N_l above 256
    assert fn(one, one, one, 200, 16, 1024, one, one, one, None) == -1
    assert fn(one, one, one, 300, 1, 64, one, one, one, None) == -1

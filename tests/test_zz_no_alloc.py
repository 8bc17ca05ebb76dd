"""zrk_rates_jac_dev_noalloc: the rates + Jacobian entry point for callers
that cannot let the library allocate device memory during a call (a CFD
code whose pool allocator owns the GPU after start-up, code where a
cudaMalloc would synchronize the device, a host with a fixed device
footprint).  It must give the results of zrk_rates_jac_dev, within the
FP64 parity tolerance of the rates tests (1e-12 of each entry's rounding
scale), on consecutive calls that share its fixed workspace.

This file is collected last so that a run stopping at the first failure
has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import have_gpu, oracle_tables, scaled_err, synth

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def torch():
    if not have_gpu():
        pytest.skip("no CUDA device")
    import torch
    return torch


def _device_inputs(torch, pm, T, P, Y, ld):
    dev = torch.device("cuda")
    n = T.shape[0]
    Tt = torch.full((ld,), 1000.0, dtype=torch.float64, device=dev)
    Pt = torch.full((ld,), 101325.0, dtype=torch.float64, device=dev)
    Yt = torch.full((pm.nsp, ld), 1.0 / pm.nsp, dtype=torch.float64, device=dev)
    Tt[:n] = torch.from_numpy(T)
    Pt[:n] = torch.from_numpy(P)
    Yt[:, :n] = torch.from_numpy(np.ascontiguousarray(Y.T))
    return Tt, Pt, Yt


def _outputs(torch, pm, ld, fill):
    dev = torch.device("cuda")
    return (torch.full((pm.nsp, ld), fill, dtype=torch.float64, device=dev),
            torch.full((pm.nnz, ld), fill, dtype=torch.float64, device=dev),
            torch.full((pm.nsp + 1, ld), fill, dtype=torch.float64, device=dev))


def _call(fn, pm, n, ld, inputs, outputs):
    import zerork_b200 as zb
    p = lambda t: C.c_void_p(t.data_ptr())
    rc = fn(pm._h, n, ld, *[p(t) for t in inputs], *[p(t) for t in outputs], None)
    assert rc == 0, zb.lib().zrk_last_error().decode()


def test_no_alloc_matches_rates_jac_dev_on_consecutive_calls(torch, mech_dir):
    import zerork_b200 as zb
    from zerork_b200 import mechgen
    L = zb.lib()
    L.zrk_rates_jac_dev_noalloc.restype = C.c_int
    L.zrk_rates_jac_dev_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_int] + [C.c_void_p] * 7
    L.zrk_last_error.restype = C.c_char_p
    g, (mf, tf) = synth("c2_53", mech_dir)
    pm = zb.Mechanism(mf, tf)
    # an explicit tile mapping, so the workspace slice size is known: rows of
    # ts doubles (C, u/RT, g/RT, one per step, two partial buffers per warp,
    # two more), ZRK_NOALLOC_SCRATCH_BYTES = 8 MiB of them
    ts, v, warps = 16, 2, 8
    pm.set_launch(ts, v, warps, False, 0)
    slice_bytes = (3 * pm.nsp + pm.nstep + 2 * warps + 2) * ts * 8
    slices = (8 << 20) // slice_bytes
    ot = oracle_tables(zb.Mechanism(mf, tf, device=False))
    # two calls in a row with different sizes and states: the second must not
    # see anything the first left in the shared workspace; 3000 states give
    # more tiles than the fixed array holds slices for, so CTAs take several
    assert -(-3000 // ts) > slices
    for n, ld, seed in ((3000, 3008, 1), (517, 517, 2)):
        T, P, Y = mechgen.rate_states(g, n, seed=seed)
        inputs = _device_inputs(torch, pm, T, P, Y, ld)
        ref = _outputs(torch, pm, ld, -3.5)
        got = _outputs(torch, pm, ld, 7.25)
        _call(L.zrk_rates_jac_dev, pm, n, ld, inputs, ref)
        _call(L.zrk_rates_jac_dev_noalloc, pm, n, ld, inputs, got)
        torch.cuda.synchronize()
        w_ref, j_ref = ref[0][:, :n].T.cpu().numpy(), ref[1][:, :n].T.cpu().numpy()
        w, j, d = (x[:, :n].T.cpu().numpy() for x in got)
        wo, jo, ws, js = ot.batch_rates_jac_scaled(T, P, Y)
        assert scaled_err(w, w_ref, ws) < TOL
        assert scaled_err(j, j_ref, js) < TOL
        d_ref = ref[2][:, :n].T.cpu().numpy()
        assert np.all(np.abs(d - d_ref) <= TOL * np.abs(d_ref).max(axis=1, keepdims=True))
        # and both against the oracle
        assert scaled_err(w, wo, ws) < TOL and scaled_err(j, jo, js) < TOL
        if ld > n:  # padding columns untouched
            assert torch.all(got[0][:, n:] == 7.25) and torch.all(got[1][:, n:] == 7.25)

"""The allocation-free force entry point (b2md_forces_noalloc).

It exists for callers that cannot allocate device memory while they call the
library: a host program that owns all device buffers and only lends a plugin
pointers, or a real-time loop that must not call cudaMalloc/cudaFree (they can
synchronise the device and take unbounded time).  The caller passes its own
device buffers; the library's only scratch is a fixed array in its device
image.  Here the test owns the buffers (allocated through torch, as such a
host program would), and the results must equal those of the engine's
b2md_calc_f on the same configuration, within the force tolerance used
throughout the tests (rms relative error <= 1e-5), on two calls in a row.

This file is collected last so that a run stopping at its first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 4000
MAX_N = 65536


def _melted_ka(capi, initconf):
    c = initconf.ka_config(N, T=2.0, seed=4)
    params = initconf.lj_params(2, initconf.KA)
    e = capi.Engine(device=0, pb=64, tp=4)
    rid = e.add(c["pos4"], c["box"], params, 2, cutoff="SF", vel4=c["vel4"])
    e.run(300)
    e.calc_f()
    out = dict(pos4=e.get(rid, "pos", N), force=e.get(rid, "force", N), stats=e.stats(rid),
               box=np.ascontiguousarray(c["box"], np.float32), params=params)
    e.close()
    return out


def test_noalloc_forces_equal_engine_forces_on_two_calls():
    import torch
    from rumd_b200 import capi, initconf
    ref = _melted_ka(capi, initconf)
    lib = capi.lib()
    dev = torch.device("cuda:0")
    pos = torch.from_numpy(ref["pos4"]).to(dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    box = ref["box"]
    params = np.ascontiguousarray(ref["params"], np.float32)
    f_ref = ref["force"].astype(np.float64)
    for call in range(2):
        force = torch.full((N, 4), float("nan"), dtype=torch.float32, device=dev)
        sums = torch.zeros(2, dtype=torch.float64, device=dev)
        rc = lib.b2md_forces_noalloc(ctypes.c_void_p(pos.data_ptr()), N, box.ctypes.data_as(ctypes.c_void_p), 2,
                                     params.ctypes.data_as(ctypes.c_void_p), capi.CUTOFF["SF"],
                                     ctypes.c_void_p(force.data_ptr()), ctypes.c_void_p(sums.data_ptr()), stream)
        assert rc == capi.B2MD_OK, lib.b2md_last_error()
        torch.cuda.synchronize(dev)
        f = force.cpu().numpy().astype(np.float64)
        s = sums.cpu().numpy()
        rms = np.sqrt(((f[:, :3] - f_ref[:, :3]) ** 2).sum() / (f_ref[:, :3] ** 2).sum())
        assert rms <= 1e-5, (call, rms)
        assert np.abs(f[:, 3] - f_ref[:, 3]).max() < 1e-4, call
        pe, vir = ref["stats"]["pe"], ref["stats"]["virial"]
        assert abs(s[0] - pe) <= 1e-5 * abs(pe), (call, s[0], pe)
        assert abs(s[1] - vir) <= 1e-5 * abs(vir) + 1e-3, (call, s[1], vir)


def test_noalloc_rejects_sizes_beyond_its_maximum():
    from rumd_b200 import capi
    lib = capi.lib()
    box = np.array([10.0, 10.0, 10.0], np.float32)
    params = np.zeros(12, np.float32)
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.b2md_forces_noalloc(dummy, MAX_N + 1, box.ctypes.data_as(ctypes.c_void_p), 1,
                                 params.ctypes.data_as(ctypes.c_void_p), 0, dummy, dummy, None)
    assert rc == capi.B2MD_ERR_ARG
    assert str(MAX_N).encode() in lib.b2md_last_error()

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
The comparison runs for every cut-off method (each packs the pair rows
differently), once on a cubic and once on a non-cubic box.

This file is collected last so that a run stopping at its first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_N = 65536
# (cut-off method, particles, box stretch per axis): the stretch keeps the
# volume, so the density stays 1.2
CASES = [("SF", 4000, (1.0, 1.0, 1.0)), ("SP", 1000, (1.25, 0.9, 1.0 / (1.25 * 0.9))),
         ("NS", 1000, (0.9, 1.2, 1.0 / (0.9 * 1.2)))]


def _melted_ka(capi, initconf, n, cutoff, stretch):
    c = initconf.ka_config(n, T=2.0, seed=4)
    params = initconf.lj_params(2, initconf.KA)
    box = (c["box"] * np.asarray(stretch, np.float32)).astype(np.float32)
    pos4 = c["pos4"].copy()
    pos4[:, :3] *= np.asarray(stretch, np.float32)
    e = capi.Engine(device=0, pb=64, tp=4)
    rid = e.add(pos4, box, params, 2, cutoff=cutoff, vel4=c["vel4"])
    e.run(300)
    e.calc_f()
    out = dict(pos4=e.get(rid, "pos", n), force=e.get(rid, "force", n), stats=e.stats(rid),
               box=np.ascontiguousarray(box, np.float32), params=params)
    e.close()
    return out


def _call(lib, pos_ptr, n, box, params, cutoff, force_ptr, sums_ptr, stream):
    return lib.b2md_forces_noalloc(pos_ptr, n, box.ctypes.data_as(ctypes.c_void_p), 2,
                                   params.ctypes.data_as(ctypes.c_void_p), cutoff, force_ptr, sums_ptr, stream)


@pytest.mark.parametrize("cutoff,n,stretch", CASES)
def test_noalloc_forces_equal_engine_forces_on_two_calls(cutoff, n, stretch):
    import torch
    from rumd_b200 import capi, initconf
    ref = _melted_ka(capi, initconf, n, cutoff, stretch)
    lib = capi.lib()
    dev = torch.device("cuda:0")
    pos = torch.from_numpy(ref["pos4"]).to(dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    params = np.ascontiguousarray(ref["params"], np.float32)
    f_ref = ref["force"].astype(np.float64)
    for call in range(2):
        force = torch.full((n, 4), float("nan"), dtype=torch.float32, device=dev)
        sums = torch.zeros(2, dtype=torch.float64, device=dev)
        rc = _call(lib, ctypes.c_void_p(pos.data_ptr()), n, ref["box"], params, capi.CUTOFF[cutoff],
                   ctypes.c_void_p(force.data_ptr()), ctypes.c_void_p(sums.data_ptr()), stream)
        assert rc == capi.B2MD_OK, lib.b2md_last_error()
        torch.cuda.synchronize(dev)
        f = force.cpu().numpy().astype(np.float64)
        s = sums.cpu().numpy()
        rms = np.sqrt(((f[:, :3] - f_ref[:, :3]) ** 2).sum() / (f_ref[:, :3] ** 2).sum())
        assert rms <= 1e-5, (cutoff, call, rms)
        assert np.abs(f[:, 3] - f_ref[:, 3]).max() < 1e-4, (cutoff, call)
        pe, vir = ref["stats"]["pe"], ref["stats"]["virial"]
        assert abs(s[0] - pe) <= 1e-5 * abs(pe), (cutoff, call, s[0], pe)
        assert abs(s[1] - vir) <= 1e-5 * abs(vir) + 1e-3, (cutoff, call, s[1], vir)


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


def test_noalloc_rejects_cutoffs_beyond_half_the_box():
    from rumd_b200 import capi, initconf
    lib = capi.lib()
    params = np.ascontiguousarray(initconf.lj_params(1, initconf.LJ), np.float32)  # rc = 2.5
    dummy = ctypes.c_void_p(16)  # never dereferenced: the argument checks come first
    box = np.array([6.0, 4.9, 6.0], np.float32)  # 2.5 > 4.9 / 2
    rc = lib.b2md_forces_noalloc(dummy, 100, box.ctypes.data_as(ctypes.c_void_p), 1,
                                 params.ctypes.data_as(ctypes.c_void_p), 0, dummy, dummy, None)
    assert rc == capi.B2MD_ERR_ARG
    assert b"half" in lib.b2md_last_error()

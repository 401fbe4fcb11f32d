"""The allocation-free entry point ngpu_run_static.

It serves callers that may not allocate device memory themselves (a fixed
device arena and budget owned by the host program, or latency limits that rule
out cudaMalloc / cudaFree): every internal buffer comes from one file-scope
device array in the library.  These tests call it through the C ABI with the
caller's own device buffers, twice in a row (the second call finds the first
call's leftovers in the shared array), and compare each result with the
regular entry point ngpu_run on the same inputs, using the FP32 parity bounds
of the other GPU tests: spike-time error <= 0.05 ms and max |dV| <= 0.1 mV
away from spikes.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from helpers import spike_time_error, subthreshold_error

pytestmark = pytest.mark.gpu

TOL_SPIKE_MS = 0.05
TOL_SUB_MV = 0.1


def _static_run(model, w, rec, stream_ptr):
    import torch
    from neurogpu_b200 import _ffi
    dev = torch.device("cuda", 0)
    params = torch.from_numpy(np.ascontiguousarray(w.params, dtype=np.float32)).to(dev)
    amps = torch.from_numpy(np.ascontiguousarray(w.amps, dtype=np.float32)).to(dev)
    dts = torch.from_numpy(w.dts).to(dev)
    out = torch.full((w.n_sets, w.n_stim, rec.size, w.nt), float("nan"), dtype=torch.float32, device=dev)
    rc = _ffi.lib().ngpu_run_static(
        model.handle, w.n_sets, C.c_void_p(params.data_ptr()), w.n_stim, w.nt,
        C.c_void_p(amps.data_ptr()), C.c_void_p(dts.data_ptr()), w.stim_node, w.stim_area,
        rec.size, _ffi.ptr(rec), w.v_init, C.c_void_p(out.data_ptr()), C.c_void_p(stream_ptr))
    _ffi.check("ngpu_run_static", rc)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_static_entry_point_matches_regular_run(ngpu_built):
    import torch
    from neurogpu_b200 import configs
    from neurogpu_b200.sim import Model, run
    w = configs.hh_active(n_sets=8, t_stop=50.0)
    rec = np.array([0, w.cell.n_nodes - 7], dtype=np.int32)
    model = Model(w.cell)
    ref = run(model, w.params, w.amps, w.dts, w.stim_node, w.stim_area, rec, w.v_init).astype(np.float64)
    stream = torch.cuda.current_stream().cuda_stream
    first = _static_run(model, w, rec, stream)
    second = _static_run(model, w, rec, stream)
    for got in (first, second):
        assert got.shape == ref.shape and np.all(np.isfinite(got))
        st, mism = spike_time_error(got.astype(np.float64), ref, w.dt)
        sub = subthreshold_error(got, ref, w.dt)
        assert mism == 0
        assert st <= TOL_SPIKE_MS
        assert sub <= TOL_SUB_MV
    assert np.array_equal(first, second)
    model.close()


def test_static_entry_point_ttpc_set_and_repeated_site(ngpu_built):
    """The TTPC mechanism set's kernel (the passive cable runs it), with a
    recording site requested twice, against ngpu_run; and a warm call leaves
    the device's free memory as it found it (no allocation)."""
    import torch
    from neurogpu_b200 import configs
    from neurogpu_b200.sim import Model, run
    w = configs.passive_cable(n_sets=6, t_stop=40.0)
    rec = np.array([0, 17, 17, w.cell.n_nodes - 1], dtype=np.int32)
    model = Model(w.cell)
    ref = run(model, w.params, w.amps, w.dts, w.stim_node, w.stim_area, rec, w.v_init).astype(np.float64)
    from neurogpu_b200 import _ffi
    stream = torch.cuda.current_stream().cuda_stream
    dev = torch.device("cuda", 0)
    params = torch.from_numpy(np.ascontiguousarray(w.params, dtype=np.float32)).to(dev)
    amps = torch.from_numpy(np.ascontiguousarray(w.amps, dtype=np.float32)).to(dev)
    dts = torch.from_numpy(w.dts).to(dev)
    outs = [torch.full((w.n_sets, w.n_stim, rec.size, w.nt), float("nan"), dtype=torch.float32, device=dev)
            for _ in range(2)]

    def call(out):
        _ffi.check("ngpu_run_static", _ffi.lib().ngpu_run_static(
            model.handle, w.n_sets, C.c_void_p(params.data_ptr()), w.n_stim, w.nt, C.c_void_p(amps.data_ptr()),
            C.c_void_p(dts.data_ptr()), w.stim_node, w.stim_area, rec.size, _ffi.ptr(rec), w.v_init,
            C.c_void_p(out.data_ptr()), C.c_void_p(stream)))
        torch.cuda.synchronize()
    call(outs[0])
    free_before = torch.cuda.mem_get_info()[0]
    call(outs[1])                                   # warm: every buffer is the caller's or the static array
    assert torch.cuda.mem_get_info()[0] == free_before
    first, second = (o.cpu().numpy() for o in outs)
    for got in (first, second):
        assert got.shape == ref.shape and np.all(np.isfinite(got))
        assert np.array_equal(got[:, :, 1], got[:, :, 2])
        assert float(np.max(np.abs(got - ref))) <= TOL_SUB_MV
    assert np.array_equal(first, second)
    model.close()


def test_static_entry_point_rejects_oversize_runs(ngpu_built):
    import torch
    from neurogpu_b200 import _ffi, configs
    from neurogpu_b200.sim import Model
    w = configs.hh_active(n_sets=100, t_stop=5.0)   # 300 instances > 256
    model = Model(w.cell)
    dummy = torch.zeros(16, device="cuda")
    rec = np.array([0], dtype=np.int32)
    p = C.c_void_p(dummy.data_ptr())
    rc = _ffi.lib().ngpu_run_static(model.handle, w.n_sets, p, w.n_stim, w.nt, p, p, 0, w.stim_area,
                                    1, _ffi.ptr(rec), w.v_init, p, None)
    assert rc == -1 and b"instances" in _ffi.lib().ngpu_last_error()
    w2 = configs.hh_active(n_sets=80, t_stop=500.0)  # 240 instances x 20000 samples: too big for the array
    rc = _ffi.lib().ngpu_run_static(model.handle, w2.n_sets, p, w2.n_stim, w2.nt, p, p, 0, w2.stim_area,
                                    1, _ffi.ptr(rec), w2.v_init, p, None)
    assert rc == -1 and b"bytes" in _ffi.lib().ngpu_last_error()
    model.close()

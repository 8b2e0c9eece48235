"""bmc_simulate_noalloc: the forward model for callers that cannot let a library allocate device memory
(a handler inside JAX/XLA, whose allocator has reserved the GPU; code under another framework's memory
budget; latency-bound pipelines, for which cudaMalloc/cudaFree synchronise the device).

Called through the C ABI, it must give bmc_simulate's results bit for bit (every chain chooses its own
Taylor degree and float32 switch point, so the cost-sorted warps of bmc_simulate and the launch-order
warps of noalloc give the same Z) on two calls in a row -- the second reuses the static scratch the first
left behind -- and refuse an event table larger than its static scratch. In a fresh process, noalloc
called first must leave the device's free memory unchanged across its second call. Named to be collected
last."""
import ctypes as C
import os
import subprocess
import sys
import textwrap
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def _inputs(torch, precision):
    import bench
    from bmc_b200.simulation import DeviceEvents, problem
    import bmc_oracle as O
    P, M0 = bench.voxel_params(96, 4, seed=11)
    ev = bench.pulse_train(7, n_pulses=3, n_samples=60)
    dev_ev = DeviceEvents(O.Events(*ev))
    pr = problem(96, 7, ev[0].shape[1], 4, 10, precision)
    dP = torch.as_tensor(P).cuda()
    dM = torch.as_tensor(M0).cuda()
    return pr, dP, dM, dev_ev


@pytest.mark.parametrize("precision", [0, 1], ids=["f64", "f32"])
def test_noalloc_matches_bmc_simulate_on_two_calls(cuda, precision):
    torch = cuda
    from bmc_b200 import _lib
    L = _lib.lib()
    pr, dP, dM, dev_ev = _inputs(torch, precision)
    ref = torch.empty((96, 7), dtype=torch.float64, device="cuda")
    _lib.check(L.bmc_simulate(pr, C.c_void_p(dP.data_ptr()), dev_ev.struct, C.c_void_p(dM.data_ptr()), None,
                              C.c_void_p(ref.data_ptr()), _lib.stream_handle()))
    outs = []
    for _ in range(2):
        z = torch.full((96, 7), float("nan"), dtype=torch.float64, device="cuda")
        _lib.check(L.bmc_simulate_noalloc(pr, C.c_void_p(dP.data_ptr()), dev_ev.struct, C.c_void_p(dM.data_ptr()),
                                          None, C.c_void_p(z.data_ptr()), _lib.stream_handle()))
        torch.cuda.synchronize()
        outs.append(z.cpu().numpy())
    want = ref.cpu().numpy()
    assert np.all(np.isfinite(want))
    for z in outs:
        np.testing.assert_array_equal(z, want)


def test_noalloc_refuses_a_table_above_its_static_scratch(cuda):
    from bmc_b200 import _lib
    L = _lib.lib()
    pr = _lib.Problem(1, 1000, 1000, 1, 4, 1, 0, 0)           # 1e6 records of 48 bytes > 32 MiB
    dummy = C.c_void_p(256)
    ev = _lib.Events(256, 256, 256, 256, 256, 256)
    st = L.bmc_simulate_noalloc(pr, dummy, ev, dummy, None, dummy, None)
    assert st == 1
    with pytest.raises(RuntimeError, match="exceeds its static scratch"):
        _lib.check(st)


_FRESH = textwrap.dedent("""
    import ctypes as C, sys
    import numpy as np, torch
    sys.path[:0] = [{root!r} + "/bmc-jax_b200", {root!r} + "/oracle", {root!r}]
    import bench, bmc_oracle as O
    from bmc_b200 import _lib
    from bmc_b200.simulation import DeviceEvents, problem
    L = _lib.lib()
    P, M0 = bench.voxel_params(64, 2, seed=5)
    ev = bench.pulse_train(9, n_pulses=2, n_samples=40)
    dev_ev = DeviceEvents(O.Events(*ev))
    pr = problem(64, 9, ev[0].shape[1], 2, 6, 0)
    dP, dM = torch.as_tensor(P).cuda(), torch.as_tensor(M0).cuda()
    z = [torch.empty((64, 9), dtype=torch.float64, device="cuda") for _ in range(3)]
    torch.cuda.synchronize()
    call = lambda out: _lib.check(L.bmc_simulate_noalloc(pr, C.c_void_p(dP.data_ptr()), dev_ev.struct,
                                  C.c_void_p(dM.data_ptr()), None, C.c_void_p(out.data_ptr()), _lib.stream_handle()))
    call(z[0])                                         # first call of the process: set-up on this device
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    call(z[1])
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    _lib.check(L.bmc_simulate(pr, C.c_void_p(dP.data_ptr()), dev_ev.struct, C.c_void_p(dM.data_ptr()), None,
                              C.c_void_p(z[2].data_ptr()), _lib.stream_handle()))
    torch.cuda.synchronize()
    a, b, c = (t.cpu().numpy() for t in z)
    assert free1 == free0, (free0, free1)
    assert np.array_equal(a, c) and np.array_equal(b, c) and np.all(np.isfinite(c))
    print("fresh ok", free0 - free1)
""")


def test_noalloc_first_in_a_fresh_process_allocates_nothing(cuda):
    """noalloc is the first library call of a new process; across its second call the device's free
    memory does not change, and both calls match bmc_simulate (called afterwards) bit for bit."""
    env = dict(os.environ)
    out = subprocess.run([sys.executable, "-c", _FRESH.format(root=str(ROOT))], capture_output=True, text=True,
                         timeout=600, env=env)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-4000:]
    assert "fresh ok 0" in out.stdout

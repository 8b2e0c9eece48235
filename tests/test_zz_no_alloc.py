"""bmc_simulate_noalloc: the forward model for callers that cannot let a library allocate device memory
(a handler inside JAX/XLA, whose allocator has reserved the GPU; code under another framework's memory
budget; latency-bound pipelines, for which cudaMalloc/cudaFree synchronise the device).

Called through the C ABI, it must give bmc_simulate's results (the tolerance of the other parity
tests, 1e-10) on two calls in a row -- the second reuses the static scratch the first left behind --
and refuse an event table larger than its static scratch. Named to be collected last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(torch, precision):
    import bench
    from bmc_b200 import _lib
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
        np.testing.assert_allclose(z, want, rtol=0, atol=1e-10)


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

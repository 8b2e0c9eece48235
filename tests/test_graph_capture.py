"""The forward entry points inside a CUDA graph: after one call of the same size on the capturing stream
(which sizes that stream's workspace and uploads the Taylor tables), bmc_simulate and bmc_uneven_simulate
enqueue only kernels and asynchronous device work, so a caller can capture them and replay the graph; the
replays reproduce the direct call bit for bit. A capture whose stream has no workspace of the size yet is
refused with a message (growing it would allocate inside the capture)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _forward_inputs(torch):
    import bench
    P, M0 = bench.voxel_params(96, 2, seed=3)
    ev = bench.pulse_train(9, n_pulses=2)
    return P, M0, ev


def test_bmc_simulate_replays_from_a_graph(cuda):
    torch = cuda
    from bmc_b200 import _lib
    from bmc_b200.simulation import DeviceEvents, problem
    P, M0, ev = _forward_inputs(torch)
    dP, dM = torch.as_tensor(P).cuda(), torch.as_tensor(M0).cuda()
    dev_ev = DeviceEvents.from_tensors(*[torch.as_tensor(a).cuda() for a in ev])
    n_off, n_ev = ev[0].shape
    pr = problem(M0.shape[0], n_off, n_ev, 2, 6, _lib.F64)
    L = _lib.lib()
    out = torch.empty((M0.shape[0], n_off), dtype=torch.float64, device="cuda")

    def call():
        _lib.check(L.bmc_simulate(pr, C.c_void_p(dP.data_ptr()), dev_ev.struct, C.c_void_p(dM.data_ptr()), None,
                                  C.c_void_p(out.data_ptr()), _lib.stream_handle()))

    call()
    torch.cuda.synchronize()
    want = out.clone()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with pytest.raises(RuntimeError, match="before capturing"):
            with torch.cuda.graph(torch.cuda.CUDAGraph(), stream=s):
                call()
        call()                                   # sizes the workspace of the capturing stream
        torch.cuda.synchronize()
        out.zero_()
        with torch.cuda.graph(g, stream=s):
            call()
    torch.cuda.current_stream().wait_stream(s)
    for _ in range(2):
        out.zero_()
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(out, want)


def test_uneven_simulate_replays_from_a_graph(cuda):
    torch = cuda
    from bmc_b200.fitting import Experiment
    from bmc_b200.simulation import SimEvent, SimParams, initial_state
    from bmc_b200.uneven import UnevenBatch
    import bench
    exps = bench.uneven_voxels(24, 5)[0]
    batch = UnevenBatch(exps)
    g0 = batch.groups[0]
    z = g0.run()
    torch.cuda.synchronize()
    want = z.clone()
    out = {}
    graph = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with torch.cuda.graph(graph, stream=s):
            out["z"] = g0.run()
    torch.cuda.current_stream().wait_stream(s)
    for _ in range(2):
        out["z"].zero_()
        graph.replay()
        torch.cuda.synchronize()
        assert torch.equal(out["z"], want)
    del Experiment, SimEvent, SimParams, initial_state

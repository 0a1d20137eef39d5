"""hp2d_cfl_dt_noalloc: the allocation-free timestep for callers that may not allocate GPU
memory while they run (a MEX gateway inside MATLAB, whose GPU memory pool owns the device).
Its scratch is a fixed array inside the library, so these checks compare it with
hp2d_cfl_dt on a context, bit for bit, over two calls in a row on different states:

* an 80-row urban grid (five 16-row blocks of partial maxima);
* a 8200 x 24 V-tilt (513 blocks, the last one 8 rows), so the final kernel's strided loop
  over more than 256 partials runs, with flag_adaptive_timestepping 1 and 0 (the wave-only
  and the speed-plus-celerity terms);
* a 65536-row V-tilt, the largest grid the scratch holds (4096 blocks).

This file is named to be collected last, and passes alone in a fresh process as well.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs_from_context(sf, case):
    """q_x, q_y and the three Hf pages as caller-owned CUDA tensors."""
    import torch
    ny, nx = case.shape
    qx = sf.download_native("qx")
    qy = sf.download_native("qy")
    hf = np.zeros((3, ny, nx), dtype=np.float32)
    hf[0] = sf.download_native("hfx")
    hf[1] = sf.download_native("hfy")
    cells = np.unique(case.outlet_rows.astype(np.int64) * nx + case.outlet_cols.astype(np.int64))
    hf[2].reshape(-1)[cells] = sf.download_native("hf3")
    dev = torch.device("cuda:0")
    return (torch.from_numpy(qx).to(dev), torch.from_numpy(qy).to(dev),
            torch.from_numpy(np.ascontiguousarray(hf)).to(dev))


def _noalloc_dt(L, case, sf, qx, qy, hf):
    import torch
    ny, nx = case.shape
    ts = C.c_double()
    vm = C.c_double()
    stream = torch.cuda.current_stream().cuda_stream
    st = L.hp2d_cfl_dt_noalloc(ny, nx, case.resolution, C.byref(sf.params), C.c_void_p(qx.data_ptr()),
                               C.c_void_p(qy.data_ptr()), C.c_void_p(hf.data_ptr()), C.c_void_p(stream),
                               C.byref(ts), C.byref(vm))
    assert st == 0, L.hp2d_noalloc_error().decode()
    return ts.value, vm.value


def _two_calls(case, steps_before=40, steps_between=25, **param_overrides):
    """Two consecutive calls, each against hp2d_cfl_dt on the same face fluxes and depths."""
    from hydropol2d_b200 import SurfaceFlow, _abi, build
    build.build()
    L = _abi.lib()
    params = dict(case.params, **param_overrides)
    sf = SurfaceFlow(*case.shape, case.resolution, "fp32", **params)
    case.apply(sf)
    sf.fused_steps(steps_before)
    results = []
    for call in range(2):
        d = sf.diag()
        ts = d["time_step"]
        sf.hydrology_step(ts)
        sf.li_step(ts)
        qx, qy, hf = _inputs_from_context(sf, case)
        ref_ts, ref_vm = sf.cfl_dt()
        got_ts, got_vm = _noalloc_dt(L, case, sf, qx, qy, hf)
        assert got_ts == ref_ts, (call, got_ts, ref_ts)
        assert got_vm == ref_vm, (call, got_vm, ref_vm)
        results.append((got_ts, got_vm))
        sf.set_clock(d["t"] + ref_ts, ref_ts, d["k"] + 1)
        sf.fused_steps(steps_between)   # a different state for the second call
    sf.close()
    return results


def test_noalloc_timestep_matches_context_timestep_twice():
    from hydropol2d_b200 import synthetic as S
    results = _two_calls(S.urban_case(80, 2.0, seed=21, hours=0.5))   # 80 rows: five 16-row blocks
    assert results[0] != results[1]
    assert results[0][1] > 0


@pytest.mark.parametrize("adaptive", [1, 0])
def test_noalloc_many_blocks_ragged_last_block(adaptive):
    from hydropol2d_b200 import synthetic as S
    case = S.vtilt_case(8200, 24, 10.0)   # 513 blocks of 16 rows, the last one 8 rows
    case.d0 = np.full(case.shape, 40.0)   # 40 mm everywhere: flowing, non-stagnant cells at once
    results = _two_calls(case, steps_before=60, steps_between=40, flag_adaptive_timestepping=adaptive)
    assert results[0] != results[1]
    assert results[1][1] > 0


def test_noalloc_largest_grid_it_holds():
    from hydropol2d_b200 import synthetic as S
    case = S.vtilt_case(65536, 8, 10.0)   # 4096 blocks: every partial slot of the scratch
    case.d0 = np.full(case.shape, 40.0)
    results = _two_calls(case, steps_before=30, steps_between=20)
    assert results[1][1] > 0


def test_noalloc_rejects_grids_beyond_its_scratch():
    from hydropol2d_b200 import _abi, build
    build.build()
    L = _abi.lib()
    p = _abi.default_params()
    ts = C.c_double()
    dummy = C.c_void_p(1)
    st = L.hp2d_cfl_dt_noalloc(65537, 4, 1.0, C.byref(p), dummy, dummy, dummy, None, C.byref(ts), None)
    assert _abi.STATUS[st] == "HP2D_INVALID_ARG"
    assert "65536 rows" in L.hp2d_noalloc_error().decode()


def test_noalloc_refuses_a_stream_under_capture():
    """The call reads its result back and synchronises, which a capturing stream does not allow:
    it refuses with HP2D_INVALID_ARG before touching the stream, and the capture stays valid."""
    import torch
    from hydropol2d_b200 import SurfaceFlow, _abi, build
    from hydropol2d_b200 import synthetic as S
    build.build()
    L = _abi.lib()
    case = S.vtilt_case(48, 32, 10.0)
    sf = SurfaceFlow(*case.shape, case.resolution, "fp32", **case.params)
    case.apply(sf)
    sf.fused_steps(10)
    ts = sf.diag()["time_step"]
    sf.hydrology_step(ts)
    sf.li_step(ts)   # the unfused step materialises the face depths the call reads
    qx, qy, hf = _inputs_from_context(sf, case)
    first = _noalloc_dt(L, case, sf, qx, qy, hf)   # resolves the scratch outside any capture
    x = torch.zeros(4, device="cuda:0")
    g = torch.cuda.CUDAGraph()
    ts = C.c_double()
    with torch.cuda.graph(g):
        stream = torch.cuda.current_stream().cuda_stream
        st = L.hp2d_cfl_dt_noalloc(*case.shape, case.resolution, C.byref(sf.params), C.c_void_p(qx.data_ptr()),
                                   C.c_void_p(qy.data_ptr()), C.c_void_p(hf.data_ptr()), C.c_void_p(stream),
                                   C.byref(ts), None)
        x.add_(1.0)
    assert _abi.STATUS[st] == "HP2D_INVALID_ARG"
    assert "captured" in L.hp2d_noalloc_error().decode()
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    assert x.cpu().tolist() == [2.0] * 4
    assert _noalloc_dt(L, case, sf, qx, qy, hf) == first   # still usable afterwards
    del g
    sf.close()

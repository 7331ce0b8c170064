"""mpm_mlp_predict_noalloc through the C ABI.

Callers that cannot allocate device memory when they need an inference (a
process whose caching allocator already holds the device, or a loop that must
not stall other streams on cudaMalloc/cudaFree) use this entry point; it stages
rows in a fixed scratch array of the library's device image. Checked here: the
same outputs as mpm_mlp_predict on two calls in a row, agreement with the
oracle's forward pass, no change in the device's free memory across calls
after the first, success while the rest of the device is reserved, the
capacity limit, and the device guard. Collected last so that it also runs
after every other GPU test in the same process."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rows(n, seed):
    rng = np.random.default_rng(seed)
    F = np.eye(3)[None] + 0.02 * rng.standard_normal((n, 3, 3))
    rows = np.zeros((n, 20), np.float32)
    rows[:, :9] = F.reshape(n, 9)
    rows[:, 9] = rng.uniform(0.5, 1.0, n)
    return rows


def _net():
    from mpm_snow_sim2d_b200.mlp import DEFAULT_WEIGHTS, Mlp
    return Mlp.load(DEFAULT_WEIGHTS)


def _noalloc(lib, net, rows):
    from mpm_snow_sim2d_b200._lib import fptr
    n = rows.shape[0]
    out = np.full((n, 10), np.nan, np.float32)
    st = lib.mpm_mlp_predict_noalloc(net._h, fptr(rows), n, rows.shape[1], fptr(out))
    return st, out


def test_noalloc_predict_matches_predict_and_oracle(gpu_lib):
    from mpm_snow_sim2d_b200 import _lib
    from oracle import mlp_ref
    lib = _lib.load()
    net = _net()
    params = net.params()
    for call, n in enumerate((5000, 777)):
        rows = _rows(n, seed=call)
        ref = net.predict(rows)
        st, out = _noalloc(lib, net, rows)
        assert st == 0, lib.mpm_mlp_last_error(net._h)
        # same kernel and inputs: equal up to 1e-6 of the output scale
        np.testing.assert_allclose(out, ref, rtol=0, atol=1e-6 * float(np.abs(ref).max()))
        # the oracle's FP64 forward pass with BF16 rounding where the kernel
        # stores BF16; differences come from FP32 accumulation order, the
        # hardware tanh and activations rounding to the other BF16 neighbour
        want, want_n = mlp_ref.forward(params, rows, net.norm)
        got_n = (out.astype(np.float64) - net.norm[2]) / net.norm[3]
        err = np.linalg.norm(got_n - want_n) / np.linalg.norm(want_n)
        print(f"call {call}: n={n} normalised-output relative L2 vs oracle {err:.2e}")
        assert err < 2e-2
    net.close()


def test_noalloc_capacity_limit(gpu_lib):
    from mpm_snow_sim2d_b200 import _lib
    lib = _lib.load()
    net = _net()
    n = 65537
    rows = np.zeros((n, 10), np.float32)
    rows[:, 9] = 1.0
    st, _ = _noalloc(lib, net, rows)
    assert st == 11  # MPM_ERR_CAPACITY
    assert b"65536" in lib.mpm_mlp_last_error(net._h)
    net.close()


def test_noalloc_allocates_nothing_after_first_call(gpu_lib):
    import torch
    from mpm_snow_sim2d_b200 import _lib
    lib = _lib.load()
    net = _net()
    dev = torch.cuda.current_device()
    st, first = _noalloc(lib, net, _rows(4096, seed=7))  # warm-up: set-up and module load
    assert st == 0, lib.mpm_mlp_last_error(net._h)
    torch.cuda.synchronize(dev)
    free0, _ = torch.cuda.mem_get_info(dev)
    for n, seed in ((4096, 7), (65536, 8), (1, 9), (3333, 10)):
        st, out = _noalloc(lib, net, _rows(n, seed))
        assert st == 0, lib.mpm_mlp_last_error(net._h)
        assert np.isfinite(out).all()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes across no-alloc calls"
    # with all but 1 GiB of the device held by torch's allocator, calls still succeed
    hold = None
    try:
        spare = free1 - (1 << 30)
        if spare > 0:
            hold = torch.empty(spare, dtype=torch.uint8, device=dev)
        for _ in range(2):
            st, out = _noalloc(lib, net, _rows(4096, seed=7))
            assert st == 0, lib.mpm_mlp_last_error(net._h)
            np.testing.assert_array_equal(out, first)
    finally:
        del hold
        torch.cuda.empty_cache()
    net.close()


def test_noalloc_refuses_another_current_device(gpu_lib):
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two visible devices")
    from mpm_snow_sim2d_b200 import _lib
    lib = _lib.load()
    net = _net()
    home = torch.cuda.current_device()
    rows = _rows(64, seed=3)
    try:
        torch.cuda.set_device(1 - home if home < 2 else 0)
        st, _ = _noalloc(lib, net, rows)
        assert st == 1  # MPM_ERR_INVALID_ARGUMENT, before any copy or launch
        assert b"device" in lib.mpm_mlp_last_error(net._h)
    finally:
        torch.cuda.set_device(home)
    net.close()

"""The learned position model: GPU forward/backward gradients against the CPU
oracle (float64), training lowers the loss, lookups stay exact, and what the
trained model gains over plain binary search."""
import ctypes as C

import numpy as np
import pytest

from conftest import to_dev
from oracle.oracle import model_gradients

pytestmark = pytest.mark.gpu

SEG_DTYPE = np.dtype([("a", np.float32), ("b", np.float32), ("err", np.uint32), ("first", np.uint32)])


def keys_dev(keys, bits):
    import torch

    a = np.ascontiguousarray(keys, dtype=np.uint64 if bits == 64 else np.uint32)
    return torch.from_numpy(a.view(np.int64 if bits == 64 else np.int32)).cuda()


def alloc_model(lib, segments):
    import torch

    return torch.zeros(int(lib.gpulsm_model_bytes(segments)), dtype=torch.uint8, device="cuda")


def parse_model(buf, segments):
    raw = buf.cpu().numpy()
    n, kmin, kmax = raw[:24].view(np.uint64)
    shift, nseg = raw[24:32].view(np.uint32)
    seg = raw[48:48 + (segments + 1) * 16].view(SEG_DTYPE)
    return int(n), int(kmin), int(kmax), int(shift), int(nseg), seg


def sorted_keys(bits, n, seed, clustered=False):
    rng = np.random.default_rng(seed)
    hi = (1 << 32) - 2 if bits == 32 else (1 << 44)
    if clustered:
        centers = rng.integers(0, hi - (1 << 20), 64, dtype=np.uint64)
        k = centers[rng.integers(0, 64, n)] + rng.integers(0, 1 << 16, n, dtype=np.uint64)
    else:
        k = rng.integers(0, hi, n, dtype=np.uint64)
    return np.unique(k)


@pytest.mark.parametrize("bits", [32, 64])
def test_gradients_match_cpu_oracle(gl, cuda, bits):
    import torch

    lib = gl.load()
    N = gl._native
    segments = 256
    keys = sorted_keys(bits, 1 << 16, 3 + bits)
    kd = keys_dev(keys, bits)
    model = alloc_model(lib, segments)
    # a partly trained model: init + 2 steps, so the residuals are not trivial
    N.check(lib.gpulsm_model_fit(kd.data_ptr(), keys.size, bits, segments, 2, model.data_ptr(), None, None))
    grad = torch.zeros(2 * segments, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    N.check(lib.gpulsm_model_gradients(kd.data_ptr(), keys.size, bits, segments, model.data_ptr(),
                                       grad.data_ptr(), loss.data_ptr(), None))
    n, kmin, kmax, shift, nseg, seg = parse_model(model, segments)
    assert n == keys.size and kmin == int(keys[0]) and kmax == int(keys[-1]) and 1 <= nseg <= segments
    ga, gb, l64 = model_gradients(keys, kmin, shift, nseg, seg["a"][:nseg].copy(), seg["b"][:nseg].copy())
    g = grad.cpu().numpy().reshape(segments, 2)[:nseg]
    # fp32 residuals against float64: relative 1e-3 of the largest gradient
    assert np.allclose(g[:, 0], ga, rtol=2e-3, atol=2e-3 * np.abs(ga).max() + 1e-6)
    assert np.allclose(g[:, 1], gb, rtol=2e-3, atol=2e-3 * np.abs(gb).max() + 1e-6)
    assert abs(float(loss.item()) - l64) <= 2e-3 * l64 + 1e-3


@pytest.mark.parametrize("bits,clustered", [(32, False), (64, False), (64, True)])
def test_training_lowers_loss_and_lookups_are_exact(gl, cuda, bits, clustered):
    import torch

    lib = gl.load()
    N = gl._native
    segments = 4096
    keys = sorted_keys(bits, 1 << 20, 17 + bits, clustered)
    kd = keys_dev(keys, bits)
    model = alloc_model(lib, segments)
    iters = 12
    hist = torch.zeros(iters + 1, dtype=torch.float32, device="cuda")
    N.check(lib.gpulsm_model_fit(kd.data_ptr(), keys.size, bits, segments, iters, model.data_ptr(),
                                 hist.data_ptr(), None))
    h = hist.cpu().numpy()
    assert h[-1] < h[0] and np.all(np.isfinite(h))
    rng = np.random.default_rng(5)
    q = np.concatenate([keys[rng.integers(0, keys.size, 50_000)],
                        rng.integers(0, int(keys[-1]) + 10, 50_000, dtype=np.uint64),
                        np.array([0, int(keys[0]), int(keys[-1]), int(keys[-1]) + 1], np.uint64)])
    if bits == 32:
        q = np.minimum(q, 0xFFFFFFFF)
    qd = keys_dev(q, bits)
    out = torch.zeros(q.size, dtype=torch.int64, device="cuda")
    N.check(lib.gpulsm_model_lower_bound(kd.data_ptr(), keys.size, bits, segments, model.data_ptr(),
                                         qd.data_ptr(), q.size, out.data_ptr(), None))
    want = np.searchsorted(keys, q, side="left")
    assert np.array_equal(out.cpu().numpy(), want)
    N.check(lib.gpulsm_binary_lower_bound(kd.data_ptr(), keys.size, bits, qd.data_ptr(), q.size,
                                          out.data_ptr(), None))
    assert np.array_equal(out.cpu().numpy(), want)


def test_trained_model_gain_over_binary_search(gl, cuda):
    """The search work the model saves: its windows vs a full binary search
    (probes per lookup), and the measured time of both on 2^24 queries."""
    import torch

    lib = gl.load()
    N = gl._native
    segments = 4096
    keys = sorted_keys(64, 1 << 24, 99)
    kd = keys_dev(keys, 64)
    model = alloc_model(lib, segments)
    N.check(lib.gpulsm_model_fit(kd.data_ptr(), keys.size, 64, segments, 12, model.data_ptr(), None, None))
    *_, nseg, seg = parse_model(model, segments)
    cnt = np.diff(seg["first"][: nseg + 1].astype(np.int64))
    window = np.minimum(2 * seg["err"][:nseg].astype(np.int64) + 3, cnt + 1)
    probes_model = float((np.log2(np.maximum(window, 1)) * cnt).sum() / cnt.sum())
    probes_binary = float(np.log2(keys.size))
    assert probes_model < probes_binary / 2
    q = keys_dev(np.random.default_rng(1).integers(0, int(keys[-1]), 1 << 24, dtype=np.uint64), 64)
    out = torch.empty(1 << 24, dtype=torch.int64, device="cuda")
    times = {}
    for name in ("model", "binary"):
        for rep in range(4):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            if name == "model":
                N.check(lib.gpulsm_model_lower_bound(kd.data_ptr(), keys.size, 64, segments, model.data_ptr(),
                                                     q.data_ptr(), q.numel(), out.data_ptr(), None))
            else:
                N.check(lib.gpulsm_binary_lower_bound(kd.data_ptr(), keys.size, 64, q.data_ptr(), q.numel(),
                                                      out.data_ptr(), None))
            e.record()
            torch.cuda.synchronize()
            times[name] = s.elapsed_time(e)
    print(f"\nprobes/lookup model={probes_model:.2f} binary={probes_binary:.2f}; "
          f"2^24 lower bounds: model {times['model']:.3f} ms, binary {times['binary']:.3f} ms")
    assert times["model"] < times["binary"]

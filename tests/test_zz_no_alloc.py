"""tamc_gpu_sa_run_noalloc: fast-mode simulated annealing whose replica words
live in a static device array instead of allocated buffers.  It must return
what tamc_gpu_sa_run returns, call after call (each call clears the words it
uses), reject shapes beyond its static scratch, and allocate nothing.

The file name sorts last so that the test also runs after every other GPU
test has used the device; it passes alone as well."""
import numpy as np
import pytest

from tamc_b200 import instances as gi

pytestmark = pytest.mark.gpu


def _device_buffers(torch, R, n):
    de = torch.full((R,), float("nan"), dtype=torch.float32, device="cuda")
    dp = torch.full((R, (n + 7) // 8), 0xA5, dtype=torch.uint8, device="cuda")  # garbage: must be overwritten
    return de, dp


def test_noalloc_matches_sa_run_on_consecutive_calls(tb, gpu):
    torch = pytest.importorskip("torch")
    calls = [  # (instance, replicas, seed): a larger anneal, then a smaller one over the same scratch
        (gi.sa_regular(700, 3, 5), 256, 11),
        (gi.sa_regular(300, 3, 6), 96, 12),
    ]
    betas = np.linspace(0.1, 6.0, 60, dtype=np.float32)
    db = torch.from_numpy(betas).cuda()
    stream = torch.cuda.Stream()
    runs = []
    for text, R, seed in calls:
        d = gpu.upload(tb.HostInstance.parse(text))
        runs.append((d, R, seed) + _device_buffers(torch, R, d.n))
    torch.cuda.synchronize()

    def call_all():
        # two calls back to back on one stream; the second reuses the scratch
        for d, R, seed, de, dp in runs:
            tb.sa_run_noalloc(d, db.data_ptr(), len(betas), R, seed, de.data_ptr(), dp.data_ptr(),
                              stream.cuda_stream)
        stream.synchronize()

    # first round: both shapes are new to the existing entry point (heuristic
    # tile); loading the kernels on first launch may take device memory
    call_all()
    free0 = torch.cuda.mem_get_info()[0]
    for d, R, seed, de, dp in runs:  # garbage again, so the repeat must rewrite every output
        de.fill_(float("nan"))
        dp.fill_(0xA5)
    torch.cuda.synchronize()
    call_all()
    call_all()
    # the defining property: calls after the first take no device memory
    assert torch.cuda.mem_get_info()[0] == free0
    for d, R, seed, de, dp in runs:
        e_ref, packed_ref = tb.sa_run(d, betas, R, 1, seed)
        assert np.array_equal(de.cpu().numpy().view(np.uint32), e_ref.view(np.uint32))
        assert np.array_equal(dp.cpu().numpy(), packed_ref)


def test_noalloc_rejects_shapes_beyond_static_scratch(tb, gpu):
    torch = pytest.importorskip("torch")
    text = gi.sa_regular(2000, 3, 7)
    d = gpu.upload(tb.HostInstance.parse(text))
    # ceil(R/32) * n * 4 bytes: 32 * 2000 * 4 fits, 1024 * 2000 * 4 does not
    assert 32 * 2000 * 4 <= tb.SA_NOALLOC_SCRATCH_BYTES < 1024 * 2000 * 4
    R = 32 * 1024
    betas = torch.ones(4, dtype=torch.float32, device="cuda")
    de, dp = _device_buffers(torch, 1, 2000)
    for R in (32 * 1024, 0xFFFFFFFF):  # the largest count must not wrap to a small need
        with pytest.raises(tb.TamcError) as err:
            tb.sa_run_noalloc(d, betas.data_ptr(), 4, R, 1, de.data_ptr(), dp.data_ptr())
        assert err.value.code == -1 and "static scratch" in str(err.value)


def test_noalloc_rejects_instances_beyond_shared_memory(tb, gpu):
    """A ring of 200000 sites fits the static scratch at 32 replicas (800 KB of
    words) but not the annealing kernel's shared memory: the call must fail
    with UNSUPPORTED, as tamc_gpu_sa_run does, before it queues any work."""
    torch = pytest.importorskip("torch")
    n = 200_000
    i = np.arange(n)
    nb = np.sort(np.stack([(i - 1) % n, (i + 1) % n], 1), axis=1)
    rp = np.arange(0, 2 * n + 1, 2, dtype=np.uint32)
    h = tb.HostInstance.from_csr(rp, nb.ravel().astype(np.uint32), np.ones(2 * n, np.float32),
                                 np.zeros(n, np.float32))
    d = gpu.upload(h)
    betas = torch.ones(4, dtype=torch.float32, device="cuda")
    de, dp = _device_buffers(torch, 32, n)
    torch.cuda.synchronize()
    with pytest.raises(tb.TamcError) as err:
        tb.sa_run_noalloc(d, betas.data_ptr(), 4, 32, 1, de.data_ptr(), dp.data_ptr())
    assert err.value.code == -7 and "too large" in str(err.value)
    torch.cuda.synchronize()
    assert torch.isnan(de).all()  # nothing ran
    with pytest.raises(tb.TamcError) as err:
        tb.sa_run(d, np.ones(4, np.float32), 32, 1, 1)
    assert err.value.code == -7

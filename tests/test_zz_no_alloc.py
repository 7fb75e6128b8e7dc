"""silk_ccd_batch_noalloc: the CCD batch on caller-owned device buffers whose
only working memory is a static device array.  Two calls in a row must give
the same hits and times of impact as silk_ccd_batch (exactly: both run the
same search in the same arithmetic), the second-pass storage must be
exercised, nothing may be allocated on the device by the second call, and
sizes beyond the scratch limits are refused before any device work.

The file name sorts last so that the test also runs after every other test
of the session; it passes alone as well."""
import numpy as np
import pytest

from silk_physics_b200 import native as N

pytestmark = pytest.mark.gpu

# Identical results are required: both entry points run ccd_batch_kernel's
# search with the same arguments.
TOI_TOL = 0.0


def _queries(rng, n, vf):
    base = rng.uniform(-1, 1, (n, 4, 3)).astype(np.float32)
    if vf:
        base[:, 1:, 2] = 0.0
        base[:, 0, 2] = rng.uniform(0.001, 0.2, n)
    motion = rng.normal(0, 0.4, (n, 4, 3)).astype(np.float32)
    motion[:, 0, 2] -= rng.uniform(0, 0.6, n)
    x = np.concatenate([base, base + motion], axis=1)
    return np.ascontiguousarray(x.reshape(n, 24), dtype=np.float32)


@pytest.mark.parametrize("vf", [True, False])
def test_noalloc_matches_ccd_batch_twice(vf):
    import torch

    rng = np.random.default_rng(142 if vf else 143)
    n = 3000
    x = _queries(rng, n, vf)
    err = np.array([4.053116e-06 if vf else 3.814698e-06] * 3, np.float32)
    ms = rng.choice([0.0, 1e-4, 1e-3], n).astype(np.float32)
    ref_hit, ref_toi, ref_tup = N.ccd_batch(vf, x, err, ms, 1e-6, 4096, 1.0)

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    xd = torch.from_numpy(x).to(dev)
    msd = torch.from_numpy(ms).to(dev)
    hit = torch.full((n,), -1, dtype=torch.int32, device=dev)
    toi = torch.full((n,), -1.0, dtype=torch.float32, device=dev)
    tup = torch.full((n,), -1.0, dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(device=dev)

    # First call: one-time setup (scratch address lookup) and a full run.
    st, spilled = N.ccd_batch_noalloc(vf, xd.data_ptr(), n, err, msd.data_ptr(),
                                      hit.data_ptr(), toi.data_ptr(), tup.data_ptr(),
                                      stream=stream.cuda_stream)
    assert st, st.to_string()
    first = (hit.cpu().numpy().copy(), toi.cpu().numpy().copy(), tup.cpu().numpy().copy())

    # Second call on fresh outputs; device free memory must not change.
    hit.fill_(-1)
    toi.fill_(-1.0)
    tup.fill_(-1.0)
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info(dev)
    st2, spilled2 = N.ccd_batch_noalloc(vf, xd.data_ptr(), n, err, msd.data_ptr(),
                                        hit.data_ptr(), toi.data_ptr(), tup.data_ptr(),
                                        stream=stream.cuda_stream)
    free_after, _ = torch.cuda.mem_get_info(dev)
    assert st2, st2.to_string()
    assert free_after == free_before
    second = (hit.cpu().numpy(), toi.cpu().numpy(), tup.cpu().numpy())

    print(f"{'VF' if vf else 'EE'}: {int(ref_hit.sum())} hits of {n}, "
          f"{spilled} queries ran in the second pass")
    assert spilled > 0 and spilled2 == spilled
    for g_hit, g_toi, g_tup in (first, second):
        np.testing.assert_array_equal(g_hit.astype(bool), ref_hit)
        np.testing.assert_allclose(g_toi, ref_toi, rtol=0, atol=TOI_TOL)
        np.testing.assert_allclose(g_tup, ref_tup, rtol=0, atol=TOI_TOL)


def test_noalloc_refuses_sizes_beyond_limits():
    import torch

    dev = torch.device("cuda", 0)
    buf = torch.zeros(24, dtype=torch.float32, device=dev)
    ibuf = torch.zeros(1, dtype=torch.int32, device=dev)
    err = np.full(3, 4e-6, np.float32)
    p, ip = buf.data_ptr(), ibuf.data_ptr()
    # Checked before any device work, so the small buffers are never read.
    for n, max_iter in ((N.CCD_NOALLOC_MAX_QUERIES + 1, 4096),
                        (1, N.CCD_NOALLOC_MAX_ITER + 1), (1, 0)):
        st, _ = N.ccd_batch_noalloc(True, p, n, err, p, ip, p, None, max_iter=max_iter)
        assert not st and st.code == N.ErrorCode.InvalidConfig
    # Host memory is refused too.
    host = np.zeros(24, np.float32)
    st, _ = N.ccd_batch_noalloc(True, host.ctypes.data, 1, err, p, ip, p, None)
    assert not st and st.code == N.ErrorCode.InvalidConfig
    # n == 0 is a valid no-op.
    st, spilled = N.ccd_batch_noalloc(True, p, 0, err, p, ip, p, None)
    assert st and spilled == 0

"""les_step_host: the time step with the velocity state in host memory equals
les_upload + les_step + les_download bit for bit, in both precisions, with
page-locked and pageable arrays, over one chunk of levels and several; the
arrays are the step's inputs; every other entry point orders itself after
the copies back."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _les(precision, nx, ny, nz):
    from new_repo_b200 import LES, RunParams, log_law_noise

    p = RunParams(nx=nx, ny=ny, nz=nz, dt=2e-4, sgs_model="dyn_LagScaleDep", dyn_init=2, cs_count=2)
    les = LES(p, precision=precision)
    les.set_initial_conditions(*log_law_noise(p, seed=5))
    return les


def _host_arrays(shape, mem):
    """u, v, w and the diagnostics buffer: page-locked by torch, numpy arrays
    page-locked through les_host_register, or plain pageable numpy arrays."""
    import torch

    if mem == "pinned":
        t = [torch.empty(shape, dtype=torch.float64, pin_memory=True) for _ in range(3)]
        t.append(torch.empty(4, dtype=torch.float64, pin_memory=True))
        return [x.numpy() for x in t[:3]], t[3].numpy(), t  # keep the tensors alive
    arrs = [np.empty(shape) for _ in range(3)] + [np.empty(4)]
    return arrs[:3], arrs[3], arrs


def _register(lib, arrs, on):
    import ctypes as C
    from new_repo_b200.les import check

    for a in arrs:
        if on:
            check(lib.les_host_register(C.c_void_p(a.ctypes.data), C.c_size_t(a.nbytes)))
        else:
            check(lib.les_host_unregister(C.c_void_p(a.ctypes.data)))


# (nx, ny, nz): one 16 MB chunk of levels; a 256 x 256 plane makes 32-level
# chunks, so 42 levels take two
GRIDS = [(64, 32, 24), (256, 256, 40)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("grid,mem", [(GRIDS[0], "pinned"), (GRIDS[0], "pageable"), (GRIDS[1], "pinned"),
                                      (GRIDS[1], "registered")])
def test_host_step_equals_the_device_step(gpu, precision, grid, mem):
    nx, ny, nz = grid
    ref, hs = _les(precision, *grid), _les(precision, *grid)
    (u, v, w), diag, keep = _host_arrays((nz + 2, ny, nx), mem)
    if mem == "registered":
        _register(hs.lib, keep, True)
    for a, n in zip((u, v, w), "uvw"):
        a[...] = hs.download(n)
    K = 5
    hs.step_host(u.ctypes.data, v.ctypes.data, w.ctypes.data, diag.ctypes.data, n=K)
    hs.sync()
    ref.step(K)
    for a, n in zip((u, v, w), "uvw"):
        r = ref.download(n)
        np.testing.assert_array_equal(a, r, err_msg=n)
        np.testing.assert_array_equal(hs.download(n), r, err_msg=n)
    np.testing.assert_array_equal(diag, np.asarray(ref.diagnostics(), dtype=np.float64))
    assert hs.jt == ref.jt and hs.jt_total == ref.jt_total

    # the host arrays are the inputs: a change made on the host between
    # steps is what the next step starts from
    u[1:-1] *= 1.01
    ref.upload("u", u)
    hs.step_host(u.ctypes.data, v.ctypes.data, w.ctypes.data, None, n=2)
    ref.step(2)
    # no sync: download orders itself after the copies back
    got = hs.download("v")
    hs.sync()
    for a, n in zip((u, v, w), "uvw"):
        np.testing.assert_array_equal(a, ref.download(n), err_msg=n)
    np.testing.assert_array_equal(got, v)
    if mem == "registered":
        _register(hs.lib, keep, False)
    del keep
    ref.close()
    hs.close()


def test_entry_points_after_host_step_see_its_copies(gpu, tmp_path):
    """Without les_sync, a checkpoint write and a precision switch right after
    les_step_host order themselves after its copies back: the checkpoint is
    byte-equal to the device-resident run's and the switched state holds the
    stepped fields."""
    grid = (64, 32, 24)
    nx, ny, nz = grid
    ref, hs = _les("fp64", *grid), _les("fp64", *grid)
    (u, v, w), diag, keep = _host_arrays((nz + 2, ny, nx), "pinned")
    for a, n in zip((u, v, w), "uvw"):
        a[...] = hs.download(n)
    hs.step_host(u.ctypes.data, v.ctypes.data, w.ctypes.data, diag.ctypes.data, n=3)
    ref.step(3)
    (tmp_path / "hs").mkdir()
    (tmp_path / "ref").mkdir()
    f_hs = hs.checkpoint_out(tmp_path / "hs")
    f_ref = ref.checkpoint_out(tmp_path / "ref")
    assert f_hs.read_bytes() == f_ref.read_bytes()
    hs.step_host(u.ctypes.data, v.ctypes.data, w.ctypes.data, diag.ctypes.data, n=2)
    ref.step(2)
    hs.set_precision("mixed")
    ref.set_precision("mixed")
    for n in ("u", "v", "w", "rhsx", "cs_opt2"):
        np.testing.assert_array_equal(hs.download(n), ref.download(n), err_msg=n)
    hs.sync()
    for a, n in zip((u, v, w), "uvw"):
        np.testing.assert_array_equal(a.astype(np.float32).astype(np.float64), hs.download(n), err_msg=n)
    del keep
    ref.close()
    hs.close()

"""mg_fftconv_compute_noalloc (the allocation-free FFTConv2D.compute on a static device scratch) through the C
ABI, against the object path mg_fftconv_create / set_kernels / compute on the same inputs. Two calls in a row
with different grids, then the limits: an FFT side above the scratch's maximum and host arrays are rejected
with MG_ERR_ARGUMENT. Collected last so that it also runs after every other test in one process."""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "lib-magnet_b200", "libmagnet_b200.so")
MG_OK, MG_ERR_ARGUMENT = 0, 1

P = ctypes.c_void_p
F32 = ctypes.c_float


def load():
    lib = ctypes.CDLL(LIB)
    lib.mg_last_error.restype = ctypes.c_char_p
    lib.mg_fftconv_compute_noalloc.argtypes = [P, P, ctypes.c_int, ctypes.c_int, P, ctypes.c_int64, F32, F32, F32,
                                               ctypes.c_int, P, P]
    lib.mg_fftconv_noalloc_max_side.restype = ctypes.c_int
    lib.mg_fftconv_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(P)]
    lib.mg_fftconv_set_kernels.argtypes = [P, P, P, ctypes.c_int64, ctypes.c_int64]
    lib.mg_fftconv_compute.argtypes = [P, P, ctypes.c_int64, F32, F32, F32, ctypes.c_int, P, P]
    lib.mg_fftconv_destroy.argtypes = [P]
    return lib


def case(seed, n, spread):
    """a layout, its grid (magnet/tsne.py:30-46) and the kernel spectra (magnet/tsne.py:48-71)"""
    rng = np.random.default_rng(seed)
    Y = rng.uniform(-spread, spread, (n, 2)).astype(np.float32)
    xmin, ymin, width, n_boxes = O.grid(Y)
    M, K1h, K2h = O.kernel_spectra(n_boxes, width, 3)
    return Y, (xmin, ymin, width, n_boxes), M, K1h, K2h


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def noalloc(lib, K1, K2, M, Yd, grid, sq, Fd):
    xmin, ymin, width, n_boxes = grid
    return lib.mg_fftconv_compute_noalloc(K1.data_ptr(), K2.data_ptr(), M, 3, Yd.data_ptr(), Yd.shape[0], xmin, ymin,
                                          width, n_boxes, sq.data_ptr(), Fd.data_ptr())


def object_path(lib, Y, grid, M, K1h, K2h):
    xmin, ymin, width, n_boxes = grid
    h = P()
    assert lib.mg_fftconv_create(M, 3, ctypes.byref(h)) == MG_OK, lib.mg_last_error()
    try:
        assert lib.mg_fftconv_set_kernels(h, K1h.ctypes.data, K2h.ctypes.data, K1h.shape[0], K1h.shape[1]) == MG_OK
        F = np.empty_like(Y)
        sq = np.zeros(1, np.float32)
        assert lib.mg_fftconv_compute(h, Y.ctypes.data, Y.shape[0], xmin, ymin, width, n_boxes, sq.ctypes.data,
                                      F.ctypes.data) == MG_OK, lib.mg_last_error()
    finally:
        lib.mg_fftconv_destroy(h)
    return float(sq[0]), F


def test_noalloc_matches_object_path_two_calls(cuda):
    import torch
    lib = load()
    assert lib.mg_fftconv_noalloc_max_side() == 512
    cases = [case(1, 3000, 15.0), case(2, 5000, 28.0)]
    assert cases[0][2] != cases[1][2] and max(c[2] for c in cases) <= 512
    # every device array exists before the first call: the calls themselves allocate nothing
    dev_args = [(dev(K1h), dev(K2h), dev(Y), torch.zeros(1, dtype=torch.float32, device=cuda),
                 torch.zeros(Y.shape, dtype=torch.float32, device=cuda)) for Y, _, _, K1h, K2h in cases]
    torch.cuda.synchronize()
    for (Y, grid, M, _, _), (K1, K2, Yd, sq, Fd) in zip(cases, dev_args):
        assert noalloc(lib, K1, K2, M, Yd, grid, sq, Fd) == MG_OK, lib.mg_last_error()
    torch.cuda.synchronize()
    for (Y, grid, M, K1h, K2h), (_, _, _, sq, Fd) in zip(cases, dev_args):
        s_obj, F_obj = object_path(lib, Y, grid, M, K1h, K2h)
        s_na, F_na = float(sq.item()), Fd.cpu().numpy()
        assert np.isfinite(F_na).all()
        # the spread's atomics sum in arrival order, and the object path runs the in-place engine (fft3.cuh) when M
        # has an in-place plan while this entry point always runs the one-radix engine (fft.cuh), so the two agree
        # to FP32 rounding, a few 1e-5 of max |F|; the bar is the FFT pass's parity tolerance against the
        # reference, 1e-4 relative
        assert abs(s_na - s_obj) <= 1e-4 * abs(s_obj), (s_na, s_obj)
        assert np.abs(F_na - F_obj).max() <= 1e-4 * np.abs(F_obj).max()
        # and both against the FP64 restatement of the pass
        s64, F64 = O.fft_repulsion_fp64(Y, *grid, n_interp=3)
        assert abs(s_na - s64) <= 1e-4 * abs(s64)
        assert np.abs(F_na - F64).max() <= 1e-4 * np.abs(F64).max()


def test_noalloc_repeat_keeps_free_memory(cuda):
    import torch
    lib = load()
    Y, grid, M, K1h, K2h = case(3, 4000, 20.0)
    K1, K2, Yd = dev(K1h), dev(K2h), dev(Y)
    sq = [torch.zeros(1, dtype=torch.float32, device=cuda) for _ in range(2)]
    Fd = [torch.zeros(Y.shape, dtype=torch.float32, device=cuda) for _ in range(2)]
    assert noalloc(lib, K1, K2, M, Yd, grid, sq[0], Fd[0]) == MG_OK, lib.mg_last_error()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    assert noalloc(lib, K1, K2, M, Yd, grid, sq[1], Fd[1]) == MG_OK, lib.mg_last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    # the spread sums with atomics in arrival order, so repeats agree to FP32 rounding (a few 1e-5 of max |F|,
    # F being a difference of large interpolated sums), not bit for bit; the bar is the 1e-4 parity tolerance
    assert abs(sq[0].item() - sq[1].item()) <= 1e-4 * abs(sq[0].item())
    assert (Fd[0] - Fd[1]).abs().max().item() <= 1e-4 * Fd[0].abs().max().item()


def test_noalloc_limits(cuda):
    import torch
    lib = load()
    # M above the scratch's maximum: n_boxes * n_interp = 540 needs M >= 540
    Y, _, _, _, _ = case(4, 100, 10.0)
    Yd = dev(Y)
    M = 1080
    K = torch.zeros((M, M // 2 + 1), dtype=torch.float32, device=cuda)
    sq = torch.zeros(1, dtype=torch.float32, device=cuda)
    Fd = torch.zeros(Y.shape, dtype=torch.float32, device=cuda)
    rc = lib.mg_fftconv_compute_noalloc(K.data_ptr(), K.data_ptr(), M, 3, Yd.data_ptr(), 100, -10.0, -10.0, 0.1, 180,
                                        sq.data_ptr(), Fd.data_ptr())
    assert rc == MG_ERR_ARGUMENT and b"exceeds the maximum FFT side 512" in lib.mg_last_error()
    # host arrays are not staged
    Y, grid, M, K1h, K2h = case(5, 500, 10.0)
    K1, K2 = dev(K1h), dev(K2h)
    F = np.zeros_like(Y)
    rc = lib.mg_fftconv_compute_noalloc(K1.data_ptr(), K2.data_ptr(), M, 3, Y.ctypes.data, Y.shape[0], grid[0],
                                        grid[1], grid[2], grid[3], sq.data_ptr(), F.ctypes.data)
    assert rc == MG_ERR_ARGUMENT and b"must be device memory" in lib.mg_last_error()
    # a grid larger than M
    Fd = torch.zeros(Y.shape, dtype=torch.float32, device=cuda)
    rc = lib.mg_fftconv_compute_noalloc(K1.data_ptr(), K2.data_ptr(), M, 3, dev(Y).data_ptr(), Y.shape[0], grid[0],
                                        grid[1], grid[2], M, sq.data_ptr(), Fd.data_ptr())
    assert rc == MG_ERR_ARGUMENT

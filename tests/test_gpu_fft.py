"""FFT-interpolated repulsion on the device against the reference (FFTConv2D.compute of the compiled reference,
golden vectors it produced) and against the FP64 all-pairs oracle. Tolerance: sumQ and F within 1e-4 relative
(F as a norm over the points) of the reference; the interpolation error against the exact sums within the
reference's own bounds (tests/test_magnet.py:230-231)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-4


def fftconv(mg, Y, grid, ni):
    xmin, ymin, width, nb = grid
    M, K1, K2 = O.kernel_spectra(int(nb), float(width), ni)
    conv = mg.FFTConv2D(M, ni)
    conv.set_kernels(K1, K2)
    return conv.compute(np.ascontiguousarray(Y, np.float32), float(xmin), float(ymin), float(width), int(nb))


@pytest.mark.parametrize("ni", [5, 3])
def test_reference_test_vector(mg, golden, ni):
    g = golden("fft_small.npz")
    sq, F = fftconv(mg, g["Y"], g[f"grid_{ni}"], ni)
    assert abs(sq - g[f"sumQ_{ni}"]) / g[f"sumQ_{ni}"] < TOL
    assert np.linalg.norm(F - g[f"F_{ni}"]) / np.linalg.norm(g[f"F_{ni}"]) < TOL
    assert abs(sq - g["sumQ_exact"]) / g["sumQ_exact"] < 1e-3
    assert np.linalg.norm(F - g["F_exact"]) / np.linalg.norm(g["F_exact"]) < 2e-2


def test_clustered_layout(mg, golden):
    g = golden("fft_small.npz")
    sq, F = fftconv(mg, g["Yc"], g["grid_c"], 3)
    assert abs(sq - g["sumQ_c"]) / g["sumQ_c"] < TOL
    assert np.linalg.norm(F - g["F_c"]) / np.linalg.norm(g["F_c"]) < TOL


@pytest.mark.parametrize("n,scale", [(20000, 25.0), (70000, 31.0)])
def test_against_compiled_reference(mg, ref, n, scale):
    if ref is None:
        pytest.skip("reference module not built")
    rng = np.random.default_rng(n)
    Y = (rng.standard_t(3, (n, 2)) * scale / 3).astype(np.float32)
    grid = O.grid(Y)
    M, K1, K2 = O.kernel_spectra(grid[3], grid[2], 3)
    conv_r = ref.FFTConv2D(M, 3)
    conv_r.set_kernels(K1, K2)
    sq_r, F_r = conv_r.compute(Y, grid[0], grid[1], grid[2], grid[3], -1)
    sq, F = fftconv(mg, Y, grid, 3)
    F_r = np.asarray(F_r)
    assert abs(sq - sq_r) / sq_r < TOL
    assert np.linalg.norm(F - F_r) / np.linalg.norm(F_r) < TOL


def test_precision_against_fp64_all_pairs(mg, ref):
    """the precision study at n = 10,000: the device's FP32 spread / FFT / gather (FP64 Z) against the direct FP64
    sums, beside the same pass with an FP64 spread / convolution / gather (the interpolation's own error) and the
    reference's FFTConv2D (its FP32 pocketfft), all on the same grid; the device's FP32 arithmetic adds nothing
    measurable to the interpolation error, which stays within the reference's own bounds"""
    rng = np.random.default_rng(7)
    Y = (rng.normal(0, 20, (10000, 2))).astype(np.float32)
    grid = O.grid(Y)
    sq, F = fftconv(mg, Y, grid, 3)
    sq_e, F_e = O.exact_repulsion(Y)
    sq_64, F_64 = O.fft_repulsion_fp64(Y, *grid, n_interp=3)
    err = lambda s, f: (abs(s - sq_e) / sq_e, np.linalg.norm(f - F_e) / np.linalg.norm(F_e))
    rows = {"device FP32": err(sq, F), "FP64 grid": err(sq_64, F_64)}
    if ref is not None:
        M, K1, K2 = O.kernel_spectra(grid[3], grid[2], 3)
        conv = ref.FFTConv2D(int(M), 3)
        conv.set_kernels(K1, K2)
        sq_r, F_r = conv.compute(Y, *grid, -1)
        rows["reference FP32"] = err(sq_r, np.asarray(F_r))
    for k, (e_s, e_f) in rows.items():
        print("%s: sumQ rel err %.3e, F rel RMS err %.3e" % (k, e_s, e_f))
    e_s, e_f = rows["device FP32"]
    assert e_s < 1e-3 and e_f < 2e-2
    assert abs(e_f - rows["FP64 grid"][1]) < 1e-4 and abs(e_s - rows["FP64 grid"][0]) < 1e-4


def test_device_tensors_in_place(mg, golden):
    import torch
    g = golden("fft_small.npz")
    xmin, ymin, width, nb = g["grid_3"]
    M, K1, K2 = O.kernel_spectra(int(nb), float(width), 3)
    conv = mg.FFTConv2D(M, 3)
    conv.set_kernels(K1, K2)
    Yd = torch.from_numpy(g["Y"]).cuda()
    sq, Fd = conv.compute(Yd, float(xmin), float(ymin), float(width), int(nb))
    assert Fd.is_cuda
    assert np.linalg.norm(Fd.cpu().numpy() - g["F_3"]) / np.linalg.norm(g["F_3"]) < TOL


def test_grid_too_large_raises(mg):
    conv = mg.FFTConv2D(120, 3)
    with pytest.raises(RuntimeError, match="grid larger than the buffer"):
        conv.compute(np.zeros((10, 2), np.float32), 0.0, 0.0, 0.7, 60)


def spectra_on_torus(M, n_boxes, width, ni, dof=1.0):
    """the kernel spectra of FFTRepulsion2D._kernels (magnet/tsne.py:48-71) on a given M torus (M >= 2N): the
    convolution of the N live nodes is the same for every such M"""
    import scipy.fft as fft
    delta = width / ni
    off = np.arange(M)
    off = np.where(off <= M // 2, off, off - M).astype(np.float64) * delta
    base = 1.0 + (off[:, None] ** 2 + off[None, :] ** 2) / dof
    K1 = (base ** (-dof)).astype(np.float32)
    K2 = (base ** (-dof - 1.0)).astype(np.float32)
    h = lambda K: np.ascontiguousarray(np.ascontiguousarray(fft.rfft2(K), dtype=np.complex64).real)
    return h(K1), h(K2)


# FFT sides covering the in-place engine's plan shapes: two stages (120 = 8 x 15), three with an even last radix
# and padding (512 = 8 x 8 x 8, 1000 = 10 x 10 x 10), three with an odd last radix (4320 = 18 x 16 x 15), four
# stages (2187 = 9 x 9 x 9 x 3; 8192 = 16 x 16 x 2 x 16, padded), and a 5-smooth side without a plan, which runs
# the one-radix engine (3125 = 5^5)
@pytest.mark.parametrize("M", [120, 512, 1000, 2187, 3125, 4320, 8192])
def test_fft_sides_against_fp64(mg, M):
    ni, nb, width = 3, 20, 0.7
    rng = np.random.default_rng(M)
    Y = rng.uniform(0.01, nb * width - 0.01, (3000, 2)).astype(np.float32)
    K1, K2 = spectra_on_torus(M, nb, width, ni)
    conv = mg.FFTConv2D(M, ni)
    conv.set_kernels(K1, K2)
    sq, F = conv.compute(Y, 0.0, 0.0, width, nb)
    sq64, F64 = O.fft_repulsion_fp64(Y, 0.0, 0.0, width, nb, n_interp=ni)
    assert abs(sq - sq64) / sq64 < TOL
    assert np.linalg.norm(F - F64) / np.linalg.norm(F64) < TOL


@pytest.mark.parametrize("ni", [2, 4, 7])
def test_other_interpolation_orders_against_fp64(mg, ni):
    """FFTConv2D at interpolation orders other than 3 and 5 (the device instantiates 1-8) against the FP64
    restatement of the pass, which matches the reference's FFTConv2D at these orders (tests/test_oracle.py)"""
    rng = np.random.default_rng(ni)
    Y = rng.normal(0, 8, (2500, 2)).astype(np.float32)
    grid = O.grid(Y)
    sq, F = fftconv(mg, Y, grid, ni)
    sq_o, F_o = O.fft_repulsion_fp64(Y, *grid, ni)
    assert abs(sq - sq_o) / abs(sq_o) < 1e-4
    assert np.linalg.norm(F - F_o) / np.linalg.norm(F_o) < 1e-4

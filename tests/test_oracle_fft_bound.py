"""How far the oracle's f32 FFT convolution can sit from any other f32 FFT
convolution, rustfft's included.

The reference's convolution (CachedConvolver, src/compute/fft.rs:288-393) runs
its complex f32 transforms through the third-party crate rustfft ("6.2",
Cargo.toml:29), whose source is not available here; the oracle restates the
same circular convolution with its own Stockham FFT.  Both compute the exact
DFT convolution with f32 rounding errors.  This test measures the oracle's
error against an FP64 pocketfft convolution (numpy) on the 512x512
multispecies workload's nine kernels, so the gap to rustfft is bounded by the
oracle's measured error plus rustfft's own, of the same order for an
O(log N)-stage f32 FFT.  The oracle's FP64 twin runs the same algorithm in
double precision; it must equal pocketfft to round-off, which pins the
algorithm itself (ordering, scaling, wrap-padding) independently of f32.
"""
import numpy as np

from autoverse_b200 import workloads as wl
from oracle import oracle as O


def test_oracle_fft_convolution_error_bound_512():
    cfg, st = wl.multispecies(512, channels=3, R=15)
    W = H = 512
    worst_rel = 0.0
    for k in cfg["kernels"]:
        kern = O.kernel_build(k, cfg["kernel_radius"])
        pad32 = O.kernel_pad(kern, W, H)
        pad64 = pad32.astype(np.float64)  # the same f32 kernel values, so only FFT arithmetic differs
        a32 = st[k["source_channel"]].reshape(H, W)
        a64 = a32.astype(np.float64)
        exact = np.fft.irfft2(np.fft.rfft2(a64) * np.fft.rfft2(pad64), s=(H, W))
        c64 = O.fft_convolve(a64, pad64)
        c32 = O.fft_convolve(a32, pad32)
        scale = np.abs(exact).max()
        # the oracle's algorithm in FP64 is the exact DFT convolution
        assert np.abs(c64 - exact).max() <= 1e-12 * max(scale, 1.0)
        # f32 rounding of a 2 x 9-stage FFT: a few ulps of the largest value (3e-7 measured)
        rel = float(np.abs(c32 - exact).max() / scale)
        worst_rel = max(worst_rel, rel)
        assert rel <= 1e-6, rel
    # Through the growth function (|dG/du| <= 2 e^-1/2 / sigma, 121 at sigma
    # = 0.01) a convolution error of worst_rel * |conv| stays near 1e-5 in U.
    assert worst_rel > 0.0

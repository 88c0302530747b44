"""Host-side logic of the package: config arithmetic and the beam generator,
checked against outputs of the reference (tests/golden)."""
import numpy as np
import pytest

from lcodepy_b200.beam_generator import generate_beam
from lcodepy_b200.config import Config, good_size


@pytest.mark.parametrize("ww,h,steps", [(6.5, 0.1, 129), (6.4, 0.1, 127),
                                        (3.25, 0.05, 129), (6.45, 0.05, 257),
                                        (5.13, 0.02, 513), (12.85, 0.05, 513),
                                        (8, 0.05, 321), (1.6, 0.05, 65)])
def test_window_snapping(ww, h, steps):
    c = Config({'geometry': '3d', 'window-width': ww, 'transverse-step': h})
    c._adjust_config_values_3d()
    assert c.getint('window-width-steps') == steps
    assert good_size(steps)


@pytest.mark.parametrize("raw,expect", [(1, 1.05), ('1', 1.05), (1.0, 1.0), (2, 2.0)])
def test_subtraction_coefficient(raw, expect):
    c = Config({'geometry': '3d', 'xi-step': 0.05,
                'field-solver-subtraction-coefficient': raw})
    c._adjust_config_values_3d()
    assert c.getfloat('field-solver-subtraction-coefficient') == pytest.approx(expect, abs=0)


def test_fineness():
    c = Config({'geometry': '3d', 'plasma-particles-per-cell': 10})
    c._adjust_config_values_3d()
    assert c.getint('plasma-fineness') == 3 and c.getint('plasma-particles-per-cell') == 9


def test_generator_matches_reference(golden):
    d = golden("gen_beams.npz")
    c1 = Config({'geometry': '3d', 'window-width': 8, 'transverse-step': 0.05,
                 'xi-step': 0.05})
    c1._adjust_config_values_3d()
    b = generate_beam(c1, {'current': 0.05, 'particles_in_layer': 150,
                           'default': {'length': 5.013256548}})
    c2 = Config({'geometry': '3d', 'window-width': 3.2, 'transverse-step': 0.05,
                 'xi-step': 0.1})
    c2._adjust_config_values_3d()
    b2 = generate_beam(c2, {'current': -0.3, 'particles_in_layer': 300, 'rng_seed': 7,
                            'seg1': {'length': 2.0, 'xishape': 'l', 'eshape': 'g',
                                     'espread': 10, 'radius': 0.5},
                            'seg2': {'length': 1.5, 'xishape': 'h', 'angspread': 1e-3,
                                     'mass_charge_ratio': 1836, 'eshape': 'u',
                                     'energy': 500, 'espread': 600}})
    for got, ref in ((b, d["test1like"]), (b2, d["twoseg"])):
        assert got.dtype == ref.dtype and got.shape == ref.shape
        for k in ref.dtype.names:
            np.testing.assert_array_equal(got[k], ref[k], err_msg=k)


def test_declustering_average_is_scipys_fourier_gaussian():
    """The solver averages the inhomogeneity by multiplying its FFT with
    exp(-2 pi^2 sigma^2 f^2) per axis (f the FFT frequencies); that is
    scipy.ndimage.fourier_gaussian, which the reference calls
    (noise_filter.py:142-143), for odd and even lattice sides."""
    import numpy as np
    import torch
    from scipy.ndimage import fourier_gaussian
    rng = np.random.default_rng(5)
    for n, sigma in ((40, 3.0), (33, 1.5)):
        a = rng.normal(size=(n, n))
        want = np.fft.ifft2(fourier_gaussian(np.fft.fft2(a), sigma=sigma)).real
        f = torch.fft.fftfreq(n, dtype=torch.float64)
        g = torch.exp(-2 * np.pi ** 2 * sigma ** 2 * f * f)
        got = torch.fft.ifft2(torch.fft.fft2(torch.tensor(a)) * (g[:, None] * g[None, :])).real
        assert np.abs(got.numpy() - want).max() < 1e-14 * np.abs(want).max()

"""Coefficient fields m(x) and c(x) of the reference's launchers, generated on
the GPU: drop-ins for generate_m_fields (scripts/m_fields_2d.py:147-238) and
generate_c_fields (scripts/c_fields_2d.py:169-248).

Every random draw is made here, with numpy's global generator, in the order
the reference makes it (so a launcher that seeds np.random gets the same
parameters and noise as with the reference's functions); the field formulas,
the Gaussian filters (scipy.ndimage.gaussian_filter's weights, computed here
exactly as scipy computes them, applied on the device in reflect mode), the
Laplacian and the normalising reductions run on the device through
nls_field2d (include/nlsb200.h). Fields agree with the reference's to about
1e-14 relative. Grids: x = linspace(-L, L, n) on both axes, X[i, j] = x[i],
Y[i, j] = x[j] (make_grid, m_fields_2d.py:8-12).
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, lib

M_PIECEWISE, M_GRADIENT, M_PHASE, M_TOPOLOGICAL, M_DEFECTS, M_QUASIPERIODIC, M_MULTISCALE = range(1, 8)
C_PERIODIC, C_PIECEWISE, C_SIGN, C_LAYERED, C_WAVEGUIDE, C_QUASIPERIODIC, C_TURBULENT = range(11, 18)
BOUNDARIES = ['circle', 'square', 'horizontal', 'vertical', 'diagonal']


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def field2d(kind: int, n: int, L: float, params, inputs=()):
    """One device evaluation (nls_field2d): params as the kind's layout, inputs
    a sequence of (n, n) arrays. Returns the (n, n) float64 field."""
    P = np.ascontiguousarray(np.asarray(params, dtype=np.float64).ravel())
    ins = [np.ascontiguousarray(a, dtype=np.float64).reshape(n, n) for a in inputs]
    inp = np.ascontiguousarray(np.stack(ins)) if ins else None
    out = np.empty((n, n))
    check(lib().nls_field2d(int(kind), int(n), float(L), _dp(P) if P.size else None, int(P.size),
                            _dp(inp) if inp is not None else None, len(ins), _dp(out)))
    return out


def gaussian_weights(sigma):
    """The taps scipy.ndimage.gaussian_filter1d correlates with (truncate 4,
    order 0): radius int(4 sigma + 0.5), exp(-0.5 / sigma^2 x^2) divided by its
    sum, reversed."""
    sd = float(sigma)
    lw = int(4.0 * sd + 0.5)
    sigma2 = sigma * sigma
    x = np.arange(-lw, lw + 1)
    phi = np.exp(-0.5 / sigma2 * x ** 2)
    phi = phi / phi.sum()
    return phi[::-1].copy()


def _filter_params(sigma):
    w = gaussian_weights(sigma)
    return [float(len(w))] + list(w)


# ----------------------------------------------------------- m fields

def constant_mass(n, L, base_value=1.0):
    return np.ones((n, n), dtype=np.float64) * base_value


def piecewise_constant_mass(n, L, m1=1.0, m2=2.0, boundary_type='circle', boundary_param=0.5, smooth_width=0.05):
    return field2d(M_PIECEWISE, n, L, [m1, m2, BOUNDARIES.index(boundary_type), boundary_param, smooth_width])


def gradient_based_mass(n, L, c_field, m0=1.0, gamma=1.0, epsilon=1e-6):
    return field2d(M_GRADIENT, n, L, [m0, gamma, epsilon], [c_field])


def phase_shifted_mass(n, L, c_field, m0=1.0, delta=0.5, shift_fraction=0.05):
    shift_pixels = max(1, int(shift_fraction * n))
    return field2d(M_PHASE, n, L, [m0, delta, shift_pixels], [c_field])


def topological_mass(n, L, c_field, m0=1.0, eta=0.8, lambda_param=0.5):
    return field2d(M_TOPOLOGICAL, n, L, [m0, eta, lambda_param] + _filter_params(1.0), [c_field])


def localized_mass_defects(n, L, m0=1.0, num_defects=10, min_strength=-0.5, max_strength=1.0, min_width=0.05,
                           max_width=0.2):
    P = [m0, num_defects]
    for _ in range(num_defects):  # draw order of m_fields_2d.py:88-95
        x0 = np.random.uniform(-L, L)
        y0 = np.random.uniform(-L, L)
        strength = np.random.uniform(min_strength, max_strength) * m0
        width = np.random.uniform(min_width, max_width) * L
        P += [x0, y0, strength, width]
    return field2d(M_DEFECTS, n, L, P)


def _wave_vectors(num_waves):
    golden_ratio = (1 + np.sqrt(5)) / 2
    out = []
    for i in range(num_waves):
        angle = i * np.pi / num_waves
        kx = np.cos(angle)
        ky = np.sin(angle)
        scale = golden_ratio ** i
        out.append((kx * scale, ky * scale))
    return out


def quasi_periodic_mass(n, L, m0=1.0, num_waves=5, min_amp=0.1, max_amp=0.5):
    P = [m0, num_waves]
    for kx, ky in _wave_vectors(num_waves):  # m_fields_2d.py:119-124
        amplitude = np.random.uniform(min_amp, max_amp) * m0
        phase = np.random.uniform(0, 2 * np.pi)
        P += [kx, ky, amplitude, phase]
    return field2d(M_QUASIPERIODIC, n, L, P)


def multiscale_mass(n, L, m0=1.0, num_scales=4, min_scale=2, max_scale=16, min_amp=0.1, max_amp=0.5):
    scale_factors = np.logspace(np.log10(min_scale), np.log10(max_scale), num_scales)
    P, noises = [m0, num_scales], []
    for scale in scale_factors:  # m_fields_2d.py:135-141: noise, then amplitude
        noises.append(np.random.randn(n, n))
        amplitude = np.random.uniform(min_amp, max_amp) * m0
        P += [amplitude] + _filter_params(scale)
    return field2d(M_MULTISCALE, n, L, P, noises)


def generate_m_fields(n, L, c_field=None, num_fields=8, field_types=None, m0=1.0):
    """Drop-in for the reference's generate_m_fields (m_fields_2d.py:147-238):
    the same draws in the same order, the fields computed on the GPU."""
    if field_types is None:
        field_types = ['constant', 'piecewise', 'gradient', 'phase', 'topological', 'defects', 'quasiperiodic',
                       'multiscale']
    fields, params = [], []
    for i, field_type in enumerate(field_types[:num_fields]):
        if field_type == 'constant':
            field = constant_mass(n, L, m0)
            param = {'type': 'constant', 'm0': m0}
        elif field_type == 'piecewise':
            m1 = m0
            m2 = np.random.uniform(1.5, 3.0) * m0
            boundary_type = np.random.choice(BOUNDARIES)
            boundary_param = np.random.uniform(0.3, 0.7)
            smooth_width = np.random.uniform(0.01, 0.1)
            field = piecewise_constant_mass(n, L, m1, m2, boundary_type, boundary_param, smooth_width)
            param = {'type': 'piecewise', 'm1': m1, 'm2': m2, 'boundary_type': boundary_type,
                     'boundary_param': boundary_param, 'smooth_width': smooth_width}
        elif field_type == 'gradient' and c_field is not None:
            gamma = np.random.uniform(0.5, 2.0)
            epsilon = np.random.uniform(1e-3, 1e-1)
            field = gradient_based_mass(n, L, c_field, m0, gamma, epsilon)
            param = {'type': 'gradient', 'm0': m0, 'gamma': gamma, 'epsilon': epsilon}
        elif field_type == 'phase' and c_field is not None:
            delta = np.random.uniform(0.3, 1.0)
            shift_fraction = np.random.uniform(0.02, 0.1)
            field = phase_shifted_mass(n, L, c_field, m0, delta, shift_fraction)
            param = {'type': 'phase', 'm0': m0, 'delta': delta, 'shift_fraction': shift_fraction}
        elif field_type == 'topological' and c_field is not None:
            eta = np.random.uniform(0.5, 1.0)
            lambda_param = np.random.uniform(0.3, 0.7)
            field = topological_mass(n, L, c_field, m0, eta, lambda_param)
            param = {'type': 'topological', 'm0': m0, 'eta': eta, 'lambda_param': lambda_param}
        elif field_type == 'defects':
            num_defects = np.random.randint(5, 20)
            min_strength = np.random.uniform(-0.5, -0.1)
            max_strength = np.random.uniform(0.5, 1.0)
            min_width = np.random.uniform(0.03, 0.08)
            max_width = np.random.uniform(0.1, 0.3)
            field = localized_mass_defects(n, L, m0, num_defects, min_strength, max_strength, min_width, max_width)
            param = {'type': 'defects', 'm0': m0, 'num_defects': num_defects, 'min_strength': min_strength,
                     'max_strength': max_strength, 'min_width': min_width, 'max_width': max_width}
        elif field_type == 'quasiperiodic':
            num_waves = np.random.randint(3, 8)
            min_amp = np.random.uniform(0.1, 0.3)
            max_amp = np.random.uniform(0.4, 0.8)
            field = quasi_periodic_mass(n, L, m0, num_waves, min_amp, max_amp)
            param = {'type': 'quasiperiodic', 'm0': m0, 'num_waves': num_waves, 'min_amp': min_amp,
                     'max_amp': max_amp}
        elif field_type == 'multiscale':
            num_scales = np.random.randint(3, 6)
            min_scale = np.random.uniform(1, 3)
            max_scale = np.random.uniform(8, 20)
            min_amp = np.random.uniform(0.1, 0.3)
            max_amp = np.random.uniform(0.4, 0.8)
            field = multiscale_mass(n, L, m0, num_scales, min_scale, max_scale, min_amp, max_amp)
            param = {'type': 'multiscale', 'm0': m0, 'num_scales': num_scales, 'min_scale': min_scale,
                     'max_scale': max_scale, 'min_amp': min_amp, 'max_amp': max_amp}
        else:
            field = constant_mass(n, L, m0)
            param = {'type': 'constant', 'm0': m0}
        fields.append(field.astype(np.float64))
        params.append(param)
    return fields, params


# ----------------------------------------------------------- c fields

def constant(n, L):
    return np.ones((n, n), dtype=np.float64)


def periodic_structure(n, L, base_value=1.0, amplitude=0.5, frequency=3):
    k = np.pi * frequency / L
    return field2d(C_PERIODIC, n, L, [base_value, amplitude, k])


def piecewise_constant(n, L, num_layers=3, base_value=1.0, contrast_factor=2.0):
    layer_width = 2 * L / num_layers
    return field2d(C_PIECEWISE, n, L, [num_layers, base_value, contrast_factor, layer_width])


def sign_changing_mass(n, L, base_value=1.0, regions='checkerboard', scale=2, sharpness=5.0):
    if regions not in ('checkerboard', 'half_space'):
        raise NotImplementedError(regions)
    cell_size = L / scale
    return field2d(C_SIGN, n, L, [base_value, 0 if regions == 'checkerboard' else 1, cell_size, sharpness])


def layered_materials(n, L, base_value=1.0, num_layers=3, min_amplitude=0.2, max_amplitude=0.8, min_freq=2,
                      max_freq=10):
    P = [base_value, num_layers]
    for _ in range(num_layers):  # c_fields_2d.py:59-67
        theta = np.random.uniform(0, np.pi)
        nx, ny = np.cos(theta), np.sin(theta)
        amplitude = np.random.uniform(min_amplitude, max_amplitude)
        freq = np.random.uniform(min_freq, max_freq)
        phase = np.random.uniform(0, 2 * np.pi)
        P += [nx, ny, amplitude, freq, phase]
    return field2d(C_LAYERED, n, L, P)


def wave_guiding_structures(n, L, base_value=1.0, min_width=0.1, max_width=0.5, guide_amplitude=0.8):
    num_guides = np.random.randint(3, 12)
    P = [base_value, guide_amplitude, num_guides, 100]
    for _ in range(num_guides):  # c_fields_2d.py:82-110
        curve_type = 'line' if np.random.random() < 0.5 else 'curve'
        width = np.random.uniform(min_width, max_width)
        if curve_type == 'line':
            x0 = np.random.uniform(-L, L)
            y0 = np.random.uniform(-L, L)
            theta = np.random.uniform(0, 2 * np.pi)
            nx, ny = np.cos(theta), np.sin(theta)
            t = np.linspace(-1.5 * L, 1.5 * L, 100)
            curve_x = x0 + t * nx
            curve_y = y0 + t * ny
        else:
            a = np.random.uniform(0.5, 2.0)
            b = np.random.uniform(0.5, 2.0)
            phi = np.random.uniform(0, 2 * np.pi)
            t = np.linspace(0, 2 * np.pi, 100)
            curve_x = a * np.cos(t + phi)
            curve_y = b * np.sin(t)
        P += [width] + list(curve_x) + list(curve_y)
    return field2d(C_WAVEGUIDE, n, L, P)


def quasi_periodic_structures(n, L, base_value=1.0, num_waves=5, min_amp=0.1, max_amp=0.5):
    P = [base_value, num_waves]
    for kx, ky in _wave_vectors(num_waves):  # c_fields_2d.py:133-138
        amplitude = np.random.uniform(min_amp, max_amp)
        phase = np.random.uniform(0, 2 * np.pi)
        P += [kx, ky, amplitude, phase]
    return field2d(C_QUASIPERIODIC, n, L, P)


def turbulent_like_fields(n, L, base_value=1.0, intensity=0.5, min_scale=2, max_scale=20, beta=5 / 3,
                          num_octaves=5):
    P, noises = [], []
    for octave in range(num_octaves):  # c_fields_2d.py:150-158: noise per octave until scale < min_scale
        scale = max_scale / (2 ** octave)
        if scale < min_scale:
            break
        noises.append(np.random.randn(n, n))
        amplitude = scale ** beta
        P += [amplitude] + _filter_params(scale)
    return field2d(C_TURBULENT, n, L, [base_value, intensity, len(noises)] + P, noises)


def generate_c_fields(n, L, num_fields=5, field_types=None, base_value=1.0, seed=None):
    """Drop-in for the reference's generate_c_fields (c_fields_2d.py:169-248):
    the same draws in the same order, the fields computed on the GPU."""
    if seed is not None:
        np.random.seed(seed)
    if field_types is None:
        field_types = ['periodic_structure', 'piecewise_constant', 'sign_changing_mass', 'layered', 'waveguide',
                       'quasiperiodic', 'turbulent']
    fields, params = [], []
    for i in range(num_fields):
        field_type = np.random.choice(field_types)
        if field_type == 'layered':
            num_layers = np.random.randint(2, 6)
            min_amp = np.random.uniform(0.1, 0.3)
            max_amp = np.random.uniform(0.4, 0.8)
            min_freq = np.random.uniform(1, 3)
            max_freq = np.random.uniform(5, 15)
            field = layered_materials(n, L, base_value, num_layers, min_amp, max_amp, min_freq, max_freq)
            param = {'type': 'layered', 'num_layers': num_layers, 'min_amp': min_amp, 'max_amp': max_amp,
                     'min_freq': min_freq, 'max_freq': max_freq}
        elif field_type == 'waveguide':
            min_width = np.random.uniform(0.1, 0.3)
            max_width = np.random.uniform(0.4, 0.8)
            guide_amp = np.random.uniform(0.5, 2.)
            field = wave_guiding_structures(n, L, base_value, min_width, max_width, guide_amp)
            param = {'type': 'waveguide', 'min_width': min_width, 'max_width': max_width, 'guide_amp': guide_amp}
        elif field_type == 'quasiperiodic':
            num_waves = np.random.randint(3, 8)
            min_amp = np.random.uniform(0.1, 0.3)
            max_amp = np.random.uniform(0.4, 0.8)
            field = quasi_periodic_structures(n, L, base_value, num_waves, min_amp, max_amp)
            param = {'type': 'quasiperiodic', 'num_waves': num_waves, 'min_amp': min_amp, 'max_amp': max_amp}
        elif field_type == 'turbulent':
            intensity = np.random.uniform(0.3, 0.8)
            min_scale = np.random.uniform(1, 3)
            max_scale = np.random.uniform(10, 30)
            beta = np.random.uniform(1, 3)
            num_octaves = np.random.randint(3, 8)
            field = turbulent_like_fields(n, L, base_value, intensity, min_scale, max_scale, beta, num_octaves)
            param = {'type': 'turbulent', 'intensity': intensity, 'min_scale': min_scale, 'max_scale': max_scale,
                     'beta': beta, 'num_octaves': num_octaves}
        elif field_type == 'periodic_structure':
            amplitude = np.random.uniform(0.2, 0.5)
            frequency = np.random.randint(1, 3)
            field = periodic_structure(n, L, amplitude=amplitude, frequency=frequency)
            param = {'type': 'periodic_structure', 'amplitude': amplitude}
        elif field_type == 'piecewise_constant':
            num_layers = np.random.randint(2, 5)
            contrast_factor = np.random.uniform(1.5, 2.5)
            field = piecewise_constant(n, L, num_layers=num_layers, contrast_factor=contrast_factor)
            param = {'type': 'piecewise_constant', 'num_layers': num_layers, 'contrast_factor': contrast_factor}
        elif field_type == 'sign_changing_mass':
            regions = np.random.choice(['checkerboard', 'half_space'])
            scale = np.random.randint(2, 3)
            sharpness = np.random.uniform(3, 6)
            field = sign_changing_mass(n, L, regions=regions, scale=scale, sharpness=sharpness)
            param = {'type': 'sign_changing_mass', 'regions': regions, 'scale': scale, 'sharpness': sharpness}
        elif field_type == 'constant':
            field = constant(n, L)
            param = {}
        else:
            raise NotImplementedError(field_type)
        fields.append(field)
        params.append(param)
    return fields, params

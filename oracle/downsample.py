"""CPU restatement (numpy) of the reference's snapshot downsampling: the
spectral crop (downsample_fft below) and the linear interpolation,
scripts/downsampling.py:68-103 (downsample_interpolation) and
:215-257 (downsample_interpolation_3d), which its HDF5 aggregation applies to
every snapshot (scripts/aggregate_single.py:61-76).

Test infrastructure only (the tests use it as the checker; the product paths
are the CUDA kernels k_downsample and k_zgemm_strided). Pinned: the linear
form equal bitwise to the reference's own outputs on
tests/golden/downsampling.npz, the spectral form within 1e-13 of them on
tests/golden/fft_downsampling.npz (both made by tests/golden/make_*_golden.py
from the reference functions).

Array axis d has the source grid linspace(-L_d, L_d, n_d) and the target grid
linspace(-L_d, L_d, t_d), L = (Lx, Ly[, Lz]) in array-axis order as the
reference pairs them. A target point q lies in source interval l, the largest
l <= n_d - 2 with x[l] <= q; y = (q - x[l]) / (x[l+1] - x[l]). The value sums
the cell's corners in the order (0,0), (0,1), (1,0), (1,1) (bit 1: index l+1,
weight y; bit 0: index l, weight 1 - y), as RegularGridInterpolator(method=
'linear') evaluates it: 2-D terms (v * w0) * w1 summed from the first corner,
3-D terms v * ((w0 * w1) * w2) summed from zero.
"""
import numpy as np


def linspace(L, n):
    """numpy.linspace(-L, L, n) arithmetic: arange(n) * step + start, last = stop."""
    if n == 1:
        return np.array([-float(L)])
    step = (L - (-L)) / (n - 1)
    x = np.arange(n, dtype=np.float64) * step + (-L)
    x[-1] = L
    return x


def axis_table(L, n, t):
    xs, xq = linspace(L, n), linspace(L, t)
    l = np.clip(np.searchsorted(xs, xq, side="right") - 1, 0, n - 2)
    return l, (xq - xs[l]) / (xs[l + 1] - xs[l])


def downsample_interpolation(u, target_shape, L):
    """u: (frames, n0, n1[, n2]); target_shape: (t0, t1[, t2]); L: half-widths per array axis."""
    u = np.asarray(u)
    dim = u.ndim - 1
    assert dim in (2, 3) and len(target_shape) == dim and len(L) == dim
    tabs = [axis_table(float(L[d]), u.shape[d + 1], int(target_shape[d])) for d in range(dim)]
    grids = np.meshgrid(*[np.arange(int(t)) for t in target_shape], indexing="ij")
    idx = [tabs[d][0][grids[d]] for d in range(dim)]
    ys = [tabs[d][1][grids[d]] for d in range(dim)]
    out = np.empty((u.shape[0],) + tuple(int(t) for t in target_shape), dtype=u.dtype)
    for f in range(u.shape[0]):
        v = u[f]
        if dim == 2:
            acc = None
            for b0 in (0, 1):
                for b1 in (0, 1):
                    w0 = ys[0] if b0 else 1 - ys[0]
                    w1 = ys[1] if b1 else 1 - ys[1]
                    term = (v[idx[0] + b0, idx[1] + b1] * w0) * w1
                    acc = term if acc is None else acc + term
        else:
            acc = 0.0
            for b0 in (0, 1):
                for b1 in (0, 1):
                    for b2 in (0, 1):
                        w0 = ys[0] if b0 else 1 - ys[0]
                        w1 = ys[1] if b1 else 1 - ys[1]
                        w2 = ys[2] if b2 else 1 - ys[2]
                        acc = acc + v[idx[0] + b0, idx[1] + b1, idx[2] + b2] * ((w0 * w1) * w2)
        out[f] = acc
    return out


def downsample_fft(u, target_shape):
    """CPU restatement of the reference's spectral downsampling,
    scripts/downsampling.py:10-35 (downsample_fft, frames of 2-D arrays) and
    :147-178 (downsample_fft_3d): per array axis the orthonormal DFT, fftshift,
    the crop of the centred target bins from (n - t) // 2, ifftshift and the
    orthonormal inverse DFT; real inputs keep the real part. u: (frames,) +
    source shape; target_shape: the frame axes' target extents."""
    u = np.asarray(u)
    cplx = np.iscomplexobj(u)
    axes = tuple(range(1, u.ndim))
    ft = np.fft.fftshift(np.fft.fftn(u.astype(np.complex128), axes=axes, norm="ortho"), axes=axes)
    sl = [slice(None)]
    for n, t in zip(u.shape[1:], target_shape):
        s = (n - t) // 2
        sl.append(slice(s, s + t))
    crop = np.fft.ifftshift(ft[tuple(sl)], axes=axes)
    out = np.fft.ifftn(crop, axes=axes, norm="ortho")
    return (out if cplx else out.real).astype(u.dtype)

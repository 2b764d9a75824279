"""Synthetic benchmark inputs: the box-mesh workloads of the flow-solver
benchmark (seeded noisy initial fields and Gaussian particle-source blobs).
No public dataset is involved; these generators stand in for the particle
solver that produces the source terms in the reference
(FlowSolver.inl:496-736)."""
import numpy as np


def noisy_fields(n, seed, t0=1500.0, u_in=50.0, p0=4000.0, amplitude=0.01):
    rng = np.random.default_rng(seed)
    out = {}
    for name, base in (("U", u_in), ("V", 0.0), ("W", 0.0), ("P", p0), ("TEM", t0)):
        noise = rng.uniform(-amplitude, amplitude, size=n)
        out[name] = u_in * noise if base == 0.0 else base * (1.0 + noise)
    return out


def blob_stencils(dims, lengths, k, seed, rel_amplitude=1e-3, rho=1.2, u_in=50.0, sigma_cells=2.0):
    """The k blobs of gaussian_blobs(dims, lengths, k, seed) kept apart:
    (cells, values, blob) triples, so that the source field of blob
    amplitudes a_b is sum over entries of a_blob * value at cell."""
    ex, ey, ez = dims
    dx, dy, dz = (lengths[0] / ex, lengths[1] / ey, lengths[2] / ez)
    amp = rel_amplitude * rho * u_in * dy * dz
    rng = np.random.default_rng(seed)
    centres = rng.choice(ex * ey * ez, size=k, replace=False)
    r = int(np.ceil(3 * sigma_cells))
    off = np.arange(-r, r + 1)
    w1 = np.exp(-0.5 * (off / sigma_cells) ** 2)
    cells, values, blob = [], [], []
    for b, c in enumerate(centres):
        x, y, z = c % ex, (c // ex) % ey, c // (ex * ey)
        xs, ys, zs = x + off, y + off, z + off
        mx, my, mz = (xs >= 0) & (xs < ex), (ys >= 0) & (ys < ey), (zs >= 0) & (zs < ez)
        Z, Y, X = np.meshgrid(zs[mz], ys[my], xs[mx], indexing="ij")
        W = amp * w1[mz][:, None, None] * w1[my][None, :, None] * w1[mx][None, None, :]
        cells.append((X + ex * (Y + ey * Z)).reshape(-1))
        values.append(W.reshape(-1))
        blob.append(np.full(W.size, b))
    return np.concatenate(cells), np.concatenate(values), np.concatenate(blob)


def blob_phases(k, seed):
    """Random phase per blob for time-varying amplitudes."""
    return np.random.default_rng(seed + 7919).uniform(0.0, 2.0 * np.pi, size=k)


def varying_sources(n_cells, stencils, phases, it, period):
    """Sources at pass `it` with blob b scaled by sin(2 pi it / period + phase_b),
    as particle_aos rows [cells][5] (momentum +x, energy, mass as in
    gaussian_blobs)."""
    cells, values, blob = stencils
    w = np.sin(2.0 * np.pi * it / period + phases)
    g = np.bincount(cells, weights=values * w[blob], minlength=n_cells)
    src = np.zeros((n_cells, 5))
    src[:, 0] = g
    src[:, 3] = 1.0e3 * g
    src[:, 4] = 1.0e-2 * g
    return src


def gaussian_blobs(dims, lengths, k, seed, rel_amplitude=1e-3, rho=1.2, u_in=50.0, sigma_cells=2.0):
    """k Gaussian blobs centred at uniform-random cells; amplitude = rel_amplitude
    x the cell inflow rho u_in A_x; momentum along +x, energy and mass scaled
    from it.  Returned as particle_aos rows [cells][5]."""
    ex, ey, ez = dims
    dx, dy, dz = (lengths[0] / ex, lengths[1] / ey, lengths[2] / ez)
    amp = rel_amplitude * rho * u_in * dy * dz
    rng = np.random.default_rng(seed)
    centres = rng.choice(ex * ey * ez, size=k, replace=False)
    g = np.zeros((ez, ey, ex))
    r = int(np.ceil(3 * sigma_cells))
    off = np.arange(-r, r + 1)
    w1 = np.exp(-0.5 * (off / sigma_cells) ** 2)
    for c in centres:
        x, y, z = c % ex, (c // ex) % ey, c // (ex * ey)
        xs, ys, zs = x + off, y + off, z + off
        mx, my, mz = (xs >= 0) & (xs < ex), (ys >= 0) & (ys < ey), (zs >= 0) & (zs < ez)
        g[np.ix_(zs[mz], ys[my], xs[mx])] += amp * w1[mz][:, None, None] * w1[my][None, :, None] * w1[mx][None, None, :]
    g = g.reshape(-1)
    src = np.zeros((ex * ey * ez, 5))
    src[:, 0] = g
    src[:, 3] = 1.0e3 * g
    src[:, 4] = 1.0e-2 * g
    return src

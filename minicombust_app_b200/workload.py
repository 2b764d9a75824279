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

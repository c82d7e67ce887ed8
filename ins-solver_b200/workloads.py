"""Seeded synthetic workloads of the benchmark configurations.

The reference's own inputs for these solves come from a running INS simulation
(pressure RHS from the velocity divergence, density from the level set); the
configurations below stand in for them with seeded synthetic fields of the
stated shapes:
  - 2D manufactured Poisson: f = 8 pi^2 sin(2 pi x) sin(2 pi y), zero Dirichlet;
  - 3D two-phase Poisson: factor 1/rho, rho = 1000 inside a sphere r=0.25 at
    (0.5,0.5,0.5), 1 outside, smoothed with tanh over 1.5h; RHS a Gaussian random
    field with correlation length 0.1 (random Fourier modes) minus its mean;
  - 3D Helmholtz: (I/(nu dt) - Laplacian) with nu = dt = 1e-3.
"""
import numpy as np

import sipg


def mass_apply(export, tables, f):
    """b = J M f per element (mesh->mass), f: (K, Np)."""
    J = export["geof"][:, -1]
    return J[:, None] * (f @ tables["M"].T)


def grf(points, corr_len=0.1, n_modes=256, seed=7):
    """Gaussian random field sampled at points (N, dim): sum of random cosines
    with wavevectors ~ N(0, 1/corr_len^2) per axis and uniform phases."""
    rng = np.random.default_rng(seed)
    dim = points.shape[1]
    k = rng.normal(0.0, 1.0 / corr_len, (n_modes, dim))
    ph = rng.uniform(0.0, 2 * np.pi, n_modes)
    out = np.zeros(points.shape[0])
    chunk = 1 << 15
    for s in range(0, points.shape[0], chunk):
        out[s:s + chunk] = np.cos(points[s:s + chunk] @ k.T + ph).sum(axis=1)
    return out * np.sqrt(2.0 / n_modes)


def two_phase_rho(x, y, z, h, ratio=1000.0, radius=0.25, center=(0.5, 0.5, 0.5), width=1.5):
    r = np.sqrt((x - center[0]) ** 2 + (y - center[1]) ** 2 + (z - center[2]) ** 2)
    return 1.0 + (ratio - 1.0) * 0.5 * (1.0 + np.tanh((radius - r) / (width * h)))


def poisson3d_two_phase(n, order=3, jitter=0.1, seed=20261203, rhs_seed=7, n_modes=256, pin=True, geometry_bits=32):
    """The 3D variable-density Poisson configuration on an n^3 x 6 tet box.
    Returns dict(mesh, export, tables, factor, rhs, bc_types, pin); geometry_bits 16: the
    FP32 kernels' geometric factors in BF16."""
    mesh = sipg.Mesh.box(3, n, jitter=jitter, seed=seed, geometry_bits=geometry_bits)
    e = mesh.export(order)
    t = sipg.ref_tables(3, order)
    h = 1.0 / n
    rho = two_phase_rho(e["x"], e["y"], e["z"], h)
    factor = 1.0 / rho
    pts = np.stack([e["x"].ravel(), e["y"].ravel(), e["z"].ravel()], 1)
    f = grf(pts, 0.1, n_modes, rhs_seed).reshape(e["K"], t["Np"])
    b = mass_apply(e, t, f)
    vol_w = mass_apply(e, t, np.ones_like(f))
    f = f - b.sum() / vol_w.sum()          # subtract the (mass-weighted) mean
    b = mass_apply(e, t, f)
    bct = np.full((1, e["Kb"]), sipg.BC_NEUMANN, np.int32)
    if pin:
        b[0, 0] = 0.0
    return dict(mesh=mesh, export=e, tables=t, factor=factor, rhs=b[None], bc_types=bct,
                pin=(0, 0) if pin else None, rho=rho)


def served_poisson(dim, n, order, two_phase, seed, n_modes=32):
    """One problem of the served stream: a box of 2 n^2 triangles or 6 n^3 tets,
    interior vertices jittered +-0.1h (seed), Neumann walls (constants projected
    out), right-hand side J M (Gaussian random field with correlation length 0.1
    minus its mean, seed + 1), factor 1/rho with rho = 1000 in a ball (disc) of
    radius 0.25 at the centre and 1 outside, or constant 1."""
    mesh = sipg.Mesh.box(dim, n, jitter=0.1, seed=seed)
    e = mesh.export(order)
    t = sipg.ref_tables(dim, order)
    coords = [e["x"], e["y"]] + ([e["z"]] if dim == 3 else [])
    factor = None
    if two_phase:
        zc = e["z"] if dim == 3 else np.full_like(e["x"], 0.5)
        factor = 1.0 / two_phase_rho(e["x"], e["y"], zc, 1.0 / n)
    pts = np.stack([c.ravel() for c in coords], 1)
    f = grf(pts, 0.1, n_modes, seed + 1).reshape(e["K"], t["Np"])
    b = mass_apply(e, t, f)
    f = f - b.sum() / mass_apply(e, t, np.ones_like(f)).sum()
    b = mass_apply(e, t, f)
    bct = np.full((1, e["Kb"]), sipg.BC_NEUMANN, np.int32)
    return dict(mesh=mesh, dim=dim, order=order, K=e["K"], factor=factor, rhs=b.reshape(-1), bc_types=bct,
                two_phase=bool(two_phase))


def served_stream_pool(n_problems, seed=4):
    """Distinct problems drawn from the served-stream distribution: 2D with
    probability 0.6 (else 3D), element count log-uniform in [2e3, 3e5] (the box
    size nearest to it), order uniform in {2, 3, 4}, two-phase coefficient with
    probability 0.5."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_problems):
        dim = 2 if rng.random() < 0.6 else 3
        K = float(np.exp(rng.uniform(np.log(2e3), np.log(3e5))))
        order = int(rng.integers(2, 5))
        two = bool(rng.random() < 0.5)
        n = max(4, int(round((K / 2) ** 0.5))) if dim == 2 else max(3, int(round((K / 6) ** (1.0 / 3.0))))
        out.append(served_poisson(dim, n, order, two, seed=1000 + 17 * i))
    return out


def poisson2d_manufactured(n, order=3):
    """2D Poisson with zero Dirichlet data and exact solution sin(2 pi x) sin(2 pi y)."""
    mesh = sipg.Mesh.box(2, n, jitter=0.0, seed=0)
    e = mesh.export(order)
    t = sipg.ref_tables(2, order)
    f = 8 * np.pi**2 * np.sin(2 * np.pi * e["x"]) * np.sin(2 * np.pi * e["y"])
    exact = np.sin(2 * np.pi * e["x"]) * np.sin(2 * np.pi * e["y"])
    b = mass_apply(e, t, f)
    bct = np.full((1, e["Kb"]), sipg.BC_DIRICHLET, np.int32)
    return dict(mesh=mesh, export=e, tables=t, rhs=b[None], exact=exact[None], bc_types=bct)


def helmholtz3d(n, order=4, nu=1e-3, dt=1e-3, seed=11, jitter=0.1, geometry_bits=32):
    """3D Helmholtz (I/(nu dt) - Laplacian) with Dirichlet walls, random input U(-1,1);
    geometry_bits 16: the FP32 kernels' geometric factors in BF16."""
    mesh = sipg.Mesh.box(3, n, jitter=jitter, seed=20261203, geometry_bits=geometry_bits)
    Np = sipg.ref_sizes(3, order)[0]
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1.0, 1.0, (1, mesh.K, Np))
    bct = np.full((1, mesh.Kb), sipg.BC_DIRICHLET, np.int32)
    return dict(mesh=mesh, x=x, bc_types=bct, mm=1.0 / (nu * dt), order=order)

"""Seeded synthetic matrices for the five workloads of this project.

Grid vertices are numbered x-fastest (index = x + nx*(y + ny*z)), the numbering
pastixOrderGrid assumes (order/order_grids.c:169).  Every generator returns a
``scipy.sparse.csc_matrix`` holding the whole matrix (both triangles).

  laplacian7      3D 7-point Laplacian, diagonal 6 + 1e-3, off-diagonals -1
  diffusion5_grf  2D 5-point variable-coefficient diffusion, k = exp(g) with g a
                  squared-exponential Gaussian random field, Dirichlet boundary
  convdiff27      3D 27-point diffusion + first-order upwind convection,
                  symmetric pattern, unsymmetric values, diagonal set from a
                  dominance ratio
  elastic27_dof3  3 unknowns per node, 27-point block stencil assembled from
                  random SPD (Wishart) coupling blocks, shifted to be indefinite
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sps


def _grid_ids(nx, ny, nz):
    return np.arange(nx * ny * nz, dtype=np.int64).reshape(nz, ny, nx)


def _pairs(nx, ny, nz, offsets):
    """(i, j) index arrays for each grid vertex i and neighbour j = i + offset (inside the grid)."""
    ids = _grid_ids(nx, ny, nz)
    out = []
    for dx, dy, dz in offsets:
        xs = slice(max(0, -dx), nx - max(0, dx))
        ys = slice(max(0, -dy), ny - max(0, dy))
        zs = slice(max(0, -dz), nz - max(0, dz))
        xt = slice(max(0, dx), nx + min(0, dx))
        yt = slice(max(0, dy), ny + min(0, dy))
        zt = slice(max(0, dz), nz + min(0, dz))
        out.append((ids[zs, ys, xs].ravel(), ids[zt, yt, xt].ravel(), (dx, dy, dz)))
    return out


FACE = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
BOX = [(dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1) if (dx, dy, dz) != (0, 0, 0)]


def laplacian7(nx: int, ny: int, nz: int, diag: float = 6.0 + 1e-3, off: float = -1.0) -> sps.csc_matrix:
    n = nx * ny * nz
    rows, cols, vals = [np.arange(n)], [np.arange(n)], [np.full(n, diag)]
    for i, j, _ in _pairs(nx, ny, nz, FACE):
        rows.append(i); cols.append(j); vals.append(np.full(i.size, off))
    A = sps.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    return A.tocsc()


def grf_2d(nx: int, ny: int, length: float, var: float, seed: int) -> np.ndarray:
    """Squared-exponential Gaussian random field by circulant embedding on a
    2x padded periodic grid (FFT), scaled to the requested variance."""
    rng = np.random.default_rng(seed)
    px, py = 2 * nx, 2 * ny
    kx = np.fft.fftfreq(px)
    ky = np.fft.fftfreq(py)
    KX, KY = np.meshgrid(kx, ky)
    spec = np.exp(-2.0 * (np.pi ** 2) * (length ** 2) * (KX ** 2 + KY ** 2))
    noise = rng.standard_normal((py, px))
    field = np.real(np.fft.ifft2(np.sqrt(spec) * np.fft.fft2(noise)))
    g = field[:ny, :nx]
    g = (g - g.mean()) / g.std() * np.sqrt(var)
    return g


def diffusion5_grf(nx: int, ny: int, kfield: np.ndarray) -> sps.csc_matrix:
    """-div(k grad u) with 5-point finite volumes, face coefficient = arithmetic
    mean of the two cells, Dirichlet boundary (boundary faces use the cell k)."""
    n = nx * ny
    k = np.asarray(kfield, dtype=np.float64).reshape(ny, nx)
    ids = np.arange(n).reshape(ny, nx)
    diag = np.zeros((ny, nx))
    rows, cols, vals = [], [], []
    # x faces
    kf = 0.5 * (k[:, :-1] + k[:, 1:])
    a, b = ids[:, :-1].ravel(), ids[:, 1:].ravel()
    rows += [a, b]; cols += [b, a]; vals += [-kf.ravel(), -kf.ravel()]
    diag[:, :-1] += kf; diag[:, 1:] += kf
    kf = 0.5 * (k[:-1, :] + k[1:, :])
    a, b = ids[:-1, :].ravel(), ids[1:, :].ravel()
    rows += [a, b]; cols += [b, a]; vals += [-kf.ravel(), -kf.ravel()]
    diag[:-1, :] += kf; diag[1:, :] += kf
    # Dirichlet boundary faces
    diag[:, 0] += k[:, 0]; diag[:, -1] += k[:, -1]; diag[0, :] += k[0, :]; diag[-1, :] += k[-1, :]
    rows.append(ids.ravel()); cols.append(ids.ravel()); vals.append(diag.ravel())
    A = sps.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    return A.tocsc()


def convdiff27(nx: int, ny: int, nz: int, vmax: float = 50.0, ratio: float = 0.95, seed: int = 3) -> sps.csc_matrix:
    """27-point diffusion (weight 1 on every neighbour) plus upwind convection on
    the 6 face neighbours with a per-cell velocity ~ U[-vmax, vmax]^3; the
    diagonal is set so that sum_j |a_ij| = ratio * a_ii."""
    n = nx * ny * nz
    rng = np.random.default_rng(seed)
    vel = rng.uniform(-vmax, vmax, size=(n, 3))
    rows, cols, vals = [], [], []
    for i, j, (dx, dy, dz) in _pairs(nx, ny, nz, BOX):
        v = -np.ones(i.size)
        if abs(dx) + abs(dy) + abs(dz) == 1:
            d = 0 if dx else (1 if dy else 2)
            s = dx + dy + dz
            # inflow from neighbour j when the velocity at i points from j to i
            v -= np.maximum(0.0, -s * vel[i, d])
        rows.append(i); cols.append(j); vals.append(v)
    r = np.concatenate(rows); c = np.concatenate(cols); v = np.concatenate(vals)
    offsum = np.bincount(r, weights=np.abs(v), minlength=n)
    diag = offsum / ratio
    A = sps.coo_matrix((np.concatenate([v, diag]), (np.concatenate([r, np.arange(n)]), np.concatenate([c, np.arange(n)]))),
                       shape=(n, n))
    return A.tocsc()


def lanczos_ritz(A: sps.spmatrix, steps: int, seed: int) -> np.ndarray:
    """Ritz values of `steps` Lanczos iterations (full reorthogonalisation)."""
    n = A.shape[0]
    rng = np.random.default_rng(seed)
    q = rng.standard_normal(n)
    q /= np.linalg.norm(q)
    Q = np.zeros((steps, n))
    al, be = np.zeros(steps), np.zeros(steps)
    b = 0.0
    qprev = np.zeros(n)
    for k in range(steps):
        Q[k] = q
        w = A @ q - b * qprev
        al[k] = q @ w
        w -= al[k] * q
        w -= Q[: k + 1].T @ (Q[: k + 1] @ w)
        b = np.linalg.norm(w)
        be[k] = b
        if b == 0:
            steps = k + 1
            break
        qprev, q = q, w / b
    T = np.diag(al[:steps]) + np.diag(be[: steps - 1], 1) + np.diag(be[: steps - 1], -1)
    return np.linalg.eigvalsh(T)


def elastic27_dof3(nx: int, ny: int, nz: int, seed: int = 4, pct: float = 5.0, lanczos_steps: int = 60):
    """3 unknowns per node; every pair of 27-point neighbours (i, j) gets a random
    SPD 3x3 block W = G G^T (G 3x6 standard normal, a Wishart(3, 6) draw),
    assembled as K_ii += W, K_jj += W, K_ij = K_ji = -W, plus 1e-2 I; the matrix
    is then shifted by -sigma I, sigma = the `pct` percentile of the Ritz values
    of a Lanczos run.  Unknown 3*v + d is component d of node v.
    Returns (K, sigma)."""
    rng = np.random.default_rng(seed)
    nn = nx * ny * nz
    half = [o for o in BOX if (o[2], o[1], o[0]) > (0, 0, 0)]
    pairs = _pairs(nx, ny, nz, half)
    rows, cols, vals = [], [], []
    dblk = np.zeros((nn, 3, 3))
    for i, j, _ in pairs:
        G = rng.standard_normal((i.size, 3, 6))
        W = G @ np.transpose(G, (0, 2, 1))
        np.add.at(dblk, i, W)
        np.add.at(dblk, j, W)
        for a in range(3):
            for b in range(3):
                rows += [3 * i + a, 3 * j + a]
                cols += [3 * j + b, 3 * i + b]
                vals += [-W[:, a, b], -W[:, b, a]]
    dblk += 1e-2 * np.eye(3)
    v = np.arange(nn)
    for a in range(3):
        for b in range(3):
            rows.append(3 * v + a); cols.append(3 * v + b); vals.append(dblk[:, a, b])
    n = 3 * nn
    K = sps.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n)).tocsc()
    ritz = lanczos_ritz(K, lanczos_steps, seed + 100)
    sigma = float(np.percentile(ritz, pct))
    K = (K - sigma * sps.identity(n, format="csc")).tocsc()
    return K, sigma


def rhs_uniform(n: int, nrhs: int, seed: int):
    """x_true ~ U[-1, 1] (Fortran order)."""
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.uniform(-1.0, 1.0, size=(n, nrhs)))


def workload(name: str, small: bool = False):
    """Matrix, grid (nx, ny, nz, dof) and factorization of a named workload.
    ``small`` gives a reduced grid of the same family for quick tests."""
    if name == "lap20":
        return laplacian7(20, 20, 20), (20, 20, 20), "POTRF"
    if name == "lap100":
        s = 24 if small else 100
        return laplacian7(s, s, s), (s, s, s), "POTRF"
    if name == "grf512":
        s = 64 if small else 512
        k = np.exp(grf_2d(s, s, 16.0, 1.0, 2))
        return diffusion5_grf(s, s, k), (s, s, 1), "POTRF"
    if name == "cd64":
        s = 16 if small else 64
        return convdiff27(s, s, s), (s, s, s), "GETRF"
    if name == "el48":
        s = 8 if small else 48
        K, _ = elastic27_dof3(s, s, s)
        return K, (s, s, s), "SYTRF"
    raise KeyError(name)

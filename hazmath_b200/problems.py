"""Seeded synthetic problem generators (host side, numpy).

Every matrix is returned as int32 CSR (``ia``, ``ja``) with float64 values,
rows sorted by column with the diagonal in place, Dirichlet vertices
eliminated (interior dofs only), vertices numbered lexicographically with x
fastest.  The same arrays feed the CUDA library and the CPU oracle, so the
generators only need to be deterministic, not bit-identical to any mesh
generator of the reference.

* ``poisson2d_5pt(m)``: P1 Laplacian on a uniform right-triangle mesh of the
  unit square with m x m interior vertices.  With one diagonal orientation
  the diagonal-edge couplings are exactly zero, so the stored operator is the
  5-point stencil [4, -1, -1, -1, -1] (h-independent in 2D).
* ``kuhn3d_p1(N, k)``: P1 stiffness matrix of -div(k grad u) on the Kuhn
  (Freudenthal) tetrahedral mesh of N^3 cubes, with one coefficient per cube.
  Each cube is split into the 6 path simplices 0 -> e_a -> e_a+e_b ->
  (1,1,1); the stored pattern is the 15-point Kuhn stencil (+-e_a,
  +-(e_a+e_b), +-(1,1,1)).  Couplings between non-adjacent path vertices are
  exactly zero (their barycentric gradients are orthogonal) and stay stored.
* ``lognormal_field(N, sigma, corr, seed)``: per-cube log-normal coefficient
  exp(sigma g) with g a unit-variance Gaussian random field (white noise
  filtered by a Gaussian kernel of the given correlation length in cells).
* ``aniso2d_p1(m, eps, theta)`` / ``aniso3d_p1``: P1 anisotropic diffusion
  K = R diag(1, eps) R^T on the same meshes (positive off-diagonals occur).
"""
from __future__ import annotations

import itertools

import numpy as np


def _csr_from_stencil(shape, offsets, coefs):
    """Build sorted CSR over the interior grid of ``shape`` (x fastest) from a
    list of integer offsets (tuples, same rank as shape, x first) and, for each
    offset, an array of coefficients indexed like the grid.  Neighbours
    outside the grid are dropped (Dirichlet elimination)."""
    dims = len(shape)
    strides = [1]
    for s in shape[:-1]:
        strides.append(strides[-1] * s)
    lin = [sum(o[d] * strides[d] for d in range(dims)) for o in offsets]
    order = np.argsort(lin, kind="stable")
    n = int(np.prod(shape))
    grid = np.indices(shape[::-1])[::-1]          # grid[d] = coordinate along d
    grid = [g.reshape(-1) for g in grid]
    cols, vals, masks = [], [], []
    for oi in order:
        o = offsets[oi]
        ok = np.ones(n, bool)
        for d in range(dims):
            c = grid[d] + o[d]
            ok &= (c >= 0) & (c < shape[d])
        masks.append(ok)
        cols.append(np.arange(n, dtype=np.int64) + lin[oi])
        vals.append(np.asarray(coefs[oi], np.float64).reshape(-1))
    mask = np.stack(masks, 1)
    col = np.stack(cols, 1)
    val = np.stack(vals, 1)
    counts = mask.sum(1)
    ia = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=ia[1:])
    ja = col[mask].astype(np.int32)
    va = val[mask]
    return ia.astype(np.int32), ja, va


def poisson2d_5pt(m: int):
    """m x m interior vertices, 5-point P1/FD Laplacian (4 on the diagonal)."""
    shape = (m, m)
    offs = [(0, 0), (1, 0), (-1, 0), (0, 1), (0, -1)]
    full = np.ones(shape[::-1])
    coefs = [4.0 * full] + [-1.0 * full] * 4
    return _csr_from_stencil(shape, offs, coefs)


def rhs_uniform(n: int, seed: int):
    """b ~ U[-1, 1] from numpy's PCG64 stream of ``seed``."""
    return np.random.default_rng(seed).uniform(-1.0, 1.0, n)


def lognormal_field(N: int, sigma: float, corr: float, seed: int):
    """Per-cube coefficient exp(sigma * g), g ~ unit-variance Gaussian random
    field with a Gaussian covariance of length ``corr`` cells (periodic FFT
    filtering of white noise).  Returned with shape (N, N, N) indexed
    [z, y, x]."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((N, N, N))
    f = np.fft.fftfreq(N)
    kz, ky, kx = np.meshgrid(f, f, np.fft.rfftfreq(N), indexing="ij")
    # Gaussian kernel exp(-r^2 / (2 corr^2)) in Fourier space
    filt = np.exp(-2.0 * (np.pi * corr) ** 2 * (kx ** 2 + ky ** 2 + kz ** 2))
    g = np.fft.irfftn(np.fft.rfftn(w) * filt, s=(N, N, N), axes=(0, 1, 2))
    g -= g.mean()
    g /= g.std()
    return np.exp(sigma * g)


# Kuhn path simplices: for each permutation p of the axes the vertices are
# v0 = 0, v1 = e_p0, v2 = e_p0 + e_p1, v3 = (1,1,1).
_KUHN_PERMS = list(itertools.permutations(range(3)))


def _kuhn_paths():
    out = []
    for p in _KUHN_PERMS:
        v = [np.zeros(3, int)]
        for a in p:
            nv = v[-1].copy()
            nv[a] += 1
            v.append(nv)
        out.append((p, v))
    return out


def _kuhn_grad_products(p, K):
    """|T| grad(lambda_i)^T K grad(lambda_j) for the reference-size path
    simplex (h = 1) of permutation p; scaled by h later."""
    # barycentric gradients in permuted coordinates (x'_0 >= x'_1 >= x'_2):
    # l0 = 1 - x'0, l1 = x'0 - x'1, l2 = x'1 - x'2, l3 = x'2
    Gp = np.array([[-1, 0, 0], [1, -1, 0], [0, 1, -1], [0, 0, 1]], float)
    G = np.zeros((4, 3))
    for c in range(3):
        G[:, p[c]] = Gp[:, c]
    return (G @ K @ G.T) / 6.0


def kuhn3d_p1(N: int, kcell=None, K=None):
    """P1 stiffness on N^3 Kuhn-split cubes of the unit cube, interior dofs
    only ((N-1)^3 rows, 15-point pattern).  ``kcell``: per-cube scalar
    coefficient, shape (N,N,N) [z,y,x] (default 1); ``K``: constant 3x3
    tensor (default identity)."""
    h = 1.0 / N
    if kcell is None:
        kcell = np.ones((N, N, N))
    K = np.eye(3) if K is None else np.asarray(K, float)
    M = N + 1
    # stencil accumulators over all vertices, keyed by offset (dx, dy, dz)
    acc = {}
    for p, verts in _kuhn_paths():
        E = _kuhn_grad_products(p, K) * h   # |T| scales h^3, gradients 1/h^2
        for a in range(4):
            for b in range(4):
                off = tuple(int(x) for x in (verts[b] - verts[a]))
                if off not in acc:
                    acc[off] = np.zeros((M, M, M))
                da = verts[a]
                sl = (slice(da[2], da[2] + N), slice(da[1], da[1] + N),
                      slice(da[0], da[0] + N))
                acc[off][sl] += E[a, b] * kcell
    inner = (slice(1, N), slice(1, N), slice(1, N))
    offs = sorted(acc.keys())
    coefs = [acc[o][inner] for o in offs]
    return _csr_from_stencil((N - 1, N - 1, N - 1), offs, coefs)


def aniso_tensor2d(eps: float, theta: float):
    c, s = np.cos(theta), np.sin(theta)
    R = np.array([[c, -s], [s, c]])
    return R @ np.diag([1.0, eps]) @ R.T


def aniso2d_p1(m: int, eps: float, theta: float):
    """P1 stiffness of -div(K grad u), K = R(theta) diag(1, eps) R^T, on the
    right-triangle mesh of (m+1)^2 squares (diagonal (0,0)-(1,1)), interior
    m x m dofs, 7-point pattern."""
    K = aniso_tensor2d(eps, theta)
    N = m + 1
    M = N + 1
    acc = {}
    # triangles of the unit square: (0,0),(1,0),(1,1) and (0,0),(1,1),(0,1)
    tris = [np.array([[0, 0], [1, 0], [1, 1]]), np.array([[0, 0], [1, 1], [0, 1]])]
    for tv in tris:
        B = np.array([tv[1] - tv[0], tv[2] - tv[0]], float).T   # 2x2
        Binv = np.linalg.inv(B)
        Gref = np.array([[-1, -1], [1, 0], [0, 1]], float)
        G = Gref @ Binv                                       # rows: grad lambda
        E = 0.5 * abs(np.linalg.det(B)) * (G @ K @ G.T)       # h-independent
        for a in range(3):
            for b in range(3):
                off = (int(tv[b][0] - tv[a][0]), int(tv[b][1] - tv[a][1]))
                if off not in acc:
                    acc[off] = np.zeros((M, M))
                sl = (slice(tv[a][1], tv[a][1] + N), slice(tv[a][0], tv[a][0] + N))
                acc[off][sl] += E[a, b]
    inner = (slice(1, N), slice(1, N))
    offs = sorted(acc.keys())
    coefs = [acc[o][inner] for o in offs]
    return _csr_from_stencil((m, m), offs, coefs)


def aniso3d_p1(m: int, eps: float, theta: float, axis):
    """3D analogue: K = R diag(1, 1, eps) R^T with R the rotation by theta
    about the unit vector ``axis``; (m+1)^3 Kuhn cubes, m^3 interior dofs."""
    a = np.asarray(axis, float)
    a /= np.linalg.norm(a)
    c, s = np.cos(theta), np.sin(theta)
    A = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    R = np.eye(3) * c + s * A + (1 - c) * np.outer(a, a)
    K = R @ np.diag([1.0, 1.0, eps]) @ R.T
    return kuhn3d_p1(m + 1, None, K)


def read_coo(path: str):
    """Read HAZmath's COO text format (header 'm n nnz', then 'i j v' lines,
    0-based) into sorted-by-row CSR, keeping the file's order within a row."""
    with open(path) as f:
        m, _n, _nnz = map(int, f.readline().split())
        d = np.loadtxt(f, ndmin=2)
    i = d[:, 0].astype(np.int64)
    j = d[:, 1].astype(np.int32)
    v = d[:, 2]
    order = np.argsort(i, kind="stable")
    ia = np.zeros(m + 1, np.int64)
    np.add.at(ia, i + 1, 1)
    return np.cumsum(ia).astype(np.int32), j[order].copy(), v[order].copy()


def batch_anisotropic(nsys: int = 512, seed: int = 11, dof_lo: int = 1000,
                      dof_hi: int = 200000):
    """nsys independent SPD systems: 2D or 3D (equal odds) P1 anisotropic
    diffusion on structured meshes, epsilon uniform in [1e-3, 1], angle
    uniform in [0, pi) (3D: about a random axis), dofs log-uniform in
    [dof_lo, dof_hi], one uniform random right-hand side each.  Returns the
    list of (ia, ja, val, b) and their block-diagonal union
    (off, ia, ja, val, b), off[k] the first row of system k."""
    rng = np.random.default_rng(seed)
    systems = []
    for _ in range(nsys):
        d = float(np.exp(rng.uniform(np.log(dof_lo), np.log(dof_hi))))
        eps = float(rng.uniform(1e-3, 1.0))
        theta = float(rng.uniform(0.0, np.pi))
        if rng.uniform() < 0.5:
            ia, ja, val = aniso2d_p1(max(2, int(round(np.sqrt(d)))), eps, theta)
        else:
            axis = rng.normal(size=3)
            ia, ja, val = aniso3d_p1(max(2, int(round(np.cbrt(d)))), eps, theta, axis)
        b = rng.uniform(-1.0, 1.0, len(ia) - 1)
        systems.append((ia, ja, val, b))
    off = np.zeros(nsys + 1, np.int64)
    eo = np.zeros(nsys + 1, np.int64)
    for k, (ia, ja, val, b) in enumerate(systems):
        off[k + 1] = off[k] + len(ia) - 1
        eo[k + 1] = eo[k] + ia[-1]
    n, nnz = int(off[-1]), int(eo[-1])
    uia = np.empty(n + 1, np.int64)
    uja = np.empty(nnz, np.int32)
    uval = np.empty(nnz)
    ub = np.empty(n)
    for k, (ia, ja, val, b) in enumerate(systems):
        r0, r1, e0, e1 = off[k], off[k + 1], eo[k], eo[k + 1]
        uia[r0:r1] = ia[:-1] + e0
        uja[e0:e1] = ja + r0
        uval[e0:e1] = val
        ub[r0:r1] = b
    uia[n] = nnz
    return systems, (off.astype(np.int32), uia.astype(np.int32), uja, uval, ub)


BLOCK_COUPLING = {
    2: np.array([[2.0, 0.5], [0.5, 1.0]]),
    3: np.array([[3.0, 0.5, 0.2], [0.5, 2.0, 0.3], [0.2, 0.3, 1.0]]),
}


def block_system(ia, ja, val, nb: int, seed: int, shift: float = 0.1):
    """Block (BSR) SPD system with the pattern of a scalar SPD CSR matrix K:
    block (I, J) = K_IJ B for the fixed SPD coupling B = BLOCK_COUPLING[nb],
    plus on every diagonal block a seeded SPD term shift G G^T / nb (G with
    standard normal entries), so that the diagonal blocks differ row by row.
    Returns (ia, ja, val) with val holding the nnz blocks row-major
    (nnz * nb^2 values)."""
    B = BLOCK_COUPLING[nb]
    ia = np.asarray(ia, np.int32)
    ja = np.asarray(ja, np.int32)
    n = len(ia) - 1
    blocks = np.asarray(val, np.float64)[:, None, None] * B[None, :, :]
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((n, nb, nb))
    M = shift * np.einsum("nij,nkj->nik", G, G) / nb
    rows = np.repeat(np.arange(n), np.diff(ia))
    diag = np.nonzero(ja == rows)[0]
    blocks[diag] += M[rows[diag]]
    return ia.copy(), ja.copy(), np.ascontiguousarray(blocks.reshape(-1))


def bsr_to_csr(ia, ja, val, nb: int):
    """Scalar CSR of a block matrix: row I nb + r lists the blocks of row I
    in order, each block's columns in order."""
    ia = np.asarray(ia, np.int64)
    ja = np.asarray(ja, np.int64)
    n = len(ia) - 1
    blocks = np.asarray(val).reshape(-1, nb, nb)
    sia = [0]
    sja, sval = [], []
    for I in range(n):
        k0, k1 = ia[I], ia[I + 1]
        for r in range(nb):
            cols = (ja[k0:k1, None] * nb + np.arange(nb)[None, :]).reshape(-1)
            sja.append(cols)
            sval.append(blocks[k0:k1, r, :].reshape(-1))
            sia.append(sia[-1] + len(cols))
    return (np.asarray(sia, np.int32), np.concatenate(sja).astype(np.int32),
            np.concatenate(sval))

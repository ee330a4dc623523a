"""Synthetic, seeded problem data for the GLR hot path.

Two families:

* ``test_glr_problem`` / ``test_prior_mat_problem``: the closed-form,
  partition-independent fixtures of the reference's own gates
  (tests/test_glr.cpp:43-65,140-141 and tests/test_prior_mat.cpp:35-73),
  regenerated exactly from their formulas.
* ``grid_problem``: the benchmark configurations.  Grid points x_i on
  [0,1]^d (n per axis, h = 1/(n-1), lexicographic with x fastest); lumped
  mass h^d halved per boundary axis; Z = h^(d-2) L + s M with L the
  Neumann graph Laplacian (5-/7-point, diag = neighbour count), the
  symmetric reading of "-Laplacian + s I, times M" (the reference's example
  assembles Z = len^2 K + M the same way, examples/heat/
  heat_source_inversion.cpp:510-518); and
  B_ij = a_i a_j M_ii M_jj exp(-|x_i-x_j|^2 / (2 l_B^2)) phi(|x_i-x_j|/rho)
  with Wendland C2 phi(t) = (1-t)^4_+ (4t+1).  Sparsity is whatever the
  radius rho gives; the measured nnz is reported, never tuned.

All arrays are numpy; CSR uses int64 row pointers and int32 column indices
with columns sorted within each row.
"""

import math

import numpy as np

# --------------------------------------------------------------------------
# the reference's gate fixtures


def factor_entry(k, i):
    """a_k[i] (tests/test_glr.cpp:43-47)."""
    return np.sin(0.1 * (i + 1) * (k + 3)) + 0.2 * np.cos(0.37 * i * k + k)


def test_glr_problem(spd=True, n=120, rank=10):
    """Dense B = sum_k s_k a_k a_k^T, diagonal Z and mass
    (tests/test_glr.cpp:43-65,140-141).  Returns a dict."""
    i = np.arange(n, dtype=np.float64)
    Bd = np.zeros((n, n))
    for k in range(rank):
        sk = 2.0 / (k + 1.0)
        if not spd and (k % 2):
            sk = -sk
        a = factor_entry(k, i)
        Bd += sk * np.outer(a, a)
    z = 1.0 + 0.01 * i
    m = 0.5 + 0.1 * (np.arange(n) % 7)
    probe = np.cos(0.05 * i + 1.0)
    return dict(n=n, B_dense=Bd, zdiag=z, mass=m, probe=probe,
                B=dense_to_csr(Bd), Z=diag_csr(z))


def test_prior_mat_problem(grid_m=24, rank=6):
    """Z = 5-point Laplacian + 0.5 I on grid_m^2 (tests/test_prior_mat.cpp:
    47-73), mass 0.5 + 0.1 (i % 7), probe cos(0.05 i + 1), and the low-rank
    B of its end-to-end gate (:234-253)."""
    n = grid_m * grid_m
    rows, cols, vals = [], [], []
    for i in range(n):
        ix, iy = i % grid_m, i // grid_m
        ent = [(i, 4.5)]
        if ix > 0:
            ent.append((i - 1, -1.0))
        if ix < grid_m - 1:
            ent.append((i + 1, -1.0))
        if iy > 0:
            ent.append((i - grid_m, -1.0))
        if iy < grid_m - 1:
            ent.append((i + grid_m, -1.0))
        ent.sort()
        for c, v in ent:
            rows.append(i)
            cols.append(c)
            vals.append(v)
    Z = coo_to_csr(n, np.array(rows), np.array(cols), np.array(vals))
    ii = np.arange(n, dtype=np.float64)
    Bd = np.zeros((n, n))
    for k in range(rank):
        a = factor_entry(k, ii)
        Bd += 2.0 / (k + 1.0) * np.outer(a, a)
    mass = 0.5 + 0.1 * (np.arange(n) % 7)
    probe = np.cos(0.05 * ii + 1.0)
    return dict(n=n, Z=Z, mass=mass, probe=probe, B_dense=Bd,
                B=dense_to_csr(Bd))


# --------------------------------------------------------------------------
# CSR helpers


def test_deflate_problem(err_scale=1.0, n=120, rank_b=10, rank_c=4):
    """The closed-form problem of the reference's deflation gates
    (tests/test_deflate.cpp:43-100): B SPD of exact rank 10, diagonal Z and
    mass, a true Hessian H_d = B + DH with a planted signed error of exact
    rank 4 (err_scale blows up the leading negative mode), deterministic
    probes, and the dense oracle of F_true = whiten(H_d), signed,
    |lambda|-descending."""
    i = np.arange(n)

    def factor(k):
        return np.sin(0.1 * (i + 1) * (k + 3)) + 0.2 * np.cos(0.37 * i * k + k)

    def perr(k):
        return np.cos(0.21 * (i + 2) * (k + 1)) + 0.3 * np.sin(0.4 * i - k)

    def terr(k):
        t = 0.08 / (k + 1.0) * (-1.0 if k % 2 else 1.0)
        return t * err_scale if k == 1 else t

    Bd = np.zeros((n, n))
    for k in range(rank_b):
        a = factor(k)
        Bd += 2.0 / (k + 1.0) * np.outer(a, a)
    Hd = Bd.copy()
    for k in range(rank_c):
        p = perr(k)
        Hd += terr(k) * np.outer(p, p)
    z = 1.0 + 0.01 * i
    m = 0.5 + 0.1 * (i % 7)
    w = np.sqrt(m) / z
    F = w[:, None] * Hd * w[None, :]
    ev = np.linalg.eigvalsh(F)
    ev = ev[np.argsort(-np.abs(ev), kind="stable")]

    def probes(k):
        jj = np.arange(k)
        return (np.sin(0.03 * (i[:, None] + 1) * (jj[None, :] + 2))
                + 0.1 * np.cos(0.7 * i[:, None] - 1.3 * jj[None, :]))

    return dict(n=n, B_dense=Bd, Hd=Hd, zdiag=z, mass=m, oracle=ev,
                probe_vec=np.cos(0.05 * i + 1.0), probes=probes,
                rank_b=rank_b, rank_c=rank_c)


def coo_to_csr(n, rows, cols, vals):
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(rowptr, rows + 1, 1)
    rowptr = np.cumsum(rowptr)
    return dict(n=n, rowptr=rowptr, colidx=cols.astype(np.int32),
                vals=np.asarray(vals, dtype=np.float64))


def dense_to_csr(D):
    n = D.shape[0]
    rows, cols = np.nonzero(np.ones_like(D, dtype=bool))
    return dict(n=n, rowptr=np.arange(0, n * n + 1, n, dtype=np.int64),
                colidx=cols.astype(np.int32).reshape(-1),
                vals=D.reshape(-1).astype(np.float64).copy())


def diag_csr(d):
    n = len(d)
    return dict(n=n, rowptr=np.arange(n + 1, dtype=np.int64),
                colidx=np.arange(n, dtype=np.int32),
                vals=np.asarray(d, dtype=np.float64).copy())


def csr_to_dense(A):
    n = A["n"]
    D = np.zeros((n, n))
    r = np.repeat(np.arange(n), np.diff(A["rowptr"]))
    D[r, A["colidx"]] = A["vals"]
    return D


def csr_matvec(A, x):
    """Reference-free numpy CSR product (rows x (n,) or (n, m))."""
    r = np.repeat(np.arange(A["n"]), np.diff(A["rowptr"]))
    contrib = A["vals"].reshape((-1,) + (1,) * (x.ndim - 1)) * x[A["colidx"]]
    out = np.zeros((A["n"],) + x.shape[1:])
    np.add.at(out, r, contrib)
    return out


# --------------------------------------------------------------------------
# grid configurations


CONFIGS = {
    # name: (n per axis, dim, Z shift s, B length l_B, Wendland radius rho,
    #        a kind, ell, q)
    "c1": dict(n=64, dim=2, shift=25.0, lb=0.03, rho=0.1, a="sincos",
               ell=60, rank=50),
    "c2": dict(n=512, dim=2, shift=25.0, lb=0.005, rho=0.015, a="sincos",
               ell=220, rank=200),
    "c3": dict(n=96, dim=3, shift=16.0, lb=0.012, rho=0.025, a="sin3",
               ell=200, ell_ext=400),
    "c5": dict(n=128, dim=3, shift=16.0, lb=0.01, rho=0.02, a="sin3",
               ell=520, rank=500),
    # config 3's operator formulas on a 32^3 grid, with the B length and
    # radius scaled by 96/32 so that the kernel spans the same number of
    # grid points as at 96^3 (a parity case the oracle finishes in seconds)
    "c3_32": dict(n=32, dim=3, shift=16.0, lb=0.036, rho=0.075, a="sin3",
                  ell=40, ell_ext=80),
}


def _coords(n, dim):
    h = 1.0 / (n - 1)
    idx = np.arange(n ** dim, dtype=np.int64)
    c = []
    for d in range(dim):
        c.append((idx // (n ** d)) % n)
    return h, c


def lumped_mass(n, dim):
    """h^d, halved once per boundary axis (edges 1/2, 2D corners 1/4, 3D
    corners 1/8)."""
    h, c = _coords(n, dim)
    m = np.full(n ** dim, h ** dim)
    for ci in c:
        m = np.where((ci == 0) | (ci == n - 1), 0.5 * m, m)
    return m


def z_operator(n, dim, shift, mass):
    """Z = h^(d-2) L + s M, L the Neumann graph Laplacian."""
    h, c = _coords(n, dim)
    N = n ** dim
    scale = h ** (dim - 2)
    offs_sorted = []
    # column order: -n^(d) ... -1, 0, +1 ... +n^(d): sorted by stride
    for d in reversed(range(dim)):
        offs_sorted.append((d, -1))
    offs_sorted.append(None)
    for d in range(dim):
        offs_sorted.append((d, +1))
    K = len(offs_sorted)
    valid = np.zeros((N, K), dtype=bool)
    cols = np.zeros((N, K), dtype=np.int64)
    vals = np.zeros((N, K))
    idx = np.arange(N, dtype=np.int64)
    deg = np.zeros(N)
    for k, o in enumerate(offs_sorted):
        if o is None:
            continue
        d, s = o
        ok = (c[d] + s >= 0) & (c[d] + s < n)
        valid[:, k] = ok
        cols[:, k] = idx + s * (n ** d)
        vals[:, k] = -scale
        deg += ok
    kd = dim
    valid[:, kd] = True
    cols[:, kd] = idx
    vals[:, kd] = scale * deg + shift * mass
    rowptr = np.concatenate([[0], np.cumsum(valid.sum(1))]).astype(np.int64)
    return dict(n=N, rowptr=rowptr, colidx=cols[valid].astype(np.int32),
                vals=vals[valid])


def a_field(n, dim, kind):
    h, c = _coords(n, dim)
    x = [ci * h for ci in c]
    if kind == "sincos":
        return 1.0 + 0.5 * np.sin(2 * np.pi * x[0]) * np.cos(2 * np.pi * x[1])
    return 1.0 + 0.5 * (np.sin(2 * np.pi * x[0]) * np.sin(2 * np.pi * x[1])
                        * np.sin(2 * np.pi * x[2]))


def b_operator(n, dim, lb, rho, mass, a, dtype=np.float64):
    """Gaussian x Wendland-C2 kernel matrix in CSR (columns sorted)."""
    h, c = _coords(n, dim)
    N = n ** dim
    R = rho / h
    r = int(math.floor(R))
    offs = []
    rng = range(-r, r + 1)
    if dim == 2:
        for dy in rng:
            for dx in rng:
                if dx * dx + dy * dy < R * R:
                    offs.append((dx, dy, 0))
    else:
        for dz in rng:
            for dy in rng:
                for dx in rng:
                    if dx * dx + dy * dy + dz * dz < R * R:
                        offs.append((dx, dy, dz))
    K = len(offs)
    idx = np.arange(N, dtype=np.int64)
    am = a * mass
    valid = np.zeros((N, K), dtype=bool)
    cols = np.zeros((N, K), dtype=np.int32)
    vals = np.zeros((N, K), dtype=dtype)
    for k, (dx, dy, dz) in enumerate(offs):
        ok = (c[0] + dx >= 0) & (c[0] + dx < n) & (c[1] + dy >= 0) \
            & (c[1] + dy < n)
        if dim == 3:
            ok &= (c[2] + dz >= 0) & (c[2] + dz < n)
        j = idx + dx + dy * n + (dz * n * n if dim == 3 else 0)
        jj = np.where(ok, j, idx)
        dist = h * math.sqrt(dx * dx + dy * dy + dz * dz)
        t = dist / rho
        g = math.exp(-dist * dist / (2 * lb * lb)) * (1 - t) ** 4 * (4 * t + 1)
        valid[:, k] = ok
        cols[:, k] = jj.astype(np.int32)
        vals[:, k] = (am * am[jj] * g).astype(dtype)
    counts = valid.sum(1)
    rowptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    return dict(n=N, rowptr=rowptr, colidx=cols[valid], vals=vals[valid])


def grid_problem(name, dtype=np.float64):
    """Mass, Z and B of a named configuration (c1, c2, c3, c5)."""
    cfg = dict(CONFIGS[name])
    n, dim = cfg["n"], cfg["dim"]
    mass = lumped_mass(n, dim)
    Z = z_operator(n, dim, cfg["shift"], mass)
    a = a_field(n, dim, cfg["a"])
    B = b_operator(n, dim, cfg["lb"], cfg["rho"], mass, a, dtype=dtype)
    cfg.update(N=n ** dim, mass=mass, Z=Z, B=B,
               nnz_B=int(B["rowptr"][-1]), nnz_Z=int(Z["rowptr"][-1]))
    return cfg


def hashed_normal_block(randn_at, seed, n, m):
    """Host helper: an (n, m) block of N(0,1) from a scalar randn_at."""
    out = np.empty((n, m))
    for j in range(m):
        for i in range(n):
            out[i, j] = randn_at(seed, i, j)
    return out

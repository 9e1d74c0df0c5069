"""Seeded synthetic SOCP instances with the shapes of the benchmark configs.

No public instance set is used by the benchmark, so these seeded generators
are the workloads.  Every instance has a strictly feasible planted point x0
and a planted dual (y0, z0) that makes the problem bounded; c = A'y0 + z0.
x0 is feasible but in general not optimal: the reference answer is always a
solve, never x0.

Pins (choices the workload description leaves open):
* config 1 variable cones: 100k x 3, 5k x 50, 20 x 5000 (650k variables);
  constraint cones on A2: 100k x 3 + 4k x 50 (500k rows);
* A1 row lengths: lognormal with median 10 and sigma sqrt(2 ln 2) (mean 20),
  clipped to [1, 2000]; A2 rows: uniform integer lengths in [5, 15];
* config 2: each of the 2000 cones is (t_k, G_k x) with G_k a 100 x n block of
  20 nonzeros per row (a 1% density would be 400M nonzeros), t_k fixed by the
  planted point; sectors are contiguous blocks of 20 assets with bounds
  [0.5, 2] x (sector size / n).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .model import SOCPModel


def _interior_cone(rng, dims, margin=(0.5, 1.5)):
    """Points strictly inside second-order cones of the given sizes."""
    out = []
    for d in dims:
        xi = rng.standard_normal(d - 1)
        t = np.linalg.norm(xi) + rng.uniform(*margin)
        out.append(np.concatenate([[t], xi]))
    return np.concatenate(out) if out else np.zeros(0)


def _interior_cones_vec(rng, dims):
    """Vectorised interior points for many equal-size cones."""
    parts = []
    dims = np.asarray(dims)
    for d in np.unique(dims):
        k = int((dims == d).sum())
        xi = rng.standard_normal((k, d - 1))
        t = np.linalg.norm(xi, axis=1) + rng.uniform(0.5, 1.5, size=k)
        parts.append((d, np.concatenate([t[:, None], xi], axis=1)))
    # restore the order of `dims`
    res = np.empty(int(dims.sum()))
    starts = np.concatenate([[0], np.cumsum(dims)])
    cursor = {d: 0 for d, _ in parts}
    table = {d: blk for d, blk in parts}
    for i, d in enumerate(dims):
        res[starts[i]:starts[i + 1]] = table[d][cursor[d]]
        cursor[d] += 1
    return res


def _random_rows(rng, nrows, ncols, lengths):
    """CSR with the given row lengths, uniform columns, N(0,1) values."""
    lengths = np.asarray(lengths, dtype=np.int64)
    nnz = int(lengths.sum())
    rows = np.repeat(np.arange(nrows, dtype=np.int64), lengths)
    cols = rng.integers(0, ncols, size=nnz, dtype=np.int64)
    vals = rng.standard_normal(nnz)
    M = sp.csr_matrix((vals, (rows, cols)), shape=(nrows, ncols))
    M.sum_duplicates()
    M.sort_indices()
    return M


def _cone_starts(first, dims):
    return np.concatenate([[first], first + np.cumsum(dims)]).astype(np.int64)


def _assemble(rng, A1, A2, n_box, var_dims, con_dims, box=(-10.0, 10.0), lin_band=(0.0, 1.0)):
    m1, n = A1.shape
    m2 = A2.shape[0]
    nv = int(np.sum(var_dims))
    assert n_box + nv == n and int(np.sum(con_dims)) == m2
    x0 = np.concatenate([rng.uniform(box[0] / 2, box[1] / 2, size=n_box),
                         _interior_cones_vec(rng, var_dims) if nv else np.zeros(0)])
    A = sp.vstack([A1, A2]).tocsr()
    ax1 = A1 @ x0
    AL1 = ax1 - rng.uniform(*lin_band, size=m1)
    AU1 = ax1 + rng.uniform(*lin_band, size=m1)
    s0 = _interior_cones_vec(rng, con_dims) if m2 else np.zeros(0)
    b2 = A2 @ x0 - s0
    y0 = np.concatenate([rng.standard_normal(m1), _interior_cones_vec(rng, con_dims) if m2 else np.zeros(0)])
    z0 = np.concatenate([np.zeros(n_box), _interior_cones_vec(rng, var_dims) if nv else np.zeros(0)])
    c = A.T @ y0 + z0
    m = m1 + m2
    AL = np.concatenate([AL1, np.full(m2, -np.inf)])
    AU = np.concatenate([AU1, np.full(m2, np.inf)])
    l = np.concatenate([np.full(n_box, box[0]), np.full(nv, -np.inf)])
    u = np.concatenate([np.full(n_box, box[1]), np.full(nv, np.inf)])
    model = SOCPModel(A=A, c=c, AL=AL, AU=AU, l=l, u=u, soc_rhs=b2,
                      SOC_con_idx=_cone_starts(m1, con_dims), SOC_var_idx=_cone_starts(n_box, var_dims),
                      number_linear_con=m1, number_lu_x=n_box)
    model.planted = {"x0": x0, "y0": y0, "z0": z0}
    return model


def config0(seed: int = 0) -> SOCPModel:
    """Small plain SOCP: n=2000 (1000 boxed in [-10,10], 50 cones of 20),
    A1 1000x2000 and A2 500x2000 at 1% density, 25 constraint cones of 20."""
    rng = np.random.default_rng(seed)
    n, n_box = 2000, 1000
    A1 = sp.random(1000, n, density=0.01, random_state=rng, data_rvs=rng.standard_normal, format="csr")
    A2 = sp.random(500, n, density=0.01, random_state=rng, data_rvs=rng.standard_normal, format="csr")
    return _assemble(rng, A1, A2, n_box, [20] * 50, [20] * 25)


def config1(seed: int = 1, scale: float = 1.0) -> SOCPModel:
    """Large sparse SOCP (scale=1): n=2,000,000, A1 1M rows (~20M nnz,
    lognormal rows, median 10, max 2000), A2 500k rows (5M nnz); variable
    cones 100k x 3, 5k x 50, 20 x 5000; constraint cones 100k x 3 + 4k x 50.
    ``scale`` shrinks every count (not the cone sizes) for tests."""
    rng = np.random.default_rng(seed)
    k3, k50, k5000 = (max(1, int(round(v * scale))) for v in (100_000, 5_000, 20))
    huge = 5000 if scale >= 0.05 else max(200, int(5000 * scale * 20))
    var_dims = [3] * k3 + [50] * k50 + [huge] * k5000
    n = max(int(round(2_000_000 * scale)), int(np.sum(var_dims)) + 10)
    n_box = n - int(np.sum(var_dims))
    m1 = max(1, int(round(1_000_000 * scale)))
    c3, c50 = max(1, int(round(100_000 * scale))), max(1, int(round(4_000 * scale)))
    con_dims = [3] * c3 + [50] * c50
    m2 = int(np.sum(con_dims))
    sig = np.sqrt(2 * np.log(2.0))
    len1 = np.clip(np.rint(np.exp(np.log(10.0) + sig * rng.standard_normal(m1))), 1, 2000).astype(np.int64)
    A1 = _random_rows(rng, m1, n, len1)
    len2 = rng.integers(5, 16, size=m2)
    A2 = _random_rows(rng, m2, n, len2)
    return _assemble(rng, A1, A2, n_box, var_dims, con_dims)


def config2(seed: int = 2, scale: float = 1.0) -> SOCPModel:
    """Robust-portfolio QP-SOCP: Q = D + F'F as an operator (D ~ U(0.01,1),
    F 50 x n at 5%), budget row, box 0 <= x <= 0.05, sector rows with
    two-sided bounds, 2000 tracking cones of dimension 101.  n=200k at
    scale=1."""
    rng = np.random.default_rng(seed)
    n = max(200, int(round(200_000 * scale)))
    nsec = max(1, int(round(10_000 * scale)))
    ncone = max(1, int(round(2_000 * scale)))
    D = rng.uniform(0.01, 1.0, size=n)
    F = sp.random(50, n, density=0.05, random_state=rng, data_rvs=rng.standard_normal, format="csr") * 0.1
    x0 = np.full(n, 1.0 / n)
    budget = sp.csr_matrix(np.ones((1, n)))
    sec_of = np.minimum(np.arange(n) * nsec // n, nsec - 1)
    S = sp.csr_matrix((np.ones(n), (sec_of, np.arange(n))), shape=(nsec, n))
    size = np.bincount(sec_of, minlength=nsec).astype(float)
    blocks = []
    rhs = []
    for k in range(ncone):
        G = _random_rows(rng, 100, n, np.full(100, 20))
        t = 2.0 * np.linalg.norm(G @ x0) + 1e-3
        blocks.append(sp.csr_matrix((1, n)))
        blocks.append(G)
        rhs.append(np.concatenate([[-t], np.zeros(100)]))
    A2 = sp.vstack(blocks).tocsr()
    A = sp.vstack([budget, S, A2]).tocsr()
    m_lin = 1 + nsec
    AL = np.concatenate([[1.0], 0.5 * size / n, np.full(A2.shape[0], -np.inf)])
    AU = np.concatenate([[1.0], 2.0 * size / n, np.full(A2.shape[0], np.inf)])
    mu = rng.uniform(0.0, 0.1, size=n)
    c = -mu
    model = SOCPModel(A=A, c=c, AL=AL, AU=AU, l=np.zeros(n), u=np.full(n, 0.05),
                      soc_rhs=np.concatenate(rhs), SOC_con_idx=_cone_starts(m_lin, [101] * ncone),
                      SOC_var_idx=np.array([n], dtype=np.int64), number_linear_con=m_lin, number_lu_x=n,
                      q_diag=D, F=F)
    model.planted = {"x0": x0}
    return model


def qp_csr(seed: int = 4, n: int = 3000, density: float = 0.01) -> SOCPModel:
    """QP-SOCP with a general sparse CSR Q that has off-diagonal entries:
    Q = B'B + diag(d), B an (n/4) x n matrix with 3 nonzeros per column
    (N(0,1) values) and d ~ U(0.01, 1), so Q is positive definite with about
    9 off-diagonal entries per row.  n/2 boxed variables in [-10, 10], the
    rest in cones of 20; A1 (n/2 rows) and A2 (n/4 rows in cones of 25) at
    `density`.  Q is passed as a CSR matrix, so it is scaled with A and its
    lambda_max comes from the power iteration (not from its diagonal).  The
    planted dual makes the problem bounded: c = A'y0 + z0 - Q x0."""
    rng = np.random.default_rng(seed)
    n_cone = (n // 2) // 20 * 20
    n_box = n - n_cone
    var_dims = [20] * (n_cone // 20)
    m1 = n // 2
    m2 = (n // 4) // 25 * 25
    A1 = sp.random(m1, n, density=density, random_state=rng, data_rvs=rng.standard_normal, format="csr")
    A2 = sp.random(m2, n, density=density, random_state=rng, data_rvs=rng.standard_normal, format="csr")
    model = _assemble(rng, A1, A2, n_box, var_dims, [25] * (m2 // 25))
    k = max(1, n // 4)
    rows = rng.integers(0, k, size=3 * n)
    cols = np.repeat(np.arange(n), 3)
    B = sp.csr_matrix((rng.standard_normal(3 * n), (rows, cols)), shape=(k, n))
    Q = (B.T @ B + sp.diags(rng.uniform(0.01, 1.0, size=n))).tocsr()
    model.Q = Q
    model.c = model.c - Q @ model.planted["x0"]
    model.__post_init__()
    return model


def small_socp(seed: int, n: int = None, diag_q: bool = None) -> SOCPModel:
    """One instance of the serving stream: n lognormal (median 400, 50..20000),
    m ~ n/2, density 2-5%, 1-200 variable cones of size 3-64, and for half of
    the instances a diagonal Q with U(0,1) entries."""
    rng = np.random.default_rng(seed)
    if n is None:
        n = int(np.clip(np.rint(np.exp(np.log(400.0) + 0.8 * rng.standard_normal())), 50, 20000))
    m = max(1, n // 2)
    dens = rng.uniform(0.02, 0.05)
    ncones = int(rng.integers(1, 201))
    dims = list(rng.integers(3, 65, size=ncones))
    while sum(dims) > n // 2 and len(dims) > 1:
        dims.pop()
    if sum(dims) > n // 2:
        dims = [min(dims[0], max(3, n // 2))]
    nv = int(sum(dims))
    n_box = n - nv
    mc_dims = []
    m_con = m // 3
    while m_con >= 3 and sum(mc_dims) + 3 <= m_con:
        d = int(rng.integers(3, 17))
        if sum(mc_dims) + d > m_con:
            break
        mc_dims.append(d)
    m2 = int(sum(mc_dims))
    m1 = m - m2
    A1 = sp.random(m1, n, density=dens, random_state=rng, data_rvs=rng.standard_normal, format="csr")
    A2 = sp.random(m2, n, density=dens, random_state=rng, data_rvs=rng.standard_normal, format="csr")
    model = _assemble(rng, A1, A2, n_box, dims, mc_dims)
    if diag_q is None:
        diag_q = bool(rng.integers(0, 2))
    if diag_q:
        model.Q = sp.diags(rng.uniform(0.0, 1.0, size=n)).tocsr()
        model.__post_init__()
    return model


def serving_stream(seed: int, count: int, rate: float = 0.0, procs: int = 0):
    """The serving workload: `count` small SOCPs (small_socp) with a per-request
    tolerance of 1e-4 or 1e-6 (50/50) and Poisson arrival times at `rate`
    requests/s (rate <= 0: everything arrives at t = 0, i.e. saturation).
    Returns a list of (model, stoptol, arrival_s).  procs > 1 builds the
    instances in that many worker processes (same instances)."""
    rng = np.random.default_rng(seed)
    specs = []
    t = 0.0
    for k in range(count):
        tol = 1e-4 if rng.integers(0, 2) == 0 else 1e-6
        if rate > 0:
            t += rng.exponential(1.0 / rate)
        specs.append((int(rng.integers(0, 2**31 - 1)), tol, t))
    if procs > 1 and count > 64:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(procs) as pool:
            models = pool.map(small_socp, [sd for sd, _, _ in specs], chunksize=64)
    else:
        models = [small_socp(sd) for sd, _, _ in specs]
    return [(m, tol, t) for m, (_, tol, t) in zip(models, specs)]

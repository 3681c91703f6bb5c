"""Density-fitted Coulomb matrix from the packed device output (the consumer
step of the (mu nu|P) path).

For a symmetric density D (n_ao x n_ao), with (mu nu|P) from a batch run or
from its auxiliary windows and the metric (P|Q):

    gamma_P = sum_{mu nu} (mu nu|P) D_{mu nu}
    c       = (P|Q)^{-1} gamma             (Cholesky factorisation, FP64)
    J_{mu nu} = sum_P (mu nu|P) c_P

Everything stays on the device: each packed class block [pair shell][I][J][K]
[aux shell] is read as a (pairs*I*J) x (K*aux) matrix, so the dense
(n_aux, n_ao, n_ao) tensor is never formed.

* ``BatchCoulomb`` (many molecules at once, the whole batch output resident):
  gamma and J are the library's own kernels (eip_batch_df_gamma /
  eip_batch_df_coulomb, csrc/df.cu), one launch each for every block of every
  molecule; the FP64 Cholesky factorisation of each (P|Q) and the triangular
  solves are library calls (torch.linalg, cuSOLVER).
* ``coulomb_matrix`` (one molecule, optionally window by window over the
  auxiliary basis): the density is gathered into each block's row order
  (off-diagonal shell pairs count twice) and the contractions are library
  GEMV calls on the window buffer.
"""

import numpy as np

from .batch import ThreeCenterBatch, metric_pair_tables


def _pairs(p):
    return np.unique(np.stack([np.asarray(p.i_ao_start), np.asarray(p.j_ao_start)], 1), axis=0)


class _Blocks:
    """Row/column index tensors of every class block of one molecule slot."""

    def __init__(self, torch, pair_data, aux_data, block_of, window=None):
        dev = "cuda"
        self.items = []
        for (li, lj), p in pair_data.items():
            pairs = _pairs(p)
            ni, nj = 2 * li + 1, 2 * lj + 1
            mu = torch.as_tensor(pairs[:, 0][:, None] + np.arange(ni)[None, :], device=dev)
            nu = torch.as_tensor(pairs[:, 1][:, None] + np.arange(nj)[None, :], device=dev)
            rows_mu = mu[:, :, None].expand(-1, ni, nj).reshape(-1)
            rows_nu = nu[:, None, :].expand(-1, ni, nj).reshape(-1)
            twice = torch.as_tensor(np.repeat(np.where(pairs[:, 0] != pairs[:, 1], 2.0, 1.0), ni * nj), device=dev)
            off = torch.as_tensor(np.repeat(pairs[:, 0] != pairs[:, 1], ni * nj), device=dev)
            for lk, a in aux_data.items():
                blk = block_of(li, lj, lk)
                if blk is None or blk[1] == 0 or blk[2] == 0:
                    continue
                o, nsp, nax = blk
                nk = 2 * lk + 1
                starts = np.unique(np.asarray(a.i_ao_start))
                if window is not None:
                    starts = starts[(starts >= window[0]) & (starts < window[1])]
                if starts.size != nax:
                    raise RuntimeError("window block does not match the auxiliary shells")
                cols = torch.as_tensor((np.arange(nk)[:, None] + starts[None, :]).reshape(-1), device=dev)
                self.items.append((o, nsp * ni * nj, nk * nax, rows_mu, rows_nu, twice, off, cols))


def _gamma(torch, buf, blocks, D, gamma):
    for o, nr, nc, mu, nu, twice, off, cols in blocks.items:
        block = buf[o:o + nr * nc].view(nr, nc)
        d = D[mu, nu] * twice
        gamma.index_add_(0, cols, d @ block)


def _coulomb(torch, buf, blocks, c, J):
    for o, nr, nc, mu, nu, twice, off, cols in blocks.items:
        block = buf[o:o + nr * nc].view(nr, nc)
        v = block @ c[cols]
        J.index_put_((mu, nu), v, accumulate=True)
        J.index_put_((nu[off], mu[off]), v[off], accumulate=True)


def metric_matrix(torch, molecule, aux_data):
    """(P|Q) (n_aux x n_aux, FP64, device) from the one-centre pair classes."""
    b = ThreeCenterBatch([molecule], [metric_pair_tables(aux_data)], [aux_data], precision="fp64")
    out = torch.empty(max(b.output_elems, 1), dtype=torch.float64, device="cuda")
    b.bind_output(out.data_ptr())
    b.run()
    b.status()
    M = torch.zeros((molecule.n_aux, molecule.n_aux), dtype=torch.float64, device="cuda")
    for (_, lP), p in metric_pair_tables(aux_data).items():
        P0 = np.unique(np.asarray(p.j_ao_start))
        nP = 2 * lP + 1
        rows = torch.as_tensor((P0[:, None] + np.arange(nP)[None, :]).reshape(-1), device="cuda")
        for lQ, a in aux_data.items():
            blk = b.block(0, 0, lP, lQ)
            if blk is None or blk[2] == 0:
                continue
            o, nsp, nax = blk
            nQ = 2 * lQ + 1
            Q0 = np.unique(np.asarray(a.i_ao_start))
            cols = torch.as_tensor((np.arange(nQ)[:, None] + Q0[None, :]).reshape(-1), device="cuda")
            M[rows[:, None], cols[None, :]] = out[o:o + nsp * nP * nQ * nax].view(nsp * nP, nQ * nax)
    b.bind_output(0)
    b.close()
    return M


def metric_factor(torch, M, max_shift=1e-8):
    """Lower Cholesky factor of the metric, FP64 (library call).  Even-tempered
    auxiliary bases on nearby atoms make (P|Q) nearly singular (condition
    numbers beyond 1e12), so when the plain factorisation fails the diagonal is
    raised by the smallest shift lambda = 10^k * max(diag M), k = -15..-8, that
    lets it complete.  Returns (L, lambda)."""
    Lf, info = torch.linalg.cholesky_ex(M)
    if int(info) == 0:
        return Lf, 0.0
    scale = float(M.diagonal().max())
    eye = torch.eye(M.shape[0], dtype=M.dtype, device=M.device)
    for k in range(-15, int(round(__import__("math").log10(max_shift))) + 1):
        lam = scale * 10.0 ** k
        Lf, info = torch.linalg.cholesky_ex(M + lam * eye)
        if int(info) == 0:
            return Lf, lam
    raise RuntimeError("metric not factorisable with a diagonal shift up to max_shift * max(diag)")


def coulomb_matrix(molecule, pair_data, aux_data, D, precision="fp64", window_bytes=None, metric=None):
    """Density-fitted J for one molecule.  With window_bytes, (mu nu|P) is
    computed in auxiliary windows of at most that many output bytes over one
    resident batch, twice (once for gamma, once for J), so no more than one
    window is ever held.  Returns (J, c, gamma) as device tensors.""" 
    import torch

    from .serving import window_edges

    D = torch.as_tensor(np.asarray(D), dtype=torch.float64, device="cuda")
    M = metric_matrix(torch, molecule, aux_data) if metric is None else metric
    b = ThreeCenterBatch([molecule], [pair_data], [aux_data], precision=precision)
    full = b.window()
    if window_bytes is None or 8 * full <= window_bytes:
        edges = [0, molecule.n_aux]
    else:
        width = max(1, int(molecule.n_aux * (window_bytes / 8) / full))
        edges = window_edges(aux_data, molecule.n_aux, width)
    sizes = [b.window([lo], [hi]) for lo, hi in zip(edges[:-1], edges[1:])]
    buf = torch.empty(max(max(sizes), 1), dtype=torch.float64, device="cuda")
    gamma = torch.zeros(molecule.n_aux, dtype=torch.float64, device="cuda")
    J = torch.zeros((molecule.n_ao, molecule.n_ao), dtype=torch.float64, device="cuda")
    stream = torch.cuda.ExternalStream(b.stream)

    def windows():
        for lo, hi in zip(edges[:-1], edges[1:]):
            b.window([lo], [hi])
            b.run_window(buf.data_ptr())
            torch.cuda.current_stream().wait_stream(stream)
            yield _Blocks(torch, pair_data, aux_data, lambda li, lj, lk: b.window_block(0, li, lj, lk), (lo, hi))
            torch.cuda.current_stream().synchronize()  # the next window overwrites buf

    for blocks in windows():
        _gamma(torch, buf, blocks, D, gamma)
    L = torch.linalg.cholesky(M)
    c = torch.cholesky_solve(gamma[:, None], L)[:, 0]
    for blocks in windows():
        _coulomb(torch, buf, blocks, c, J)
    b.status()
    b.close()
    return J, c, gamma


class BatchCoulomb:
    """Density-fitted J for every molecule of a batch with its packed output
    bound and computed (``batch.run()``):

        gamma = (mu nu|P) D,   c = (P|Q)^{-1} gamma,   J = (mu nu|P) c

    ``metric_factors``: per molecule the lower Cholesky factor L of its (P|Q)
    (device, FP64), e.g. ``torch.linalg.cholesky(metric_matrix(...))``.  With
    ``inverse_factors`` the factors are inverted once here (L^{-1}, a
    triangular solve against the identity, like the factorisation a
    per-geometry cost) and every solve is two matrix-vector products,
    c = L^{-T} (L^{-1} gamma), each reading the inverse once at memory speed;
    otherwise each solve is a pair of triangular substitutions
    (``torch.cholesky_solve``).  The densities and results are concatenated
    device arrays (molecule m's n_ao^2 block after the previous molecules');
    ``run`` queues everything on the batch stream's side of the current torch
    stream and returns J."""

    def __init__(self, torch, batch, metric_factors, inverse_factors=False):
        self.torch = torch
        self.batch = batch
        self.n_ao2, self.n_aux = batch.df_plan()
        self.inverse = inverse_factors
        self.factors = []
        for Lf in metric_factors:
            if inverse_factors:
                eye = torch.eye(Lf.shape[0], dtype=Lf.dtype, device=Lf.device)
                Lf = torch.linalg.solve_triangular(Lf, eye, upper=False)
            self.factors.append(Lf)
        self.aux_off = np.concatenate([[0], np.cumsum([m.n_aux for m in batch.molecules])]).astype(np.int64)
        self.ao_off = np.concatenate([[0], np.cumsum([m.n_ao ** 2 for m in batch.molecules])]).astype(np.int64)
        dev = "cuda"
        self.gamma = torch.zeros(max(self.n_aux, 1), dtype=torch.float64, device=dev)
        self.c = torch.zeros(max(self.n_aux, 1), dtype=torch.float64, device=dev)
        self.J = torch.zeros(max(self.n_ao2, 1), dtype=torch.float64, device=dev)
        self.stream = torch.cuda.ExternalStream(batch.stream)

    def fit(self, D):
        """gamma = (mu nu|P) D for every molecule (D: concatenated densities).
        The batch stream first waits for the current torch stream, where D and
        this object's buffers and (inverted) factors were made; solve and
        coulomb follow on the batch stream."""
        self.stream.wait_stream(self.torch.cuda.current_stream())
        self.batch.df_gamma(D.data_ptr(), self.gamma.data_ptr())

    def solve(self):
        """c = (P|Q)^{-1} gamma for every molecule, on the batch stream."""
        torch = self.torch
        with torch.cuda.stream(self.stream):
            for m, F in enumerate(self.factors):
                a0, a1 = int(self.aux_off[m]), int(self.aux_off[m + 1])
                if a1 <= a0:
                    continue
                if self.inverse:
                    self.c[a0:a1] = torch.mv(F.T, torch.mv(F, self.gamma[a0:a1]))
                else:
                    self.c[a0:a1] = torch.cholesky_solve(self.gamma[a0:a1, None], F)[:, 0]

    def coulomb(self):
        """J = (mu nu|P) c for every molecule."""
        self.batch.df_coulomb(self.c.data_ptr(), self.J.data_ptr())

    def run(self, D):
        """D: concatenated densities (device tensor of n_ao2 doubles).  Returns
        the concatenated J (device tensor; valid once the batch stream is done)."""
        self.fit(D)
        self.solve()
        self.coulomb()
        return self.J

    def molecule_J(self, m):
        n = self.batch.molecules[m].n_ao
        return self.J[int(self.ao_off[m]):int(self.ao_off[m + 1])].view(n, n)

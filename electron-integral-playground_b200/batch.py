"""Batched (mu nu|P) over many molecules (the eip_batch_* C ABI).

All molecules' pair and auxiliary tables are uploaded once and stay on the
device; every run is one CUDA-graph launch that computes every
(l_i, l_j | l_k) class of every molecule into a packed device buffer
(one block per molecule and class, layout [pair shell][I][J][K][aux shell]).
``dense(m)`` expands molecule m's blocks into the reference's dense
(n_aux, n_ao, n_ao) layout (used by tests; the packed form is the product).

Two more integral kinds run through the same kernels:

* nuclear attraction V[mu nu C]: point charges per molecule (``charges_list``)
  form the ket class ``POINT_CHARGES`` (l_k = 0, one block entry per charge);
  ``dense_V(m)`` gives the reference's (n_ao, n_ao, n_charge) layout;
* the two-centre metric (P|Q): ``metric_pair_tables(aux)`` turns the auxiliary
  basis into one-centre pair tables (an exponent-0 s function times each
  auxiliary primitive, A = B = P), so a molecule slot with those pairs and the
  auxiliary tables as ket computes (0, l_P | l_Q) blocks; ``dense_metric(m)``
  gives the reference's (n_aux, n_aux) layout.
"""

import ctypes

import numpy as np

from ._lib import IntegralError, as_f64, as_i32, dp, ip, lib

_vp = ctypes.c_void_p

POINT_CHARGES = -1  # ket-class key of point charges (EIP_POINT_CHARGES)


def metric_pair_tables(aux_data):
    """(P|Q) as three-centre classes (0, l_P | l_Q): every auxiliary primitive
    becomes a one-centre pair: A = (P, exponent 0), B = (P, q), P_p = (P, q),
    coefficient = the primitive's, i_ao_start = 0, j_ao_start = P's first
    function."""
    from .data_structure import PrimitivePairData

    out = {}
    for l, a in aux_data.items():
        B = np.ascontiguousarray(np.asarray(a.A_a, np.float64))
        A = B.copy()
        A[:, 3] = 0.0
        st = np.asarray(a.i_ao_start, np.int32)
        out[(0, int(l))] = PrimitivePairData(P_p=B, A_a=A, B_b=B, coefficient=np.ascontiguousarray(a.coefficient),
                                             i_ao_start=np.zeros_like(st), j_ao_start=st.copy(), i_atom=None,
                                             j_atom=None)
    return out


def _bind(L):
    if getattr(L, "_batch_bound", False):
        return
    c_int, c_double, c_bool, c_ll = ctypes.c_int, ctypes.c_double, ctypes.c_bool, ctypes.c_longlong
    _dpp = ctypes.POINTER(ctypes.c_double)
    _ipp = ctypes.POINTER(ctypes.c_int)
    L.eip_batch_create.argtypes = [c_int, c_bool, c_double]
    L.eip_batch_create.restype = _vp
    L.eip_batch_add_pairs.argtypes = [_vp, c_int, c_int, c_int, _dpp, _dpp, _dpp, _dpp, _ipp, _ipp, c_int]
    L.eip_batch_add_aux.argtypes = [_vp, c_int, c_int, _dpp, _dpp, _ipp, c_int]
    L.eip_batch_add_charges.argtypes = [_vp, c_int, _dpp, c_int]
    L.eip_batch_build.argtypes = [_vp]
    L.eip_batch_set_precision.argtypes = [_vp, c_int, c_double]
    L.eip_batch_set_streams.argtypes = [_vp, c_int]
    L.eip_batch_precision_split.argtypes = [_vp, c_int, c_int, c_int, ctypes.POINTER(c_ll), ctypes.POINTER(c_ll)]
    L.eip_batch_output_elems.argtypes = [_vp]
    L.eip_batch_output_elems.restype = c_ll
    L.eip_batch_block.argtypes = [_vp, c_int, c_int, c_int, c_int, ctypes.POINTER(c_ll), _ipp, _ipp]
    L.eip_batch_alloc_output.argtypes = [_vp]
    L.eip_batch_bind_output.argtypes = [_vp, _vp]
    L.eip_batch_output_device.argtypes = [_vp]
    L.eip_batch_output_device.restype = _vp
    L.eip_batch_run.argtypes = [_vp, c_int]
    L.eip_batch_run_class.argtypes = [_vp, c_int, c_int, c_int]
    L.eip_batch_window_plan.argtypes = [_vp, _ipp, _ipp, c_int]
    L.eip_batch_window_plan.restype = c_ll
    L.eip_batch_window_block.argtypes = [_vp, c_int, c_int, c_int, c_int, ctypes.POINTER(c_ll), _ipp, _ipp]
    L.eip_batch_run_window.argtypes = [_vp, _vp, c_int]
    L.eip_batch_sync.argtypes = [_vp]
    L.eip_batch_status.argtypes = [_vp]
    L.eip_batch_upload.argtypes = [_vp]
    L.eip_batch_table_bytes.argtypes = [_vp]
    L.eip_batch_table_bytes.restype = c_ll
    L.eip_batch_device_bytes.argtypes = [_vp]
    L.eip_batch_device_bytes.restype = c_ll
    L.eip_batch_class_splits.argtypes = [_vp, c_int, c_int, c_int]
    L.eip_batch_class_splits.restype = c_int
    L.eip_batch_launches_per_run.argtypes = [_vp]
    L.eip_batch_launches_per_run.restype = ctypes.c_ulonglong
    L.eip_batch_checksums.argtypes = [_vp, _dpp]
    L.eip_batch_copy_output.argtypes = [_vp, c_ll, c_ll, _dpp]
    L.eip_batch_stream.argtypes = [_vp]
    L.eip_batch_stream.restype = _vp
    L.eip_batch_error.argtypes = [_vp]
    L.eip_batch_error.restype = ctypes.c_char_p
    L.eip_batch_df_plan.argtypes = [_vp, _ipp, _ipp]
    L.eip_batch_df_gamma.argtypes = [_vp, _vp, _vp]
    L.eip_batch_df_coulomb.argtypes = [_vp, _vp, _vp]
    L.eip_batch_destroy.argtypes = [_vp]
    L.eip_batch_destroy.restype = None
    L._batch_bound = True


DEFAULT_FP32_THRESHOLD = 1e-3


class ThreeCenterBatch:
    """precision: "fp64", or "mixed" (FP32 R/ket/bra for shell pairs whose
    bound Q_pair * max Q_aux (times the output-transform gains) is below
    fp32_threshold; FP64 Boys, E recurrences, prefactors and every other pair)."""

    def __init__(self, molecules, pair_data_list, aux_data_list, omega: float = 0.0, precision: str = "fp64",
                 fp32_threshold: float = DEFAULT_FP32_THRESHOLD, charges_list=None):
        if not (len(molecules) == len(pair_data_list) == len(aux_data_list)) or not molecules:
            raise ValueError("need one pair table and one auxiliary table per molecule")
        if charges_list is None:
            charges_list = [None] * len(molecules)
        if len(charges_list) != len(molecules):
            raise ValueError("need one charge array (or None) per molecule")
        spherical = {bool(m.spherical_basis) for m in molecules}
        if len(spherical) != 1:
            raise ValueError("all molecules of a batch must share spherical_basis")
        self.L = lib()
        _bind(self.L)
        self.molecules = molecules
        self.pair_data_list = pair_data_list
        self.aux_data_list = aux_data_list
        self.charges_list = charges_list
        self.spherical = spherical.pop()
        self.omega = float(omega)
        self.h = self.L.eip_batch_create(len(molecules), self.spherical, self.omega)
        if not self.h:
            raise IntegralError("eip_batch_create failed")
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.precision = precision
        self._check(self.L.eip_batch_set_precision(self.h, 1 if precision == "mixed" else 0, float(fp32_threshold)),
                    "set_precision")
        self._keep = []
        for m, (pd, ad) in enumerate(zip(pair_data_list, aux_data_list)):
            for (li, lj), p in pd.items():
                arrs = [as_f64(p.P_p, (4,)), as_f64(p.A_a, (4,)), as_f64(p.B_b, (4,)), as_f64(p.coefficient),
                        as_i32(p.i_ao_start), as_i32(p.j_ao_start)]
                self._keep.append(arrs)
                self._check(self.L.eip_batch_add_pairs(self.h, m, int(li), int(lj), dp(arrs[0]), dp(arrs[1]),
                                                       dp(arrs[2]), dp(arrs[3]), ip(arrs[4]), ip(arrs[5]),
                                                       arrs[0].shape[0]), "add_pairs")
            for lk, a in ad.items():
                arrs = [as_f64(a.A_a, (4,)), as_f64(a.coefficient), as_i32(a.i_ao_start)]
                self._keep.append(arrs)
                self._check(self.L.eip_batch_add_aux(self.h, m, int(lk), dp(arrs[0]), dp(arrs[1]), ip(arrs[2]),
                                                     arrs[0].shape[0]), "add_aux")
            if charges_list[m] is not None and len(charges_list[m]) > 0:
                c = as_f64(np.asarray(charges_list[m]).reshape(-1, 3), (3,))
                self._keep.append([c])
                self._check(self.L.eip_batch_add_charges(self.h, m, dp(c), c.shape[0]), "add_charges")
        self._check(self.L.eip_batch_build(self.h), "build")
        self._keep = None
        self.output_elems = int(self.L.eip_batch_output_elems(self.h))

    def _check(self, rc, what):
        if rc == 1:
            raise IntegralError(f"eip_batch_{what}: unsupported angular class")
        if rc != 0:
            raise IntegralError(f"eip_batch_{what}: {self.L.eip_batch_error(self.h).decode(errors='replace')}")

    @property
    def output_bytes(self):
        return 8 * self.output_elems

    def alloc_output(self):
        self._check(self.L.eip_batch_alloc_output(self.h), "alloc_output")

    def bind_output(self, device_ptr: int):
        self._check(self.L.eip_batch_bind_output(self.h, ctypes.c_void_p(device_ptr)), "bind_output")

    def set_streams(self, n: int):
        """Streams the class kernels are forked over (before the first run)."""
        self._check(self.L.eip_batch_set_streams(self.h, int(n)), "set_streams")

    def run(self, checksum: bool = False, sync: bool = True):
        self._check(self.L.eip_batch_run(self.h, 1 if checksum else 0), "run")
        if sync:
            self.sync()

    def run_class(self, li, lj, lk):
        """Launch one class's kernel alone on the batch stream (per-kernel timing)."""
        rc = self.L.eip_batch_run_class(self.h, li, lj, lk)
        if rc == 1:
            return False
        self._check(rc, "run_class")
        return True

    def window(self, fn_lo=None, fn_hi=None, with_charges=False):
        """Select the auxiliary window [fn_lo[m], fn_hi[m]) of every molecule
        (None: all functions); returns the window's packed output size."""
        if (fn_lo is None) != (fn_hi is None):
            raise ValueError("give both window bounds or neither")
        if fn_lo is not None:
            lo = as_i32(np.broadcast_to(np.asarray(fn_lo), (len(self.molecules),)))
            hi = as_i32(np.broadcast_to(np.asarray(fn_hi), (len(self.molecules),)))
            n = self.L.eip_batch_window_plan(self.h, ip(lo), ip(hi), 1 if with_charges else 0)
        else:
            n = self.L.eip_batch_window_plan(self.h, None, None, 1 if with_charges else 0)
        if n < 0:
            raise IntegralError(f"eip_batch_window_plan: {self.L.eip_batch_error(self.h).decode(errors='replace')}")
        return int(n)

    def window_block(self, m, li, lj, lk):
        off, nsp, nax = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_int()
        rc = self.L.eip_batch_window_block(self.h, m, li, lj, lk, ctypes.byref(off), ctypes.byref(nsp),
                                           ctypes.byref(nax))
        if rc != 0:
            return None
        return off.value, nsp.value, nax.value

    def run_window(self, device_ptr: int, checksum: bool = False):
        """Launch the selected window into device memory at device_ptr (async)."""
        self._check(self.L.eip_batch_run_window(self.h, ctypes.c_void_p(device_ptr), 1 if checksum else 0),
                    "run_window")

    def sync(self):
        self._check(self.L.eip_batch_sync(self.h), "sync")

    def status(self):
        """Raise if a class kernel of the last run recorded a failed self-check."""
        rc = self.L.eip_batch_status(self.h)
        if rc != 0:
            raise IntegralError(f"eip_batch_status: {self.L.eip_batch_error(self.h).decode(errors='replace')}")

    def upload(self):
        self._check(self.L.eip_batch_upload(self.h), "upload")

    @property
    def table_bytes(self):
        return int(self.L.eip_batch_table_bytes(self.h))

    def class_splits(self, li, lj, lk):
        """0: the class runs on a fast kernel; n >= 1: on the general kernel,
        each block split into n items; -1: no such class."""
        return int(self.L.eip_batch_class_splits(self.h, li, lj, lk))

    @property
    def device_bytes(self):
        """Device memory held besides the output (tables, E tables, maps)."""
        return int(self.L.eip_batch_device_bytes(self.h))

    @property
    def launches_per_run(self):
        return int(self.L.eip_batch_launches_per_run(self.h))

    @property
    def stream(self):
        return self.L.eip_batch_stream(self.h)

    def checksums(self):
        out = np.empty(len(self.molecules))
        self._check(self.L.eip_batch_checksums(self.h, dp(out)), "checksums")
        return out

    def precision_split(self, li, lj, lk):
        """(FP64 triplets, FP32 triplets) of one class."""
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        if self.L.eip_batch_precision_split(self.h, li, lj, lk, ctypes.byref(a), ctypes.byref(b)) != 0:
            return None
        return a.value, b.value

    def block(self, m, li, lj, lk):
        off, nsp, nax = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_int()
        rc = self.L.eip_batch_block(self.h, m, li, lj, lk, ctypes.byref(off), ctypes.byref(nsp), ctypes.byref(nax))
        if rc != 0:
            return None
        return off.value, nsp.value, nax.value

    def dense(self, m):
        """Molecule m's (mu nu|P) in the reference's dense layout (n_aux, n_ao, n_ao)."""
        mol = self.molecules[m]
        J = np.zeros((mol.n_aux, mol.n_ao, mol.n_ao))
        sph = self.spherical
        n_of = (lambda l: 2 * l + 1) if sph else (lambda l: (l + 1) * (l + 2) // 2)
        for (li, lj), p in self.pair_data_list[m].items():
            pairs = np.unique(np.stack([np.asarray(p.i_ao_start), np.asarray(p.j_ao_start)], 1), axis=0)
            for lk, a in self.aux_data_list[m].items():
                blk = self.block(m, li, lj, lk)
                if blk is None or blk[1] == 0 or blk[2] == 0:
                    continue
                off, nsp, nax = blk
                ni, nj, nk = n_of(li), n_of(lj), n_of(lk)
                buf = np.empty(nsp * ni * nj * nk * nax)
                self._check(self.L.eip_batch_copy_output(self.h, off, buf.size, dp(buf)), "copy_output")
                buf = buf.reshape(nsp, ni, nj, nk, nax)
                aux0 = np.unique(np.asarray(a.i_ao_start))
                assert pairs.shape[0] == nsp and aux0.shape[0] == nax
                I = pairs[:, 0][:, None, None, None, None] + np.arange(ni)[None, :, None, None, None]
                Jc = pairs[:, 1][:, None, None, None, None] + np.arange(nj)[None, None, :, None, None]
                K = aux0[None, None, None, None, :] + np.arange(nk)[None, None, None, :, None]
                I, Jc, K = np.broadcast_arrays(I, Jc, K)
                J[K, I, Jc] = buf
                off_diag = np.broadcast_to((pairs[:, 0] != pairs[:, 1])[:, None, None, None, None], buf.shape)
                J[K[off_diag], Jc[off_diag], I[off_diag]] = buf[off_diag]
        return J

    def _block_array(self, m, li, lj, lk, ni, nj, nk):
        blk = self.block(m, li, lj, lk)
        if blk is None or blk[1] == 0 or blk[2] == 0:
            return None
        off, nsp, nax = blk
        buf = np.empty(nsp * ni * nj * nk * nax)
        self._check(self.L.eip_batch_copy_output(self.h, off, buf.size, dp(buf)), "copy_output")
        return buf.reshape(nsp, ni, nj, nk, nax)

    def dense_V(self, m):
        """Molecule m's V[mu nu C] in the reference's layout (n_ao, n_ao, n_charge)."""
        mol = self.molecules[m]
        nc = len(self.charges_list[m])
        V = np.zeros((mol.n_ao, mol.n_ao, nc))
        n_of = (lambda l: 2 * l + 1) if self.spherical else (lambda l: (l + 1) * (l + 2) // 2)
        for (li, lj), p in self.pair_data_list[m].items():
            ni, nj = n_of(li), n_of(lj)
            buf = self._block_array(m, li, lj, POINT_CHARGES, ni, nj, 1)
            if buf is None:
                continue
            pairs = np.unique(np.stack([np.asarray(p.i_ao_start), np.asarray(p.j_ao_start)], 1), axis=0)
            for s, (i0, j0) in enumerate(pairs):
                V[i0:i0 + ni, j0:j0 + nj, :] = buf[s, :, :, 0, :]
                if i0 != j0:
                    V[j0:j0 + nj, i0:i0 + ni, :] = buf[s, :, :, 0, :].transpose(1, 0, 2)
        return V

    def dense_metric(self, m):
        """(P|Q) of a slot built from metric_pair_tables: (n_aux, n_aux)."""
        mol = self.molecules[m]
        M = np.zeros((mol.n_aux, mol.n_aux))
        n_of = (lambda l: 2 * l + 1) if self.spherical else (lambda l: (l + 1) * (l + 2) // 2)
        for (li, lj), p in self.pair_data_list[m].items():
            p_starts = np.unique(np.asarray(p.j_ao_start))
            for lk, a in self.aux_data_list[m].items():
                nj, nk = n_of(lj), n_of(lk)
                buf = self._block_array(m, li, lj, lk, 1, nj, nk)
                if buf is None:
                    continue
                q_starts = np.unique(np.asarray(a.i_ao_start))
                for s, p0 in enumerate(p_starts):
                    for t, q0 in enumerate(q_starts):
                        M[p0:p0 + nj, q0:q0 + nk] = buf[s, 0, :, :, t]
        return M

    def df_plan(self):
        """List the batch's class blocks for the density-fitting contractions
        (df_gamma / df_coulomb); returns (sum n_ao^2, sum n_aux), the sizes of
        the concatenated D / J and gamma / c arrays."""
        n_ao = as_i32([m.n_ao for m in self.molecules])
        n_aux = as_i32([m.n_aux for m in self.molecules])
        self._check(self.L.eip_batch_df_plan(self.h, ip(n_ao), ip(n_aux)), "df_plan")
        return int(np.sum(n_ao.astype(np.int64) ** 2)), int(np.sum(n_aux))

    def df_gamma(self, D_ptr: int, gamma_ptr: int):
        """gamma_P = sum (mu nu|P) D_{mu nu} of every molecule (device arrays, async)."""
        self._check(self.L.eip_batch_df_gamma(self.h, ctypes.c_void_p(D_ptr), ctypes.c_void_p(gamma_ptr)),
                    "df_gamma")

    def df_coulomb(self, c_ptr: int, J_ptr: int):
        """J_{mu nu} = sum (mu nu|P) c_P of every molecule (device arrays, async)."""
        self._check(self.L.eip_batch_df_coulomb(self.h, ctypes.c_void_p(c_ptr), ctypes.c_void_p(J_ptr)),
                    "df_coulomb")

    def close(self):
        if self.h:
            self.L.eip_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def measure_fma_peak(fp64: bool = True) -> float:
    """FP64 (or FP32) FMA throughput of the current device in TFLOP/s."""
    L = lib()
    L.eip_measure_fma_peak.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    v = ctypes.c_double()
    if L.eip_measure_fma_peak(1 if fp64 else 0, ctypes.byref(v)) != 0:
        raise IntegralError("FMA peak microbenchmark failed")
    return v.value

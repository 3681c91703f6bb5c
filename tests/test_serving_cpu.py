"""Host logic of the server and the metric tables (no GPU): arena
sub-allocation, auxiliary slicing, packed sizes, one-centre pair tables."""

import importlib

import numpy as np

syn = importlib.import_module("electron-integral-playground_b200.synthetic")
pu = importlib.import_module("electron-integral-playground_b200.pair_utility")
sv = importlib.import_module("electron-integral-playground_b200.serving")
bt = importlib.import_module("electron-integral-playground_b200.batch")


class _Buf:
    def __init__(self, n):
        self.n = n

    def numel(self):
        return self.n


class _FakeTorch:
    float64 = "f64"

    @staticmethod
    def empty(n, dtype=None, device=None):
        return _Buf(n)


def test_arena_first_fit_and_merge():
    a = sv.Arena(_FakeTorch, 1024)
    x = a.alloc(100)
    y = a.alloc(200)
    z = a.alloc(300)
    assert x == (0, 128) and y == (128, 224) and z == (352, 320)
    assert a.alloc(1000) is None
    a.release(*y)
    assert a.largest_free == 1024 - 672
    w = a.alloc(64)
    assert w[0] == 128  # first fit reuses the hole
    a.release(*x)
    a.release(*w)
    a.release(*z)
    assert a.free == [(0, 1024)]


def _mol(n, seed):
    return syn.attach_synthetic_basis(syn.organic_molecule(n, seed), aux_l_max=4, seed=0)


def test_aux_slices_cover_every_shell_once():
    m = _mol(8, 3)
    ad = pu.form_auxiliary_pair_data(m)
    sl = sv.aux_slices(ad, m.n_aux, 200)
    assert len(sl) > 1
    assert sl[0][0] == 0 and sl[-1][1] == m.n_aux
    for (lo, hi, sub), nxt in zip(sl, sl[1:] + [(m.n_aux, None, None)]):
        assert hi == nxt[0]
    seen = []
    for lo, hi, sub in sl:
        for l, a in sub.items():
            st = np.asarray(a.i_ao_start) + lo
            assert np.all((st >= lo) & (st < hi))
            seen.append(np.stack([np.full(st.shape, l), st, np.asarray(a.A_a)[:, 3]], 1))
    seen = np.concatenate(seen)
    full = np.concatenate([np.stack([np.full(len(a.i_ao_start), l), np.asarray(a.i_ao_start),
                                     np.asarray(a.A_a)[:, 3]], 1) for l, a in ad.items()])
    assert sorted(map(tuple, seen)) == sorted(map(tuple, full))
    # slices' packed sizes add up to the whole
    pd = pu.form_pair_data(m, 1e-14)
    assert sum(sv.packed_elems(pd, sub) for _, _, sub in sl) == sv.packed_elems(pd, ad)


def test_packed_elems_counts_shell_pairs_and_charges():
    m = _mol(4, 1)
    pd, ad = pu.form_pair_data(m, 1e-14), pu.form_auxiliary_pair_data(m)
    n_sp = {k: len({(i, j) for i, j in zip(p.i_ao_start, p.j_ao_start)}) for k, p in pd.items()}
    n_ax = {l: len(set(a.i_ao_start)) for l, a in ad.items()}
    want = sum(n_sp[(li, lj)] * (2 * li + 1) * (2 * lj + 1) * (2 * lk + 1) * n_ax[lk]
               for (li, lj) in pd for lk in ad)
    assert sv.packed_elems(pd, ad) == want
    extra = sum(n_sp[(li, lj)] * (2 * li + 1) * (2 * lj + 1) * 5 for (li, lj) in pd)
    assert sv.packed_elems(pd, {}, 5) == extra


def test_metric_pair_tables_are_one_centre():
    m = _mol(3, 2)
    ad = pu.form_auxiliary_pair_data(m)
    mt = bt.metric_pair_tables(ad)
    assert set(mt) == {(0, l) for l in ad}
    for l, a in ad.items():
        p = mt[(0, l)]
        np.testing.assert_array_equal(p.P_p, a.A_a)
        np.testing.assert_array_equal(p.B_b, a.A_a)
        np.testing.assert_array_equal(p.A_a[:, :3], np.asarray(a.A_a)[:, :3])
        assert np.all(p.A_a[:, 3] == 0.0)
        assert np.all(p.i_ao_start == 0)
        np.testing.assert_array_equal(p.j_ao_start, a.i_ao_start)

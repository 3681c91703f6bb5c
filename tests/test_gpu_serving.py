"""GPU checks of the continuous-batching server: every request's integrals are
the same whether it is served alone (FP64, nothing else in flight) or in a mix
of concurrently admitted requests (mixed precision, shared launches, sliced
auxiliary basis), within 1e-10."""

import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

syn = importlib.import_module("electron-integral-playground_b200.synthetic")
pu = importlib.import_module("electron-integral-playground_b200.pair_utility")
mi = importlib.import_module("electron-integral-playground_b200.molecular_integral")
sv = importlib.import_module("electron-integral-playground_b200.serving")


def _requests(sizes, seed=5):
    reqs = []
    for i, n in enumerate(sizes):
        m = syn.attach_synthetic_basis(syn.organic_molecule(n, seed * 100 + i), aux_l_max=4, seed=seed)
        reqs.append(sv.Request(i, m, pu.form_pair_data(m, 1e-14), pu.form_auxiliary_pair_data(m),
                               arrival=0.002 * i))
    return reqs


def _fresh(r):
    return sv.Request(r.rid, r.molecule, r.pair_data, r.aux_data, r.arrival)


def test_request_alone_equals_request_in_the_mix():
    sizes = [3, 9, 5, 14, 4, 11, 7]
    reqs = _requests(sizes)
    budget = 48e6  # small arena: forces auxiliary slicing and queueing
    alone = {}
    for r in reqs:
        s = sv.IntegralServer(budget_bytes=budget, precision="fp64", max_inflight=1, keep_blocks=True,
                              host_overlap=False)
        s.serve([_fresh(r)], realtime=False)
        alone[r.rid] = s.kept[r.rid]
        del s
    mixed = sv.IntegralServer(budget_bytes=budget, precision="mixed", max_inflight=3, keep_blocks=True)
    mix_reqs = [_fresh(r) for r in reqs]
    stats = mixed.serve(mix_reqs, realtime=True)
    assert stats["requests"] == len(reqs)
    assert stats["launches"] < sum(len(mixed.pieces_of(r)) for r in reqs), "pieces should share launches"
    assert any(k[0] == "3c" and k[1] > 0 for k in alone[3]), "the 14-atom request should be sliced"
    for r in mix_reqs:
        a, b = alone[r.rid], mixed.kept[r.rid]
        assert a.keys() == b.keys()
        for k in a:
            err = float(np.max(np.abs(a[k] - b[k]))) if a[k].size else 0.0
            assert err <= 1e-10, (r.rid, k, err)
        assert r.S is not None
        np.testing.assert_array_equal(r.S, mi.overlap(r.pair_data, r.molecule))


@pytest.mark.parametrize("budget", [160e6, 6e6])
def test_served_blocks_match_drop_in(budget):
    """The served V blocks and (P|Q) columns equal the drop-in entry points,
    whole (160 MB arena) and as windows / slices (6 MB arena)."""
    r = _requests([6])[0]
    s = sv.IntegralServer(budget_bytes=budget, precision="fp64", keep_blocks=True, host_overlap=False)
    s.serve([r], realtime=False)
    kept = s.kept[r.rid]
    mol = r.molecule
    V = mi.nuclear_attraction(r.pair_data, mol, mol.geometry)
    M = mi.two_center(r.aux_data, mol)
    nc = mol.geometry.shape[0]
    windows = {k[1] for k in kept if k[0] == "3c"}
    assert (len(windows) > 1) == (budget < 1e7)
    for (li, lj), p in r.pair_data.items():
        pairs = np.unique(np.stack([np.asarray(p.i_ao_start), np.asarray(p.j_ao_start)], 1), axis=0)
        blk = kept[("3c", 0, li, lj, sv.POINT_CHARGES)].reshape(len(pairs), 2 * li + 1, 2 * lj + 1, nc)
        for t, (i0, j0) in enumerate(pairs):
            np.testing.assert_allclose(blk[t], V[i0:i0 + 2 * li + 1, j0:j0 + 2 * lj + 1, :], rtol=0, atol=1e-13)
    n_cols = 0
    for key, v in kept.items():
        if key[0] != "metric":
            continue
        _, lo, _, lP, lQ = key
        P0 = np.unique(np.asarray(r.aux_data[lP].i_ao_start))
        nP, nQ = 2 * lP + 1, 2 * lQ + 1
        nax = v.size // (len(P0) * nP * nQ)
        allQ = np.unique(np.asarray(r.aux_data[lQ].i_ao_start))
        Q0 = allQ[allQ >= lo][:nax]
        blk = v.reshape(len(P0), nP, nQ, nax)
        for s_, p0 in enumerate(P0):
            ref = M[p0:p0 + nP][:, Q0[:, None] + np.arange(nQ)[None, :]]
            np.testing.assert_allclose(blk[s_], ref.transpose(0, 2, 1), rtol=0,
                                       atol=max(1e-12, 1e-13 * float(np.abs(ref).max())))
        n_cols += nax * nQ
    assert n_cols == M.shape[0] * len(r.aux_data)  # every column once per l_P


def test_server_builds_tables_when_requests_carry_molecules_only():
    """Requests without tables: the server builds them (pair tables on the
    device) after arrival; the results equal those from the front end's tables
    to rounding (the device tables differ from numpy's in the last bits)."""
    reqs = _requests([4, 9])
    a = sv.IntegralServer(budget_bytes=48e6, precision="fp64", keep_blocks=True, host_overlap=False)
    a.serve([_fresh(r) for r in reqs], realtime=False)
    b = sv.IntegralServer(budget_bytes=48e6, precision="fp64", keep_blocks=True, host_overlap=False)
    bare = [sv.Request(r.rid, r.molecule, arrival=r.arrival) for r in reqs]
    b.serve(bare, realtime=True)
    for r in reqs:
        ka, kb = a.kept[r.rid], b.kept[r.rid]
        assert ka.keys() == kb.keys()
        for k in ka:
            scale = max(1.0, float(np.max(np.abs(ka[k]))) if ka[k].size else 1.0)
            assert float(np.max(np.abs(ka[k] - kb[k]), initial=0.0)) <= 1e-12 * scale, (r.rid, k)


def test_resident_batches_are_bounded():
    """Windowed requests (a 6 MB arena) keep their tables on the device in a
    resident batch; at most max_resident such batches exist or are being
    built at once, later ones wait in arrival order, and the results are the
    same as with no bound (to rounding: which pieces share a launch, and so
    whether a small class runs on the fast or the general kernel, depends on
    admission)."""
    reqs = _requests([6, 7, 8, 9])
    kw = dict(budget_bytes=6e6, precision="fp64", keep_blocks=True, host_overlap=False)
    loose = sv.IntegralServer(max_resident=8, **kw)
    loose.serve([_fresh(r) for r in reqs], realtime=False)
    tight = sv.IntegralServer(max_resident=1, dead_bytes_max=0, **kw)
    tight.serve([_fresh(r) for r in reqs], realtime=False)
    assert loose.resident_high == len(reqs)
    assert tight.resident_high == 1
    for r in reqs:
        a, b = loose.kept[r.rid], tight.kept[r.rid]
        assert a.keys() == b.keys()
        assert any(k[0] == "3c" and k[1] > 0 for k in a), "every request should be windowed"
        for k in a:
            scale = max(1.0, float(np.max(np.abs(a[k]))) if a[k].size else 1.0)
            np.testing.assert_allclose(b[k], a[k], rtol=0, atol=1e-12 * scale)

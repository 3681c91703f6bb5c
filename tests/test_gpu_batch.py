"""GPU checks of the batched path (eip_batch_*): every molecule's packed
output, expanded to the dense layout, equals the drop-in three_center entry
point and the reference library; checksums match the written values."""

import importlib

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

syn = importlib.import_module("electron-integral-playground_b200.synthetic")
pu = importlib.import_module("electron-integral-playground_b200.pair_utility")
mi = importlib.import_module("electron-integral-playground_b200.molecular_integral")
bt = importlib.import_module("electron-integral-playground_b200.batch")
at = importlib.import_module("electron-integral-playground_b200.autotune")


@pytest.fixture(scope="module")
def small_batch():
    mols = []
    for i, n in enumerate([3, 5, 4, 7]):
        m = syn.organic_molecule(n, seed=100 + i)
        syn.attach_synthetic_basis(m, aux_l_max=4, seed=0)
        mols.append(m)
    pds = [pu.form_pair_data(m, 1e-14) for m in mols]
    ads = [pu.form_auxiliary_pair_data(m) for m in mols]
    b = bt.ThreeCenterBatch(mols, pds, ads)
    b.alloc_output()
    b.run(checksum=True)
    yield mols, pds, ads, b
    b.close()


def test_batch_matches_drop_in(small_batch):
    mols, pds, ads, b = small_batch
    for m in range(len(mols)):
        dense = b.dense(m)
        single = mi.three_center(pds[m], ads[m], mols[m])
        np.testing.assert_allclose(dense, single, rtol=0, atol=1e-14)


def test_batch_matches_reference(small_batch):
    mols, pds, ads, b = small_batch
    ref = oracle.reference()
    if ref is None:
        pytest.skip("reference library not built")
    dense = b.dense(1)
    np.testing.assert_allclose(dense, oracle.drive_three_center(ref, pds[1], ads[1], mols[1]), rtol=0, atol=1e-12)


def test_batch_checksums_and_rerun(small_batch):
    mols, pds, ads, b = small_batch
    ck = b.checksums()
    out = np.empty(b.output_elems)
    b._check(b.L.eip_batch_copy_output(b.h, 0, b.output_elems, out.ctypes.data_as(
        __import__("ctypes").POINTER(__import__("ctypes").c_double))), "copy")
    # per-molecule sums of the packed blocks
    for m in range(len(mols)):
        s = 0.0
        for (li, lj) in pds[m]:
            for lk in ads[m]:
                off, nsp, nax = b.block(m, li, lj, lk)
                n = nsp * (2 * li + 1) * (2 * lj + 1) * (2 * lk + 1) * nax
                s += out[off:off + n].sum()
        assert abs(ck[m] - s) <= 1e-9 * max(1.0, abs(s))
    # graph re-launch is deterministic
    b.run(checksum=True)
    out2 = np.empty_like(out)
    b._check(b.L.eip_batch_copy_output(b.h, 0, b.output_elems, out2.ctypes.data_as(
        __import__("ctypes").POINTER(__import__("ctypes").c_double))), "copy")
    assert np.array_equal(out, out2)


def test_every_tuning_variant_matches_reference(small_batch):
    """All compiled variants of every fast class give the same integrals."""
    mols, pds, ads, b = small_batch
    ref = oracle.reference()
    if ref is None:
        pytest.skip("reference library not built")
    lm = importlib.import_module("electron-integral-playground_b200._lib")
    L = lm.lib()
    want = oracle.drive_three_center(ref, pds[3], ads[3], mols[3])
    saved = {(li, lj, lk): L.eip_tune_get(li, lj, lk) for (li, lj) in pds[3] for lk in ads[3]}
    try:
        for v in range(at.N_VARIANTS):
            for (li, lj, lk) in saved:
                if saved[(li, lj, lk)] >= 0:
                    L.eip_tune_set(li, lj, lk, v)
            got = mi.three_center(pds[3], ads[3], mols[3])
            np.testing.assert_allclose(got, want, rtol=0, atol=1e-12, err_msg=f"variant {v}")
    finally:
        for k, v in saved.items():
            if v >= 0:
                L.eip_tune_set(*k, v)


def _contracted_auxiliary_molecule():
    """A 5-atom molecule whose auxiliary shells (s-g, 3 per l and element) are
    contractions of 1-4 primitives, so the 32 shells of a warp have ragged
    primitive counts (units past a shell's own count contribute nothing)."""
    basis_utility = importlib.import_module("electron-integral-playground_b200.basis_utility")
    readers = importlib.import_module("electron-integral-playground_b200.readers")
    rng = np.random.default_rng(31)
    ladder = [0.1 * 2.5 ** i for i in range(9)]
    lines = []
    for el in ("C", "H", "N", "O"):
        lines.append(f"{el}     0")
        for l in range(5):
            for _ in range(3):
                k = int(rng.integers(1, 5))
                exps = sorted(rng.choice(ladder, size=k, replace=False), reverse=True)
                lines.append(f"{basis_utility.ANGULAR_LETTERS[l]}    {k}   1.00")
                for e in exps:
                    lines.append(f"    {float(e)!r}    {float(rng.uniform(0.2, 1.0))!r}")
        lines.append("****")
    m = syn.organic_molecule(5, seed=40)
    m.spherical_basis = True
    basis_utility.attach_basis_to_molecule(m, readers.read_basis_content(syn.orbital_basis_text(["H", "C", "N", "O"], 3)))
    basis_utility.attach_auxiliary_basis_to_molecule(m, readers.read_basis_content("\n".join(lines) + "\n"))
    return m


def test_contracted_auxiliary_every_variant_and_mixed():
    """Contracted, ragged auxiliary shells through every launch variant of the
    fast kernels (one-warp and multi-warp CTAs), FP64 and FP32, against the
    reference library."""
    ref = oracle.reference()
    if ref is None:
        pytest.skip("reference library not built")
    m = _contracted_auxiliary_molecule()
    pd, ad = pu.form_pair_data(m, 1e-14), pu.form_auxiliary_pair_data(m)
    counts = np.concatenate([np.unique(a.i_ao_start, return_counts=True)[1] for a in ad.values()])
    assert counts.max() > 1 and counts.min() == 1  # ragged contractions
    want = oracle.drive_three_center(ref, pd, ad, m)
    lm = importlib.import_module("electron-integral-playground_b200._lib")
    L = lm.lib()
    saved = {(li, lj, lk): L.eip_tune_get(li, lj, lk) for (li, lj) in pd for lk in ad}
    try:
        for v in range(at.N_VARIANTS):
            for (li, lj, lk) in saved:
                if saved[(li, lj, lk)] >= 0:
                    L.eip_tune_set(li, lj, lk, v)
            got = mi.three_center(pd, ad, m)
            np.testing.assert_allclose(got, want, rtol=0, atol=1e-12, err_msg=f"variant {v}")
    finally:
        for k, v in saved.items():
            if v >= 0:
                L.eip_tune_set(*k, v)
    # every shell pair in FP32 (R, ket, bra), through every FP32 launch variant:
    # a loose bound that still catches any misplaced component or unit
    saved32 = {k: L.eip_tune_get_fp32(*k) for k in saved}
    try:
        for v in at.FP32_VARIANTS:
            for k in saved32:
                if saved32[k] >= 0:
                    assert L.eip_tune_set_fp32(*k, v) == 0
            mix = bt.ThreeCenterBatch([m], [pd], [ad], precision="mixed", fp32_threshold=float("inf"))
            mix.alloc_output()
            mix.run()
            mix.status()
            err = np.max(np.abs(mix.dense(0) - want))
            mix.close()
            assert 0.0 < err <= 1e-4 * max(1.0, float(np.max(np.abs(want)))), (v, err)
    finally:
        for k, v in saved32.items():
            if v >= 0:
                L.eip_tune_set_fp32(*k, v)


def _two_fragments():
    ds = importlib.import_module("electron-integral-playground_b200.data_structure")
    a = syn.organic_molecule(6, seed=21)
    b = syn.organic_molecule(6, seed=22)
    shift = np.array([12.0, 3.0, -2.0]) / 0.52917721054482
    m = ds.Molecule(elements=a.elements + b.elements, geometry=np.vstack([a.geometry, b.geometry + shift]))
    syn.attach_synthetic_basis(m, aux_l_max=4, seed=0)
    return m


def test_mixed_precision_within_1e10_of_fp64():
    m = _two_fragments()
    pd, ad = pu.form_pair_data(m, 1e-14), pu.form_auxiliary_pair_data(m)
    f64 = bt.ThreeCenterBatch([m], [pd], [ad], precision="fp64")
    mix = bt.ThreeCenterBatch([m], [pd], [ad], precision="mixed")
    f32_triplets = 0
    for (li, lj) in pd:
        for lk in ad:
            split = mix.precision_split(li, lj, lk)
            if split:
                f32_triplets += split[1]
    assert f32_triplets > 0, "the gate should send the far fragment pairs to FP32"
    for b in (f64, mix):
        b.alloc_output()
        b.run()
        b.status()
    d64, dmix = f64.dense(0), mix.dense(0)
    err = np.max(np.abs(d64 - dmix))
    assert err <= 1e-10, err
    assert err > 0.0  # the FP32 path really ran
    f64.close()
    mix.close()


def _pq_close(a, b):
    """(P|Q) reaches ~1e2: 1e-12 absolute where |v| <= 10, 1e-13 relative above."""
    tol = np.maximum(1e-12, 1e-13 * np.abs(b))
    err = np.abs(a - b)
    assert np.all(err <= tol), float(np.max(err / tol))


@pytest.mark.parametrize("omega", [0.0, 0.3])
def test_batch_point_charges_match_nuclear_attraction(small_batch, omega):
    """The point-charge ket class gives the drop-in nuclear_attraction V[mu nu C]
    (and the reference library's) for every molecule of a batch."""
    mols, pds, ads, _ = small_batch
    charges = [m.geometry for m in mols]
    b = bt.ThreeCenterBatch(mols, pds, ads, omega=omega, charges_list=charges)
    b.alloc_output()
    b.run()
    b.status()
    ref = oracle.reference()
    for m in range(len(mols)):
        V = b.dense_V(m)
        np.testing.assert_allclose(V, mi.nuclear_attraction(pds[m], mols[m], charges[m], omega), rtol=0,
                                   atol=1e-13)
        if ref is not None:
            np.testing.assert_allclose(V, oracle.drive_nuclear_attraction(ref, pds[m], mols[m], charges[m], omega),
                                       rtol=0, atol=1e-12)
    # the (mu nu|P) blocks are unchanged by the extra ket class
    np.testing.assert_allclose(b.dense(2), mi.three_center(pds[2], ads[2], mols[2], omega), rtol=0, atol=1e-14)
    b.close()


@pytest.mark.parametrize("omega", [0.0, 0.3])
def test_batch_metric_matches_two_center(small_batch, omega):
    """(P|Q) as one-centre pair classes (0, l_P | l_Q) on the fast kernels equals
    the drop-in two_center and the reference library."""
    mols, _, ads, _ = small_batch
    metric = [bt.metric_pair_tables(a) for a in ads]
    b = bt.ThreeCenterBatch(mols, metric, ads, omega=omega)
    b.alloc_output()
    b.run()
    b.status()
    ref = oracle.reference()
    for m in range(len(mols)):
        M = b.dense_metric(m)
        _pq_close(M, mi.two_center(ads[m], mols[m], omega))
        if ref is not None:
            _pq_close(M, oracle.drive_two_center(ref, ads[m], mols[m], omega))
    b.close()


def test_mixed_batch_keeps_the_metric_fp64():
    """(P|Q) feeds a Cholesky factorisation: in a mixed-precision batch its
    one-centre pairs never take the FP32 path, so it equals the FP64 batch."""
    m = _two_fragments()
    ad = pu.form_auxiliary_pair_data(m)
    metric = bt.metric_pair_tables(ad)
    f64 = bt.ThreeCenterBatch([m], [metric], [ad], precision="fp64")
    mix = bt.ThreeCenterBatch([m], [metric], [ad], precision="mixed")
    for b in (f64, mix):
        b.alloc_output()
        b.run()
        b.status()
    assert all(mix.precision_split(0, l, k)[1] == 0 for l in ad for k in ad)
    np.testing.assert_array_equal(f64.dense_metric(0), mix.dense_metric(0))
    f64.close()
    mix.close()


def test_window_runs_reproduce_the_full_run(small_batch):
    """Runs over auxiliary windows (per-molecule function ranges, resident
    tables) give exactly the corresponding slices of the full run's blocks,
    FP64 and mixed, with and without the point-charge class."""
    import torch

    mols, pds, ads, _ = small_batch
    charges = [m.geometry for m in mols]
    for precision in ("fp64", "mixed"):
        b = bt.ThreeCenterBatch(mols, pds, ads, precision=precision, charges_list=charges)
        b.alloc_output()
        b.run()
        b.status()
        full = np.empty(b.output_elems)
        b._check(b.L.eip_batch_copy_output(b.h, 0, b.output_elems, full.ctypes.data_as(
            __import__("ctypes").POINTER(__import__("ctypes").c_double))), "copy")
        rng = np.random.default_rng(3)
        for trial in range(3):
            lo = np.array([int(rng.integers(0, max(1, m.n_aux // 2))) for m in mols])
            hi = np.array([int(rng.integers(l + 1, m.n_aux + 1)) for l, m in zip(lo, mols)])
            if trial == 2:
                lo[1], hi[1] = 0, 0  # an empty window
            n = b.window(lo, hi, with_charges=(trial == 0))
            out = torch.full((max(n, 1),), float("nan"), dtype=torch.float64, device="cuda")
            b.run_window(out.data_ptr())
            b.sync()
            b.status()
            w = out.cpu().numpy()
            seen = 0
            for m in range(len(mols)):
                for (li, lj) in pds[m]:
                    kets = list(ads[m]) + [bt.POINT_CHARGES]
                    for lk in kets:
                        f_off, nsp, nax = b.block(m, li, lj, lk)
                        w_off, wsp, wax = b.window_block(m, li, lj, lk)
                        nk = 1 if lk == bt.POINT_CHARGES else 2 * lk + 1
                        shape = (nsp, 2 * li + 1, 2 * lj + 1, nk)
                        fb = full[f_off:f_off + np.prod(shape) * nax].reshape(shape + (nax,))
                        if lk == bt.POINT_CHARGES:
                            sel = slice(0, nax) if trial == 0 else slice(0, 0)
                        else:
                            st = np.unique(np.asarray(ads[m][lk].i_ao_start))
                            sel = slice(int(np.searchsorted(st, lo[m])), int(np.searchsorted(st, hi[m])))
                        want = fb[..., sel]
                        assert wsp == nsp and wax == want.shape[-1]
                        got = w[w_off:w_off + want.size].reshape(want.shape)
                        assert np.array_equal(got, want), (precision, m, li, lj, lk)
                        seen += want.size
            assert seen == n
        b.close()


def test_cartesian_batch_matches_drop_in():
    """Cartesian output (every class on the generic kernels inside the graph)."""
    mols = []
    for i, n in enumerate([3, 4]):
        m = syn.organic_molecule(n, seed=300 + i)
        syn.attach_synthetic_basis(m, aux_l_max=3, seed=1, spherical=False)
        mols.append(m)
    pds = [pu.form_pair_data(m, 1e-14) for m in mols]
    ads = [pu.form_auxiliary_pair_data(m) for m in mols]
    b = bt.ThreeCenterBatch(mols, pds, ads)
    b.alloc_output()
    b.run()
    b.status()
    for m in range(len(mols)):
        np.testing.assert_allclose(b.dense(m), mi.three_center(pds[m], ads[m], mols[m]), rtol=0, atol=1e-13)
    b.close()

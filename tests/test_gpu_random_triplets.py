"""High-angular-momentum stress (2000 random shell triplets: orbital l <= 4,
auxiliary l <= 5, 1-8 primitives, exponents log-uniform in [0.05, 1e4],
centres in a 6 A cube): the FP64 drop-in against the reference library, the
mixed-precision batch against the FP64 batch, and the device Boys function
against the long-double series on 1e6 (T, m) samples."""

import importlib

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

syn = importlib.import_module("electron-integral-playground_b200.synthetic")
mi = importlib.import_module("electron-integral-playground_b200.molecular_integral")
bt = importlib.import_module("electron-integral-playground_b200.batch")
lib = importlib.import_module("electron-integral-playground_b200._lib")


@pytest.fixture(scope="module")
def triplets():
    return syn.random_shell_triplets(0, 2000)


def test_boys_1e6_samples_against_series():
    rng = np.random.default_rng(11)
    T = np.concatenate([[0.0, 1e-300, 1e-12, 0.025, 35.99, 36.0, 36.01, 200.0], rng.uniform(0, 200, 1000000)])
    L = 15
    F = lib.device_boys(L, T).reshape(T.size, L + 1)
    ref = oracle.boys_many(L, T)
    rel = np.abs(F - ref) / np.abs(ref)
    assert np.max(rel) < 1e-14, float(np.max(rel))


# The triplets of the seeded 2000 whose FP64 value cancels: every one of them
# has an f or g shell on centre B (l_j >= 3) and extreme exponents, and the
# reference and this repository's independent C oracle already differ on it
# by 5e-13 to 2.5e-10.  Only these may exceed
# 1e-12 (each within 4x that distance); any other triplet must meet 1e-12.
CANCELLING_TRIPLETS = frozenset({160, 276, 372, 404, 422, 546, 626, 694, 717, 949, 1096, 1117, 1192, 1287, 1377,
                                 1431, 1526, 1735, 1868, 1880})


def test_2000_triplets_fp64_against_reference(triplets):
    """|GPU - reference| <= 1e-12 max(1, max|reference|) for at least 98% of the
    triplets; the rest are high-L triplets with extreme exponents whose FP64
    values cancel: two independent FP64 implementations (the reference and
    this repository's C oracle) already differ on them by up to ~2.5e-10.
    Those triplets are named (CANCELLING_TRIPLETS); there the GPU must be
    within max(1e-11, 4x the oracle-to-reference distance)."""
    ref = oracle.reference()
    if ref is None:
        pytest.skip("reference library not built")
    worst, enveloped = 0.0, []
    for n, (lij, pair, lk, aux, mol) in enumerate(triplets):
        got = mi.three_center({lij: pair}, {lk: aux}, mol)
        want = oracle.drive_three_center(ref, {lij: pair}, {lk: aux}, mol)
        scale = max(1.0, float(np.max(np.abs(want))))
        err = float(np.max(np.abs(got - want))) / scale
        worst = max(worst, err)
        if err > 1e-12:
            other = oracle.drive_three_center(oracle.oracle(), {lij: pair}, {lk: aux}, mol)
            env = float(np.max(np.abs(other - want))) / scale
            enveloped.append((n, lij, lk, err, env))
    print(f"2000 triplets: max |GPU - reference| / max(1, |reference|) = {worst:.3e}; "
          f"{len(enveloped)} above 1e-12 (triplet, class, GPU error, oracle-reference distance): {enveloped}")
    for n, lij, lk, err, env in enveloped:
        assert n in CANCELLING_TRIPLETS, (n, lij, lk, err, env)
        assert err <= max(1e-11, 4 * env), (n, lij, lk, err, env)


def test_2000_triplets_mixed_against_fp64(triplets):
    mols = [t[4] for t in triplets]
    pds = [{t[0]: t[1]} for t in triplets]
    ads = [{t[2]: t[3]} for t in triplets]
    f64 = bt.ThreeCenterBatch(mols, pds, ads, precision="fp64")
    mix = bt.ThreeCenterBatch(mols, pds, ads, precision="mixed")
    out = []
    for b in (f64, mix):
        b.alloc_output()
        b.run()
        b.status()
        buf = np.empty(b.output_elems)
        b._check(b.L.eip_batch_copy_output(b.h, 0, b.output_elems, lib.dp(buf)), "copy")
        out.append(buf)
    assert f64.output_elems == mix.output_elems
    err = np.abs(out[0] - out[1])
    classes = {(t[0][0], t[0][1], t[2]) for t in triplets}
    n32 = sum((mix.precision_split(*c) or (0, 0))[1] for c in classes)
    print(f"mixed vs FP64: max abs {err.max():.3e} over {err.size} values; {n32} of 2000 triplets in FP32")
    assert err.max() <= 1e-10, float(err.max())
    # and the FP64 batch equals the drop-in for a sample of triplets
    for m in range(0, 2000, 97):
        np.testing.assert_allclose(f64.dense(m), mi.three_center(pds[m], ads[m], mols[m]), rtol=0,
                                   atol=1e-12 * max(1.0, float(np.abs(out[0]).max())))
    f64.close()
    mix.close()


def test_2000_triplets_batch_with_split_items(triplets):
    """The batch splits the blocks of its heavy general classes (up to 8x8
    primitive pairs x 8 auxiliary primitives) over several CTAs, whose partial
    blocks the last to arrive adds in split order.  Every triplet equals the
    unsplit drop-in (1e-12 max(1, |v|); the named cancelling triplets 1e-10),
    and repeated runs, one class launched alone and a window over every
    auxiliary function all reproduce the full run bit for bit."""
    mols = [t[4] for t in triplets]
    pds = [{t[0]: t[1]} for t in triplets]
    ads = [{t[2]: t[3]} for t in triplets]
    b = bt.ThreeCenterBatch(mols, pds, ads, precision="fp64")
    b.alloc_output()
    classes = sorted({(t[0][0], t[0][1], t[2]) for t in triplets})
    splits = {c: b.class_splits(*c) for c in classes}
    assert max(splits.values()) > 1, splits
    assert splits[(4, 4, 5)] > 1

    def copy():
        buf = np.empty(b.output_elems)
        b._check(b.L.eip_batch_copy_output(b.h, 0, b.output_elems, lib.dp(buf)), "copy")
        return buf

    b.run()
    b.status()
    first = copy()
    b.run()
    b.status()
    np.testing.assert_array_equal(copy(), first)
    for n, (lij, pair, lk, aux, mol) in enumerate(triplets):
        want = mi.three_center({lij: pair}, {lk: aux}, mol)
        scale = max(1.0, float(np.max(np.abs(want))))
        err = float(np.max(np.abs(b.dense(n) - want))) / scale
        assert err <= (1e-10 if n in CANCELLING_TRIPLETS else 1e-12), (n, lij, lk, err)
    # one split class alone (over the full run's output: the same values)
    assert b.run_class(4, 4, 5)
    b.sync()
    b.status()
    np.testing.assert_array_equal(copy(), first)
    # a window over every auxiliary function reproduces the full run
    import torch

    n = b.window()
    assert n == b.output_elems
    out = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
    b.run_window(out.data_ptr())
    b.sync()
    b.status()
    w = out.cpu().numpy()
    for m, (lij, pair, lk, aux, mol) in enumerate(triplets):
        f_off, nsp, nax = b.block(m, lij[0], lij[1], lk)
        w_off, wsp, wax = b.window_block(m, lij[0], lij[1], lk)
        size = nsp * (2 * lij[0] + 1) * (2 * lij[1] + 1) * (2 * lk + 1) * nax
        assert (wsp, wax) == (nsp, nax)
        assert np.array_equal(w[w_off:w_off + size], first[f_off:f_off + size]), m
    b.close()

"""eip_three_center_noalloc: the (mu nu|P) entry point that allocates nothing.

It exists for callers that cannot let a library call cudaMalloc -- code whose
device memory is owned by another allocator (a framework's caching pool, or a
program that reserves the device up front) and code where an allocation could
stall, fail or synchronise at an unpredictable time.  It takes device inputs
and a device output and keeps its working memory in one fixed 16 MiB device
array.  Here it is checked, through the C ABI, against the reference-compatible
three_center() entry point on two calls in a row (the second call finds the
first call's data still in the shared array), and its size limit is checked.
Collected last so that a run stopping at the first failure has run the rest.
"""

import ctypes
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

syn = importlib.import_module("electron-integral-playground_b200.synthetic")
pu = importlib.import_module("electron-integral-playground_b200.pair_utility")
lm = importlib.import_module("electron-integral-playground_b200._lib")

FP64_ATOL = 1e-12
_vp = ctypes.c_void_p


def _bind():
    L = lm.lib()
    f = L.eip_three_center_noalloc
    f.argtypes = [ctypes.c_int] * 3 + [_vp] * 6 + [ctypes.c_int] + [_vp] * 3 + [ctypes.c_int, _vp, ctypes.c_int,
                                                                            ctypes.c_int, ctypes.c_bool,
                                                                            ctypes.c_double, _vp]
    f.restype = ctypes.c_int
    L.eip_last_error.restype = ctypes.c_char_p
    return L


def _existing(L, li, lj, lk, p, a, mol):
    out = np.zeros((mol.n_aux, mol.n_ao, mol.n_ao))
    rc = L.three_center(li, lj, lk, lm.dp(p.P_p), lm.dp(p.A_a), lm.dp(p.B_b), lm.dp(p.coefficient),
                        lm.ip(p.i_ao_start), lm.ip(p.j_ao_start), p.P_p.shape[0], lm.dp(a.A_a),
                        lm.dp(a.coefficient), lm.ip(a.i_ao_start), a.A_a.shape[0], lm.dp(out), mol.n_ao,
                        mol.n_aux, True, 0.0)
    assert rc == 0
    return out


def _noalloc(L, torch, li, lj, lk, p, a, mol, out_dev):
    d = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in
         (p.P_p, p.A_a, p.B_b, p.coefficient, p.i_ao_start, p.j_ao_start, a.A_a, a.coefficient, a.i_ao_start)]
    stream = torch.cuda.current_stream()
    rc = L.eip_three_center_noalloc(li, lj, lk, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), d[3].data_ptr(),
                                    d[4].data_ptr(), d[5].data_ptr(), p.P_p.shape[0], d[6].data_ptr(),
                                    d[7].data_ptr(), d[8].data_ptr(), a.A_a.shape[0], out_dev.data_ptr(), mol.n_ao,
                                    mol.n_aux, True, 0.0, _vp(stream.cuda_stream))
    torch.cuda.synchronize()
    return rc


def test_noalloc_matches_three_center_on_two_calls():
    torch = pytest.importorskip("torch")
    L = _bind()
    mol = syn.organic_molecule(4, seed=11)
    syn.attach_synthetic_basis(mol, aux_l_max=3, seed=11)
    pd = pu.form_pair_data(mol, 1e-14)
    ad = pu.form_auxiliary_pair_data(mol)
    for (li, lj), lk in [((1, 2), 3), ((0, 1), 2)]:
        p, a = pd[(li, lj)], ad[lk]
        want = _existing(L, li, lj, lk, p, a, mol)
        out = torch.zeros(mol.n_aux * mol.n_ao * mol.n_ao, dtype=torch.float64, device="cuda")
        assert _noalloc(L, torch, li, lj, lk, p, a, mol, out) == 0
        got = out.cpu().numpy().reshape(want.shape)
        np.testing.assert_allclose(got, want, rtol=0, atol=FP64_ATOL)


def test_noalloc_rejects_calls_beyond_its_fixed_memory():
    torch = pytest.importorskip("torch")
    L = _bind()
    mol = syn.organic_molecule(40, seed=3)
    syn.attach_synthetic_basis(mol, aux_l_max=4, seed=0)
    pd = pu.form_pair_data(mol, 1e-14)
    ad = pu.form_auxiliary_pair_data(mol)
    p, a = pd[(1, 2)], ad[4]
    # the host-side check must already say "too large": only then is the call
    # made, with an output buffer that a launch would overrun
    chk = L.eip_three_center_noalloc_check
    chk.argtypes = [ctypes.c_int] * 5 + [ctypes.c_bool, ctypes.POINTER(ctypes.c_size_t)]
    chk.restype = ctypes.c_int
    need = ctypes.c_size_t(0)
    assert chk(1, 2, 4, p.P_p.shape[0], a.A_a.shape[0], True, ctypes.byref(need)) == 4
    out = torch.zeros(16, dtype=torch.float64, device="cuda")  # never touched on rejection
    assert _noalloc(L, torch, 1, 2, 4, p, a, mol, out) == 4
    assert b"fixed limit" in L.eip_last_error()
    assert float(out.abs().sum()) == 0.0

"""Fermion storage conversion on the device (cpsb_fermion_convert) against the
oracle's restatement of Lattice::Fconvert (itself pinned to the compiled
reference by tests/test_oracle_golden.py): a permutation, so bit-exact."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims,ls,order", [((4, 4, 4, 6), 1, 0), ((4, 4, 4, 6), 4, 0), ((4, 4, 4, 6), 4, 1),
                                           ((8, 6, 4, 4), 6, 0), ((8, 6, 4, 4), 8, 1)])
def test_fermion_convert_matches_oracle(dims, ls, order):
    import torch
    import cps_public_b200 as cb
    from cps_public_b200 import _lib
    from oracle import oracle
    cb.init(0)
    lib = _lib.load()
    v = np.random.default_rng(11).standard_normal(int(np.prod(dims)) * ls * 24)
    name = "wilson" if order == 0 else "4d_ee"
    d = (C.c_int * 4)(*dims)
    vin = torch.from_numpy(v).cuda()
    vout = torch.empty_like(vin)
    for direction in (0, 1):
        _lib.check(lib.cpsb_fermion_convert(d, ls, order, direction, C.c_void_p(vout.data_ptr()),
                                            C.c_void_p(vin.data_ptr()), None), "cpsb_fermion_convert")
        want = oracle.fermion_convert(v, dims, ls, name, inverse=bool(direction))
        np.testing.assert_array_equal(vout.cpu().numpy(), want)
    # round trip
    _lib.check(lib.cpsb_fermion_convert(d, ls, order, 0, C.c_void_p(vout.data_ptr()), C.c_void_p(vin.data_ptr()),
                                        None), "cpsb_fermion_convert")
    back = torch.empty_like(vin)
    _lib.check(lib.cpsb_fermion_convert(d, ls, order, 1, C.c_void_p(back.data_ptr()), C.c_void_p(vout.data_ptr()),
                                        None), "cpsb_fermion_convert")
    np.testing.assert_array_equal(back.cpu().numpy(), v)

"""GPU test of tild_bond_observables_noalloc, the entry point for callers that cannot allocate
device memory (it keeps its partial sums in a fixed device array instead of cudaMalloc'd
scratch).  Its bond energy and virial must equal those of tild_observables for the same
positions, on two calls in a row (the second call reuses the array the first left behind).

Device buffers for the inputs come from torch here only because the test needs somewhere to put
them; the entry point itself allocates nothing.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import tild
from helpers import small_diblock

pytestmark = pytest.mark.gpu


def _entry():
    L = tild.lib()
    f = L.tild_bond_observables_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_float),
                  C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_void_p, C.c_void_p]
    f.restype = C.c_int32
    return f


@pytest.mark.parametrize("dim", [3, 2])
def test_noalloc_bond_observables_match_context(dim):
    torch = pytest.importorskip("torch")
    s = small_diblock(dim, 1)
    with tild.Context(s) as ctx:
        ctx.step(5)
        ref = ctx.observables()
        x, _, _ = ctx.get_state()
    dev = torch.device("cuda:0")
    d_x = torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    d_nb = torch.from_numpy(np.ascontiguousarray(s.n_bonds, np.int32)).to(dev)
    d_bt = torch.from_numpy(np.ascontiguousarray(s.bonded_to, np.int32)).to(dev)
    d_by = torch.from_numpy(np.ascontiguousarray(s.bond_type, np.int32)).to(dev)
    box = (C.c_float * 3)(*[float(s.box[d]) if d < dim else 1.0 for d in range(3)])
    bk = (C.c_float * len(s.bond_k))(*s.bond_k)
    br = (C.c_float * len(s.bond_req))(*s.bond_req)
    f = _entry()
    stream = torch.cuda.current_stream().cuda_stream
    np_comps = 6 if dim == 3 else 3
    results = []
    for _ in range(2):  # two calls in a row share the fixed scratch
        d_out = torch.full((1 + np_comps,), float("nan"), dtype=torch.float64, device=dev)
        st = f(d_x.data_ptr(), d_nb.data_ptr(), d_bt.data_ptr(), d_by.data_ptr(), s.ns, dim, box, len(s.bond_k), bk, br,
               d_out.data_ptr(), stream)
        assert st == tild.OK
        torch.cuda.synchronize()
        results.append(d_out.cpu().numpy())
    for out in results:
        assert out[0] == pytest.approx(ref["ubond"], rel=1e-12)
        np.testing.assert_allclose(out[1:], ref["bond_vir"], rtol=1e-10, atol=1e-14)
    np.testing.assert_array_equal(results[0], results[1])


def test_noalloc_rejects_sizes_beyond_its_scratch():
    f = _entry()
    box = (C.c_float * 3)(1.0, 1.0, 1.0)
    one = (C.c_float * 1)(1.0)
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    max_beads = 4096 * 256  # TILD_NOALLOC_MAX_BEADS
    st = f(dummy, dummy, dummy, dummy, max_beads + 1, 3, box, 1, one, one, dummy, None)
    assert st == tild.ERR_BAD_INPUT


@pytest.mark.parametrize("fault", ["negative_partner", "partner_past_end", "bond_count"])
def test_noalloc_corrupt_topology_gives_nan_energy(fault):
    """A partner id or bond count out of range poisons the energy instead of giving a plausible
    wrong number (a negative partner would otherwise be skipped by the j < i test)."""
    torch = pytest.importorskip("torch")
    s = small_diblock(3, 1)
    nb = np.ascontiguousarray(s.n_bonds, np.int32).copy()
    bt = np.ascontiguousarray(s.bonded_to, np.int32).copy()
    i = int(np.nonzero(nb > 0)[0][5])
    if fault == "negative_partner":
        bt[i, 0] = -3
    elif fault == "partner_past_end":
        bt[i, 0] = s.ns + 7
    else:
        nb[i] = 4
    dev = torch.device("cuda:0")
    d_x = torch.from_numpy(np.ascontiguousarray(s.x)).to(dev)
    d_nb = torch.from_numpy(nb).to(dev)
    d_bt = torch.from_numpy(bt).to(dev)
    d_by = torch.from_numpy(np.ascontiguousarray(s.bond_type, np.int32)).to(dev)
    box = (C.c_float * 3)(*[float(v) for v in s.box[:3]])
    bk = (C.c_float * len(s.bond_k))(*s.bond_k)
    br = (C.c_float * len(s.bond_req))(*s.bond_req)
    d_out = torch.zeros(7, dtype=torch.float64, device=dev)
    st = _entry()(d_x.data_ptr(), d_nb.data_ptr(), d_bt.data_ptr(), d_by.data_ptr(), s.ns, 3, box, len(s.bond_k), bk,
                  br, d_out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == tild.OK
    torch.cuda.synchronize()
    assert np.isnan(d_out.cpu().numpy()[0])

"""gr_lj_crf_innerloop_noalloc against gr_lj_crf_innerloop.

The allocation-free entry point takes device buffers (allocated here by
torch: the test may allocate, the entry point may not) and keeps its scratch
in a static device array.  Two calls in a row must both match the allocating
entry point on the same inputs; the file name sorts last so the test also runs
after every other GPU test has used the library.
"""
import ctypes as C

import numpy as np
import pytest

from golden_loader import load_fixture
import oracle_binding as ob

pytestmark = pytest.mark.gpu


def _inputs():
    s, _ = load_fixture("nacl_water_box")
    lists = ob.pairlist(s, algorithm=0)
    pairs = np.ascontiguousarray(np.concatenate([lists[0], lists[1], lists[3]]), dtype=np.uint32)
    lj = np.ascontiguousarray(s.topo.lj[:, :, :2], dtype=np.float64)
    return s, pairs, lj


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    from gromos_nb import _lib
    from gromos_nb.nonbonded import CRFParameters, lj_crf_innerloop

    s, pairs, lj = _inputs()
    crf = CRFParameters.new(s.params.rcutl, 1.0, s.params.epsrf, 0.0)
    f_ref, elj_ref, ecrf_ref, vir_ref = lj_crf_innerloop(s.pos, s.topo.charge, s.topo.iac, pairs, lj, crf, box=s.box)

    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    n = s.pos.shape[0]
    pos = torch.tensor(np.asarray(s.pos, dtype=np.float32), device=dev).contiguous()
    q = torch.tensor(np.asarray(s.topo.charge, dtype=np.float32), device=dev)
    iac = torch.tensor(np.asarray(s.topo.iac, dtype=np.int32), device=dev)
    pl = torch.tensor(pairs.astype(np.int32), device=dev).contiguous()
    ljd = torch.tensor(lj.reshape(-1), device=dev)
    # outputs start as garbage: the entry point clears forces and overwrites the rest
    forces = torch.full((n, 3), 7.0, dtype=torch.float32, device=dev)
    energies = torch.full((2,), 7.0, dtype=torch.float64, device=dev)
    virial = torch.full((9,), 7.0, dtype=torch.float64, device=dev)
    box = np.ascontiguousarray(s.box, dtype=np.float64)
    stream = torch.cuda.current_stream(dev)

    fn = _lib.lib().gr_lj_crf_innerloop_noalloc
    for _ in range(2):
        st = fn(pos.data_ptr(), q.data_ptr(), iac.data_ptr(), n, pl.data_ptr(), pairs.shape[0], ljd.data_ptr(),
                lj.shape[0], box.ctypes.data_as(C.c_void_p), 1, crf.crf_cut, crf.crf_2cut3i, crf.crf_cut3i,
                forces.data_ptr(), energies.data_ptr(), virial.data_ptr(), C.c_void_p(stream.cuda_stream))
        _lib.check(st)
        stream.synchronize()
        f = forces.cpu().numpy().astype(np.float64)
        e = energies.cpu().numpy()
        v = virial.cpu().numpy().reshape(3, 3)
        # both paths run the same FP32 pair kernel; only the order of the
        # float/double atomic additions differs between launches
        ref = f_ref.astype(np.float64)
        rms = np.sqrt(np.mean((f - ref) ** 2) / np.mean(ref ** 2))
        assert rms < 1e-5
        assert abs(e[0] - elj_ref) <= 1e-6 * max(1.0, abs(elj_ref))
        assert abs(e[1] - ecrf_ref) <= 1e-6 * max(1.0, abs(ecrf_ref))
        assert np.max(np.abs(v - vir_ref)) <= 1e-5 * max(1.0, np.max(np.abs(vir_ref)))


def test_noalloc_rejects_too_many_types():
    from gromos_nb import _lib

    # rejected before any device work: every pointer may be null here
    st = _lib.lib().gr_lj_crf_innerloop_noalloc(None, None, None, 0, None, 0, None, 65, None, 0, 0.0, 0.0, 0.0,
                                               None, None, None, None)
    assert st == _lib.GR_ERR_INVALID
    assert b"64" in _lib.lib().gr_last_error()

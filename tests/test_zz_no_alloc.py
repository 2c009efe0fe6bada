"""lmc_deryr2_noalloc: the compact y-derivative for callers that may not
allocate device memory (a fixed device-memory budget handed over by the
driver, or a time loop that cannot afford cudaFree's device-wide
synchronisation).  Its operator tables live in a fixed per-device array
inside the library, so it must give the same result as the handle-based
operator (lmc_op_y, op 1) and as the FP64 oracle's deryr -- here on two
calls in a row, and after a call on another grid has overwritten that
array.  The file sorts last so that a run stopping at the first failure has
already run every other test."""
import numpy as np
import pytest

from loma_phd_b200 import Lomacte, stretched_mesh
from loma_phd_b200 import lomacte as lm
from tests.helpers import case, oracle_for, rel_l2

pytestmark = pytest.mark.gpu
OP_TOL = 1e-12  # the single-operator tolerance of the parity tests


def _field(p, y, seed):
    rng = np.random.default_rng(seed)
    shp = p.shape
    return (rng.standard_normal(shp) + 1j * rng.standard_normal(shp)) * np.exp(-(y / 6.0) ** 2)


@pytest.mark.parametrize("ny", [65, 257])
def test_noalloc_matches_handle_operator(gpu, ny):
    import torch
    p, y, st = case(nx=16, nz=16, ny=ny)
    g = Lomacte(p, y)
    f = _field(p, y, ny)
    fin = torch.from_numpy(f.view(np.float64).copy()).cuda()
    ref = torch.empty_like(fin)  # op_y writes every entry on the handle's stream
    torch.cuda.synchronize()
    g.op_y(1, fin, ref)
    torch.cuda.synchronize()
    ref_h = ref.cpu().numpy().view(np.complex128)
    # the oracle's deryr, pencil by pencil
    o = oracle_for(p, y, st, nthreads=2)
    fo = f.reshape(-1, p.my)
    ref_o = np.array([o.deryr(u.real) + 1j * o.deryr(u.imag) for u in fo])
    npencil = p.nplanes * p.mz
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # two calls in a row share the scratch array
        out = torch.full_like(fin, float("nan"))
        rc = lm.deryr2_noalloc(y, npencil, fin.data_ptr(), out.data_ptr(), stream)
        assert rc == lm.LMC_OK
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.complex128)
        e = rel_l2(got, ref_h)
        assert e < OP_TOL, e
        e = rel_l2(got.reshape(-1, p.my), ref_o)
        assert e < OP_TOL, e
    g.close()


def test_noalloc_after_other_grid_and_limits(gpu):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    # a call on another grid rewrites the shared array first
    y1 = stretched_mesh(129)
    a = torch.zeros(2 * 129 * 5, dtype=torch.float64, device="cuda")
    b = torch.zeros_like(a)
    assert lm.deryr2_noalloc(y1, 5, a.data_ptr(), b.data_ptr(), stream) == lm.LMC_OK
    p, y, _ = case(nx=16, nz=16, ny=33)
    g = Lomacte(p, y)
    f = _field(p, y, 3)
    fin = torch.from_numpy(f.view(np.float64).copy()).cuda()
    ref = torch.empty_like(fin)
    torch.cuda.synchronize()
    g.op_y(1, fin, ref)
    out = torch.zeros_like(fin)
    assert lm.deryr2_noalloc(y, p.nplanes * p.mz, fin.data_ptr(), out.data_ptr(), stream) == lm.LMC_OK
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), ref.cpu().numpy()) < OP_TOL
    # beyond the scratch limit: rejected before any launch
    big = stretched_mesh(545)
    assert lm.deryr2_noalloc(big, 1, fin.data_ptr(), out.data_ptr(), stream) == lm.LMC_EINVAL
    # in place, and an output shifted by one double: rejected, nothing launched
    n = p.nplanes * p.mz
    assert lm.deryr2_noalloc(y, n, fin.data_ptr(), fin.data_ptr(), stream) == lm.LMC_EINVAL
    assert lm.deryr2_noalloc(y, n - 1, fin.data_ptr(), out.data_ptr() + 8, stream) == lm.LMC_EINVAL
    g.close()


def test_noalloc_refuses_a_capturing_stream(gpu):
    """The table upload reads a host buffer released on return, so a call on
    a stream under capture is refused rather than recorded."""
    import torch
    p, y, _ = case(nx=16, nz=16, ny=33)
    n = p.nplanes * p.mz
    a = torch.zeros(2 * p.my * n, dtype=torch.float64, device="cuda")
    b = torch.zeros_like(a)
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    # the first call in this context, outside any capture
    assert lm.deryr2_noalloc(y, n, a.data_ptr(), b.data_ptr(), s.cuda_stream) == lm.LMC_OK
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        rc = lm.deryr2_noalloc(y, n, a.data_ptr(), b.data_ptr(), s.cuda_stream)
        b.add_(0.0)  # the capture holds one node of its own
    assert rc == lm.LMC_EINVAL
    del graph

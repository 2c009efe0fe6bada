"""lmc_deryr2_noalloc: the compact y-derivative for callers that may not
allocate device memory (a fixed device-memory budget handed over by the
driver, or a time loop that cannot afford cudaFree's device-wide
synchronisation).  Its operator tables live in a fixed per-device array
inside the library, so it must give the same result as the handle-based
operator (lmc_op_y, op 1) -- here on two calls in a row, and after a call
on another grid has overwritten that array.  The file sorts last so that a
run stopping at the first failure has already run every other test."""
import numpy as np
import pytest

from loma_phd_b200 import Lomacte, stretched_mesh
from loma_phd_b200 import lomacte as lm
from tests.helpers import case, rel_l2

pytestmark = pytest.mark.gpu
OP_TOL = 1e-12  # the single-operator tolerance of the parity tests


def _field(p, y, seed):
    rng = np.random.default_rng(seed)
    shp = p.shape
    return (rng.standard_normal(shp) + 1j * rng.standard_normal(shp)) * np.exp(-(y / 6.0) ** 2)


@pytest.mark.parametrize("ny", [65, 257])
def test_noalloc_matches_handle_operator(gpu, ny):
    import torch
    p, y, _ = case(nx=16, nz=16, ny=ny)
    g = Lomacte(p, y)
    f = _field(p, y, ny)
    fin = torch.from_numpy(f.view(np.float64).copy()).cuda()
    ref = torch.zeros_like(fin)
    g.op_y(1, fin, ref)
    torch.cuda.synchronize()
    ref_h = ref.cpu().numpy().view(np.complex128)
    npencil = p.nplanes * p.mz
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # two calls in a row share the scratch array
        out = torch.full_like(fin, float("nan"))
        rc = lm.deryr2_noalloc(y, npencil, fin.data_ptr(), out.data_ptr(), stream)
        assert rc == lm.LMC_OK
        torch.cuda.synchronize()
        e = rel_l2(out.cpu().numpy().view(np.complex128), ref_h)
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
    ref = torch.zeros_like(fin)
    g.op_y(1, fin, ref)
    out = torch.zeros_like(fin)
    assert lm.deryr2_noalloc(y, p.nplanes * p.mz, fin.data_ptr(), out.data_ptr(), stream) == lm.LMC_OK
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), ref.cpu().numpy()) < OP_TOL
    # beyond the scratch limit: rejected before any launch
    big = stretched_mesh(545)
    assert lm.deryr2_noalloc(big, 1, fin.data_ptr(), out.data_ptr(), stream) == lm.LMC_EINVAL
    g.close()

"""Pencil assembly on the GPU (amls_hex_assemble): element integration of
8- and 27-node hex elasticity elements and CSR assembly on the device, in
the pattern of amls_element_pattern, against the host assembly of the same
seeded pencils (1e-13 relative), and a solve from the device-assembled
values against the host-assembled solve."""
import numpy as np
import pytest

from amls_b200 import AmlsOptions, cases
from amls_b200.solver import element_pattern

from .helpers import rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,order", [((4, 3, 5), 1), ((3, 2, 3), 2), ((7, 7, 7), 2)])
def test_gpu_assembly_matches_host(solver, shape, order):
    p = cases.hex_pencil(*shape, order, seed=5)
    rp, ci = element_pattern(p.n, p.dofmap)
    assert np.array_equal(rp, p.K.indptr) and np.array_equal(ci, p.K.indices)
    K, M = solver.assemble_hex(p, rp, ci)
    for A, B in ((K, p.K), (M, p.M)):
        assert np.max(np.abs(A.data - B.data)) <= 1e-13 * np.max(np.abs(B.data))


def test_solve_from_device_assembled_values(solver):
    import torch
    p = cases.config_pencil("C2", seed=0)
    rp, ci = element_pattern(p.n, p.dofmap)
    kv = torch.zeros(ci.size, dtype=torch.float64, device="cuda")
    mv = torch.zeros(ci.size, dtype=torch.float64, device="cuda")
    solver.assemble_hex(p, rp, ci, on_device=True, k_ptr=kv.data_ptr(), m_ptr=mv.data_ptr())
    o = AmlsOptions(nev=100, nLevels=6, leafSize=500, recoverVectors=False)
    ref = solver.solve(p.K, p.M, o)
    solver.analyze(p.K, p.M, o)
    th = torch.zeros(100, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    solver.solve_values(kv.data_ptr(), mv.data_ptr(), True, th.data_ptr(), None, True)
    torch.cuda.synchronize()
    assert rel_err(th.cpu().numpy(), ref.theta) < 1e-11

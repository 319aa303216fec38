"""Known-answer energies of small chains where DMRG is exact (bond dimension at
the full Hilbert-space size): the GPU chain (iDMRG + sweeps, FP64 and mixed)
against exact diagonalisation (oracle/ed.py, pinned against the reference's own
runs in test_ed_cpu.py), including the triplet sector (SU(2) 2J = 2, U(1)
2Sz = 2) and open chains.  Tolerance 1e-9 relative.
"""
import pytest

from oracle import ed

pytestmark = pytest.mark.gpu

CASES = [
    # sym, cplx, L, D, open, totspin
    (1, False, 12, 64, False, 2),
    (0, False, 12, 64, False, 2),
    (0, True, 12, 64, False, 2),
    (1, False, 12, 64, True, 0),
    (0, False, 12, 64, True, 0),
    (1, True, 8, 16, True, 0),
    (0, False, 8, 16, True, 0),
]


@pytest.mark.parametrize("sym,cplx,L,D,open_bc,totspin", CASES,
                         ids=lambda v: str(v))
@pytest.mark.parametrize("prec", ["fp64", "tf32x3"])
def test_chain_energy_known_answer(sym, cplx, L, D, open_bc, totspin, prec):
    import sadmrg
    h = sadmrg.Handle(sym=sym, cplx=cplx)
    h.chain_create(1, L, D, 1, totspin, open_bc, 0.0)
    h.chain_set_precision(sadmrg.PREC_FP64 if prec == "fp64" else sadmrg.PREC_TF32X3)
    h.set_lanczos_tol(1e-12)
    h.chain_idmrg()
    e = None
    for _ in range(2):
        e = h.chain_sweep()
    ref = ed.ground_energy(L, periodic=not open_bc, two_sz=totspin)
    assert abs(e - ref) <= 1e-9 * abs(ref), (e, ref)
    assert h.device_status() == 0
